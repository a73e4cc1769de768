"""Checkpoint / restart in the reference's pio state format.

A checkpoint is a directory snapshot.<loop, 12 digits> holding
  state#000000   a pio file: the FILEHEADER object, a blank line, then one
                 fixed-length record per cell (gid, Vm, the 18 BetterTT06
                 states in checkpoint order);
  restart        "<name> SIMULATE { loop=..; time=..; stateFile=..; }".
The layout, header keys, field names, types and units and the record
formats follow writeCheckpoint / writeHeader / writeRestart
(elec/checkpointIO.cc:57-202): ASCII records "%12llu %21.13e" then
" %21.13e" per state and "\\n" (lossy: 14 significant digits), or BINARY
records of little-endian u8 gid and f8 values (exact).  Reading follows
readCheckpoint (elec/checkpointIO.cc:205-268): fields are matched by name,
converted from the file's units, records matched to cells by gid; Vm is
loaded when present.  The reference's own reader (simUtil pio.c,
elec/readPioFile.cc) reads what `write` produces.
"""
import os
import struct
import time as _time
from dataclasses import dataclass, field

import numpy as np

from . import pio, tt06

ENDIAN_KEY = struct.unpack("<i", b"1234")[0]     # 875770417, memcpy of "1234" on a little-endian host


def field_units():
    """Units of the checkpointed states (BetterTT06 getUnit, elec/BetterTT06.cc:1773-1790)."""
    return [tt06.STATE_UNITS.get(n, "1") for n in tt06.STATE_NAMES]


def header_text(nrecord, loop, time, nx, ny, nz, binary, reaction_method="BetterTT06", nfiles=1, create_time=None):
    names = ["gid", "Vm"] + list(tt06.STATE_NAMES)
    nstate = len(tt06.STATE_NAMES)
    if binary:
        dtype, lrec, types = "FIXRECORDBINARY", 8 * (nstate + 2), ["u8", "f8"] + ["f8"] * nstate
    else:
        dtype, lrec, types = "FIXRECORDASCII", 34 + 22 * nstate + 1, ["u", "f"] + ["f"] * nstate
    units = ["1", "mV"] + field_units()
    ct = create_time or _time.asctime()
    return ("state FILEHEADER {\n"
            "   create_time = %s;\n"
            "   user = %s;   host = %s;\n"
            "   exe_version = %s;   srcpath = %s;\n"
            "   compile_time = %s;\n"
            "   datatype = %s;\n"
            "   nfiles = %d;\n"
            "   nrecord = %d;\n"
            "   lrec = %d;\n"
            "   endian_key = %d;\n"
            "   time = %f;\n"
            "   loop = %d;\n"
            "   reactionMethod = %s;\n"
            "   nfields = %d;\n"
            "   field_names = %s;\n"
            "   field_types = %s;\n"
            "   field_units = %s;\n"
            "   nx = %u; ny = %u; nz = %u;\n"
            "}\n\n") % (ct, os.environ.get("USER", "unknown"), "b200", "cardioid_b200", "cardioid_b200", ct, dtype,
                        nfiles, nrecord, lrec, ENDIAN_KEY, time, loop, reaction_method, len(names), " ".join(names),
                        " ".join(types), " ".join(units), nx, ny, nz), lrec


def write(directory, gid, vm, states, loop, time, nx, ny, nz, binary=True, name="simulate",
          reaction_method="BetterTT06", create_time=None):
    """Writes directory/state#000000 and directory/restart.  states: 18 x n
    in checkpoint order.  Returns the state file's pio name (ending '#')."""
    gid = np.ascontiguousarray(gid, dtype=np.uint64)
    vm = np.ascontiguousarray(vm, dtype=np.float64)
    states = np.ascontiguousarray(states, dtype=np.float64)
    n = gid.shape[0]
    assert vm.shape == (n,) and states.shape == (len(tt06.STATE_NAMES), n)
    os.makedirs(directory, exist_ok=True)
    head, lrec = header_text(n, loop, time, nx, ny, nz, binary, reaction_method, create_time=create_time)
    path = os.path.join(directory, "state#000000")
    with open(path, "wb") as f:
        f.write(head.encode())
        if binary:
            rec = np.empty(n, dtype=np.dtype([("gid", "<u8"), ("vm", "<f8"), ("s", "<f8", (states.shape[0],))]))
            rec["gid"], rec["vm"], rec["s"] = gid, vm, states.T
            assert rec.dtype.itemsize == lrec
            f.write(rec.tobytes())
        else:
            fmt = "%12d %21.13e" + " %21.13e" * states.shape[0] + "\n"
            rows = np.column_stack([vm, states.T])
            f.write("".join(fmt % ((int(g),) + tuple(r)) for g, r in zip(gid, rows)).encode())
    with open(os.path.join(directory, "restart"), "w") as f:
        f.write("%s SIMULATE {\n   loop=%d; time=%f; stateFile=%s;\n}\n" % (name, loop, time,
                                                                            os.path.join(directory, "state")))
    return os.path.join(directory, "state#")


@dataclass
class Checkpoint:
    header: dict
    fields: dict = field(default_factory=dict)     # name -> float64 array (gid as int64)
    units: dict = field(default_factory=dict)

    @property
    def loop(self):
        return int(self.header.get("loop", 0))

    @property
    def time(self):
        return float(self.header.get("time", 0.0))


def read(name):
    """Reads a pio state file; name is the file name without the
    #000000 suffix, with or without its trailing '#'."""
    f = pio.read(name)
    return Checkpoint(f.header, f.fields, f.units)


# units_convert (simUtil/src/units.c) for the units BetterTT06 states use
_SCALE = {"mM": 1e-3, "uM": 1e-6, "nM": 1e-9, "M": 1.0, "mV": 1e-3, "V": 1.0, "1": 1.0}


def unit_factor(src, dst):
    if src == dst:
        return 1.0
    if src in _SCALE and dst in _SCALE and (src in ("mV", "V")) == (dst in ("mV", "V")):
        return _SCALE[src] / _SCALE[dst]
    raise ValueError("cannot convert %s to %s" % (src, dst))


def save(engine, tid, tissue, directory=None, binary=True, name="simulate", reaction_method=None, root="."):
    """Writes the tissue's checkpoint at its current step; returns the
    directory (default root/snapshot.<loop, 12 digits>)."""
    loop, time = engine.time(tid)
    directory = directory or os.path.join(root, "snapshot.%012d" % loop)
    write(directory, tissue.gid, engine.read_vm(tid), engine.read_states(tid), loop, time, tissue.nx, tissue.ny,
          tissue.nz, binary=binary, name=name, reaction_method=reaction_method or "BetterTT06")
    return directory


def restore(engine, tid, tissue, name, time=None):
    """Loads a checkpoint into a tissue already added to the engine: Vm and
    every state the file holds (by name, converted from its units), cells
    matched by gid; then the tissue's clock (the header's loop and time, or
    `time` when given).  Returns (loop, time)."""
    ck = read(name)
    gid = ck.fields["gid"]
    order = np.argsort(gid, kind="stable")
    pos = np.searchsorted(gid[order], tissue.gid)
    if np.any(pos >= len(gid)) or np.any(gid[order][np.minimum(pos, len(gid) - 1)] != tissue.gid):
        raise ValueError("the checkpoint does not hold every cell of the tissue")
    take = order[pos]
    units = dict(zip(tt06.STATE_NAMES, field_units()))
    for nm, vals in ck.fields.items():
        if nm in units:
            engine.write_state(tid, nm, vals[take] * unit_factor(ck.units.get(nm, "1"), units[nm]))
    if "Vm" in ck.fields:
        engine.write_vm(tid, ck.fields["Vm"][take] * unit_factor(ck.units.get("Vm", "mV"), "mV"))
    t = ck.time if time is None else time
    engine.set_clock(tid, ck.loop, t)
    return ck.loop, t
