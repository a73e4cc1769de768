"""Python face of the fused B200 engine (libcardioid_b200.so, cdb_engine_*).

    eng = Engine(dt=0.02, precision="fp64")
    rx = [eng.add_reaction(p) for p in params]           # BetterTT06 parameter sets
    tid = eng.add_tissue(tissue, reaction=rx_per_cell)    # a cardioid_b200.tissue.Tissue
    eng.step(1000)
    vm = eng.read_vm(tid)

One engine drives any number of tissues (instances) in one launch per
step; tissues join and retire between steps.
"""
import ctypes
import os

import numpy as np

from . import _lib, objectdb, tt06
from .tissue import Tissue

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
PRECISIONS = {"fp64": _lib.CDB_FP64, "mixed": _lib.CDB_MIXED}


def shipped_fit_path(dt, celltype):
    return os.path.join(DATA, "tt06_dt%g_celltype%d.fit.data" % (dt, int(celltype)))


def default_params(celltype, dt, g_K1=None):
    """BetterTT06 defaults for a celltype with fits: the shipped fit file when
    one matches dt, celltype and g_K1 (the reference's reuse rule), else
    freshly generated (cardioid_b200.fitgen)."""
    p = tt06.TT06Params.defaults(celltype)
    if g_K1 is not None:
        p.g_K1 = g_K1
    path = shipped_fit_path(dt, celltype)
    if os.path.exists(path):
        db = objectdb.ObjectDB().compile_file(path)
        names = db.names("FIT")
        fobj = db.find(names[0], "FIT")
        if (objectdb.get_float(fobj, "dt") == dt and objectdb.get_float(fobj, "celltype") == p.celltype
                and objectdb.get_float(fobj, "g_K1") == p.g_K1):
            p.fits = tt06.fits_from_fit_object(db, names[0])
            return p
    from . import fitgen
    p.fits = fitgen.generate(dt, p)
    return p


class Engine:
    def __init__(self, dt, precision="fp64", device=0, use_graphs=True):
        L = _lib.load()
        cfg = _lib.EngineConfig()
        cfg.device = device
        cfg.precision = PRECISIONS[precision]
        cfg.dt = dt
        cfg.use_graphs = 1 if use_graphs else 0
        h = ctypes.c_void_p()
        _lib.check(L.cdb_engine_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.dt = dt
        self.precision = precision
        self.tissues = {}

    def close(self):
        if getattr(self, "h", None):
            _lib.load().cdb_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_reaction(self, params):
        """Registers a TT06Params (with its 30 fits); returns its id."""
        fits = _lib.to_fit_array(params.fits)
        cp = _lib.to_params(params)
        rid = ctypes.c_int32()
        _lib.check(_lib.load().cdb_engine_add_reaction(self.h, ctypes.byref(cp), fits, ctypes.byref(rid)))
        return rid.value

    def _desc(self, t, reaction, scales):
        n = t.n
        keep = {}
        d = _lib.TissueDesc()
        d.nx, d.ny, d.nz = t.nx, t.ny, t.nz
        d.dx, d.dy, d.dz = t.dx, t.dy, t.dz
        d.nCells = n
        full = n == t.nx * t.ny * t.nz and np.array_equal(t.gid, np.arange(n))
        if full:
            d.gid = None
        else:
            keep["gid"] = np.ascontiguousarray(t.gid, dtype=np.int64)
            d.gid = keep["gid"].ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        keep["ct"] = np.ascontiguousarray(t.cell_type, dtype=np.int32)
        d.cellType = keep["ct"].ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        keep["rx"] = np.ascontiguousarray(reaction, dtype=np.uint8)
        d.reaction = keep["rx"].ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        keep["sig"] = np.ascontiguousarray(t.sigma, dtype=np.float64)
        d.sigma6 = _lib.dptr(keep["sig"])
        if t.vm0 is not None:
            keep["vm0"] = np.ascontiguousarray(t.vm0, dtype=np.float64)
            d.vm0 = _lib.dptr(keep["vm0"])
        d.diffusionScale = t.diffusion_scale
        d.g_Kr_scale, d.g_CaL_scale, d.g_Na_scale = scales
        d.nStim = len(t.stimuli)
        keep["stim"] = (_lib.Stimulus * max(1, len(t.stimuli)))(*[_lib.to_stimulus(s) for s in t.stimuli])
        d.stim = keep["stim"]
        return d, keep

    def tissue_bytes(self, t, reaction=None, scales=(1.0, 1.0, 1.0)):
        reaction = np.zeros(t.n, np.uint8) if reaction is None else reaction
        d, keep = self._desc(t, reaction, scales)
        b = ctypes.c_int64()
        _lib.check(_lib.load().cdb_engine_tissue_bytes(self.h, ctypes.byref(d), ctypes.byref(b)))
        return b.value

    def free_bytes(self):
        f, t = ctypes.c_int64(), ctypes.c_int64()
        _lib.check(_lib.load().cdb_engine_free_bytes(self.h, ctypes.byref(f), ctypes.byref(t)))
        return f.value, t.value

    def add_tissue(self, t, reaction, scales=(1.0, 1.0, 1.0)):
        """Adds a Tissue; ``reaction`` gives the reaction id of every cell."""
        d, keep = self._desc(t, reaction, scales)
        tid = ctypes.c_int32()
        _lib.check(_lib.load().cdb_engine_add_tissue(self.h, ctypes.byref(d), ctypes.byref(tid)))
        self.tissues[tid.value] = t.n
        return tid.value

    def remove_tissue(self, tid):
        _lib.check(_lib.load().cdb_engine_remove_tissue(self.h, tid))
        del self.tissues[tid]

    def step(self, n=1):
        _lib.check(_lib.load().cdb_engine_step(self.h, int(n)))

    def sync(self):
        _lib.check(_lib.load().cdb_engine_sync(self.h))

    def test_bounded_wait(self):
        """The next step batch withholds its bulk copies after each warp's
        first tile, so its bounded waits run out (about a second) and sync
        raises a CdbError with status TIMEOUT; for testing the failure path."""
        _lib.check(_lib.load().cdb_engine_test_bounded_wait(self.h))

    def time(self, tid):
        s, t = ctypes.c_int64(), ctypes.c_double()
        _lib.check(_lib.load().cdb_engine_tissue_time(self.h, tid, ctypes.byref(s), ctypes.byref(t)))
        return s.value, t.value

    def set_clock(self, tid, loop, time):
        """A restart: the tissue continues from step `loop` at `time` (ms)."""
        _lib.check(_lib.load().cdb_engine_set_clock(self.h, tid, int(loop), float(time)))

    def set_ecg(self, tid, points, eval_rate, kconst=1.0):
        """Fused ECG pseudo-sensor: electrodes points (n x 3, mm), evaluated
        every eval_rate steps (ECGSensor)."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        self._ecg_n = {**getattr(self, "_ecg_n", {}), tid: len(pts)}
        _lib.check(_lib.load().cdb_engine_set_ecg(self.h, tid, len(pts), _lib.dptr(pts), int(eval_rate),
                                                  float(kconst)))

    def read_ecg(self, tid, max_entries=1024):
        """(loops, values[entries, electrodes]) of the evaluations not read yet."""
        n = self._ecg_n.get(tid, 0)
        loops = np.empty(max_entries, np.int64)
        vals = np.empty(max_entries * max(n, 1))
        cnt = ctypes.c_int64()
        _lib.check(_lib.load().cdb_engine_read_ecg(
            self.h, tid, max_entries, ctypes.byref(cnt), loops.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            _lib.dptr(vals)))
        k = cnt.value
        return loops[:k].copy(), vals[:k * n].reshape(k, n)

    def read_vm(self, tid):
        out = np.empty(self.tissues[tid])
        _lib.check(_lib.load().cdb_engine_read_vm(self.h, tid, _lib.dptr(out)))
        return out

    def write_vm(self, tid, vm):
        v = np.ascontiguousarray(vm, dtype=np.float64)
        _lib.check(_lib.load().cdb_engine_write_vm(self.h, tid, _lib.dptr(v)))

    def read_state(self, tid, var):
        k = tt06.STATE_NAMES.index(var) if isinstance(var, str) else int(var)
        out = np.empty(self.tissues[tid])
        _lib.check(_lib.load().cdb_engine_read_state(self.h, tid, k, _lib.dptr(out)))
        return out

    def write_state(self, tid, var, values):
        k = tt06.STATE_NAMES.index(var) if isinstance(var, str) else int(var)
        v = np.ascontiguousarray(values, dtype=np.float64)
        _lib.check(_lib.load().cdb_engine_write_state(self.h, tid, k, _lib.dptr(v)))

    def read_states(self, tid):
        return np.stack([self.read_state(tid, k) for k in range(tt06.NSTATE)])

    def read_activation(self, tid):
        out = np.empty(self.tissues[tid])
        _lib.check(_lib.load().cdb_engine_read_activation(self.h, tid, _lib.dptr(out)))
        return out

    def minmax(self, tid):
        lo, hi = ctypes.c_double(), ctypes.c_double()
        _lib.check(_lib.load().cdb_engine_minmax(self.h, tid, ctypes.byref(lo), ctypes.byref(hi)))
        return lo.value, hi.value

    def read_weights(self, tid):
        out = np.empty(self.tissues[tid] * 19)
        _lib.check(_lib.load().cdb_engine_read_weights(self.h, tid, _lib.dptr(out)))
        return out.reshape(-1, 19)

    def step_host(self, tid, vm_in, vm_out):
        _lib.check(_lib.load().cdb_engine_step_host(self.h, tid, _lib.dptr(vm_in), _lib.dptr(vm_out)))

    def set_tuning(self, stage, ctas_per_sm):
        """stage: how each warp gets its next tile's inputs while it computes
        the current one: 0 = direct loads, 1 = per-lane cp.async into shared
        memory, 2 = bulk (TMA) copies into shared memory completing on an
        mbarrier, 3 = as 2, plus the Vm tile and halo of each row tile (the
        nine stencil rows of 32 consecutive voxels of a volume tissue) copied
        into shared memory while the reaction computes (defaults: 2 mixed,
        0 FP64; every stage gives the same bits); ctas_per_sm sizes the
        persistent grid (0: as many CTAs per SM as are resident)."""
        _lib.check(_lib.load().cdb_engine_set_tuning(self.h, int(stage), int(ctas_per_sm)))

    def set_layout(self, layout):
        """Warp-tile layout of tissues added from now on: "cells" (each
        reaction type's cells in cell order, 32 per tile) or "rows" (the
        default: every x-row run of a type cut into whole 32-cell row tiles,
        remainders packed).  Same results bit for bit."""
        code = {"cells": 0, "rows": 1}[layout]
        _lib.check(_lib.load().cdb_engine_set_layout(self.h, code))

    def get_layout(self):
        v = ctypes.c_int32()
        _lib.check(_lib.load().cdb_engine_get_layout(self.h, ctypes.byref(v)))
        return ("cells", "rows")[v.value]

    def get_tuning(self):
        p, c = ctypes.c_int32(), ctypes.c_int32()
        _lib.check(_lib.load().cdb_engine_get_tuning(self.h, ctypes.byref(p), ctypes.byref(c)))
        return p.value, c.value

    def launch_count(self):
        c = ctypes.c_int64()
        _lib.check(_lib.load().cdb_engine_launch_count(self.h, ctypes.byref(c)))
        return c.value

    def stream(self):
        s = ctypes.c_void_p()
        _lib.check(_lib.load().cdb_engine_stream(self.h, ctypes.byref(s)))
        return s.value


def transmural_setup(eng, tissue, dt):
    """Registers the endo/mid/epi BetterTT06 types (celltype 0/1/2) and maps
    anatomy cellType 100/101/102 onto them; returns the per-cell reaction ids
    and the TT06Params used."""
    params = [default_params(ct, dt) for ct in (0, 1, 2)]
    ids = [eng.add_reaction(p) for p in params]
    ct = np.asarray(tissue.cell_type)
    if ((ct < 100) | (ct > 102)).any():
        raise ValueError("transmural tissues use anatomy cellType 100/101/102")
    lut = np.array(ids, dtype=np.uint8)
    return lut[ct - 100], params
