"""Reader for the reference's pio files (simUtil/src/pio.c): a FILEHEADER
object, a blank line, then records, split over files name#000000,
name#000001, ... (the header is in the first).  Data types FIXRECORDASCII,
FIXRECORDBINARY (little-endian, endian_key 875770417) and VARRECORDASCII
(one record per line), the three readPioFile handles
(elec/readPioFile.cc:33-66).  Field types: u / i (integers), f (float) in
ASCII; u8, u4, i8, i4, f8, f4 in binary."""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class PioFile:
    header: dict
    fields: dict = field(default_factory=dict)      # name -> array (int64 or float64)
    units: dict = field(default_factory=dict)

    @property
    def names(self):
        return self.header["field_names"].split()


def parse_header(text):
    body = text[text.index("{") + 1:text.rindex("}")]
    out = {}
    for item in body.replace("\n", " ").split(";"):
        if "=" in item:
            k, v = item.split("=", 1)
            out[k.strip()] = v.strip()
    return out


def split_header(raw):
    """(header text, its length): lines up to and including the first line
    of at most one character, as readPheader counts them
    (simUtil/src/pio.c:642-703)."""
    pos = 0
    while True:
        nl = raw.index(b"\n", pos)
        line = raw[pos:nl + 1]
        pos = nl + 1
        if len(line) <= 1:
            return raw[:pos].decode(), pos


_BIN = {"u8": "<u8", "u4": "<u4", "i8": "<i8", "i4": "<i4", "f8": "<f8", "f4": "<f4"}
_INT = ("u", "i", "u8", "u4", "i8", "i4")


def read(name):
    """name: the file name without the #000000 suffix, with or without
    its trailing '#'."""
    base = name[:-1] if name.endswith("#") else name
    with open(base + "#000000", "rb") as f:
        raw = f.read()
    head, hlen = split_header(raw)
    hdr = parse_header(head)
    chunks = [raw[hlen:]]
    for k in range(1, int(hdr.get("nfiles", "1"))):
        with open(base + "#%06d" % k, "rb") as f:
            chunks.append(f.read())
    data = b"".join(chunks)
    names = hdr["field_names"].split()
    types = hdr["field_types"].split()
    units = hdr.get("field_units", " ".join(["1"] * len(names))).split()
    n = int(hdr.get("nrecord", hdr.get("nrecords", "-1")))
    out = PioFile(hdr, units=dict(zip(names, units)))
    kind = hdr["datatype"]
    if kind == "FIXRECORDBINARY":
        dt = np.dtype([(nm, _BIN[t]) for nm, t in zip(names, types)])
        if "lrec" in hdr and dt.itemsize != int(hdr["lrec"]):
            raise ValueError("record length does not match the field types")
        rec = np.frombuffer(data, dtype=dt, count=n)
        for nm, t in zip(names, types):
            out.fields[nm] = rec[nm].astype(np.int64 if t in _INT else np.float64)
        return out
    if kind == "FIXRECORDASCII":
        lrec = int(hdr["lrec"])
        tok = np.array(data[:n * lrec].split())
    elif kind == "VARRECORDASCII":
        lines = [ln for ln in data.split(b"\n") if ln.strip()]
        if n >= 0:
            lines = lines[:n]
        n = len(lines)
        tok = np.array(b" ".join(lines).split())
    else:
        raise ValueError("unsupported pio datatype " + kind)
    tok = tok.reshape(n, len(names))
    for j, (nm, t) in enumerate(zip(names, types)):
        out.fields[nm] = tok[:, j].astype(np.int64 if t in _INT else np.float64)
    return out
