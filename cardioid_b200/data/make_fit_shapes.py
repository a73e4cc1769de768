"""Writes cardioid_b200/csrc/fit_shapes.h: the compile-time fit shapes of the
specialised step kernels, from the shipped fit files.

Per fit slot the header holds the largest numerator and denominator term
counts over the shipped celltypes; a reaction type whose fits are no longer
than these is packed zero-padded at the header's fixed offsets (leading zero
coefficients leave Horner's result unchanged) and runs the fully unrolled
kernel; any other fit set runs the generic kernel.  The header also lists
the fits the mixed kernel evaluates in FP64 (those whose monomial form
loses more than 1e-5 of their range in FP32, as decided at registration).

    python -m cardioid_b200.data.make_fit_shapes
"""
import os

import numpy as np

from cardioid_b200 import engine, tt06

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(HERE), "csrc", "fit_shapes.h")


def fp32_loses(f, slot):
    lo, hi = (1e-7, 0.1) if slot == 0 else (-100.0, 100.0)
    x = np.linspace(lo, hi, 4001)
    v = f.eval(x)
    c = np.array(f.coeff, dtype=np.float32)
    xf = x.astype(np.float32)
    num = np.full_like(xf, c[f.numer - 1])
    for k in range(f.numer - 2, -1, -1):
        num = (xf * num + c[k]).astype(np.float32)
    vf = num
    if f.denom > 1:
        d = c[f.numer:]
        den = np.full_like(xf, d[f.denom - 2])
        for k in range(f.denom - 3, -1, -1):
            den = (xf * den + d[k]).astype(np.float32)
        den = (xf * den + 1).astype(np.float32)
        with np.errstate(all="ignore"):
            vf = num / den
    err = np.abs(vf.astype(np.float64) - v)
    return (not np.isfinite(err).all()) or err.max() > 1e-5 * np.abs(v).max()


def main(dt=0.02):
    numer = [0] * tt06.NFIT
    denom = [0] * tt06.NFIT
    mask = 0
    for ct in (0, 1, 2):
        p = engine.default_params(ct, dt)
        for i, f in enumerate(p.fits):
            numer[i] = max(numer[i], f.numer)
            denom[i] = max(denom[i], f.denom)
            if fp32_loses(f, i):
                mask |= 1 << i
    offset, off = [], 0
    for i in range(tt06.NFIT):
        offset.append(off)
        off += numer[i] + denom[i] - 1
    lines = [
        "// Generated by cardioid_b200/data/make_fit_shapes.py from the shipped",
        "// dt = %g BetterTT06 fit files; do not edit." % dt,
        "#pragma once",
        "namespace cdb {",
        "constexpr int kSpecNumer[30] = {%s};" % ", ".join(map(str, numer)),
        "constexpr int kSpecDenom[30] = {%s};" % ", ".join(map(str, denom)),
        "constexpr int kSpecOffset[30] = {%s};" % ", ".join(map(str, offset)),
        "constexpr int kSpecPool = %d;" % off,
        "constexpr unsigned kSpecFp64Mask = 0x%08xu;" % mask,
        "}  // namespace cdb",
        "",
    ]
    with open(HEADER, "w") as f:
        f.write("\n".join(lines))
    print("wrote", HEADER, "pool", off, "fp64 mask 0x%x" % mask)


if __name__ == "__main__":
    main()
