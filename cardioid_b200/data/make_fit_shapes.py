"""Writes cardioid_b200/csrc/fit_shapes.h: the compile-time fit shapes of the
specialised step kernels, from the shipped fit files.

Per fit slot the header holds the largest numerator and denominator term
counts over the shipped celltypes; a reaction type whose fits are no longer
than these is packed zero-padded at the header's fixed offsets (leading zero
coefficients leave Horner's result unchanged) and runs the fully unrolled
kernel; any other fit set runs the generic kernel.

The header also holds, per fit, the FP32 form the mixed kernels evaluate:
fits whose monomial form stays within half the 1e-5 tolerance in FP32
(relative to their range) are evaluated as written (kSpecShift = 0 and
their bit in kSpecShiftMask clear), so that registration, which accepts
up to 1e-5, has a margin; the others (high-degree rational fits whose numerator and
denominator span many decades: the h and m Rush-Larsen rates, the j rate's
b, the s rate of the non-endo types, the p_K term and the K1 current) are evaluated in the shifted argument
t = (x - s) / 128, with s chosen here from a 5 mV grid as the shift giving
the smallest FP32 error over the shipped celltypes.  Registration rewrites
those fits' FP32 coefficients in t (common.cuh, spec_pool32).

    python -m cardioid_b200.data.make_fit_shapes
"""
import os
from fractions import Fraction
from math import comb

import numpy as np

from cardioid_b200 import engine, tt06

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(HERE), "csrc", "fit_shapes.h")
SHIFT_SCALE = 128.0     # a power of two: t = x / 128 - s / 128 is one exactly-scaled FMA
TOL = 1e-5          # FP32 error allowed, as a fraction of the fit's largest magnitude


def domain(slot):
    lo, hi = (1e-7, 0.1) if slot == 0 else (-100.0, 100.0)
    return np.linspace(lo, hi, 4001)


def _horner32(c, x):
    """FP32 Horner with fused multiply-adds (each step rounded once)."""
    c = np.asarray(c, np.float32)
    x = np.asarray(x, np.float32)
    r = np.full_like(x, c[-1])
    for a in c[-2::-1]:
        r = (r.astype(np.float64) * x + np.float64(a)).astype(np.float32)
    return r.astype(np.float64)


def _pow32(c, x):
    """FP32 power basis, low terms first: sum of fma(x^k, c_k, acc), x^k by
    repeated products (each step rounded once)."""
    c = np.asarray(c, np.float32)
    x = np.asarray(x, np.float32)
    p = np.ones_like(x)
    r = np.full_like(x, c[0])
    for a in c[1:]:
        p = (p * x).astype(np.float32)
        r = (p.astype(np.float64) * np.float64(a) + r).astype(np.float32)
    return r.astype(np.float64)


def horner_slot(slot):
    """Whether the compiled mixed kernels evaluate fit `slot` by Horner when
    it is not shifted: every fit (fit_pair32 runs each numerator and
    denominator chain pair by Horner in two-lane FMAs; a shifted fit runs
    the same in the shifted argument).  _pow32 remains for comparing the
    power basis."""
    return True


def _poly64(c, x):
    r = np.zeros_like(x)
    for a in c[::-1]:
        r = r * x + a
    return r


def taylor_shift(c, s, h=SHIFT_SCALE):
    """Coefficients q of p(x) = sum_j q_j t^j, t = (x - s) / h, exactly."""
    q = [Fraction(0)] * len(c)
    for k, ck in enumerate(c):
        for j in range(k + 1):
            q[j] += Fraction(float(ck)) * comb(k, j) * Fraction(float(s)) ** (k - j) * Fraction(h) ** j
    return np.array([float(v) for v in q])


def fp32_error(f, slot, shift=None):
    """Largest FP32 error of the fit over its domain, relative to its largest
    magnitude, evaluated as the compiled mixed kernels do: as written (shift
    None; Horner or power basis, horner_slot) or by Horner in the shifted
    argument."""
    x = domain(slot)
    c = np.array(f.coeff)
    num, den = c[:f.numer], np.concatenate([[1.0], c[f.numer:]])
    v = _poly64(num, x) / _poly64(den, x)
    if shift is None:
        ev = _horner32 if horner_slot(slot) else _pow32
        n32, d32 = ev(num, x), ev(den, x)
    else:
        t = ((x - shift) / SHIFT_SCALE).astype(np.float32)
        qn, qd = taylor_shift(num, shift), taylor_shift(den, shift)
        n32, d32 = _horner32(qn / qd[0], t), _horner32(qd / qd[0], t)
    with np.errstate(all="ignore"):
        vf = (n32.astype(np.float32) / d32.astype(np.float32)).astype(np.float64)
        err = np.abs(vf - v).max() / np.abs(v).max()
    return float(err) if np.isfinite(err) else np.inf


def main(dt=0.02):
    numer = [0] * tt06.NFIT
    denom = [0] * tt06.NFIT
    fits = [engine.default_params(ct, dt).fits for ct in (0, 1, 2)]
    shift = [0.0] * tt06.NFIT
    mask = 0
    for i in range(tt06.NFIT):
        for fs in fits:
            numer[i] = max(numer[i], fs[i].numer)
            denom[i] = max(denom[i], fs[i].denom)
        if i == 0 or max(fp32_error(fs[i], i) for fs in fits) <= TOL / 2:
            continue
        best = min(((max(fp32_error(fs[i], i, s) for fs in fits), s) for s in np.arange(-100.0, 100.1, 5.0)))
        if best[0] > TOL:
            raise RuntimeError("fit %d: no shift keeps the FP32 error under %g (best %.3g)" % (i, TOL, best[0]))
        shift[i] = float(best[1])
        mask |= 1 << i
        print("fit %2d: shift %g mV, FP32 error %.3g of range" % (i, shift[i], best[0]))
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
        "// FP32 form of the mixed kernels: fits in kSpecShiftMask take t = (x - kSpecShift) / kSpecShiftScale",
        "constexpr float kSpecShift[30] = {%s};" % ", ".join("%.1ff" % s for s in shift),
        "constexpr float kSpecShiftScale = %.1ff;" % SHIFT_SCALE,
        "constexpr unsigned kSpecShiftMask = 0x%08xu;" % mask,
        "}  // namespace cdb",
        "",
    ]
    with open(HEADER, "w") as f:
        f.write("\n".join(lines))
    print("wrote", HEADER, "pool", off, "shift mask 0x%x" % mask)


if __name__ == "__main__":
    main()
