"""The FP32 fit forms of the compiled mixed kernels (host side, CPU).

The mixed step evaluates every BetterTT06 fit (Interpolation::eval,
elec/Interpolation.hh:11-99) in FP32.  Fits whose monomial form loses
accuracy in FP32 are rewritten at registration in a shifted argument
t = (x - s) / 128 (cardioid_b200/csrc/common.cuh, spec_pool32).  These
tests check, through cdb_diag_fit_forms, that the shipped dt = 0.02 fits
run the compiled kernels, that the registered FP32 coefficients are the
exact Taylor shift rounded to FP32, that every fit's FP32 form stays within
1e-5 of its range against the FP64 monomial form, and that an ill-conditioned
fit set is sent to the generic kernel instead.
"""
import ctypes

import numpy as np
import pytest

from cardioid_b200 import _lib, engine, tt06
from cardioid_b200.data import make_fit_shapes as mfs


def forms(fits):
    L = _lib.load()
    pool = (ctypes.c_float * 640)()
    shift = (ctypes.c_float * 30)()
    scale = ctypes.c_float()
    compiled = ctypes.c_int32()
    _lib.check(L.cdb_diag_fit_forms(_lib.to_fit_array(fits), 640, pool, shift, ctypes.byref(scale),
                                    ctypes.byref(compiled)))
    return np.array(pool[:], np.float32), np.array(shift[:], np.float32), scale.value, compiled.value


def offsets():
    """Compiled shapes (numer, denom, offset per fit) read from fit_shapes.h."""
    import os
    import re
    src = open(os.path.join(os.path.dirname(mfs.HEADER), "fit_shapes.h")).read()
    get = lambda name: [int(v) for v in re.search(name + r"\[30\] = \{([^}]*)\}", src).group(1).split(",")]
    return get("kSpecNumer"), get("kSpecDenom"), get("kSpecOffset")


def eval32(pool, N, D, O, xf, horner):
    """One packed fit (numerator N terms, denominator 1 + x (D - 1 terms))
    in FP32 as the compiled mixed kernels evaluate it: Horner or the power
    basis (mfs._horner32 / mfs._pow32), FP32 quotient."""
    ev = mfs._horner32 if horner else mfs._pow32
    num = ev(pool[O:O + N], xf)
    den = ev(np.concatenate([[1.0], pool[O + N:O + N + D - 1]]), xf) if D > 1 else np.ones_like(num)
    return (num.astype(np.float32) / den.astype(np.float32)).astype(np.float64)


@pytest.mark.parametrize("celltype", [0, 1, 2])
def test_shipped_fits_run_compiled_and_stay_accurate(celltype):
    fits = engine.default_params(celltype, 0.02).fits
    pool, shift, scale, compiled = forms(fits)
    assert compiled == 1
    assert scale == 128.0
    numer, denom, off = offsets()
    for i, f in enumerate(fits):
        x = mfs.domain(i)
        v = f.eval(x)
        shifted = shift[i] != 0.0
        xf = ((x - shift[i]) / scale).astype(np.float32) if shifted else x.astype(np.float32)
        vf = eval32(pool, numer[i], denom[i], off[i], xf, horner=mfs.horner_slot(i) or shifted)
        err = np.abs(vf - v).max() / np.abs(v).max()
        assert err <= 1e-5, (i, err)
        if shifted:
            # the registered coefficients are the exact shift, rounded once to FP32
            c = np.array(f.coeff)
            qn = mfs.taylor_shift(c[:f.numer], shift[i], scale)
            qd = mfs.taylor_shift(np.concatenate([[1.0], c[f.numer:]]), shift[i], scale)
            want = np.zeros(numer[i] + denom[i] - 1, np.float32)
            want[:f.numer] = (qn / qd[0]).astype(np.float32)
            want[numer[i]:numer[i] + f.denom - 1] = (qd[1:] / qd[0]).astype(np.float32)
            got = pool[off[i]:off[i] + numer[i] + denom[i] - 1]
            np.testing.assert_array_max_ulp(got, want, maxulp=1)


def test_shifted_fits_are_the_ill_conditioned_ones():
    """The fits the generator shifted are exactly those whose monomial FP32
    form exceeds half the tolerance (h, m Rush-Larsen rates, j's b, s for
    the non-endo types, p_K term, K1)."""
    _, shift, _, _ = forms(engine.default_params(0, 0.02).fits)
    fits = [engine.default_params(ct, 0.02).fits for ct in (0, 1, 2)]
    for i in range(1, tt06.NFIT):
        worst = max(mfs.fp32_error(fs[i], i) for fs in fits)
        assert (shift[i] != 0.0) == (worst > mfs.TOL / 2), (i, worst)


def test_ill_conditioned_fit_set_runs_generic_kernel():
    """A fit in an unshifted slot whose monomial form cancels badly in FP32
    (T_18(x / 100) written in monomials) makes the set fall back to the
    generic kernel, which evaluates such fits in FP64."""
    fits = list(engine.default_params(1, 0.02).fits)
    cheb = np.polynomial.chebyshev.cheb2poly([0] * 18 + [1])          # T_18(z), z = x / 100
    mono = cheb / 100.0 ** np.arange(19)
    fits[15] = tt06.Fit(19, 1, [float(v) for v in mono])
    _, _, _, compiled = forms(fits)
    assert compiled == 0
    fits[15] = engine.default_params(1, 0.02).fits[15]
    assert forms(fits)[3] == 1
