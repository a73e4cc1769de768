"""Rational-fit generator for the 30 BetterTT06 lookup functions.

The reference builds these at start-up when no reusable FIT object exists
(ThisReaction::createInterpolants, elec/BetterTT06.cc:206-1002) with
Interpolation::create (elec/Interpolation.cc:115-423):
  1. sample the function at the midpoints of a uniform grid
     (V in [-100, 100] mV at 0.01 mV; Ca_ss in [1e-7, 0.1] at 1e-6 mM);
  2. for growing "cost" = numerator terms + denominator terms, least-squares
     fit every split of that cost in a Chebyshev basis on [lb, ub], the
     rational form linearised as  p(z) - y q~(z) = y  with q = 1 + q~;
  3. score each fit by the L2 norm of the error divided by a moving-window
     range of the function (window = rangeWindow * samples, odd), floored at
     1e-7 of the largest range; keep the best, stop at the first cost whose
     best error is under the tolerance;
  4. convert the Chebyshev coefficients to monomials in x and normalise the
     denominator's constant term to 1.
Each least-squares problem is solved as the reference's DGELS call does
(elec/Interpolation.cc:276-292): Householder QR of the (overdetermined,
full-rank) matrix, then R x = Q^T y.  The cost search stops at the first
cost whose best error is under the tolerance, so a solver with different
rounding (an SVD, say) can stop one cost earlier or later on a fit whose
error sits at the tolerance; with QR the generated shapes are the
reference generator's.  Fits are only ever shared through FIT files, so the
engine and the oracle always evaluate the same coefficients.
"""
import numpy as np
from scipy.linalg import solve_triangular

from .tt06 import Fit, NFIT

MAX_TERM_COUNT = 32

# Model constants used by the sampled functions (elec/BetterTT06.cc:206-1002).
_F, _R, _T = 96485.3415, 8314.472, 310.0


def _rl_a(dt, tau):
    return np.exp(-dt / tau) - 1.0


def sample(index, dt, params):
    """Inputs and outputs of fit ``index`` (slot order of _interpolant[]),
    and its (tolerance, rangeWindow)."""
    if index == 0:
        n = int((1e-1 - 1e-7) / 1e-6)
        x = 1e-7 + (1e-1 - 1e-7) * (np.arange(n) + 0.5) / n
        tau = 2 + 80 / (400.0 * (x * x) + 1)
        return x, _rl_a(dt, tau), 1e-4, 0.1
    n = int((100 - -100) / 1e-2)
    V = -100 + (100 - -100) * (np.arange(n) + 0.5) / n
    e = np.exp
    ct = params.celltype
    if index == 1:
        a = 450 / (e(-V / 10.0 - 4.5) + 1)
        b = 6 / (13.5813245225782 * e(0.0869565217391304 * V) + 1)
        y, w = _rl_a(dt, a * b), 0.1
    elif index == 2:
        y, w = -(1.0 / (e(-V / 7.0 - 26.0 / 7.0) + 1)), 1
    elif index == 3:
        a = 3 / (e(-V / 20.0 - 3) + 1)
        b = 1.12 / (e(V / 20.0 - 3) + 1)
        y, w = _rl_a(dt, a * b), 0.1
    elif index == 4:
        y, w = -(1.0 / (e(V / 24.0 + 11.0 / 3.0) + 1)), 1
    elif index == 5:
        a = 1400 * (e(-V / 6.0 + 5.0 / 6.0) + 1) ** -0.5
        b = 1.0 / (e(V / 15.0 - 7.0 / 3.0) + 1)
        y, w = _rl_a(dt, a * b + 80), 0.1
    elif index == 6:
        y, w = -(1.0 / (e(-V / 14.0 - 5.0 / 14.0) + 1)), 1
    elif index == 7:
        a = 0.25 + 1.4 / (e(-V / 13.0 - 35.0 / 13.0) + 1)
        b = 1.4 / (e(V / 5.0 + 1) + 1)
        g = 1.0 / (e(-V / 20.0 + 2.5) + 1)
        y, w = _rl_a(dt, a * b + g), 0.1
    elif index == 8:
        y, w = -(1.0 / (0.344153786865412 * e(-0.133333333333333 * V) + 1)), 1
    elif index == 9:
        tau = 562 * e(-((V + 27) ** 2) / 240.0) + 80 / (e(V / 10.0 + 3) + 1) + 31 / (e(-V / 10.0 + 2.5) + 1)
        y, w = _rl_a(dt, tau), 0.1
    elif index == 10:
        y, w = -(0.33 + 0.67 / (e(V / 7.0 + 5) + 1)), 1
    elif index == 11:
        tau = 1102.5 * e(-((V + 27) ** 2) / 225.0) + 20 + 200 / (e(-V / 10.0 + 1.3) + 1) + 180 / (e(V / 10.0 + 3) + 1)
        y, w = _rl_a(dt, tau), 0.1
    elif index == 12:
        y, w = -(1.0 / (e(V / 7.0 + 20.0 / 7.0) + 1)), 1
    elif index == 13:
        lo = V < -40
        ah = np.where(lo, 4.43126792958051e-7 * e(-0.147058823529412 * V), 0.0)
        bh = np.where(lo, 310000 * e(0.3485 * V) + 2.7 * e(0.079 * V),
                      0.77 / (0.0497581410839387 * e(-0.0900900900900901 * V) + 0.13))
        y, w = _rl_a(dt, 1.0 / (ah + bh)), 0.1
    elif index in (14, 16):
        t = 15212.5932856544 * e(0.134589502018843 * V) + 1
        y, w = -(1.0 / t / t), 1
    elif index == 15:
        lo = V < -40
        aj = np.where(lo, (-25428 * e(0.2444 * V) - 6.948e-6 * e(-0.04391 * V)) * (V + 37.78) /
                      (50262745825.954 * e(0.311 * V) + 1), 0.0)
        bj = np.where(lo, 0.02424 * e(-0.01052 * V) / (0.00396086833990426 * e(-0.1378 * V) + 1),
                      0.6 * e(0.057 * V) / (0.0407622039783662 * e(-0.1 * V) + 1))
        y, w = _rl_a(dt, 1.0 / (aj + bj)), 0.1
    elif index == 17:
        am = 1.0 / (e(-V / 5.0 - 12) + 1)
        bm = 0.1 / (e(V / 200.0 - 0.25) + 1) + 0.1 / (e(V / 5.0 + 7) + 1)
        y, w = _rl_a(dt, am * bm), 0.1
    elif index == 18:
        t = 0.00184221158116513 * e(-0.110741971207087 * V) + 1
        y, w = -(1.0 / t / t), 1
    elif index == 19:
        y, w = _rl_a(dt, 9.5 * e(-((V + 40) ** 2) / 1800.0) + 0.8), 0.1
    elif index == 20:
        y, w = -(1.0 / (e(-V / 6.0 + 10.0 / 3.0) + 1)), 1
    elif index == 21:
        if ct == 0:
            tau = 1000 * e(-((V + 67) ** 2) / 1000.0) + 8
        else:
            tau = 85 * e(-((V + 45) ** 2) / 320.0) + 3 + 5 / (e(V / 5.0 - 4) + 1)
        y, w = _rl_a(dt, tau), 0.1
    elif index == 22:
        y = -(1.0 / (e(V / 5.0 + (28.0 / 5.0 if ct == 0 else 4.0)) + 1))
        w = 1
    elif index == 23:
        y, w = e(_F * V * 0.35 / (_R * _T)), 0.1
    elif index == 24:
        y, w = e(_F * V * (0.35 - 1) / (_R * _T)), 0.1
    elif index in (25, 26):
        t1 = (_F * _F) * (4 * V - 60) / (_R * _T)
        t2 = e(_F * (2 * V - 30) / (_R * _T))
        with np.errstate(divide="ignore", invalid="ignore"):
            t3 = np.where(V == 15, 2 * _F, t1 / (t2 - 1))
        y, w = (t3 if index == 25 else t2 * t3), 0.1
    elif index == 27:
        ko, kmk, pnak = 5.4, 1.0, 2.724
        y = ko * pnak / ((ko + kmk) * (0.0353 * e(-_F * V / (_R * _T)) + 0.1245 * e(-0.1 * _F * V / (_R * _T)) + 1))
        w = 0.1
    elif index == 28:
        y, w = 1.0 / (65.4052157419383 * e(-0.167224080267559 * V) + 1), 0.1
    elif index == 29:
        vek = V
        a = 0.1 / (6.14421235332821e-6 * e(0.06 * vek) + 1)
        b = (0.367879441171442 * e(0.1 * vek) + 3.06060402008027 * e(0.0002 * vek)) / (e(-0.5 * vek) + 1)
        y, w = 0.430331482911935 * vek * np.sqrt(5.4) * params.g_K1 * (a / (a + b)), 0.1
    else:
        raise IndexError(index)
    return V, np.asarray(y, dtype=np.float64), 1e-3, w


def _moving_range(y, window):
    n = len(y)
    f = int(n * window)
    if f % 2 == 0:
        f += 1
    if f > n:
        f = n if n % 2 else n - 1
    h = f // 2
    # range over the clamped window [i-h, i+h], shifted at the ends exactly
    # as the reference's sliding multiset (elec/Interpolation.cc:205-225)
    from numpy.lib.stride_tricks import sliding_window_view
    win = sliding_window_view(y, f)
    rmax, rmin = win.max(axis=1), win.min(axis=1)
    idx = np.clip(np.arange(n) - h, 0, n - f)
    r = rmax[idx] - rmin[idx]
    return np.maximum(r, r.max() * 1e-7)


def _lstsq_qr(A, y):
    """min ||A x - y||_2 by Householder QR (A of full column rank)."""
    Q, R = np.linalg.qr(A, mode="reduced")
    return solve_triangular(R, Q.T @ y)


def _cheb_to_mono(c, lb, ub):
    """Chebyshev series on z = (2x - (ub+lb))/(ub-lb) -> monomials in x."""
    n = len(c)
    zc = np.polynomial.chebyshev.cheb2poly(c)
    M, B = 2.0 / (ub - lb), -(ub + lb) / (ub - lb)
    xc = np.zeros(n)
    # sum_k zc[k] (M x + B)^k
    poly = np.array([1.0])
    for k in range(n):
        xc[:len(poly)] += zc[k] * poly
        poly = np.convolve(poly, [B, M])
    return xc


def fit_samples(x, y, tol, window):
    """Interpolation::create: returns (Fit, achieved error)."""
    lb, ub = x[0], x[-1]
    n = len(x)
    z = (x - (ub + lb) / 2) * 2 / (ub - lb)
    T = np.empty((MAX_TERM_COUNT, n))
    T[0] = 1
    T[1] = z
    for j in range(2, MAX_TERM_COUNT):
        T[j] = 2 * T[1] * T[j - 1] - T[j - 2]
    rng = _moving_range(y, window)
    best = (1e30, None, -1, -1)
    cost = 2
    while best[0] >= tol and cost <= 2 * MAX_TERM_COUNT:
        for nd in range(1, cost):
            nn = cost if nd == 1 else cost - nd
            if nn > MAX_TERM_COUNT or nd > MAX_TERM_COUNT:
                continue
            A = np.empty((n, nn + nd - 1))
            A[:, :nn] = T[:nn].T
            if nd > 1:
                A[:, nn:] = (-y[None, :] * T[1:nd]).T
            coef = _lstsq_qr(A, y)
            num = T[:nn].T @ coef[:nn]
            den = 1 + (T[1:nd].T @ coef[nn:] if nd > 1 else 0)
            err = np.sqrt(np.sum(((y - num / den) / rng) ** 2) / n)
            if err < best[0]:
                best = (err, coef, nn, nd)
        cost += 1
    err, coef, nn, nd = best
    hn = _cheb_to_mono(coef[:nn], lb, ub)
    hd = _cheb_to_mono(np.concatenate([[1.0], coef[nn:]]), lb, ub)
    out = list(hn / hd[0]) + list(hd[1:] / hd[0])
    return Fit(nn, nd, [float(v) for v in out]), float(err)


def generate(dt, params, verbose=False):
    """All 30 fits for one BetterTT06 parameter set at time step dt."""
    fits = []
    for i in range(NFIT):
        x, y, tol, w = sample(i, dt, params)
        f, err = fit_samples(x, y, tol, w)
        if verbose:
            print("fit %2d numer=%2d denom=%2d err=%.3g" % (i, f.numer, f.denom, err))
        fits.append(f)
    return fits
