"""The engine's branch-free FP64 quotient (div64: hardware reciprocal seed,
one Newton-Raphson step, one residual correction) against CUDA's IEEE
a / b on operands spanning the model's range: at most 2 ulp away."""
import ctypes

import numpy as np
import pytest

from cardioid_b200 import _lib

pytestmark = pytest.mark.gpu
MAX_ULP = 2


def test_div64_within_two_ulp_of_ieee(cdb_lib):
    import torch
    rng = np.random.default_rng(1)
    n = 1 << 20
    mag_a = 10.0 ** rng.uniform(-12, 12, n)
    mag_b = 10.0 ** rng.uniform(-12, 12, n)
    a = mag_a * rng.choice([-1.0, 1.0], n)
    b = mag_b * rng.choice([-1.0, 1.0], n)
    a[:4] = [1.0, 3.0, 0.6, 5.4]
    b[:4] = [3.0, 7.0, 1.0 + 400.0 * 1.7e-4 ** 2, 138.4]
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    q = torch.empty_like(da)
    _lib.check(cdb_lib.cdb_diag_div64(0, n, ctypes.c_void_p(da.data_ptr()), ctypes.c_void_p(db.data_ptr()),
                                      ctypes.c_void_p(q.data_ptr()), None))
    ieee = (da / db).cpu().numpy()
    got = q.cpu().numpy()
    ulp = np.abs(got.view(np.int64) - ieee.view(np.int64))
    assert ulp.max() <= MAX_ULP, ulp.max()
    assert (ulp == 0).mean() > 0.9
