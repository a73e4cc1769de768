"""cdb_fgr_calc_static, the FGR stencil for callers that cannot allocate
device memory (it keeps its padded Vm block in a static device array),
against the allocating entry points cdb_fgr_create / _update_local_voltage /
_calc on the same box, for two calls in a row with different voltages (the
second call must not see the first call's block).

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest

from cardioid_b200 import _lib, plugins, tissue

pytestmark = pytest.mark.gpu
REL_TOL = 1e-12     # relative to max |dVm|; both paths use the same weights and order


def _static_calc(lib, t, w19_dev, vm_dev, out_dev, stream):
    return lib.cdb_fgr_calc_static(0, t.nx, t.ny, t.nz, ctypes.c_void_p(w19_dev.data_ptr()),
                                   ctypes.c_void_p(vm_dev.data_ptr()), ctypes.c_void_p(out_dev.data_ptr()),
                                   t.diffusion_scale, ctypes.c_void_p(stream))


def test_static_scratch_stencil_matches_allocating_path_twice(cdb_lib):
    import torch
    t = tissue.box(23, 17, 11, seed=9)
    ref = plugins.FGRDiffusion(t)
    w19 = torch.from_numpy(np.ascontiguousarray(ref.weights().T)).cuda()   # 19 rows of n
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(4)
    for call in range(2):
        vm = torch.from_numpy(t.vm0 + rng.uniform(-20.0, 60.0, t.n) * (call + 1)).cuda()
        want = torch.empty_like(vm)
        ref.updateLocalVoltage(vm)
        ref.calc(want)
        got = torch.full_like(vm, float("nan"))
        _lib.check(_static_calc(cdb_lib, t, w19, vm, got, stream))
        torch.cuda.synchronize()
        w, g = want.cpu().numpy(), got.cpu().numpy()
        assert np.isfinite(g).all()
        assert np.abs(g - w).max() <= REL_TOL * np.abs(w).max(), call


def test_static_scratch_rejects_boxes_beyond_its_block(cdb_lib):
    import torch
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    st = cdb_lib.cdb_fgr_calc_static(0, 200, 200, 200, p, p, p, 1.0, None)
    assert st == _lib.CDB_INVALID_ARG
    assert b"static block" in cdb_lib.cdb_last_error()
