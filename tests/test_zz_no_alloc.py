"""cdb_fgr_calc_static, the FGR stencil for callers that cannot allocate
device memory (it keeps its padded Vm block in a static device array),
against the allocating entry points cdb_fgr_create / _update_local_voltage /
_calc and against the oracle's stencil, for two calls in a row: first on a
larger box, then on a smaller one, so the first call's values sit where the
second call's halo is (the second call must clear them).  A warmed-up call leaves the device's free memory
unchanged and the calling thread's current device as it was.

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


def _case(t, scale, seed):
    """Weights (19 rows of n on the device), a voltage and the allocating
    path's dVm for box t."""
    import torch
    ref = plugins.FGRDiffusion(t)
    w19 = torch.from_numpy(np.ascontiguousarray(ref.weights().T)).cuda()
    rng = np.random.default_rng(seed)
    vm = torch.from_numpy(t.vm0 + rng.uniform(-20.0, 60.0, t.n) * scale).cuda()
    want = torch.empty_like(vm)
    ref.updateLocalVoltage(vm)
    ref.calc(want)
    torch.cuda.synchronize()
    return w19, vm, want.cpu().numpy()


def _oracle_dvmd(oracle_port, fits, t, vm):
    """The oracle's diffusion term for voltage vm (the FGR stencil of one
    step taken from vm, elec/FGRDiffusionOMP.cc:109-131)."""
    sim = oracle_port.PortSim(t, fits, (t.cell_type - 100).astype(np.uint8), 0.02)
    sim.set_vm(vm)
    sim.step(1)
    return sim.dvm()[1]


def test_static_scratch_stencil_matches_allocating_path_twice(cdb_lib, oracle_port, fits002):
    """Each call against the allocating plugin and against the oracle."""
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    for call, t in enumerate((tissue.box(23, 17, 11, seed=9), tissue.box(11, 9, 7, seed=10))):
        w19, vm, want = _case(t, call + 1, 4 + call)
        got = torch.full_like(vm, float("nan"))
        _lib.check(_static_calc(cdb_lib, t, w19, vm, got, stream))
        torch.cuda.synchronize()
        g = got.cpu().numpy()
        assert np.isfinite(g).all()
        assert np.abs(g - want).max() <= REL_TOL * np.abs(want).max(), call
        ref = _oracle_dvmd(oracle_port, fits002, t, vm.cpu().numpy())
        assert np.abs(g - ref).max() <= REL_TOL * np.abs(ref).max(), call


def test_static_scratch_allocates_nothing(cdb_lib):
    """After a first call (which may load the library's module on this
    device), another call leaves the device's free memory unchanged."""
    import torch
    t = tissue.box(15, 13, 9, seed=11)
    w19, vm, want = _case(t, 1, 12)
    got = torch.empty_like(vm)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_static_calc(cdb_lib, t, w19, vm, got, stream))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    _lib.check(_static_calc(cdb_lib, t, w19, vm, got, stream))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.current_device() == 0
    assert np.abs(got.cpu().numpy() - want).max() <= REL_TOL * np.abs(want).max()


def test_static_scratch_rejects_boxes_beyond_its_block(cdb_lib):
    import torch
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    st = cdb_lib.cdb_fgr_calc_static(0, 200, 200, 200, p, p, p, 1.0, None)
    assert st == _lib.CDB_INVALID_ARG
    assert b"static block" in cdb_lib.cdb_last_error()
