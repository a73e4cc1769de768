"""The irregular shell anatomy: its generator on the CPU, and the engine on
it against the oracle on the GPU (coarse voxels so the oracle finishes in
seconds; the bench runs the 0.25 mm shell).

Tolerances as in test_engine_gpu: FP64 max |dVm| <= 1e-6 mV and identical
activation times; mixed activation-time error <= 0.5 ms."""
import numpy as np
import pytest

from cardioid_b200 import shell


def test_shell_cell_count_matches_wall_volume():
    t = shell.prolate_shell(dx=1.0)
    exact = shell.shell_volume_mm3() / 1.0 ** 3
    assert abs(t.n - exact) / exact < 0.01
    assert (t.nx, t.ny, t.nz) == shell.grid_shape(1.0)
    assert t.gid.dtype == np.int64 and (np.diff(t.gid) > 0).all()
    # cell types follow depth
    assert (t.cell_type[t.depth < 0.30] == 100).all()
    assert (t.cell_type[(t.depth >= 0.30) & (t.depth < 0.65)] == 101).all()
    assert (t.cell_type[t.depth >= 0.65] == 102).all()
    for ct in (100, 101, 102):
        assert (t.cell_type == ct).sum() > 0.15 * t.n


def test_shell_conductivity_is_the_fibre_tensor():
    t = shell.prolate_shell(dx=1.0)
    s = t.sigma
    m = np.stack([s[:, [0, 1, 2]], s[:, [1, 3, 4]], s[:, [2, 4, 5]]], axis=1)
    ev = np.linalg.eigvalsh(m)
    np.testing.assert_allclose(ev[:, 2], shell.SIGMA_L, rtol=1e-9)
    np.testing.assert_allclose(ev[:, :2], shell.SIGMA_T, rtol=1e-9)


def test_shell_pacing_sites_are_endocardial_and_seeded():
    a = shell.prolate_shell(dx=1.0, seed=7)
    b = shell.prolate_shell(dx=1.0, seed=7)
    c = shell.prolate_shell(dx=1.0, seed=8)
    assert len(a.stimuli) == 20
    np.testing.assert_array_equal(a.sites, b.sites)
    assert not np.array_equal(a.sites, c.sites)
    pos = np.searchsorted(a.gid, a.sites)
    assert (a.depth[pos] < 1.0 / shell.WALL).all()


@pytest.mark.gpu
def test_shell_fp64_matches_oracle_and_mixed_within_tolerance(cdb_lib, oracle_port, fits002):
    from cardioid_b200 import engine as eng_mod
    t = shell.prolate_shell(dx=1.0, duration=2.0)
    rx = (t.cell_type - 100).astype(np.uint8)
    sim = oracle_port.PortSim(t, fits002, rx, 0.02)
    sim.step(600)
    ref_act = sim.activation()
    assert (ref_act > 0).sum() > 1000
    for precision in ("fp64", "mixed"):
        with eng_mod.Engine(0.02, precision=precision) as e:
            for p in fits002:
                e.add_reaction(p)
            tid = e.add_tissue(t, rx)
            e.step(600)
            vm = e.read_vm(tid)
            act = e.read_activation(tid)
        if precision == "fp64":
            assert np.abs(vm - sim.vm()).max() <= 1e-6
            np.testing.assert_array_equal(act, ref_act)
        else:
            assert ((act > 0) == (ref_act > 0)).mean() > 0.999
            both = (act > 0) & (ref_act > 0)
            assert np.abs(act[both] - ref_act[both]).max() <= 0.5
