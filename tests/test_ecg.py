"""The ECG pseudo-sensor fused into the step against the reference's rule
(ECGSensor::calcInvR / eval / calcEcg, elec/ECGSensor.cc:46-78 and 231-320):
ecg_j = kconst dx dy dz sum over cells of dVmD / |r - p_j|, r = (x dx, y dy,
z dz), evaluated every evalRate steps on that step's dVmD.  The oracle's
dVmD (oracle port) feeds a numpy restatement of that rule: the 1/r table of
the reference's calcInvr kernel (elec/ECGSensor.cu:9-40, restated: it is
CUDA code) and the sum, which is pinned on the CPU to the reference's own
calcEcg run by the oracle build.

Tolerance: FP64 relative 1e-9 of the largest |ecg| (the sum runs in another
order); mixed relative 2e-3."""
import numpy as np
import pytest

from cardioid_b200 import tissue

POINTS = np.array([[-2.0, 1.0, 1.2], [1.5, 1.4, 3.0], [5.0, -1.0, 0.7], [1.1, 1.3, 1.0]])
KCONST = 0.37


def _ref_built():
    from oracle import refsim
    return refsim.available()


def invr_table(t, points):
    """[cell, electrode] 1 / |r - p| with r = (x dx, y dy, z dz) from the
    cell's gid (the reference's calcInvr_kernel)."""
    x, y, z = t.tuples()
    r = np.stack([x * t.dx, y * t.dy, z * t.dz], axis=1)
    return 1.0 / np.sqrt(((r[:, None, :] - points[None, :, :]) ** 2).sum(axis=2))


def ecg_sum(invr, dvmd):
    """ecg_j = sum_i invr[i, j] dvmd[i] (the reference's calcEcg)."""
    return (invr * dvmd[:, None]).sum(axis=0)


def ecg_reference(t, dvmd, points, kconst):
    return kconst * t.dx * t.dy * t.dz * ecg_sum(invr_table(t, points), dvmd)


@pytest.mark.skipif(not _ref_built(), reason="needs the reference build (oracle/_ref)")
def test_ecg_sum_is_the_references():
    """The restatement's sum against the reference's calcEcg on a 1/r table
    of a masked box and random dVmD: within 1e-13 of the sum of |terms|
    (numpy sums pairwise, the reference in cell order)."""
    from oracle import refsim
    t = tissue.box(13, 9, 7, seed=2)
    keep = np.random.default_rng(5).random(t.n) > 0.2
    t = tissue.Tissue(t.nx, t.ny, t.nz, t.dx, t.dy, t.dz, t.gid[keep], t.cell_type[keep], t.sigma[keep],
                      t.vm0[keep], [])
    invr = invr_table(t, POINTS)
    dvmd = np.random.default_rng(6).normal(size=t.n)
    want = refsim.calc_ecg(invr, dvmd)
    got = ecg_sum(invr, dvmd)
    bound = 1e-13 * (np.abs(invr) * np.abs(dvmd)[:, None]).sum(axis=0)
    assert (np.abs(got - want) <= bound).all(), np.abs(got - want) / bound


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 2e-3)])
def test_fused_ecg_matches_reference_rule(cdb_lib, oracle_port, fits002, precision, tol):
    from cardioid_b200 import engine as eng_mod
    t = tissue.box(16, 14, 12, period=6.0)
    rx = (t.cell_type - 100).astype(np.uint8)
    sim = oracle_port.PortSim(t, fits002, rx, 0.02)
    rate, steps = 5, 300
    want_loops, want = [], []
    for s in range(1, steps + 1):
        sim.step(1)
        if s % rate == 0:
            want_loops.append(s)
            want.append(ecg_reference(t, sim.dvm()[1], POINTS, KCONST))
    want = np.array(want)
    with eng_mod.Engine(0.02, precision=precision) as e:
        for p in fits002:
            e.add_reaction(p)
        tid = e.add_tissue(t, rx)
        e.set_ecg(tid, POINTS, rate, KCONST)
        got_loops, got = [], []
        for chunk in (7, 93, 200):          # reads between launch batches of different lengths
            e.step(chunk)
            lp, v = e.read_ecg(tid)
            got_loops.append(lp)
            got.append(v)
        got_loops, got = np.concatenate(got_loops), np.concatenate(got)
    np.testing.assert_array_equal(got_loops, want_loops)
    scale = np.abs(want).max()
    assert scale > 0
    assert np.abs(got - want).max() <= tol * scale, np.abs(got - want).max() / scale


@pytest.mark.gpu
def test_ecg_ring_keeps_the_latest_evaluations(cdb_lib, fits002):
    from cardioid_b200 import engine as eng_mod
    t = tissue.box(8, 6, 5)
    with eng_mod.Engine(0.02, precision="fp64") as e:
        for p in fits002:
            e.add_reaction(p)
        tid = e.add_tissue(t, (t.cell_type - 100).astype(np.uint8))
        e.set_ecg(tid, POINTS[:2], 1, 1.0)
        e.step(1100)                         # more evaluations than the ring holds (1023)
        loops, v = e.read_ecg(tid, max_entries=2048)
        assert len(loops) == 1023 and loops[0] == 1100 - 1022 and loops[-1] == 1100
        e.step(3)
        loops, _ = e.read_ecg(tid)
        np.testing.assert_array_equal(loops, [1101, 1102, 1103])
        e.set_ecg(tid, POINTS[:0], 1, 1.0)   # off
        e.step(2)
        assert len(e.read_ecg(tid)[0]) == 0


@pytest.mark.gpu
def test_reference_gpu_ecg_kernels(cdb_lib, oracle_port, fits002):
    """The reference's own ECG kernels (calcInvrCUDA, calcEcgCUDA of
    elec/ECGSensor.cu, built from its source by oracle/ref/Makefile and run
    on the GPU) against the restatement above and the fused sensor:
    - the 1/r table equals the restatement's to 1e-15 relative (the kernel
      contracts the squared distance into FMAs; IEEE sqrt and division);
    - its sum over the oracle's dVmD equals the restatement's within 1e-13
      of the sum of |terms| (atomic, blocked summation order);
    - the fused sensor's FP64 trace at the same step equals kconst dx dy dz
      times that sum, within 1e-9 of its size (the FP64 tolerance above).
    The box's 2688 cells are a multiple of 112, where the reference's sum
    kernel stays inside the cell array."""
    from cardioid_b200 import engine as eng_mod
    from oracle import refgpu
    if not refgpu.ecg_available():
        pytest.skip("oracle/_ref/ref_gpu_ecg not built (needs the reference checkout at build time)")
    t = tissue.box(16, 14, 12, period=6.0)
    assert t.n % 112 == 0
    rx = (t.cell_type - 100).astype(np.uint8)
    sim = oracle_port.PortSim(t, fits002, rx, 0.02)
    steps = 40
    sim.step(steps)
    dvmd = sim.dvm()[1]
    invr, sums = refgpu.ecg(t, POINTS, dvmd)
    np.testing.assert_allclose(invr, invr_table(t, POINTS), rtol=1e-15, atol=0)
    bound = 1e-13 * (np.abs(invr) * np.abs(dvmd)[:, None]).sum(axis=0)
    assert (np.abs(sums - ecg_sum(invr, dvmd)) <= bound).all()
    want = KCONST * t.dx * t.dy * t.dz * sums
    with eng_mod.Engine(0.02, precision="fp64") as e:
        for p in fits002:
            e.add_reaction(p)
        tid = e.add_tissue(t, rx)
        e.set_ecg(tid, POINTS, steps, KCONST)
        e.step(steps)
        loops, got = e.read_ecg(tid)
    np.testing.assert_array_equal(loops, [steps])
    assert np.abs(got[0] - want).max() <= 1e-9 * np.abs(want).max()
