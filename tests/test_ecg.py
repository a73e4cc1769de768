"""The ECG pseudo-sensor fused into the step against the reference's rule
(ECGSensor::calcInvR / eval / calcEcg, elec/ECGSensor.cc:46-78 and 231-320):
ecg_j = kconst dx dy dz sum over cells of dVmD / |r - p_j|, r = (x dx, y dy,
z dz), evaluated every evalRate steps on that step's dVmD.  The oracle's
dVmD (oracle port) feeds a numpy restatement of that sum.

Tolerance: FP64 relative 1e-9 of the largest |ecg| (the sum runs in another
order); mixed relative 2e-3."""
import numpy as np
import pytest

from cardioid_b200 import tissue

pytestmark = pytest.mark.gpu

POINTS = np.array([[-2.0, 1.0, 1.2], [1.5, 1.4, 3.0], [5.0, -1.0, 0.7], [1.1, 1.3, 1.0]])
KCONST = 0.37


def ecg_reference(t, dvmd, points, kconst):
    x, y, z = t.tuples()
    r = np.stack([x * t.dx, y * t.dy, z * t.dz], axis=1)
    d = np.linalg.norm(r[:, None, :] - points[None, :, :], axis=2)
    return kconst * t.dx * t.dy * t.dz * (dvmd[:, None] / d).sum(axis=0)


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
