"""The reference's multipleReaction test end to end: its pio anatomy (40 x 5
x 5, three cell types, conductivity tensors in mS/mm), three BetterTT06
reaction objects with dt 0.01 fit files and SINGLECELL initial states, a box
stimulus, 30 000 steps; expected Vm of three cells every 200 steps from the
reference's results (fixture: tests/golden/multiple_reaction.npz, made by
make_multiple_reaction.py).  The reference checks these traces to 1e-14.

CPU: the anatomy reader, and the oracle against the expected traces.  GPU:
the fused engine (FP64) against the same traces."""
import os

import numpy as np
import pytest

from cardioid_b200 import anatomy, tissue, tt06
from conftest import REFERENCE

FIX = os.path.join(os.path.dirname(__file__), "golden", "multiple_reaction.npz")
REF_ANATOMY = os.path.join(REFERENCE, "test", "tests", "multipleReaction", "snapshot.initial", "anatomy#")
# The reference compares these traces to 1e-14 on its own platform; the
# oracle (glibc libm) lands 9e-6 mV from them after 30 000 steps, the spread
# of one-ulp differences in exp/log through the upstrokes.
TRACE_TOL_ORACLE = 2e-5     # mV
TRACE_TOL_FP64 = 1e-4       # mV


def case():
    d = np.load(FIX)
    s = d["stim"]
    stim = tissue.BoxStim(xMin=s[0], xMax=s[1], yMin=s[2], yMax=s[3], zMin=s[4], zMax=s[5], vStim=s[6],
                          tStart=s[7], duration=s[8], period=s[9], t0=s[10], tf=s[11])
    rx = np.searchsorted(d["reaction_cell_types"], d["cell_type"]).astype(np.uint8)
    t = tissue.Tissue(int(d["nx"]), int(d["ny"]), int(d["nz"]), float(d["dx"]), float(d["dx"]), float(d["dx"]),
                      d["gid"], d["cell_type"], d["sigma"], d["vm0"][rx], [stim], float(d["diffusion_scale"]))
    params = []
    for r in range(len(d["params"])):
        p = tt06.TT06Params(*d["params"][r])
        p.fits = [tt06.Fit(int(f[0]), int(f[1]), list(f[2:2 + int(f[0]) + int(f[1]) - 1])) for f in d["fits"][r]]
        params.append(p)
    states = d["states"][rx].T           # 18 x n: each cell starts in its reaction's SINGLECELL state
    pos = np.searchsorted(t.gid, d["sensor"])
    return t, params, rx, states, float(d["dt"]), int(d["steps"]), pos, d["traces"]


@pytest.mark.skipif(not (REFERENCE and os.path.exists(REF_ANATOMY + "000000")), reason="needs the reference checkout")
def test_anatomy_reader_matches_fixture():
    t = anatomy.read_anatomy(REF_ANATOMY)
    d = np.load(FIX)
    np.testing.assert_array_equal(t.gid, d["gid"])
    np.testing.assert_array_equal(t.cell_type, d["cell_type"])
    np.testing.assert_array_equal(t.sigma, d["sigma"])
    assert t.sigma[0, 0] == pytest.approx(0.1334177e-3)     # mS/mm in the file


def test_ibt_fibre_tensor():
    s = anatomy.ibt_sigma(np.array([np.pi / 2, 0.0, np.pi / 3]), np.array([0.0, 0.4, 1.1]), 3.0, 1.0)
    m = np.stack([s[:, [0, 1, 2]], s[:, [1, 3, 4]], s[:, [2, 4, 5]]], axis=1)
    np.testing.assert_allclose(np.linalg.eigvalsh(m), [[1, 1, 3]] * 3, rtol=1e-12)
    th, ph = np.pi / 3, 1.1
    f = np.array([np.cos(ph) * np.sin(th), np.sin(ph) * np.sin(th), np.cos(th)])
    np.testing.assert_allclose(m[2] @ f, 3 * f, rtol=1e-12)


def _run(step, vm, every, n_rows, pos):
    rows = []
    for _ in range(n_rows):
        step(every)
        rows.append(vm()[pos])
    return np.array(rows)


def test_oracle_reproduces_reference_multiple_reaction_traces(oracle_port):
    t, params, rx, states, dt, steps, pos, traces = case()
    sim = oracle_port.PortSim(t, params, rx, dt)
    for k in range(tt06.NSTATE):
        sim.set_state(k, states[k])
    every = steps // len(traces)
    got = _run(sim.step, sim.vm, every, len(traces), pos)
    err = np.abs(got - traces[:, 1:]).max()
    assert err <= TRACE_TOL_ORACLE, err


@pytest.mark.gpu
def test_engine_reproduces_reference_multiple_reaction_traces(cdb_lib):
    from cardioid_b200 import engine as eng_mod
    t, params, rx, states, dt, steps, pos, traces = case()
    with eng_mod.Engine(dt, precision="fp64") as e:
        rid = [e.add_reaction(p) for p in params]
        tid = e.add_tissue(t, np.array(rid, np.uint8)[rx])
        for k in range(tt06.NSTATE):
            e.write_state(tid, k, states[k])
        every = steps // len(traces)
        got = _run(e.step, lambda: e.read_vm(tid), every, len(traces), pos)
    err = np.abs(got - traces[:, 1:]).max()
    assert err <= TRACE_TOL_FP64, err


@pytest.mark.skipif(not (lambda: __import__("oracle.refsim", fromlist=["x"]).available())(),
                    reason="needs the reference build (oracle/_ref)")
@pytest.mark.parametrize("rot,homog,sheet", [(1, False, 45.0), (1, False, 30.0), (1, True, 45.0)])
def test_jhu_conductivity_is_the_references(rot, homog, sheet):
    """anatomy.jhu_sigma against the reference's JHUConductivity::compute
    (built into the oracle), bit for bit, on every cell of a 7 x 11 x 5
    grid, for two sheet angles and the homogeneous fibre."""
    from cardioid_b200 import anatomy
    from oracle import refsim
    nx, ny, nz = 7, 11, 5
    gid = np.arange(nx * ny * nz)
    want = refsim.jhu_sigma(gid, nx, ny, nz, 0.3e-3, 0.0315e-3, sheet, rot, homog)
    got = anatomy.jhu_sigma(gid, nx, ny, nz, 0.3e-3, 0.0315e-3, sheet, rot, homog)
    np.testing.assert_array_equal(got, want)


def test_jhu_reflection_convention_is_rejected():
    """Rotation convention 0 is a reflection; the reference's determinant
    assert aborts on it, anatomy.jhu_sigma raises."""
    from cardioid_b200 import anatomy
    with pytest.raises(ValueError, match="determinant"):
        anatomy.jhu_sigma(np.arange(10), 7, 11, 5, rotation_matrix=0)
