"""Pins the oracle (the C restatement in oracle/port) against the reference:
the reference's own golden outputs (singleCell, Niederer), the committed
fixture made by the reference code (tests/golden), and the reference code
itself compiled here (oracle/_ref) where it is built."""
import os

import numpy as np
import pytest

from conftest import REFERENCE

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
HAVE_REF_TREE = bool(REFERENCE) and os.path.exists(os.path.join(REFERENCE, "test", "tests"))


def _ref_built():
    from oracle import refsim
    return refsim.available()


def test_port_matches_committed_reference_fixture(oracle_port, fits002):
    """Bit-exact against the reference code's run of a 10x8x6 box
    (three cell types, FGR, box stimulus, dt = 0.02)."""
    from golden.make_golden import box_case, DT
    g = np.load(os.path.join(GOLDEN, "ref_box_dt002.npz"))
    t = box_case()
    rx = (t.cell_type - 100).astype(np.uint8)
    sim = oracle_port.PortSim(t, fits002, rx, DT)
    done = 0
    for s in (25, 50, 100):
        sim.step(s - done)
        done = s
        np.testing.assert_array_equal(sim.vm(), g["vm_%d" % s])
    np.testing.assert_array_equal(sim.states(), g["states"])
    np.testing.assert_array_equal(sim.activation(), g["activation"])
    r, d, i = sim.dvm()
    np.testing.assert_array_equal(r, g["dvmR"])
    np.testing.assert_array_equal(d, g["dvmD"])
    np.testing.assert_array_equal(i, g["iStim"])
    assert sim.time == float(g["time"])


@pytest.mark.skipif(not HAVE_REF_TREE, reason="reference checkout not present")
def test_port_reproduces_reference_singlecell_golden(oracle_port):
    """test/results/osx/seq/singleCell/BetterTT06.stdOut: 4 cells, dt 0.01,
    a 60 mV/ms stimulus for 1 ms, Vm every 1 ms for 1000 ms (the reference's
    numCompare tolerance is 1e-7 of the column range)."""
    from cardioid_b200 import objectdb, tt06, tissue
    T = os.path.join(REFERENCE, "test")
    db = objectdb.ObjectDB().compile_file(os.path.join(T, "tests", "singleCell", "BetterTT06.data"))
    p = tt06.TT06Params.defaults(0)
    p.fits = tt06.fits_from_fit_object(db, "BetterTT06_fit")
    golden = np.loadtxt(os.path.join(T, "results", "osx", "seq", "singleCell", "BetterTT06.stdOut"))
    # singleCell.cc: iStim = stim-strength (60) for round(1 ms / dt) steps from step 0
    stim = tissue.BoxStim(xMin=-1, xMax=1e9, yMin=-1, yMax=1e9, zMin=-1, zMax=1e9, vStim=-60.0,
                          tStart=0.0, duration=1.0, period=1e9)
    t = tissue.Tissue(4, 1, 1, 1.0, 1.0, 1.0, np.arange(4), np.full(4, 100, np.int32), np.zeros((4, 6)),
                      np.full(4, -83.0), [stim])
    sim = oracle_port.PortSim(t, [p], np.zeros(4, np.uint8), 0.01, diffusion=False)
    vm = [sim.vm()[0]]
    for _ in range(1000):
        sim.step(100)
        vm.append(sim.vm()[0])
    vm = np.array(vm)
    assert np.abs(vm - golden[:, 1]).max() < 1e-12


@pytest.mark.skipif(not HAVE_REF_TREE, reason="reference checkout not present")
def test_port_reproduces_reference_niederer_golden(oracle_port):
    """test/results/osx/seq/Niederer/data: 200x70x30 brick at 0.1 mm, uniform
    conductivity, BetterTT06 celltype 2, two box stimuli, dt 0.01; Vm and
    dVm_r of gid 0 at loops 5 and 10 (printed to 15 decimals)."""
    from cardioid_b200 import objectdb, tt06, tissue
    T = os.path.join(REFERENCE, "test")
    db = objectdb.ObjectDB().compile_file(os.path.join(T, "tests", "Niederer", "tt06.fit.data"))
    p = tt06.TT06Params.defaults(2)
    p.fits = tt06.fits_from_fit_object(db, "tt06_fit")
    nx, ny, nz = 200, 70, 30
    n = nx * ny * nz
    sig = np.zeros((n, 6))
    sig[:, 0], sig[:, 3], sig[:, 5] = 0.0001334177, 0.0000176062, 0.0000176062
    s1 = tissue.BoxStim(xMin=-1, xMax=15, yMin=-1, yMax=15, zMin=-1, zMax=15, vStim=-35.71429, tStart=0,
                        duration=2, period=10000)
    s2 = tissue.BoxStim(xMin=14, xMax=nx, yMin=54, yMax=ny, zMin=184, zMax=nz, vStim=-35.71429, tStart=565,
                        duration=2, period=10000)
    t = tissue.Tissue(nx, ny, nz, 0.1, 0.1, 0.1, np.arange(n), np.full(n, 102, np.int32), sig,
                      np.full(n, -83.0), [s1, s2], diffusion_scale=714.2857143)
    sim = oracle_port.PortSim(t, [p], np.zeros(n, np.uint8), 0.01)
    rows = np.loadtxt(os.path.join(T, "results", "osx", "seq", "Niederer", "data"))
    for loop, vm, dvmr, dvmd in [(int(r[0]), r[3], r[4], r[5]) for r in rows[1:]]:
        sim.step(5)
        r, d, _ = sim.dvm()
        assert abs(sim.vm()[0] - vm) < 1e-13
        assert abs(r[0] - dvmr) < 1e-13
        assert abs(d[0] - dvmd) < 1e-12


@pytest.mark.skipif(not _ref_built(), reason="oracle/_ref not built")
@pytest.mark.parametrize("shape", [(7, 6, 5), (9, 1, 1), (8, 7, 1)])
def test_port_bit_exact_vs_reference_build(oracle_port, fits002, shape):
    """The port against the reference's own code on boxes, a cable and a
    sheet, 300 steps: every Vm, state and activation time identical."""
    from golden.make_golden import reference_sim
    from cardioid_b200 import tissue
    t = tissue.box(*shape, dx=0.2, seed=11)
    ref = reference_sim(t)
    ref.set_vm(t.vm0)
    sim = oracle_port.PortSim(t, fits002, (t.cell_type - 100).astype(np.uint8), 0.02)
    for _ in range(3):
        ref.step(100)
        sim.step(100)
        np.testing.assert_array_equal(sim.vm(), ref.vm())
    names = ref.field_names()
    for k, name in enumerate(names):
        np.testing.assert_array_equal(sim.state(k), ref.state(name))
    np.testing.assert_array_equal(sim.activation(), ref.activation())


@pytest.mark.skipif(not _ref_built(), reason="oracle/_ref not built")
def test_port_bit_exact_vs_reference_build_config0(oracle_port, fits002):
    """Config 0 itself: the 64^3 box (the GPU parity test's input,
    tissue.box(64, 64, 64)) for 1000 steps, the reference's own code against
    the port: every Vm, state and activation time identical (so the GPU's
    config-0 parity against the port is parity against the reference
    build).  About a minute and a half on 8 cores."""
    from golden.make_golden import reference_sim
    from cardioid_b200 import tissue
    from oracle import refsim
    refsim.set_threads(os.cpu_count() or 1)
    t = tissue.box(64, 64, 64)
    ref = reference_sim(t)
    ref.set_vm(t.vm0)
    sim = oracle_port.PortSim(t, fits002, (t.cell_type - 100).astype(np.uint8), 0.02)
    ref.step(1000)
    sim.step(1000)
    np.testing.assert_array_equal(sim.vm(), ref.vm())
    for k, name in enumerate(ref.field_names()):
        np.testing.assert_array_equal(sim.state(k), ref.state(name))
    act = ref.activation()
    assert (act > 0).sum() > 1000
    np.testing.assert_array_equal(sim.activation(), act)


@pytest.mark.skipif(not _ref_built(), reason="oracle/_ref not built")
def test_port_masked_tissue_vs_reference_build(oracle_port, fits002):
    """Irregular tissue (a hollow box): FGR boundary weights on an irregular
    mask, bit-exact against the reference."""
    from golden.make_golden import reference_sim
    from cardioid_b200 import tissue
    full = tissue.box(9, 8, 7, dx=0.2, seed=5)
    x, y, z = full.tuples()
    keep = ~((x >= 3) & (x <= 5) & (y >= 2) & (y <= 5) & (z >= 2) & (z <= 4))
    keep &= ~((x == 8) & (y == 0))
    t = tissue.Tissue(full.nx, full.ny, full.nz, full.dx, full.dy, full.dz, full.gid[keep], full.cell_type[keep],
                      full.sigma[keep], full.vm0[keep], full.stimuli)
    ref = reference_sim(t)
    ref.set_vm(t.vm0)
    sim = oracle_port.PortSim(t, fits002, (t.cell_type - 100).astype(np.uint8), 0.02)
    ref.step(150)
    sim.step(150)
    np.testing.assert_array_equal(sim.vm(), ref.vm())
    r1, d1, _ = ref.dvm()
    r2, d2, _ = sim.dvm()
    np.testing.assert_array_equal(d2, d1)


def _point_stim_tissue():
    """A masked 9x8x6 box with box and point stimuli in an order that
    exercises assign-then-add, add-then-assign and a point on a non-tissue
    voxel (which the reference ignores)."""
    from cardioid_b200 import tissue
    full = tissue.box(9, 8, 6, dx=0.2, seed=21)
    x, y, z = full.tuples()
    keep = ~((x == 4) & (y == 4) & (z == 3))
    pulse = dict(vStim=-30.0, duration=1.0, period=3.0)
    face = tissue.BoxStim(xMin=-1, xMax=1, vStim=-52.0, duration=1.0, period=1000.0)
    stims = [
        tissue.point_stim(0 + 9 * (2 + 8 * 1), 9, 8, tStart=0.0, **pulse),   # on the face, then overwritten
        face,
        tissue.point_stim(0 + 9 * (3 + 8 * 2), 9, 8, tStart=0.0, **pulse),   # on the face: adds to it
        tissue.point_stim(6 + 9 * (5 + 8 * 4), 9, 8, tStart=0.4, **pulse),   # interior, later phase
        tissue.point_stim(4 + 9 * (4 + 8 * 3), 9, 8, tStart=0.0, **pulse),   # removed voxel: no cell
    ]
    return tissue.Tissue(full.nx, full.ny, full.nz, full.dx, full.dy, full.dz, full.gid[keep], full.cell_type[keep],
                         full.sigma[keep], full.vm0[keep], stims)


@pytest.mark.skipif(not _ref_built(), reason="oracle/_ref not built")
def test_port_point_stimuli_vs_reference_build(oracle_port, fits002):
    """PointStimulus adds its pulse to one cell, BoxStimulus assigns, in
    list order: port and reference agree bit for bit over 250 steps."""
    from golden.make_golden import reference_sim
    t = _point_stim_tissue()
    ref = reference_sim(t)
    ref.set_vm(t.vm0)
    sim = oracle_port.PortSim(t, fits002, (t.cell_type - 100).astype(np.uint8), 0.02)
    ref.step(1)
    sim.step(1)
    _, _, s_ref = ref.dvm()
    _, _, s_port = sim.dvm()
    np.testing.assert_array_equal(s_port, s_ref)
    cell = {int(g): i for i, g in enumerate(t.gid)}
    assert s_port[cell[9 * (2 + 8 * 1)]] == 52.0            # assigned over the earlier point
    assert s_port[cell[9 * (3 + 8 * 2)]] == 52.0 + 30.0     # point after the box adds
    assert s_port[cell[6 + 9 * (5 + 8 * 4)]] == 0.0          # not yet on (tStart 0.4)
    ref.step(249)
    sim.step(249)
    np.testing.assert_array_equal(sim.vm(), ref.vm())
    np.testing.assert_array_equal(sim.activation(), ref.activation())


def test_fit_eval_port_matches_python(oracle_port, fits002):
    """Interpolation::eval restated in C and in numpy agree bit for bit."""
    x = np.linspace(-100, 100, 37)
    for f in fits002[0].fits[1:]:
        np.testing.assert_array_equal(oracle_port.fit_eval(f, x), f.eval(x))
