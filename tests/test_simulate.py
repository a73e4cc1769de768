"""The deck runner (cardioid_b200.simulate): a Cardioid object.data deck
turned into engine inputs and run.

CPU: the reference's multipleReaction deck gives exactly the inputs of the
committed fixture (made by tests/golden/make_multiple_reaction.py from the
same deck), and its Niederer deck, run by the oracle from the loaded inputs,
reproduces the reference's golden Vm and dVm_r (test/results/osx/seq/
Niederer/data).  GPU: a deck written here (brick anatomy, uniform
conductivity, BetterTT06 with the shipped fits, a box stimulus, the
activation and min/max sensors, printRate) run on the fused engine matches
the oracle on the same inputs."""
import os

import numpy as np
import pytest

from cardioid_b200 import engine, simulate, tissue
from conftest import REFERENCE

TESTS = os.path.join(REFERENCE, "test", "tests")
HAVE_DECKS = bool(REFERENCE) and os.path.exists(os.path.join(TESTS, "Niederer", "object.data"))


@pytest.mark.skipif(not HAVE_DECKS, reason="reference checkout not present")
def test_multiple_reaction_deck_loads_as_the_fixture():
    d = os.path.join(TESTS, "multipleReaction")
    files = [os.path.join(d, f) for f in ("object.data", "tt06Endo.fit.data", "tt06Mid.fit.data", "tt06Epi.fit.data",
                                          "tt06Endo.sv", "tt06Mid.sv", "tt06Epi.sv")]
    sim = simulate.load(files)
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "multiple_reaction.npz"))
    t = sim.tissue
    np.testing.assert_array_equal(t.gid, g["gid"])
    np.testing.assert_array_equal(t.cell_type, g["cell_type"])
    np.testing.assert_array_equal(t.sigma, g["sigma"])
    rx = np.searchsorted(g["reaction_cell_types"], g["cell_type"])
    np.testing.assert_array_equal(sim.reaction_of_cell, rx)
    np.testing.assert_array_equal(t.vm0, g["vm0"][rx])
    np.testing.assert_array_equal(sim.states, g["states"][rx].T)
    assert (sim.dt, sim.steps, t.diffusion_scale) == (float(g["dt"]), int(g["steps"]), float(g["diffusion_scale"]))
    np.testing.assert_array_equal(np.array([p.as_array() for p in sim.params]), g["params"])


@pytest.mark.skipif(not HAVE_DECKS, reason="reference checkout not present")
def test_niederer_deck_through_the_oracle_reproduces_its_golden(oracle_port):
    d = os.path.join(TESTS, "Niederer")
    sim = simulate.load([os.path.join(d, "object.data"), os.path.join(d, "tt06.fit.data")])
    t = sim.tissue
    assert (t.nx, t.ny, t.nz, sim.steps, sim.print_rate) == (200, 70, 30, 10, 5)
    port = oracle_port.PortSim(t, sim.params, sim.reaction_of_cell, sim.dt)
    rows = np.loadtxt(os.path.join(REFERENCE, "test", "results", "osx", "seq", "Niederer", "data"))
    for loop, vm, dvmr in [(int(r[0]), r[3], r[4]) for r in rows[1:]]:
        port.step(sim.print_rate)
        r, _, _ = port.dvm()
        assert abs(port.vm()[0] - vm) < 1e-13
        assert abs(r[0] - dvmr) < 1e-13


def _write_deck(tmp_path):
    dt = 0.02
    with open(engine.shipped_fit_path(dt, 1)) as f:
        fits = f.read()
    fit_name = [w for w in fits.split() if w.endswith("_fit")][0] if "_fit" in fits else None
    deck = """
run SIMULATE { anatomy = slab; diffusion = fgr; reaction = mid; stimulus = s1 pt; sensor = act mm;
               dt = %g; maxLoop = 240; printRate = 40; printGid = 130; }
slab ANATOMY { method = brick; cellType = 101; dx = 0.2; dy = 0.2; dz = 0.2; nx = 18; ny = 9; nz = 7;
               conductivity = cond; }
cond CONDUCTIVITY { method = uniform; sigma11 = 0.000133; sigma22 = 0.0000176; sigma33 = 0.0000176;
                    sigma12 = 0.00001; }
fgr DIFFUSION { method = FGR; diffusionScale = 714.2857143; }
mid REACTION { method = BetterTT06; cellTypes = 101; celltype = 1; %s }
s1 STIMULUS { method = box; xMax = 2; vStim = -52; duration = 1; period = 1000; }
pt STIMULUS { method = point; cell = 500; vStim = -30; tStart = 2; duration = 0.5; }
act SENSOR { method = activationTime; }
mm SENSOR { method = minMax; printRate = 60; }
""" % (dt, ("fit = %s;" % fit_name) if fit_name else "")
    path = tmp_path / "object.data"
    path.write_text(deck)
    fpath = tmp_path / "mid.fit.data"
    fpath.write_text(fits)
    return [str(path), str(fpath)]


def test_written_deck_loads(tmp_path):
    sim = simulate.load(_write_deck(tmp_path))
    t = sim.tissue
    assert (t.nx, t.ny, t.nz, t.n, sim.steps, sim.print_rate, sim.print_gid) == (18, 9, 7, 1134, 240, 40, 130)
    assert sim.sensors == ["activationTime", "minMax"]
    assert t.stimuli[1].mode == 1 and t.stimuli[1].cell == 500
    np.testing.assert_array_equal(t.sigma[7], [0.000133, 0.00001, 0.0, 0.0000176, 0.0, 0.0000176])


@pytest.mark.gpu
def test_written_deck_runs_on_the_engine_as_the_oracle(cdb_lib, oracle_port, tmp_path):
    sim = simulate.load(_write_deck(tmp_path))
    out = sim.run("fp64", out_dir=str(tmp_path))
    port = oracle_port.PortSim(sim.tissue, sim.params, sim.reaction_of_cell, sim.dt)
    pos = int(np.searchsorted(sim.tissue.gid, sim.print_gid))
    for row in out["print"]:
        port.step(sim.print_rate)
        assert abs(row[3] - port.vm()[pos]) <= 1e-6
    assert out["steps"] == 240 and abs(out["time"] - port.time) < 1e-12
    assert np.abs(out["vm"] - port.vm()).max() <= 1e-6
    np.testing.assert_array_equal(out["activation"], port.activation())
    from cardioid_b200 import pio
    f = pio.read(out["activation_file"][:-len("#000000")])
    np.testing.assert_array_equal(f.fields["gid"], sim.tissue.gid)
    np.testing.assert_allclose(f.fields["tActiv"], np.maximum(out["activation"], 0.0), rtol=0, atol=1e-12)
    assert (out["activation"] > 0).any()
    assert out["minmax"] == (out["vm"].min(), out["vm"].max())
    mm = np.loadtxt(out["minmax_file"])          # time, min, max, max - min every 60 steps
    assert mm.shape == (4, 4)
    np.testing.assert_allclose(mm[-1, 1:3], [out["vm"].min(), out["vm"].max()], rtol=1e-9)


@pytest.mark.gpu
def test_written_deck_checkpoints_and_restarts(cdb_lib, tmp_path):
    """checkpointRate writes the reference's snapshot.<loop> directories; the
    deck plus one of their restart files (merged into its SIMULATE object,
    as the reference reads it) continues from that loop to the same Vm and
    printed rows, bit for bit (binary checkpoints are exact)."""
    files = _write_deck(tmp_path)
    extra = tmp_path / "checkpoint.data"
    extra.write_text("run SIMULATE { checkpointRate = 120; }")
    full = simulate.load(files + [str(extra)]).run("fp64", out_dir=str(tmp_path))
    assert [os.path.basename(d) for d in full["checkpoints"]] == ["snapshot.000000000120", "snapshot.000000000240"]
    restart = os.path.join(str(tmp_path), "snapshot.000000000120", "restart")
    again = simulate.load(files + [restart]).run("fp64", out_dir=str(tmp_path / "again"))
    assert (again["loop"], again["steps"]) == (240, 120)
    np.testing.assert_array_equal(again["vm"], full["vm"])
    tail = full["print"][-len(again["print"]):]
    np.testing.assert_array_equal(again["print"][:, [0, 2, 3]], tail[:, [0, 2, 3]])
    # a restart takes its time from the checkpoint, as the reference's does:
    # the accumulated time may differ in its last bits
    np.testing.assert_allclose(again["print"][:, 1], tail[:, 1], rtol=0, atol=1e-12)


@pytest.mark.gpu
def test_cuda_diffusion_deck_runs_the_split_loop_as_the_oracle(cdb_lib, oracle_port, tmp_path):
    """A deck whose DIFFUSION is the 6-face "cuda" rule runs the split loop on
    the drop-in plugins (BetterTT06 per reaction, CUDADiffusion); against the
    oracle's reaction with the 6-face restatement added each step (same
    inputs, 60 steps): Vm within 1e-6 mV (ulp-level differences grow to a few
    1e-9 mV through the upstrokes), the same activation times."""
    from oracle import diff6
    files = _write_deck(tmp_path)
    extra = tmp_path / "cuda.data"
    extra.write_text("fgr DIFFUSION { method = cuda; }\nrun SIMULATE { maxLoop = 60; printRate = 0; }")
    sim = simulate.load(files + [str(extra)])
    assert sim.diffusion_method == "cuda"
    out = sim.run("fp64", out_dir=str(tmp_path / "cuda"))
    assert np.loadtxt(out["minmax_file"], ndmin=2).shape == (1, 4)     # printRate 60 over 60 steps
    t = sim.tissue
    port = oracle_port.PortSim(t, sim.params, sim.reaction_of_cell, sim.dt, diffusion=False)
    act = np.full(t.n, -1.0)
    for _ in range(60):
        v0 = port.vm()
        d = diff6.calc(t, v0, t.diffusion_scale)
        port.step(1)
        v = port.vm() + sim.dt * d
        port.set_vm(v)
        act[(act < 0) & (v > 0)] = port.time
    assert np.abs(out["vm"] - port.vm()).max() <= 1e-6      # the FP64 parity tolerance
    np.testing.assert_array_equal(out["activation"], act)


@pytest.mark.parametrize("patch,match", [
    ("slab ANATOMY { method = simple; }", "ANATOMY method simple"),
    ("fgr DIFFUSION { method = gpu; }", "DIFFUSION method gpu"),
    ("s1 STIMULUS { method = test; }", "method test"),
    ("s1 STIMULUS { pulse = random; }", "pulse random"),
    ("mid REACTION { method = TT06Dev; }", "only BetterTT06"),
    ("slab ANATOMY { cellType = 102; }", "no reaction for cellTypes"),
])
def test_unsupported_deck_items_raise(tmp_path, patch, match):
    """What the engine does not run is refused with ValueError, never
    replaced by something else."""
    files = _write_deck(tmp_path)
    extra = tmp_path / "patch.data"
    extra.write_text(patch)
    with pytest.raises(ValueError, match=match):
        simulate.load(files + [str(extra)])
