"""The B200TT06 adapter (cardioid_b200/adapter/B200TT06.cc) inside the
reference's own code: built as a dynamic reaction against the reference
sources (oracle/ref/Makefile), loaded by the reference's reactionFactory
(dlopen of the REACTION's method, elec/reactionFactory.cc:48-70), driven by
the reference's ReactionManager, FGRDiffusionOMP, BoxStimulus and omp-loop
integrator (oracle/ref/ref_driver.cc), and computing on the GPU through the
C ABI.  Against the same simulation with the reference's own BetterTT06:
FP64 max |dVm| <= 1e-6 mV after 300 steps, identical activation times."""
import os

import numpy as np
import pytest

from cardioid_b200 import engine, tissue

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER = os.path.join(ROOT, "oracle", "_ref", "libb200tt06.so")


def _built():
    from oracle import refsim
    return refsim.available() and os.path.exists(ADAPTER)


@pytest.mark.skipif(not _built(), reason="oracle/_ref with the adapter not built")
def test_adapter_in_reference_reaction_manager(cdb_lib):
    from golden.make_golden import reference_sim
    from oracle import refsim
    t = tissue.box(10, 8, 6, dx=0.2, seed=17)
    ref = reference_sim(t)           # compiles the shipped fits and the BetterTT06 objects
    text = ""
    for name, ct, fit in (("b200Endo", 0, "tt06Endo_fit"), ("b200Mid", 1, "tt06Mid_fit"), ("b200Epi", 2, "tt06Epi_fit")):
        text += "%s REACTION { method = %s; cellTypes = %d; celltype = %d; fit = %s; }\n" % (name, ADAPTER, 100 + ct,
                                                                                          ct, fit)
    refsim.compile_once("b200-adapter", text)
    prefix = refsim.unique_prefix()
    refsim.compile_objects(tissue.stimulus_objects_text(t.stimuli, prefix=prefix))
    gpu = refsim.RefSim(["b200Endo", "b200Mid", "b200Epi"], ["%s%d" % (prefix, i) for i in range(len(t.stimuli))],
                        (t.nx, t.ny, t.nz), (t.dx, t.dy, t.dz), t.gid, t.cell_type, t.sigma, 0.02, t.diffusion_scale)
    # both start from the reactions' own initial Vm (initializeMembraneVoltage)
    np.testing.assert_array_equal(gpu.vm(), ref.vm())
    ref.set_vm(t.vm0)
    gpu.set_vm(t.vm0)
    for _ in range(3):
        ref.step(100)
        gpu.step(100)
    assert np.abs(gpu.vm() - ref.vm()).max() <= 1e-6
    np.testing.assert_array_equal(gpu.activation(), ref.activation())
    assert (ref.activation() > 0).any()
    for name in ("Ca_i", "m", "h"):
        r = ref.state(name)
        assert np.abs(gpu.state(name) - r).max() <= 1e-8 * max(1e-12, np.abs(r).max())


@pytest.mark.skipif(not _built(), reason="oracle/_ref with the adapter not built")
def test_mixed_adapter_in_reference_loop_over_one_beat(cdb_lib):
    """REACTION objects with precision = mixed: the adapter's mixed-precision
    reactions inside the reference's time loop for one paced beat (20000
    steps, 400 ms) against the reference's own BetterTT06 (FP64): every cell
    activates in both, activation times within 0.5 ms, APD90 within 1 ms at
    probe cells (the mixed path's tolerances)."""
    from golden.make_golden import reference_sim
    from oracle import refsim
    from cardioid_b200.sensors import apd90
    t = tissue.box(10, 8, 6, dx=0.2, seed=29)
    ref = reference_sim(t)
    text = ""
    for name, ct, fit in (("b200mEndo", 0, "tt06Endo_fit"), ("b200mMid", 1, "tt06Mid_fit"),
                          ("b200mEpi", 2, "tt06Epi_fit")):
        text += "%s REACTION { method = %s; cellTypes = %d; celltype = %d; fit = %s; precision = mixed; }\n" % (
            name, ADAPTER, 100 + ct, ct, fit)
    refsim.compile_once("b200-adapter-mixed", text)
    prefix = refsim.unique_prefix()
    refsim.compile_objects(tissue.stimulus_objects_text(t.stimuli, prefix=prefix))
    gpu = refsim.RefSim(["b200mEndo", "b200mMid", "b200mEpi"], ["%s%d" % (prefix, i) for i in range(len(t.stimuli))],
                        (t.nx, t.ny, t.nz), (t.dx, t.dy, t.dz), t.gid, t.cell_type, t.sigma, 0.02, t.diffusion_scale)
    ref.set_vm(t.vm0)
    gpu.set_vm(t.vm0)
    probes = np.array([0, 9, t.n // 2, t.n - 1])
    tr_r, tr_g, times = [], [], []
    for _ in range(2000):
        ref.step(10)
        gpu.step(10)
        tr_r.append(ref.vm()[probes])
        tr_g.append(gpu.vm()[probes])
        times.append(ref.time)
    act_r, act_g = ref.activation(), gpu.activation()
    assert (act_r > 0).all() and (act_g > 0).all()
    assert np.abs(act_g - act_r).max() <= 0.5
    tr_r, tr_g, times = np.array(tr_r), np.array(tr_g), np.array(times)
    for j in range(len(probes)):
        a_r, a_g = apd90(tr_r[:, j], times), apd90(tr_g[:, j], times)
        assert len(a_r) == len(a_g) and len(a_r) >= 1
        assert np.abs(a_r - a_g).max() <= 1.0


FGR_ADAPTER = os.path.join(ROOT, "oracle", "_ref", "libb200fgr.so")


def _holed(t):
    """The tissue with a block of cells removed (anatomy holes: the stencil
    sees non-tissue neighbours)."""
    x, y, z = t.tuples()
    keep = ~((x >= 3) & (x < 6) & (y >= 2) & (y < 5) & (z >= 1) & (z < 4))
    return tissue.Tissue(t.nx, t.ny, t.nz, t.dx, t.dy, t.dz, t.gid[keep], t.cell_type[keep], t.sigma[keep],
                         t.vm0[keep], t.stimuli)


def _b200_reaction_sim(t):
    """A RefSim whose three reactions are the B200TT06 adapter (loaded by
    the reference's reactionFactory) on the shipped fits."""
    from golden.make_golden import reference_sim
    from oracle import refsim
    reference_sim(t).close()          # compiles the shipped fits into the object database
    text = ""
    for name, ct, fit in (("b200Endo", 0, "tt06Endo_fit"), ("b200Mid", 1, "tt06Mid_fit"), ("b200Epi", 2, "tt06Epi_fit")):
        text += "%s REACTION { method = %s; cellTypes = %d; celltype = %d; fit = %s; }\n" % (name, ADAPTER, 100 + ct,
                                                                                          ct, fit)
    refsim.compile_once("b200-adapter", text)
    prefix = refsim.unique_prefix()
    refsim.compile_objects(tissue.stimulus_objects_text(t.stimuli, prefix=prefix))
    return refsim.RefSim(["b200Endo", "b200Mid", "b200Epi"], ["%s%d" % (prefix, i) for i in range(len(t.stimuli))],
                         (t.nx, t.ny, t.nz), (t.dx, t.dy, t.dz), t.gid, t.cell_type, t.sigma, 0.02,
                         t.diffusion_scale)


@pytest.mark.skipif(not (_built() and os.path.exists(FGR_ADAPTER)), reason="oracle/_ref with the adapters not built")
@pytest.mark.parametrize("holes,reactions", [(False, "reference"), (True, "reference"), (True, "b200")])
def test_fgr_adapter_in_reference_time_loop(cdb_lib, holes, reactions):
    """The B200FGR Diffusion adapter (cardioid_b200/adapter/B200FGR.cc) in
    place of the reference's FGRDiffusionOMP inside its own time loop, with
    the reference's BetterTT06 or with the B200TT06 reaction adapter (the
    whole step then on the GPU through the two adapters): FP64 max |dVm| <=
    1e-6 mV after 300 steps against the all-reference simulation, identical
    activation times."""
    from golden.make_golden import reference_sim
    t = tissue.box(10, 8, 6, dx=0.2, seed=23)
    if holes:
        t = _holed(t)
    ref = reference_sim(t)
    gpu = reference_sim(t) if reactions == "reference" else _b200_reaction_sim(t)
    gpu.use_diffusion_plugin(FGR_ADAPTER)
    for s in (ref, gpu):
        s.set_vm(t.vm0)
    for _ in range(3):
        ref.step(100)
        gpu.step(100)
    assert np.abs(gpu.vm() - ref.vm()).max() <= 1e-6
    np.testing.assert_array_equal(gpu.activation(), ref.activation())
    assert (ref.activation() > 0).any()
