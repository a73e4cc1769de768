"""The drop-in Reaction / Diffusion plugins against the oracle: the same data
flow as the reference's omp loop (elec/simulationLoop.cc:183-231) driven
through BetterTT06.calc with an index array and FGRDiffusion.calc."""
import numpy as np
import pytest

from cardioid_b200 import objectdb, plugins, tissue

pytestmark = pytest.mark.gpu
DT = 0.02


def test_reaction_plugin_index_gather_scatter(cdb_lib, oracle_port, fits002):
    """A permuted index array: every cell keeps its own state, dVm lands at
    indexArray[i] (bit-exact index handling, FP64 values within 1e-9)."""
    import torch
    n = 257
    rng = np.random.default_rng(0)
    perm = rng.permutation(n).astype(np.int32)
    vm = -83.0 + rng.uniform(-1, 1, n)
    t = tissue.Tissue(n, 1, 1, 1.0, 1.0, 1.0, np.arange(n), np.full(n, 101, np.int32), np.zeros((n, 6)), vm, [])
    sim = oracle_port.PortSim(t, [fits002[1]], np.zeros(n, np.uint8), DT, diffusion=False)
    r = plugins.BetterTT06(fits002[1], n, DT)
    idx = torch.from_numpy(perm).cuda()
    Vm = torch.from_numpy(vm.copy()).cuda()
    dVm = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
    iStim = torch.zeros(n, dtype=torch.float64, device="cuda")
    for _ in range(50):
        r.calc(DT, idx, Vm, iStim, dVm)
        Vm += DT * dVm
        sim.step(1)
    torch.cuda.synchronize()
    got = Vm.cpu().numpy()
    assert np.abs(got - sim.vm()).max() <= 1e-9
    st = sim.states()
    for k in range(18):
        ours = r.getValues(k)   # reaction-local order: cell i of the reaction is Vm[perm[i]]
        np.testing.assert_allclose(ours, st[k][perm], rtol=1e-9, atol=1e-15)


def _masked_box(nx, ny, nz):
    """A box with a hole through its middle and one missing edge column."""
    full = tissue.box(nx, ny, nz)
    x, y, z = full.tuples()
    keep = ~((x >= nx // 3) & (x < 2 * nx // 3) & (y >= ny // 3) & (y < 2 * ny // 3))
    keep &= ~((x == nx - 1) & (y == 0))
    return tissue.Tissue(full.nx, full.ny, full.nz, full.dx, full.dy, full.dz, full.gid[keep], full.cell_type[keep],
                         full.sigma[keep], full.vm0[keep], full.stimuli)


@pytest.mark.parametrize("kind", ["box", "cable", "sheet", "masked"])
def test_fgr_plugin_matches_oracle_weights_and_dvm(cdb_lib, oracle_port, fits002, kind):
    """FGRDiffusion's 19 weights bit for bit and its dVm within 1e-12 of the
    largest |dVm| against the oracle, on a box, a cable and a sheet (the
    missing neighbours get no weight) and a box with a hole (no-flux faces
    inside the grid)."""
    import torch
    t = {"box": lambda: tissue.box(11, 9, 7), "cable": lambda: tissue.box(40, 1, 1),
         "sheet": lambda: tissue.box(20, 16, 1), "masked": lambda: _masked_box(12, 11, 9)}[kind]()
    d = plugins.FGRDiffusion(t)
    sim = oracle_port.PortSim(t, fits002, (t.cell_type - 100).astype(np.uint8), DT)
    np.testing.assert_array_equal(d.weights(), sim.weights())
    sim.step(1)   # dVmD of the first step is computed from vm0
    Vm = torch.from_numpy(t.vm0.copy()).cuda()
    dVm = torch.empty_like(Vm)
    d.updateLocalVoltage(Vm)
    d.updateRemoteVoltage(None)
    d.calc(dVm)
    _, ref, _ = sim.dvm()
    assert np.abs(dVm.cpu().numpy() - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def _split_loop(t, steps, precision="fp64", probes=None, every=10):
    """The omp loop's step order on the drop-in plugins (ReactionManager over
    the three declared reactions, FGR diffusion, box stimulus, integrator).
    Returns the final Vm, the reaction manager, the activation times (first
    post-step time with Vm > 0, -1 if none) and, with probes, their Vm and
    the time every `every` steps."""
    import torch
    from cardioid_b200 import engine
    db = objectdb.ObjectDB()
    for ct in (0, 1, 2):
        db.compile_file(engine.shipped_fit_path(DT, ct))
    db.compile(tissue.reaction_objects_text(["tt06Endo_fit", "tt06Mid_fit", "tt06Epi_fit"]))
    db.compile("fgr DIFFUSION { method = FGR; diffusionScale = %r; }" % t.diffusion_scale)
    rm = plugins.ReactionManager(db, ["tt06Endo", "tt06Mid", "tt06Epi"], DT, t.cell_type, precision=precision)
    diff = plugins.diffusionFactory(db, "fgr", t)
    x, y, z = t.tuples()
    s = t.stimuli[0]
    inbox = torch.from_numpy((x > s.xMin) & (x < s.xMax) & (y > s.yMin) & (y < s.yMax) & (z > s.zMin) &
                             (z < s.zMax)).cuda()
    Vm = torch.from_numpy(t.vm0.copy()).cuda()
    dVmR, dVmD = torch.zeros_like(Vm), torch.zeros_like(Vm)
    iStim = torch.zeros_like(Vm)
    act = torch.full_like(Vm, -1.0)
    trace, times = [], []
    time = 0.0
    for k in range(steps):
        iStim.zero_()
        v = s.value(time)
        if v != 0:
            iStim[inbox] = v
        rm.calc(DT, Vm, iStim, dVmR)
        diff.updateLocalVoltage(Vm)
        diff.calc(dVmD)
        Vm += DT * (dVmR + dVmD + iStim)
        time += DT
        act = torch.where((act < 0) & (Vm > 0), torch.full_like(act, time), act)
        if probes is not None and (k + 1) % every == 0:
            trace.append(Vm[probes].cpu().numpy())
            times.append(time)
    out = (Vm.cpu().numpy(), rm, act.cpu().numpy())
    return out + ((np.array(trace), np.array(times)) if probes is not None else ())


def test_split_plugins_loop_matches_oracle(cdb_lib, oracle_port, fits002):
    """ReactionManager + FGRDiffusion + stimulus + integrator, step by step
    as the omp loop, for 300 steps: within the FP64 parity tolerance
    (1e-6 mV) of the oracle."""
    t = tissue.box(10, 8, 6)
    vm, _, _ = _split_loop(t, 300)
    sim = oracle_port.PortSim(t, fits002, (t.cell_type - 100).astype(np.uint8), DT)
    sim.step(300)
    assert np.abs(vm - sim.vm()).max() <= 1e-6


def test_mixed_reaction_plugins_vs_fp64_oracle(cdb_lib, oracle_port, fits002):
    """The split loop with the mixed-precision plugin reactions (FP64 FGR
    diffusion) on a 12x10x8 box for 20000 steps (400 ms, one paced beat)
    against the FP64 oracle: every cell activates, activation times within
    0.5 ms, APD90 within 1 ms at probe cells (the mixed path's tolerances)."""
    from cardioid_b200.sensors import apd90
    t = tissue.box(12, 10, 8, period=1000.0)
    probes = np.array([0, 7, t.n // 3, t.n // 2, t.n - 1])
    steps, every = 20000, 10
    _, _, act_m, tr_m, times = _split_loop(t, steps, "mixed", probes, every)
    sim = oracle_port.PortSim(t, fits002, (t.cell_type - 100).astype(np.uint8), DT)
    tr_o = []
    for _ in range(0, steps, every):
        sim.step(every)
        tr_o.append(sim.vm()[probes])
    tr_o = np.array(tr_o)
    act_o = sim.activation()
    assert (act_o > 0).all() and (act_m > 0).all()
    assert np.abs(act_m - act_o).max() <= 0.5
    for j in range(len(probes)):
        a_o, a_m = apd90(tr_o[:, j], times), apd90(tr_m[:, j], times)
        assert len(a_o) == len(a_m) and len(a_o) >= 1
        assert np.abs(a_o - a_m).max() <= 1.0


def test_reaction_without_cells_is_a_no_op(cdb_lib, oracle_port, fits002):
    """A declared REACTION whose cellTypes the tissue lacks (here the mid
    type: its cells made endo) is created with no cells, as
    ReactionManager::create does; its init and calc return without touching
    anything, even with empty (null) arrays, and the loop over the other two
    matches the oracle (1e-6 mV after 200 steps)."""
    import torch
    t = tissue.box(10, 8, 6)
    t.cell_type[t.cell_type == 101] = 100
    vm, rm, _ = _split_loop(t, 200)
    assert [r.nCells for r in rm.reactions] == [int((t.cell_type == 100).sum()), 0, int((t.cell_type == 102).sum())]
    sim = oracle_port.PortSim(t, fits002, (t.cell_type - 100).astype(np.uint8), DT)
    sim.step(200)
    assert np.abs(vm - sim.vm()).max() <= 1e-6
    empty = rm.reactions[1]
    idx = torch.zeros(0, dtype=torch.int32, device="cuda")
    Vm = torch.zeros(0, dtype=torch.float64, device="cuda")
    empty.calc(DT, idx, Vm, Vm, Vm)
    empty.initializeMembraneVoltage(idx, Vm)
    # the same through the real arrays of the loop: dVm keeps its NaNs
    Vm = torch.from_numpy(vm).cuda()
    dVm = torch.full_like(Vm, float("nan"))
    empty.calc(DT, idx, Vm, torch.zeros_like(Vm), dVm)
    torch.cuda.synchronize()
    assert bool(torch.isnan(dVm).all())
    assert empty.getValues(0).shape == (0,)


def _single_type(n, vm):
    return tissue.Tissue(n, 1, 1, 1.0, 1.0, 1.0, np.arange(n), np.full(n, 101, np.int32), np.zeros((n, 6)), vm, [])


def test_reaction_slots_past_the_last_and_shared(cdb_lib, oracle_port, fits002):
    """Eight plugin reactions with distinct g_Kr alive at once: the first
    take constant-memory slots (the compiled per-slot kernel), the rest run
    the generic kernel; each matches the oracle with its own parameters.
    A ninth with the first one's content shares its slot."""
    import dataclasses
    import torch
    n = 96
    rng = np.random.default_rng(1)
    base = fits002[1]
    variants = [dataclasses.replace(base, g_Kr=base.g_Kr * (1 + 0.25 * k)) for k in range(8)] + [base]
    vm0 = -83.0 + rng.uniform(-1, 1, n)
    vm0[:8] = 20.0      # a few cells depolarised, so g_Kr matters within the run
    rx = [plugins.BetterTT06(p, n, DT) for p in variants]
    idx = torch.arange(n, dtype=torch.int32, device="cuda")
    iStim = torch.zeros(n, dtype=torch.float64, device="cuda")
    finals = []
    for r, p in zip(rx, variants):
        sim = oracle_port.PortSim(_single_type(n, vm0), [p], np.zeros(n, np.uint8), DT, diffusion=False)
        Vm = torch.from_numpy(vm0.copy()).cuda()
        dVm = torch.empty_like(Vm)
        for _ in range(40):
            r.calc(DT, idx, Vm, iStim, dVm)
            Vm += DT * dVm
        sim.step(40)
        got = Vm.cpu().numpy()
        assert np.abs(got - sim.vm()).max() <= 1e-9
        finals.append(got)
    assert np.abs(finals[0] - finals[1]).max() > 1e-6      # the variants differ
    np.testing.assert_array_equal(finals[-1], finals[0])   # same content, same slot, same bits


def test_engine_shares_slots_with_plugin_reactions(cdb_lib, fits002):
    """Plugin reactions for the three shipped types hold three slots; an
    engine registering the same three types shares them, so three more
    distinct plugin reactions still get slots and the engine still steps."""
    import dataclasses
    from cardioid_b200 import engine
    keep = [plugins.BetterTT06(p, 32, DT) for p in fits002]
    extra = [plugins.BetterTT06(dataclasses.replace(fits002[0], g_Kr=0.1 * (k + 1)), 32, DT) for k in range(3)]
    t = tissue.box(12, 10, 8)
    with engine.Engine(DT, precision="fp64") as e:
        rx, _ = engine.transmural_setup(e, t, DT)
        e.add_tissue(t, rx)
        e.step(20)
        e.sync()
        assert np.isfinite(e.read_vm(0)).all()
    del keep, extra
