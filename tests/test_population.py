"""Populations of independent instances stepped together by one engine.

CPU: the seeded population draw.  GPU: a small heterogeneous population
(cables, sheets and boxes; per-instance cell type, conductance scales and
pacing cycle length) in one engine, with a seeded sample of instances
checked one by one against the oracle run alone (FP64: max |dVm| <= 1e-6
mV, identical activation times)."""
import numpy as np
import pytest

from cardioid_b200 import population as pop

# scales from 0.7 so that the sampled instances fire (Vm above 0 mV)
SMALL = pop.PopulationSpec(n=14, cable=(60, 300), sheet=(12, 40), box=(6, 14), cl=(8.0, 20.0), scale=(0.7, 1.0))


def test_population_draw_is_seeded_and_within_ranges():
    a = pop.draw(seed=3)
    b = pop.draw(seed=3)
    assert a == b
    assert len(a) == 4096
    kinds = [i.kind for i in a]
    assert (kinds.count("cable"), kinds.count("sheet"), kinds.count("box")) == (2048, 1638, 410)
    for i in a:
        lo, hi = {"cable": (100, 5000), "sheet": (64, 512), "box": (32, 96)}[i.kind]
        assert lo <= i.dims[0] <= hi
        assert 0 <= min(i.scales) and max(i.scales) <= 1 and 400 <= i.cl <= 2000
    assert 1.8e8 < pop.total_cells(a) < 2.4e8


def test_population_tissue_paces_at_its_cycle_length():
    inst = pop.draw(SMALL, seed=5)[0]
    t = pop.build(inst)
    assert t.n == inst.cells and (t.cell_type == 100 + inst.celltype).all()
    assert t.stimuli[0].period == inst.cl and t.stimuli[0].xMax == 3


@pytest.mark.gpu
def test_population_in_one_engine_matches_oracle_per_instance(cdb_lib, oracle_port, fits002):
    import copy
    from cardioid_b200 import engine as eng_mod
    insts = pop.draw(SMALL, seed=11)
    steps = 1500
    with eng_mod.Engine(0.02, precision="fp64") as e:
        rid = [e.add_reaction(p) for p in fits002]
        tids = []
        for inst in insts:
            t = pop.build(inst)
            tids.append(e.add_tissue(t, np.full(t.n, rid[inst.celltype], np.uint8), scales=inst.scales))
        e.step(steps)
        got = {k: (e.read_vm(tids[k]), e.read_activation(tids[k])) for k in range(len(insts))}
    rng = np.random.default_rng(2)
    activated = 0
    for k in rng.choice(len(insts), size=4, replace=False):
        inst = insts[k]
        t = pop.build(inst)
        p = copy.deepcopy(fits002[inst.celltype])
        p.g_Kr *= inst.scales[0]
        p.g_CaL *= inst.scales[1]
        p.g_Na *= inst.scales[2]
        sim = oracle_port.PortSim(t, [p], np.zeros(t.n, np.uint8), 0.02)
        sim.step(steps)
        vm, act = got[k]
        assert np.abs(vm - sim.vm()).max() <= 1e-6, inst
        np.testing.assert_array_equal(act, sim.activation())
        activated += int((act > 0).any())
    # a small g_Na scale can leave an instance unexcitable; most fire
    assert activated >= 2


@pytest.mark.gpu
def test_mixed_population_in_one_engine_within_tolerance(cdb_lib, oracle_port, fits002):
    """The same heterogeneous population in one mixed-precision engine: each
    sampled instance against the FP64 oracle run alone, activation times
    within 0.5 ms (the mixed path's tolerance) wherever both activate, and
    the same cells activated (at most 0.1 % may differ, a cell crossing 0 mV
    at the last step in one precision only)."""
    import copy
    from cardioid_b200 import engine as eng_mod
    insts = pop.draw(SMALL, seed=11)
    steps = 1500
    with eng_mod.Engine(0.02, precision="mixed") as e:
        rid = [e.add_reaction(p) for p in fits002]
        tids = []
        for inst in insts:
            t = pop.build(inst)
            tids.append(e.add_tissue(t, np.full(t.n, rid[inst.celltype], np.uint8), scales=inst.scales))
        e.step(steps)
        got = {k: e.read_activation(tids[k]) for k in range(len(insts))}
    rng = np.random.default_rng(2)
    compared = 0
    for k in rng.choice(len(insts), size=4, replace=False):
        inst = insts[k]
        t = pop.build(inst)
        p = copy.deepcopy(fits002[inst.celltype])
        p.g_Kr *= inst.scales[0]
        p.g_CaL *= inst.scales[1]
        p.g_Na *= inst.scales[2]
        sim = oracle_port.PortSim(t, [p], np.zeros(t.n, np.uint8), 0.02)
        sim.step(steps)
        act, ref = got[k], sim.activation()
        assert ((act > 0) == (ref > 0)).mean() >= 0.999, inst
        both = (act > 0) & (ref > 0)
        if both.any():
            assert np.abs(act[both] - ref[both]).max() <= 0.5, inst
            compared += 1
    assert compared >= 2
