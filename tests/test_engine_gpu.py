"""Parity of the fused B200 engine with the oracle (oracle/port, pinned to
the reference by tests/test_oracle.py) through the C ABI.

Tolerances (written here, checked below):
  FP64 path  max |dVm| <= 1e-6 mV after 1000 steps; activation times
             identical (same step); FGR weights bit-exact; cell-type and
             index handling bit-exact (each cell keeps its own state).
  mixed path activation-time error <= 0.5 ms, APD90 error <= 1 ms.
"""
import numpy as np
import pytest
import torch

from cardioid_b200 import engine as eng_mod
from cardioid_b200 import tissue, tt06
from cardioid_b200.sensors import apd90

pytestmark = pytest.mark.gpu

DT = 0.02
VM_TOL_FP64 = 1e-6       # mV, after 1000 steps
ACT_TOL_MIXED = 0.5      # ms
APD_TOL_MIXED = 1.0      # ms


def _reaction_ids(t):
    return (t.cell_type - 100).astype(np.uint8)


def _engine(fits, precision="fp64", graphs=True):
    e = eng_mod.Engine(DT, precision=precision, use_graphs=graphs)
    for p in fits:
        e.add_reaction(p)
    return e


def _masked(nx, ny, nz, seed=3):
    full = tissue.box(nx, ny, nz, dx=0.2, seed=seed)
    x, y, z = full.tuples()
    keep = ~((x >= nx // 3) & (x < 2 * nx // 3) & (y >= ny // 3) & (y < 2 * ny // 3) & (z >= 1) & (z < nz - 1))
    keep &= ~((x == nx - 1) & (y == 0))
    return tissue.Tissue(full.nx, full.ny, full.nz, full.dx, full.dy, full.dz, full.gid[keep], full.cell_type[keep],
                         full.sigma[keep], full.vm0[keep], full.stimuli)


@pytest.mark.parametrize("kind", ["box", "cable", "sheet", "masked"])
def test_weights_bit_exact(cdb_lib, oracle_port, fits002, kind):
    t = {"box": lambda: tissue.box(12, 10, 8), "cable": lambda: tissue.box(40, 1, 1),
         "sheet": lambda: tissue.box(20, 16, 1), "masked": lambda: _masked(12, 11, 9)}[kind]()
    with _engine(fits002) as e:
        tid = e.add_tissue(t, _reaction_ids(t))
        w = e.read_weights(tid)
    ref = oracle_port.PortSim(t, fits002, _reaction_ids(t), DT).weights()
    np.testing.assert_array_equal(w, ref)


@pytest.mark.parametrize("kind,steps", [("box", 1000), ("cable", 1000), ("sheet", 1000), ("masked", 600)])
def test_fp64_fused_matches_oracle(cdb_lib, oracle_port, fits002, kind, steps):
    t = {"box": lambda: tissue.box(16, 14, 12), "cable": lambda: tissue.box(300, 1, 1),
         "sheet": lambda: tissue.box(48, 40, 1), "masked": lambda: _masked(16, 14, 12)}[kind]()
    rx = _reaction_ids(t)
    sim = oracle_port.PortSim(t, fits002, rx, DT)
    with _engine(fits002) as e:
        tid = e.add_tissue(t, rx)
        for chunk in (100, 400, steps - 500):
            e.step(chunk)
            sim.step(chunk)
        vm = e.read_vm(tid)
        act = e.read_activation(tid)
        states = e.read_states(tid)
        s, time = e.time(tid)
    ref = sim.vm()
    assert s == steps and time == sim.time
    assert np.abs(vm - ref).max() <= VM_TOL_FP64
    np.testing.assert_array_equal(act, sim.activation())
    assert (act > 0).any()
    rs = sim.states()
    for k, name in enumerate(tt06.STATE_NAMES):
        scale = max(1e-12, np.abs(rs[k]).max())
        assert np.abs(states[k] - rs[k]).max() <= 1e-8 * scale, name


def test_config0_fp64_parity_64cubed_1000_steps(cdb_lib, oracle_port, fits002):
    """The 64^3 box, dt 0.02, 1000 steps, face stimulus at t = 0: max |dVm|
    <= 1e-6 mV and identical activation times."""
    t = tissue.box(64, 64, 64)
    rx = _reaction_ids(t)
    sim = oracle_port.PortSim(t, fits002, rx, DT)
    sim.step(1000)
    with _engine(fits002) as e:
        tid = e.add_tissue(t, rx)
        e.step(1000)
        vm = e.read_vm(tid)
        act = e.read_activation(tid)
        lo, hi = e.minmax(tid)
    assert np.abs(vm - sim.vm()).max() <= VM_TOL_FP64
    np.testing.assert_array_equal(act, sim.activation())
    assert lo == vm.min() and hi == vm.max()
    assert (act > 0).sum() > t.n // 4


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_tissues_equal_alone(cdb_lib, fits002, precision):
    """Index handling: tissues packed into one launch give bit-identical
    results to each tissue run alone, per-tissue drug block included, in
    both precisions."""
    ts = [tissue.box(20, 1, 1, seed=1), tissue.box(10, 9, 1, seed=2), tissue.box(7, 6, 5, seed=3),
          _masked(9, 8, 7, seed=4)]
    scales = [(1.0, 1.0, 1.0), (0.5, 1.0, 1.0), (1.0, 0.3, 0.8), (0.2, 0.9, 0.1)]
    alone = []
    for t, sc in zip(ts, scales):
        with _engine(fits002, precision) as e:
            tid = e.add_tissue(t, _reaction_ids(t), sc)
            e.step(300)
            alone.append((e.read_vm(tid), e.read_states(tid), e.read_activation(tid)))
    with _engine(fits002, precision) as e:
        ids = [e.add_tissue(t, _reaction_ids(t), sc) for t, sc in zip(ts, scales)]
        e.step(300)
        for tid, (vm, st, act) in zip(ids, alone):
            np.testing.assert_array_equal(e.read_vm(tid), vm)
            np.testing.assert_array_equal(e.read_states(tid), st)
            np.testing.assert_array_equal(e.read_activation(tid), act)


def test_join_and_retire_between_steps(cdb_lib, fits002):
    """A tissue that joins late runs from its own t = 0 and ends equal to the
    same tissue run alone; retiring one tissue leaves the others unchanged."""
    a, b = tissue.box(8, 7, 6, seed=5), tissue.box(30, 1, 1, seed=6)
    with _engine(fits002) as e:
        ib = e.add_tissue(b, _reaction_ids(b))
        e.step(200)
        vb = e.read_vm(ib)
    with _engine(fits002) as e:
        ia = e.add_tissue(a, _reaction_ids(a))
        e.step(150)
        ib = e.add_tissue(b, _reaction_ids(b))
        e.step(120)
        e.remove_tissue(ia)
        e.step(80)
        assert e.time(ib)[0] == 200
        np.testing.assert_array_equal(e.read_vm(ib), vb)


def test_graphs_and_plain_launches_agree(cdb_lib, fits002):
    t = tissue.box(10, 9, 8)
    out = []
    for graphs in (True, False):
        with _engine(fits002, graphs=graphs) as e:
            tid = e.add_tissue(t, _reaction_ids(t))
            e.step(37)
            e.step(37)
            out.append(e.read_vm(tid))
    np.testing.assert_array_equal(out[0], out[1])


def test_step_host_equals_device_step(cdb_lib, fits002):
    t = tissue.box(9, 8, 7)
    with _engine(fits002) as e:
        tid = e.add_tissue(t, _reaction_ids(t))
        e.step(5)
        ref = e.read_vm(tid)
    with _engine(fits002) as e:
        tid = e.add_tissue(t, _reaction_ids(t))
        vm = np.ascontiguousarray(t.vm0, dtype=np.float64)
        out = np.empty_like(vm)
        for _ in range(5):
            e.step_host(tid, vm, out)
            vm, out = out, vm
        np.testing.assert_array_equal(vm, ref)


def _host_pair(vm0, locked):
    """Two host Vm buffers, the first holding vm0: plain numpy arrays, or
    page-locked ones (the chunked host step then replays captured graphs)."""
    if not locked:
        return np.ascontiguousarray(vm0, dtype=np.float64), np.empty(len(vm0))
    a, b = (torch.empty(len(vm0), dtype=torch.float64, pin_memory=True) for _ in range(2))
    a.numpy()[:] = vm0
    return a.numpy(), b.numpy()


@pytest.mark.parametrize("kind,precision,host", [("box", "fp64", "pageable"), ("box", "mixed", "pageable"),
                                                 ("sheet", "mixed", "pageable"), ("masked", "fp64", "pageable"),
                                                 ("box", "mixed", "locked"), ("masked", "fp64", "locked")])
def test_chunked_step_host_equals_device_steps(cdb_lib, fits002, kind, precision, host):
    """cdb_engine_step_host on tissues large enough for its chunked pipeline
    (64^3 box: 4 chunks of z-planes; a 512 x 256 sheet: 8 chunks of rows; a
    masked box: 2 chunks): Vm, activation times and states bit-identical to
    device-resident steps, across the stimulus and the wave it starts; with
    page-locked buffers through the two captured graphs of the alternating
    buffer pair (the same kernels launched per step as issued directly)."""
    t = {"box": lambda: tissue.box(64, 64, 64), "sheet": lambda: tissue.box(512, 256, 1),
         "masked": lambda: _masked(64, 48, 40)}[kind]()
    steps = 120
    with _engine(fits002, precision) as e:
        tid = e.add_tissue(t, _reaction_ids(t))
        e.step(steps)
        ref = (e.read_vm(tid), e.read_activation(tid), e.read_states(tid))
    per_step = []
    with _engine(fits002, precision) as e:
        tid = e.add_tissue(t, _reaction_ids(t))
        vm, out = _host_pair(t.vm0, host == "locked")
        for _ in range(steps):
            before = e.launch_count()
            e.step_host(tid, vm, out)
            per_step.append(e.launch_count() - before)
            vm, out = out, vm
        np.testing.assert_array_equal(vm, ref[0])
        np.testing.assert_array_equal(e.read_vm(tid), ref[0])
        np.testing.assert_array_equal(e.read_activation(tid), ref[1])
        np.testing.assert_array_equal(e.read_states(tid), ref[2])
        assert e.time(tid)[0] == steps
    assert (ref[1] > 0).any()
    assert len(set(per_step[1:])) == 1 and per_step[-1] > 3


@pytest.mark.parametrize("host", ["pageable", "locked"])
def test_chunked_step_host_in_place(cdb_lib, fits002, host):
    """vm_in and vm_out may be one buffer: each output range goes down only
    after every chunk it overlaps has gone up."""
    t = tissue.box(64, 64, 64)
    with _engine(fits002, "mixed") as e:
        tid = e.add_tissue(t, _reaction_ids(t))
        e.step(40)
        ref = e.read_vm(tid)
    with _engine(fits002, "mixed") as e:
        tid = e.add_tissue(t, _reaction_ids(t))
        vm, _ = _host_pair(t.vm0, host == "locked")
        for _ in range(40):
            e.step_host(tid, vm, vm)
        np.testing.assert_array_equal(vm, ref)


def test_host_step_graphs_follow_changes(cdb_lib, fits002):
    """Captured host-step graphs are dropped when what they captured changes:
    a retuned launch, a Vm written from the host and a second buffer pair
    between host steps give the same Vm as device-resident steps with the
    same changes."""
    t = tissue.box(64, 64, 64)
    vm_set = np.full(t.n, -20.0)
    with _engine(fits002, "mixed") as e:
        tid = e.add_tissue(t, _reaction_ids(t))
        e.step(30)
        e.set_tuning(0, 0)
        e.step(30)
        e.write_vm(tid, vm_set)
        e.step(30)
        ref = e.read_vm(tid)
    with _engine(fits002, "mixed") as e:
        tid = e.add_tissue(t, _reaction_ids(t))
        vm, out = _host_pair(t.vm0, True)
        for k in range(90):
            if k == 30:
                e.set_tuning(0, 0)
            if k == 60:
                vm2, out = _host_pair(vm_set, True)
                vm = vm2
            e.step_host(tid, vm, out)
            vm, out = out, vm
        np.testing.assert_array_equal(vm, ref)


@pytest.mark.parametrize("graphs", [True, False])
def test_activation_after_host_vm_writes(cdb_lib, oracle_port, fits002, graphs):
    """The engine reads a cell's activation time only on upward crossings of
    0 mV, plus every cell in the first step after the host wrote Vm.  Cells
    the host puts above 0 mV (from the start, between steps, or through
    cdb_engine_step_host) must still get the reference's activation time: the
    first post-step time with Vm > 0."""
    t = tissue.box(16, 12, 10)
    x, _, _ = t.tuples()
    far = np.flatnonzero(x >= 12)
    t.vm0 = t.vm0.copy()
    t.vm0[far[::41]] = 15.0
    rx = _reaction_ids(t)
    sim = oracle_port.PortSim(t, fits002, rx, DT)
    with _engine(fits002, graphs=graphs) as e:
        tid = e.add_tissue(t, rx)
        e.step(30)
        sim.step(30)
        v = e.read_vm(tid)
        v[far[7::29]] = 20.0
        e.write_vm(tid, v)
        sim.set_vm(v)
        e.step(40)
        sim.step(40)
        v = e.read_vm(tid)
        v[far[3::31]] = 25.0
        out = np.empty_like(v)
        e.step_host(tid, v, out)
        sim.set_vm(v)
        sim.step(1)
        e.step(20)
        sim.step(20)
        act = e.read_activation(tid)
        vm = e.read_vm(tid)
    ref = sim.activation()
    assert (ref[far[::41]] > 0).all() and (ref[far[7::29]] > 0).all() and (ref[far[3::31]] > 0).all()
    np.testing.assert_array_equal(act, ref)
    assert np.abs(vm - sim.vm()).max() <= VM_TOL_FP64


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_point_and_box_stimuli_match_oracle(cdb_lib, oracle_port, fits002, precision):
    """Point stimuli add, box stimuli assign, in list order (the port is
    pinned to the reference on this tissue by test_oracle)."""
    from test_oracle import _point_stim_tissue
    t = _point_stim_tissue()
    rx = _reaction_ids(t)
    sim = oracle_port.PortSim(t, fits002, rx, DT)
    sim.step(400)
    with _engine(fits002, precision=precision) as e:
        tid = e.add_tissue(t, rx)
        e.step(400)
        vm = e.read_vm(tid)
        act = e.read_activation(tid)
    ref_act = sim.activation()
    if precision == "fp64":
        assert np.abs(vm - sim.vm()).max() <= VM_TOL_FP64
        np.testing.assert_array_equal(act, ref_act)
    else:
        both = (act > 0) & (ref_act > 0)
        assert (both == (ref_act > 0)).all()
        assert np.abs(act[both] - ref_act[both]).max() <= ACT_TOL_MIXED


def test_mixed_precision_errors_vs_fp64_oracle(cdb_lib, oracle_port, fits002):
    """Mixed path on a 24x20x16 box for 20000 steps (400 ms, one paced beat):
    activation-time error <= 0.5 ms, APD90 error <= 1 ms at probe cells."""
    t = tissue.box(24, 20, 16, period=1000.0)
    rx = _reaction_ids(t)
    sim = oracle_port.PortSim(t, fits002, rx, DT)
    probes = np.array([0, 5, t.n // 3, t.n // 2, t.n - 1])
    steps, every = 20000, 10
    tr_o, tr_m, times = [], [], []
    with _engine(fits002, precision="mixed") as e:
        tid = e.add_tissue(t, rx)
        for k in range(0, steps, every):
            e.step(every)
            sim.step(every)
            tr_m.append(e.read_vm(tid)[probes])
            tr_o.append(sim.vm()[probes])
            times.append(sim.time)
        act_m = e.read_activation(tid)
    act_o = sim.activation()
    assert ((act_o > 0) == (act_m > 0)).all()
    assert np.abs(act_m - act_o)[act_o > 0].max() <= ACT_TOL_MIXED
    tr_o, tr_m, times = np.array(tr_o), np.array(tr_m), np.array(times)
    for j in range(len(probes)):
        a_o, a_m = apd90(tr_o[:, j], times), apd90(tr_m[:, j], times)
        assert len(a_o) == len(a_m) and len(a_o) >= 1
        assert np.abs(a_o - a_m).max() <= APD_TOL_MIXED


def test_full_size_box_mixed_vs_fp64_and_repeatable(cdb_lib):
    """At the benchmark's size (256^3, three transmural types, S1 pacing):
    two FP64 runs agree bit for bit (no order-dependent reductions in the
    step), and the mixed run's activation times stay within 0.5 ms of FP64
    over the first 5 ms of the wave."""
    t = tissue.box(256, 256, 256, period=500.0)
    steps = 250
    acts, vms = {}, {}
    for run, precision in (("a", "fp64"), ("b", "fp64"), ("m", "mixed")):
        with eng_mod.Engine(DT, precision=precision) as e:
            rx, _ = eng_mod.transmural_setup(e, t, DT)
            tid = e.add_tissue(t, rx)
            e.step(steps)
            acts[run], vms[run] = e.read_activation(tid), e.read_vm(tid)
    np.testing.assert_array_equal(vms["a"], vms["b"])
    np.testing.assert_array_equal(acts["a"], acts["b"])
    a, m = acts["a"], acts["m"]
    assert (a > 0).sum() > 100_000
    both = (a > 0) & (m > 0)
    assert ((a > 0) != (m > 0)).mean() < 1e-3
    assert np.abs(a[both] - m[both]).max() <= ACT_TOL_MIXED


def _rows_box(nx, ny, nz, seed):
    """A box of one cell type whose x-rows are whole warp tiles (nx a
    multiple of 32, even padded strides): every tile is a row tile, which
    stage 3 stages through the Vm window; each row's last window reaches
    past the padded block's x extent (read as zeros)."""
    t = tissue.box(nx, ny, nz, seed=seed)
    t.cell_type[:] = 101
    return t


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_staging_modes_agree(cdb_lib, fits002, precision):
    """Direct loads (0), per-lane cp.async staging (1), bulk-copy staging on
    mbarriers (2) and bulk-copy staging with the Vm tile and halo of row
    tiles in shared memory (3) compute the same bits, on a mix of tissue
    classes (row tiles, multi-row tiles, a cable, a masked tissue) and with
    several tiles per warp (small grid)."""
    # the row-tile box dominates its reaction type's tiles (640 of about 770),
    # so stage 3 runs that type's launches with Vm windows
    ts = [tissue.box(40, 33, 9, seed=8), tissue.box(300, 1, 1, seed=9), _masked(13, 12, 11, seed=10),
          _rows_box(128, 16, 10, seed=11)]
    out = {}
    for stage in (0, 1, 2, 3):
        with _engine(fits002, precision=precision) as e:
            e.set_tuning(stage, 1)
            ids = [e.add_tissue(t, _reaction_ids(t)) for t in ts]
            e.step(60)
            e.sync()
            out[stage] = [(e.read_vm(i), e.read_states(i), e.read_activation(i)) for i in ids]
    for stage in (1, 2, 3):
        for a, b in zip(out[0], out[stage]):
            for x, y in zip(a, b):
                np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tile_layouts_agree(cdb_lib, fits002, precision):
    """The two warp-tile layouts (cells in cell order; x-row runs cut into
    whole row tiles with packed remainders) give the same bits, with bulk
    staging (2) and with the Vm windows of row tiles (3), on a box whose
    type slabs are 25 / 35 / 40 cells wide along x, a masked tissue and a
    cable, in one engine."""
    ts = [tissue.box(100, 7, 6, seed=12), _masked(70, 6, 5, seed=13), tissue.box(150, 1, 1, seed=14)]
    out = {}
    for layout in ("cells", "rows"):
        for stage in (2, 3):
            with _engine(fits002, precision=precision) as e:
                e.set_tuning(stage, 1)
                e.set_layout(layout)
                assert e.get_layout() == layout
                ids = [e.add_tissue(t, _reaction_ids(t)) for t in ts]
                e.step(40)
                e.sync()
                out[layout, stage] = [(e.read_vm(i), e.read_states(i), e.read_activation(i)) for i in ids]
    for key in out:
        for a, b in zip(out["cells", 2], out[key]):
            for x, y in zip(a, b):
                np.testing.assert_array_equal(x, y, err_msg=str(key))


def test_rows_layout_host_step_matches_device_steps(cdb_lib, fits002):
    """The chunked host step on a rows-layout tissue (tiles reordered by the
    chunk they need) matches steps on device-resident Vm bit for bit."""
    t = tissue.box(96, 40, 36, seed=15)
    res = {}
    for mode in ("device", "host"):
        with _engine(fits002, precision="mixed") as e:
            e.set_layout("rows")
            tid = e.add_tissue(t, _reaction_ids(t))
            if mode == "device":
                e.step(12)
                res[mode] = e.read_vm(tid)
            else:
                vm = np.ascontiguousarray(t.vm0)
                o = np.empty_like(vm)
                for _ in range(12):
                    e.step_host(tid, vm, o)
                    vm, o = o, vm
                res[mode] = vm
    np.testing.assert_array_equal(res["device"], res["host"])


def _cube_in(n_box, off, side=8, seed=5):
    """A side^3 cube of tissue (transmural slabs, x = 0 face paced) placed at
    offset `off` inside an n_box^3 grid (a masked tissue)."""
    import dataclasses
    c = tissue.box(side, side, side, dx=0.2, seed=seed)
    x, y, z = c.tuples()
    gid = (x + off) + n_box * ((y + off) + n_box * (z + off).astype(np.int64))
    s = dataclasses.replace(c.stimuli[0], xMin=off - 1, xMax=off + 1, yMin=off - 1, yMax=off + side,
                            zMin=off - 1, zMax=off + side)
    return tissue.Tissue(n_box, n_box, n_box, c.dx, c.dy, c.dz, gid.astype(np.int64), c.cell_type, c.sigma, c.vm0,
                         [s])


def test_64bit_voxel_indices_far_corner(cdb_lib, fits002):
    """The same 8^3 cube in a 10^3 grid and at the far corner of a 1300^3
    grid (cell gids and padded-voxel indices above 2^31; ~35 GB of padded
    Vm blocks): bit-identical Vm and activation times after 300 steps."""
    small = _cube_in(10, 1)
    big = _cube_in(1300, 1290)
    assert big.gid.max() > 2 ** 31
    out = []
    for t in (small, big):
        with _engine(fits002) as e:
            tid = e.add_tissue(t, _reaction_ids(t))
            e.step(300)
            e.sync()
            out.append((e.read_vm(tid), e.read_activation(tid)))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    assert (out[0][1] > 0).any()     # the wave started


@pytest.mark.parametrize("shape", [(1, 1, 1), (33, 1, 1), (5, 7, 1), (3, 3, 3), (31, 2, 1)])
def test_tiny_and_ragged_tissues_match_oracle(cdb_lib, oracle_port, fits002, shape):
    """A single cell, and tissues whose type groups end mid-tile (ragged 32-slot
    blocks, one-cell groups): FP64 parity with the oracle after 400 steps."""
    t = tissue.box(*shape, seed=11)
    rx = _reaction_ids(t)
    sim = oracle_port.PortSim(t, fits002, rx, DT)
    sim.step(400)
    with _engine(fits002) as e:
        tid = e.add_tissue(t, rx)
        e.step(400)
        vm = e.read_vm(tid)
        act = e.read_activation(tid)
    assert np.abs(vm - sim.vm()).max() <= VM_TOL_FP64
    np.testing.assert_array_equal(act, sim.activation())
    assert (act > 0).any()


def test_non_finite_vm_reported_by_sync(cdb_lib, fits002):
    """A NaN that the host writes into Vm (the failure is made on the host;
    NaN arithmetic faults nothing on the device) is reported by
    cdb_engine_sync as CDB_NUMERIC_FAULT after the next launch batch, once;
    a clean engine's sync stays OK."""
    from cardioid_b200 import _lib
    t = tissue.box(12, 10, 8)
    with _engine(fits002) as e:
        tid = e.add_tissue(t, _reaction_ids(t))
        e.step(10)
        e.sync()
        vm = e.read_vm(tid)
        vm[5] = np.nan
        e.write_vm(tid, vm)
        e.step(10)
        with pytest.raises(_lib.CdbError) as err:
            e.sync()
        assert err.value.status == _lib.CDB_NUMERIC_FAULT
        e.sync()                      # read once, then cleared
    with _engine(fits002) as e:
        e.add_tissue(t, _reaction_ids(t))
        e.step(50)
        e.sync()


@pytest.mark.parametrize("stage", [2, 3])
def test_bounded_wait_runs_out_and_engine_recovers(cdb_lib, fits002, stage):
    """The failure path of the step's bounded waits, made without a fault:
    one batch withholds its bulk copies after each warp's first tile (a wait
    that nothing completes), its waits give up after about a second, the
    warps leave, and cdb_engine_sync reports CDB_TIMEOUT; the next batches
    run normally on the same context.  Bulk-copy staging (2) and the same
    with the Vm windows of row tiles (3)."""
    from cardioid_b200 import _lib
    t = tissue.box(96, 96, 96)          # about 9000 tiles per type: several per warp
    with eng_mod.Engine(DT, precision="mixed") as e:
        e.set_tuning(stage, 0)
        e.set_layout("rows")
        rx, _ = eng_mod.transmural_setup(e, t, DT)
        tid = e.add_tissue(t, rx)
        e.step(5)
        e.sync()
        e.test_bounded_wait()
        e.step(1)
        with pytest.raises(_lib.CdbError) as err:
            e.sync()
        assert err.value.status == _lib.CDB_TIMEOUT
        e.step(20)
        e.sync()
        assert np.isfinite(e.read_vm(tid)).all()
