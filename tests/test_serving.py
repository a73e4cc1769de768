"""The serving loop (continuous batching of simulation jobs).

CPU: the scheduler against a fake engine (memory admission, FIFO order,
batches cut at job ends, rejection of jobs that never fit, percentiles),
and the multi-GPU job partition over two gloo ranks.  GPU: a job's
activation map is the same served in a mix as run alone (FP64, bit-exact)."""
import os

import numpy as np
import pytest

from cardioid_b200 import population as pop
from cardioid_b200 import serving


class FakeTissue:
    def __init__(self, inst):
        self.n = inst.cells
        self.inst = inst


class FakeEngine:
    """Memory of 100 bytes per cell; a clock that advances 1 ns per cell-step."""

    def __init__(self, total):
        self.total = total
        self.used = 0
        self.tissues = {}
        self.next = 0
        self.now = 0.0
        self.peak = 0
        self.log = []

    def clock(self):
        return self.now

    def tissue_bytes(self, t, rx, scales):
        return 100 * t.n

    def free_bytes(self):
        return self.total - self.used, self.total

    def add_tissue(self, t, rx, scales):
        assert self.used + 100 * t.n <= self.total
        tid = self.next
        self.next += 1
        self.tissues[tid] = {"n": t.n, "steps": 0, "id": t.inst.index}
        self.used += 100 * t.n
        self.peak = max(self.peak, self.used)
        self.log.append(("add", t.inst.index))
        return tid

    def remove_tissue(self, tid):
        self.used -= 100 * self.tissues[tid]["n"]
        del self.tissues[tid]

    def step(self, k):
        for s in self.tissues.values():
            s["steps"] += k
            self.now += 1e-9 * k * s["n"]

    def sync(self):
        pass

    def read_activation(self, tid):
        s = self.tissues[tid]
        return np.full(s["n"], float(s["steps"]))


def _jobs(n=40, seed=1, rate=2000.0):
    spec = serving.JobSpec(rate=rate, median_cells=3000, sigma=1.0, max_cells=60000, steps=None, beats=1,
                           population=pop.PopulationSpec(cl=(2.0, 10.0)))
    return serving.draw_jobs(n, spec, seed=seed)


def _server(eng, **kw):
    return serving.Server(eng, [0, 1, 2], clock=eng.clock, sleep=lambda s: setattr(eng, "now", eng.now + s),
                          build=FakeTissue, reserve=0, **kw)


def test_server_runs_every_job_to_its_length_within_memory():
    jobs = _jobs()
    eng = FakeEngine(total=100 * 120000)
    srv = _server(eng, batch=97)
    res = srv.run(jobs)
    assert sorted(r.id for r in res) == [j.id for j in jobs]
    by_id = {j.id: j for j in jobs}
    for r in res:
        # the fake's activation map holds the steps the tissue took
        assert r.steps == by_id[r.id].steps and r.finished >= r.admitted >= r.arrival - 1e-12
    assert eng.peak <= eng.total
    assert [i for op, i in eng.log] == sorted(i for op, i in eng.log)   # FIFO admission
    assert srv.cell_steps == sum(j.steps * j.instance.cells for j in jobs)


def test_server_batches_stop_at_job_ends():
    jobs = _jobs(n=12, seed=4)
    eng = FakeEngine(total=100 * 10 ** 7)
    srv = serving.Server(eng, [0, 1, 2], batch=1000, keep=True, clock=eng.clock,
                         sleep=lambda s: setattr(eng, "now", eng.now + s), build=FakeTissue, reserve=0)
    res = srv.run(jobs)
    for r in res:
        assert (r.activation == r.steps).all()


def test_server_rejects_jobs_larger_than_the_device():
    jobs = _jobs(n=10, seed=2)
    big = max(jobs, key=lambda j: j.instance.cells)
    eng = FakeEngine(total=100 * (big.instance.cells - 1))
    srv = _server(eng)
    res = srv.run(jobs)
    assert big.id in srv.rejected
    assert len(res) + len(srv.rejected) == len(jobs)


def test_summary_percentiles():
    rs = [serving.JobResult(i, 1, 1, 0.0, 0.0, float(i + 1), 0, float("nan")) for i in range(100)]
    s = serving.summary(rs, 10.0, 500)
    assert s["p50_s"] == pytest.approx(50.5) and s["p99_s"] == pytest.approx(99.01)
    assert s["cell_steps_per_s"] == 50.0


def test_job_draw_shapes_and_lengths():
    jobs = serving.draw_jobs(500, serving.JobSpec(rate=10.0), seed=9)
    cells = np.array([j.instance.cells for j in jobs])
    assert cells.max() <= 30_000_000 and 5e4 < np.median(cells) < 8e5
    assert all(j.steps == round(5 * j.instance.cl / 0.02) for j in jobs)
    assert np.all(np.diff([j.arrival for j in jobs]) > 0)


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    jobs = _jobs(n=30, seed=6)
    mine = serving.partition(jobs, rank, world)
    eng = FakeEngine(total=100 * 10 ** 7)
    res = _server(eng).run(mine)
    t = torch.tensor([len(res), sum(r.id for r in res), srv_cells(res)], dtype=torch.float64)
    dist.all_reduce(t)
    out.put((rank, t.tolist()))
    dist.destroy_process_group()


def srv_cells(res):
    return sum(r.cells for r in res)


def test_partition_over_two_gloo_ranks_serves_every_job_once():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    jobs = _jobs(n=30, seed=6)
    want = [len(jobs), sum(j.id for j in jobs), sum(j.instance.cells for j in jobs)]
    for _, t in got:
        assert t == want


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_served_job_equals_job_alone(cdb_lib, fits002, precision):
    """A job served among others (joining and retiring between batches)
    activates bit for bit as the same job run alone, in both precisions."""
    from cardioid_b200 import engine as eng_mod
    spec = serving.JobSpec(rate=1e6, median_cells=2000, sigma=0.8, max_cells=20000, steps=700,
                           population=pop.PopulationSpec(cl=(5.0, 12.0)))
    jobs = serving.draw_jobs(8, spec, seed=3)
    with eng_mod.Engine(0.02, precision=precision) as e:
        rid = [e.add_reaction(p) for p in fits002]
        res = serving.Server(e, rid, batch=150, keep=True, reserve=0).run(jobs)
    assert len(res) == len(jobs)
    for r in res[:3]:
        inst = jobs[r.id].instance
        with eng_mod.Engine(0.02, precision=precision) as e:
            rid = [e.add_reaction(p) for p in fits002]
            t = pop.build(inst)
            tid = e.add_tissue(t, np.full(t.n, rid[inst.celltype], np.uint8), scales=inst.scales)
            e.step(700)
            np.testing.assert_array_equal(e.read_activation(tid), r.activation)


def test_server_builds_on_worker_threads_with_the_same_results():
    """Tissues built on worker threads (the default) or at admission serve
    the same jobs to the same results, first come first served."""
    jobs = _jobs(n=30, seed=7)
    out = {}
    for workers in (0, 2):
        eng = FakeEngine(total=100 * 120000)
        srv = _server(eng, batch=97, keep=True, workers=workers)
        res = srv.run(jobs)
        assert [i for op, i in eng.log] == sorted(i for op, i in eng.log)
        out[workers] = sorted((r.id, r.cells, r.steps, r.activated, tuple(r.activation)) for r in res)
    assert out[0] == out[2]
    assert [r[0] for r in out[0]] == [j.id for j in jobs]


def test_server_build_errors_reach_the_caller():
    """A tissue that fails to build on a worker thread raises from run(), and
    the workers are shut down."""
    jobs = _jobs(n=6, seed=3)
    bad = jobs[2].id

    def build(inst):
        if inst.index == bad:
            raise ValueError("no tissue for instance %d" % inst.index)
        return FakeTissue(inst)

    eng = FakeEngine(total=100 * 120000)
    srv = serving.Server(eng, [0, 1, 2], clock=eng.clock, sleep=lambda s: setattr(eng, "now", eng.now + s),
                         build=build, reserve=0, workers=2)
    with pytest.raises(ValueError, match="no tissue"):
        srv.run(jobs)
    assert srv._pool is None
