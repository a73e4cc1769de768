"""Serving loop: simulation jobs (one tissue each) arrive over time and are
stepped together by one engine — continuous batching.  Between launch
batches the loop admits waiting jobs first come, first served while the
device has memory for them (cdb_engine_tissue_bytes against free memory),
steps every active job, and retires the finished ones, reading back their
activation maps.  Worker threads build arrived jobs' tissues on the host
meanwhile, so a large job's set-up does not stall the active ones.  Reports time-to-result percentiles and the aggregate
cell-steps/s.

The engine runs each tissue on its own clock and step count, so a job's
result does not depend on which other jobs share its launches.

On N GPUs, one process per GPU serves its own share of the jobs
(partition(): round robin by job id); the shares need no exchange.
"""
import collections
import math
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import population as pop


@dataclass
class Job:
    id: int
    arrival: float               # seconds after the start of serving
    instance: pop.Instance       # geometry, cell type, scales, cycle length
    steps: int


@dataclass
class JobResult:
    id: int
    cells: int
    steps: int
    arrival: float
    admitted: float
    finished: float
    activated: int               # cells with an activation time
    mean_activation: float       # ms, over activated cells (nan if none)
    activation: np.ndarray = None

    @property
    def time_to_result(self):
        return self.finished - self.arrival


@dataclass
class JobSpec:
    """Jobs: Poisson arrivals at `rate` per second; cell counts log-normal
    (median 2e5, sigma 1.5, at most 3e7) shaped as a cable, sheet or box with
    the population's kind fractions; cell type, scales and cycle length as
    in population.PopulationSpec; length `beats` cycles (steps = beats CL /
    dt) unless `steps` is given."""
    rate: float = 1.0
    median_cells: float = 2e5
    sigma: float = 1.5
    max_cells: int = 30_000_000
    min_cells: int = 32
    beats: int = 5
    steps: int = None
    dt: float = 0.02
    population: pop.PopulationSpec = field(default_factory=pop.PopulationSpec)


def _dims(kind, cells):
    if kind == "cable":
        return (cells, 1, 1)
    if kind == "sheet":
        s = max(2, int(round(math.sqrt(cells))))
        return (s, s, 1)
    s = max(2, int(round(cells ** (1.0 / 3.0))))
    return (s, s, s)


def draw_jobs(n, spec=None, seed=20240611):
    spec = spec or JobSpec()
    rng = np.random.default_rng(seed)
    ps = spec.population
    t = 0.0
    jobs = []
    for i in range(n):
        t += rng.exponential(1.0 / spec.rate)
        kind = pop.KINDS[int(rng.choice(3, p=np.asarray(ps.fractions) / sum(ps.fractions)))]
        cells = int(min(spec.max_cells, max(spec.min_cells, round(spec.median_cells * math.exp(spec.sigma *
                                                                                            rng.standard_normal())))))
        celltype = int(rng.integers(0, 3))
        scales = tuple(float(v) for v in rng.uniform(ps.scale[0], ps.scale[1], size=3))
        cl = float(rng.uniform(*ps.cl))
        inst = pop.Instance(i, kind, _dims(kind, cells), celltype, scales, cl)
        steps = spec.steps if spec.steps is not None else int(round(spec.beats * cl / spec.dt))
        jobs.append(Job(i, t, inst, steps))
    return jobs


def partition(jobs, rank, world):
    """This rank's share of the jobs: round robin by id."""
    return [j for j in jobs if j.id % world == rank]


class Server:
    """Continuous batching over one engine.

    engine     a cardioid_b200.engine.Engine (or anything with its
               tissue_bytes / free_bytes / add_tissue / remove_tissue /
               step / sync / read_activation methods)
    reactions  engine reaction ids by BetterTT06 celltype 0/1/2
    batch      most steps per launch batch; a batch never runs a job past
               its end, so it is cut to the fewest steps any job has left
    reserve    device bytes kept free beyond each admitted tissue
    keep       keep each job's activation map in its result
    workers    threads that build arrived jobs' tissues on the host while
               the device steps the active ones (0: build at admission)
    """

    def __init__(self, engine, reactions, batch=200, reserve=1 << 30, keep=False, clock=time.perf_counter,
                 sleep=time.sleep, build=pop.build, workers=2):
        self.engine = engine
        self.reactions = list(reactions)
        self.batch = int(batch)
        self.reserve = int(reserve)
        self.keep = keep
        self.clock = clock
        self.sleep = sleep
        self.build = build
        self.workers = int(workers)
        self.cell_steps = 0
        self.rejected = []
        self._built = {}
        self._pool = None

    def _arrived(self, job):
        if self._pool is not None:
            self._built[job.id] = self._pool.submit(self.build, job.instance)

    def _admit(self, job, now, alone):
        """(tissue id, state) once admitted, None to wait (for memory, or for
        the job's tissue to be built), or "reject" when the job cannot fit
        even alone."""
        inst = job.instance
        entry = self._built.get(job.id)
        if entry is None or isinstance(entry, Future):
            if entry is None:
                t = self.build(inst)
            elif not entry.done():
                return None
            else:
                t = entry.result()
            rx = np.full(t.n, self.reactions[inst.celltype], np.uint8)
            self._built[job.id] = (t, rx, self.engine.tissue_bytes(t, rx, inst.scales))
        t, rx, need = self._built[job.id]
        free, total = self.engine.free_bytes()
        if need + self.reserve > free:
            return "reject" if alone or need + self.reserve > total else None
        tid = self.engine.add_tissue(t, rx, scales=inst.scales)
        del self._built[job.id]
        return tid, {"job": job, "left": job.steps, "admitted": now, "cells": t.n}

    def run(self, jobs, max_seconds=None):
        """Serves jobs (arrival times relative to the call) to completion, or
        until max_seconds, and returns their JobResults in finishing order."""
        pending = collections.deque(sorted(jobs, key=lambda j: j.arrival))
        waiting = collections.deque()
        active = {}
        results = []
        if self.workers > 0:
            self._pool = ThreadPoolExecutor(max_workers=self.workers)
        try:
            return self._serve(pending, waiting, active, results, max_seconds)
        finally:
            if self._pool is not None:
                self._pool.shutdown(wait=True, cancel_futures=True)
                self._pool = None

    def _serve(self, pending, waiting, active, results, max_seconds):
        t0 = self.clock()
        while pending or waiting or active:
            now = self.clock() - t0
            if max_seconds is not None and now > max_seconds:
                break
            while pending and pending[0].arrival <= now:
                job = pending.popleft()
                waiting.append(job)
                self._arrived(job)
            while waiting:
                got = self._admit(waiting[0], now, alone=not active)
                if got is None:
                    break
                job = waiting.popleft()
                if got == "reject":
                    self.rejected.append(job.id)
                    self._built.pop(job.id, None)
                    continue
                tid, state = got
                active[tid] = state
            if not active:
                if waiting:
                    self.sleep(0.001)      # the head of the queue is being built
                elif pending:
                    self.sleep(max(0.0, min(0.01, pending[0].arrival - (self.clock() - t0))))
                continue
            k = min(self.batch, min(s["left"] for s in active.values()))
            self.engine.step(k)
            self.engine.sync()
            for tid, s in list(active.items()):
                s["left"] -= k
                self.cell_steps += k * s["cells"]
                if s["left"] == 0:
                    act = self.engine.read_activation(tid)
                    self.engine.remove_tissue(tid)
                    done = self.clock() - t0
                    hit = act > 0
                    results.append(JobResult(s["job"].id, s["cells"], s["job"].steps, s["job"].arrival,
                                             s["admitted"], done, int(hit.sum()),
                                             float(act[hit].mean()) if hit.any() else float("nan"),
                                             act if self.keep else None))
                    del active[tid]
        self.elapsed = self.clock() - t0
        return results


def summary(results, elapsed, cell_steps):
    """p50 / p99 time-to-result (s) and aggregate cell-steps/s."""
    ttr = np.array([r.time_to_result for r in results]) if results else np.array([np.nan])
    return {"jobs": len(results), "p50_s": float(np.percentile(ttr, 50)), "p99_s": float(np.percentile(ttr, 99)),
            "cell_steps_per_s": cell_steps / elapsed if elapsed > 0 else float("nan"), "elapsed_s": elapsed,
            "cell_steps": int(cell_steps)}
