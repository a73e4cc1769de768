"""Autotuner for the fused step: warp-tile layout, staging mode and the
persistent grid.

Candidates (every one gives the same results bit for bit, so the choice is
timing alone):
  layout        "cells" (each reaction type's cells in cell order, 32 per
                warp tile) or "rows" (every x-row run cut into whole 32-cell
                row tiles, remainders packed): the stencil tile shape;
  stage         0 direct loads, 1 cp.async staging, 2 bulk (TMA) staging of
                the next tile's state and weights, 3 = 2 plus the Vm tile and
                halo of row tiles loaded by one TMA tensor copy;
  ctas_per_sm   the persistent grid (SMs x this CTAs of 128 threads; 0 = as
                many as are resident): with the grid fixed, each thread
                walks cells / (grid x 128) cells per launch, so this sets the
                cells per thread against the number of resident warps.

tune() builds a representative tissue set on one scratch engine per layout
(all alive at once), then times every (layout, stage, ctas_per_sm) with
CUDA events on its engine's stream, `repeats` rounds in round-robin order
so slow drifts of the clock (the power cap) fall on every candidate alike,
and keeps each candidate's fastest round; it returns the fastest candidate.
Results are cached per (precision, workload key) for the process.  apply()
sets a choice on an engine; the layout applies to tissues added
afterwards, so apply before adding them.
"""
import itertools

LAYOUTS = ("cells", "rows")
STAGE_MODES = (0, 1, 2, 3)
CTAS_PER_SM = (0, 3, 4)     # 0: as many as are resident

_cache = {}


def time_steps(eng, steps):
    """ms per step of `steps` steps (one captured graph), CUDA events on the
    engine's stream; the graph is captured and run once outside the timed
    region."""
    import torch
    stream = torch.cuda.ExternalStream(eng.stream())
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    eng.step(steps)
    eng.sync()
    start.record(stream)
    eng.step(steps)
    stop.record(stream)
    stop.synchronize()
    return start.elapsed_time(stop) / steps


def autotune(eng, steps=10, stage_modes=STAGE_MODES, ctas_per_sm=CTAS_PER_SM, repeats=3, verbose=False):
    """Times every (stage, ctas_per_sm) on the engine's current tissues,
    `repeats` round-robin rounds, fastest round per candidate; returns (best
    (stage, ctas), {candidate: ms per step}) and leaves the engine on the
    best.  Timing advances the tissues: run it during warm-up, or on a
    scratch engine."""
    cands = list(itertools.product(stage_modes, ctas_per_sm))
    times = {c: [] for c in cands}
    for _ in range(repeats):
        for c in cands:
            eng.set_tuning(*c)
            times[c].append(time_steps(eng, steps))
    results = {c: min(v) for c, v in times.items()}
    if verbose:
        for (st, cta), ms in results.items():
            print("stage %d ctas/SM %d: %.4f ms/step" % (st, cta, ms))
    best = min(results, key=results.get)
    eng.set_tuning(*best)
    return best, results


def tune(make_engine, add_tissues, key, steps=10, layouts=LAYOUTS, stage_modes=STAGE_MODES,
         ctas_per_sm=CTAS_PER_SM, repeats=3, verbose=False):
    """The fastest (layout, stage, ctas_per_sm) for a workload.

    make_engine() returns a new engine with the workload's reaction types
    (used as a context manager); add_tissues(engine) adds a representative
    tissue set to it (with the engine's reaction types registered by it or
    by make_engine).  key names the workload (with the engine's precision
    it keys the cache).  Returns {"layout", "stage", "ctas_per_sm",
    "ms_per_step", "table": {"layout/stage/ctas": ms}}."""
    import contextlib
    probe = make_engine()
    precision = probe.precision
    probe.close()
    ck = (precision, key)
    if ck in _cache:
        return _cache[ck]
    cands = list(itertools.product(layouts, stage_modes, ctas_per_sm))
    times = {c: [] for c in cands}
    with contextlib.ExitStack() as stack:
        engines = {}
        for layout in layouts:
            e = stack.enter_context(make_engine())
            e.set_layout(layout)
            add_tissues(e)
            e.step(3)
            engines[layout] = e
        for _ in range(repeats):
            for layout, st, cta in cands:
                e = engines[layout]
                e.set_tuning(st, cta)
                times[(layout, st, cta)].append(time_steps(e, steps))
    table = {"%s/%d/%d" % c: min(v) for c, v in times.items()}
    if verbose:
        for k, ms in table.items():
            print("%s: %.4f ms/step" % (k, ms))
    best = min(table, key=table.get)
    layout, st, cta = best.split("/")
    out = {"layout": layout, "stage": int(st), "ctas_per_sm": int(cta), "ms_per_step": table[best],
           "table": table, "key": key, "precision": precision, "repeats": repeats, "steps": steps}
    _cache[ck] = out
    return out


def apply(eng, choice):
    """Sets a tune() choice on an engine (before its tissues are added)."""
    eng.set_layout(choice["layout"])
    eng.set_tuning(choice["stage"], choice["ctas_per_sm"])
