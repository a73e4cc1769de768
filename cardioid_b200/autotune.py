"""Autotuner for the fused step's launch shape.

For each candidate (shared-memory staging mode, CTAs per SM of the
persistent grid) it times a few steps of the engine's current tissues with
CUDA events on the engine's stream and keeps the fastest.  Timing advances
the tissues: run it during warm-up, or on a scratch engine holding a tissue
of the same shape.
"""
import itertools

STAGE_MODES = (0, 1, 2)    # direct loads, cp.async, bulk copies
CTAS_PER_SM = (0, 4, 8)     # 0: as many as are resident


def time_steps(eng, steps):
    import torch
    stream = torch.cuda.ExternalStream(eng.stream())
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    eng.step(steps)        # capture the graph of this length outside the timed region
    eng.sync()
    start.record(stream)
    eng.step(steps)
    stop.record(stream)
    stop.synchronize()
    return start.elapsed_time(stop) / steps


def autotune(eng, steps=10, stage_modes=STAGE_MODES, ctas_per_sm=CTAS_PER_SM, verbose=False):
    """Returns (best (stage, ctas), {candidate: ms per step}) and leaves the
    engine on the best candidate."""
    results = {}
    for st, cta in itertools.product(stage_modes, ctas_per_sm):
        eng.set_tuning(st, cta)
        results[(st, cta)] = time_steps(eng, steps)
        if verbose:
            print("stage %d ctas/SM %d: %.4f ms/step" % (st, cta, results[(st, cta)]))
    best = min(results, key=results.get)
    eng.set_tuning(*best)
    return best, results
