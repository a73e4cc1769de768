"""Host-side measures on Vm traces.

APD90 is not a sensor of the reference; it is defined here and applied the
same way to every trace it is compared on (the oracle's, the FP64 and the
mixed engine's): per beat, activation at the first sample with Vm > 0
(the ActivationTimeSensor rule, elec/ActivationTimeSensor.cc:99-111),
V_rest the sample just before it, V_peak the maximum after it, and
repolarisation at the first sample after the peak below
V_rest + 0.1 (V_peak - V_rest).
"""
import numpy as np


def apd90(trace, times):
    """APD90 (ms) of every complete beat in one cell's Vm trace sampled at
    `times` (ms)."""
    trace = np.asarray(trace)
    times = np.asarray(times)
    up = np.flatnonzero((trace[1:] > 0) & (trace[:-1] <= 0)) + 1
    out = []
    for u in up:
        vrest = trace[u - 1]
        peak_i = u + np.argmax(trace[u:])
        thr = vrest + 0.1 * (trace[peak_i] - vrest)
        below = np.flatnonzero(trace[peak_i:] < thr)
        if len(below):
            out.append(times[peak_i + below[0]] - times[u])
    return np.array(out)
