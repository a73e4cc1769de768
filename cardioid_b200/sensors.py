"""Host-side measures on Vm traces, and sensor output files.

APD90 is not a sensor of the reference; it is defined here and applied the
same way to every trace it is compared on (the oracle's, the FP64 and the
mixed engine's): per beat, activation at the first sample with Vm > 0
(the ActivationTimeSensor rule, elec/ActivationTimeSensor.cc:99-111),
V_rest the sample just before it, V_peak the maximum after it, and
repolarisation at the first sample after the peak below
V_rest + 0.1 (V_peak - V_rest).
"""
import os

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


def write_activation(directory, gid, activation, loop, time, grid, spacing, filename="activationTime",
                     print_rate=0, eval_rate=1):
    """Writes directory/<filename>#000000 as the reference's
    ActivationTimeSensor::print does (elec/ActivationTimeSensor.cc:39-96): a
    FIXRECORDASCII pio file of 32-byte records "%12llu %18.12f" (gid,
    activation time in ms) padded with blanks and a newline; cells that never
    activated hold 0, the reference's initial value.  Returns the path."""
    os.makedirs(directory, exist_ok=True)
    gid = np.asarray(gid, dtype=np.int64)
    act = np.where(np.asarray(activation) > 0, activation, 0.0)
    nx, ny, nz = grid
    dx, dy, dz = spacing
    header = ("activationTime FILEHEADER {\n"
              "   datatype = FIXRECORDASCII;\n"
              "   nfiles = 1;\n"
              "   nrecord = %d;\n"
              "   lrec = 32;\n"
              "   time = %f;\n"
              "   loop = %d;\n"
              "   nfields = 2;\n"
              "   field_names = gid tActiv;\n"
              "   field_types = u f;\n"
              "   field_units = 1 ms;\n"
              "   nx = %d; ny = %d; nz = %d;\n"
              "   dx = %g; dy = %g; dz = %g;\n"
              "   printRate = %d; evalRate = %d;\n"
              "}\n\n") % (len(gid), time, loop, nx, ny, nz, dx, dy, dz, print_rate, eval_rate)
    rows = "".join(("%12d %18.12f" % (g, a)).ljust(31) + "\n" for g, a in zip(gid, act))
    path = os.path.join(directory, filename + "#000000")
    with open(path, "w") as f:
        f.write(header + rows)
    return path


def write_minmax(path, rows):
    """Writes the rows (time, min Vm, max Vm) as MinMaxSensor::print does
    (elec/MinMaxSensor.cc:30-68): a header line, then time, min, max and
    max - min in scientific notation with 10 digits.  Returns the path."""
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "w") as f:
        f.write("#    time   min V_m    max V_m    max-min\n")
        for time, lo, hi in rows:
            f.write(" %.10e     %.10e      %.10e    %.10e\n" % (time, lo, hi, hi - lo))
    return path
