"""Builds the CUDA library libcardioid_b200.so in-tree (cardioid_b200/_lib/)
for sm_100a with nvcc.

    python -m cardioid_b200.build [--force] [--checked] [-v]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libcardioid_b200.so")
# The same library with every index of the step kernel checked
# (CDB_BOUNDS_CHECK): for tests only, loaded through CARDIOID_B200_LIB.
CHECKED_LIB = os.path.join(OUT_DIR, "libcardioid_b200_checked.so")
SOURCES = ["engine_host.cu", "plugins.cu", "static_scratch.cu", "diff6.cu"]
HEADERS = ["common.cuh", "tt06_device.cuh", "tt06_step.cuh", "fgr_device.cuh", "step_kernel.cuh", "fit_shapes.h",
           os.path.join("..", "..", "include", "cardioid_b200.h")]

NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--extended-lambda", "-gencode", "arch=compute_100a,code=sm_100a",
              "-Xcompiler", "-fPIC", "-shared"]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def up_to_date(lib=LIB):
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    for f in SOURCES + HEADERS:
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return False
    return True


def _start(lib, extra, verbose):
    tmp = lib + ".tmp"
    cmd = [nvcc()] + NVCC_FLAGS + extra + (["-Xptxas", "-v"] if verbose else []) + \
          ["-o", tmp] + [os.path.join(CSRC, s) for s in SOURCES]
    return subprocess.Popen(cmd, cwd=CSRC, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True), tmp


def build(force=False, verbose=False, checked=False):
    """Builds libcardioid_b200.so (and, with checked, the bounds-checked
    variant alongside it, compiled at the same time)."""
    os.makedirs(OUT_DIR, exist_ok=True)
    jobs = []
    if force or not up_to_date(LIB):
        jobs.append((LIB,) + _start(LIB, [], verbose))
    if checked and (force or not up_to_date(CHECKED_LIB)):
        jobs.append((CHECKED_LIB,) + _start(CHECKED_LIB, ["-DCDB_BOUNDS_CHECK"], False))
    for lib, proc, tmp in jobs:
        out, err = proc.communicate()
        if proc.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s%s" % (os.path.basename(lib), out, err))
        if verbose and lib == LIB:
            sys.stderr.write(err)
        os.replace(tmp, lib)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, checked="--checked" in sys.argv))
