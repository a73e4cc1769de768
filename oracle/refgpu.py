"""Runs the reference's own GPU code in child processes: its reaction path
(oracle/_ref/ref_gpu_reaction: BetterTT06 compiled with USE_CUDA, its NVRTC
kernel driven through the reference's ReactionManager::calc,
elec/BetterTT06.cc:1004-1410 and elec/ReactionManager.cc:14-27) and its ECG
kernels (oracle/_ref/ref_gpu_ecg: elec/ECGSensor.cu) and "cuda" Diffusion
(oracle/_ref/ref_gpu_diff6: elec/CUDADiffusion.cc with its kernels).

TEST AND MEASUREMENT INFRASTRUCTURE.  Only tests/ and bench.py use it, as
a checker and as the reference's GPU comparison point; the product never
imports it.
"""
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BINARY = os.path.join(HERE, "_ref", "ref_gpu_reaction")
NAMES = ("tt06Endo", "tt06Mid", "tt06Epi")


def available():
    return os.path.exists(BINARY)


def objects_text(dt):
    """The three transmural BetterTT06 REACTION objects on the shipped fits
    (anatomy cellType 100/101/102 -> celltype 0/1/2)."""
    from cardioid_b200 import engine, tissue
    text = ""
    for ct in (0, 1, 2):
        with open(engine.shipped_fit_path(dt, ct)) as f:
            text += f.read()
    return text + tissue.reaction_objects_text(["tt06Endo_fit", "tt06Mid_fit", "tt06Epi_fit"])


def run(cell_type, dt, steps, warmup=0, vm=None, outputs=False, timeout=600):
    """Steps the reference's GPU reaction `warmup` + `steps` times with Vm
    and iStim fixed (cells in the given order, anatomy cellTypes 100-102).

    Returns (info, dvm, states): info is the driver's JSON line (cells,
    ms_per_step over the `steps` timed calls, cell_steps_per_s); with
    `outputs`, dvm (float64[n]) and the checkpoint states after the last
    call ({name: float64[n]}, the reference's getCheckpointInfo order).
    """
    if not available():
        raise RuntimeError("oracle/_ref/ref_gpu_reaction is not built (make -C oracle/ref gpu)")
    ct = np.ascontiguousarray(cell_type, dtype=np.int32)
    n = ct.size
    with tempfile.TemporaryDirectory() as tmp:
        obj = os.path.join(tmp, "objects.data")
        with open(obj, "w") as f:
            f.write(objects_text(dt))
        ct_path = os.path.join(tmp, "celltype.bin")
        ct.tofile(ct_path)
        vm_path = "-"
        if vm is not None:
            vm_path = os.path.join(tmp, "vm.bin")
            np.ascontiguousarray(vm, dtype=np.float64).tofile(vm_path)
        out_path = os.path.join(tmp, "out.bin") if outputs else "-"
        cmd = [BINARY, obj, repr(dt), str(steps), str(warmup), ct_path, vm_path, out_path] + list(NAMES)
        # cwd: a fit the reference had to generate would be written there
        res = subprocess.run(cmd, cwd=tmp, capture_output=True, text=True, timeout=timeout)
        if res.returncode != 0:
            raise RuntimeError("ref_gpu_reaction failed (%d): %s" % (res.returncode, res.stderr[-2000:]))
        info = json.loads(res.stdout.strip().splitlines()[-1])
        if not outputs:
            return info, None, None
        raw = np.fromfile(out_path, dtype=np.float64)
    from cardioid_b200 import tt06
    names = list(tt06.STATE_NAMES)
    if raw.size != n * (1 + len(names)):
        raise RuntimeError("ref_gpu_reaction wrote %d values, expected %d" % (raw.size, n * (1 + len(names))))
    cols = raw.reshape(1 + len(names), n)
    return info, cols[0].copy(), {nm: cols[1 + k].copy() for k, nm in enumerate(names)}


ECG_BINARY = os.path.join(HERE, "_ref", "ref_gpu_ecg")


def ecg_available():
    return os.path.exists(ECG_BINARY)


def ecg(t, points, dvmd=None, timeout=300):
    """The reference's own ECG kernels on the GPU (oracle/_ref/ref_gpu_ecg:
    calcInvrCUDA and calcEcgCUDA of elec/ECGSensor.cu) for tissue t's cells
    and the electrodes `points` ([m, 3], mm): returns (invr [n, m], sums [m]
    or None), sums[j] = sum over cells of dvmd[i] invr[i, j] when dvmd is
    given (no kconst or voxel-volume factor: ECGSensor applies those)."""
    if not ecg_available():
        raise RuntimeError("oracle/_ref/ref_gpu_ecg is not built (make -C oracle/ref gpu)")
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    n, m = len(t.gid), len(pts)
    with tempfile.TemporaryDirectory() as tmp:
        gp, pp, op = (os.path.join(tmp, f) for f in ("gid.bin", "points.bin", "out.bin"))
        np.ascontiguousarray(t.gid, dtype=np.int64).tofile(gp)
        pts.tofile(pp)
        dp = "-"
        if dvmd is not None:
            dp = os.path.join(tmp, "dvmd.bin")
            np.ascontiguousarray(dvmd, dtype=np.float64).tofile(dp)
        cmd = [ECG_BINARY, str(t.nx), str(t.ny), str(t.nz), repr(t.dx), repr(t.dy), repr(t.dz), gp, pp, dp, op]
        res = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        if res.returncode != 0:
            raise RuntimeError("ref_gpu_ecg failed (%d): %s" % (res.returncode, res.stderr[-2000:]))
        raw = np.fromfile(op, dtype=np.float64)
    invr = raw[:n * m].reshape(n, m)
    return invr, (raw[n * m:n * m + m].copy() if dvmd is not None else None)


DIFF6_BINARY = os.path.join(HERE, "_ref", "ref_gpu_diff6")


def diff6_available():
    return os.path.exists(DIFF6_BINARY)


def diff6(t, vm, scale, timeout=300, steps=0):
    """dVm from the reference's own "cuda" Diffusion on the GPU
    (oracle/_ref/ref_gpu_diff6: CUDADiffusion with diff_6face_v1, one
    updateLocalVoltage + calc as the omp loop calls them) for tissue t and
    Vm `vm`, diffusion scale `scale`.  t's extents in y and z must be
    multiples of 30 (the driver refuses other shapes: there the reference
    kernel returns from threads before its barriers).  With `steps`, also
    returns the driver's JSON line (ms per updateLocalVoltage + calc)."""
    if not diff6_available():
        raise RuntimeError("oracle/_ref/ref_gpu_diff6 is not built (make -C oracle/ref gpu)")
    n = len(t.gid)
    with tempfile.TemporaryDirectory() as tmp:
        paths = [os.path.join(tmp, f) for f in ("gid.bin", "ct.bin", "sigma.bin", "vm.bin", "out.bin")]
        np.ascontiguousarray(t.gid, dtype=np.int64).tofile(paths[0])
        np.ascontiguousarray(t.cell_type, dtype=np.int32).tofile(paths[1])
        np.ascontiguousarray(t.sigma, dtype=np.float64).reshape(-1).tofile(paths[2])
        np.ascontiguousarray(vm, dtype=np.float64).tofile(paths[3])
        cmd = [DIFF6_BINARY, str(t.nx), str(t.ny), str(t.nz), repr(t.dx), repr(t.dy), repr(t.dz), repr(scale)] + paths
        if steps:
            cmd.append(str(steps))
        res = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        if res.returncode != 0:
            raise RuntimeError("ref_gpu_diff6 failed (%d): %s" % (res.returncode, res.stderr[-2000:]))
        out = np.fromfile(paths[4], dtype=np.float64)
    if out.size != n:
        raise RuntimeError("ref_gpu_diff6 wrote %d values, expected %d" % (out.size, n))
    if steps:
        return out, json.loads(res.stdout.strip().splitlines()[-1])
    return out
