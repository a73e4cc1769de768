"""Small and edge-case runs of the fused engine, saved to an .npz: run once
with the normal library and once with the bounds-checked one
(CARDIOID_B200_LIB) by tests/test_bounds_gpu.py, each in its own process.

    python tests/bounds_cases.py OUT.npz
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from cardioid_b200 import engine, tissue  # noqa: E402

DT = 0.02


def masked(nx, ny, nz, seed=3):
    full = tissue.box(nx, ny, nz, dx=0.2, seed=seed)
    x, y, z = full.tuples()
    keep = ~((x >= nx // 3) & (x < 2 * nx // 3) & (y >= ny // 3) & (y < 2 * ny // 3) & (z >= 1) & (z < nz - 1))
    return tissue.Tissue(full.nx, full.ny, full.nz, full.dx, full.dy, full.dz, full.gid[keep], full.cell_type[keep],
                         full.sigma[keep], full.vm0[keep], full.stimuli)


def rows(nx, ny, nz):
    """One cell type, x-rows of whole warp tiles: stage 3's Vm windows, the
    last one's TMA box reaching past the padded block's x extent (read as
    zeros)."""
    t = tissue.box(nx, ny, nz)
    t.cell_type[:] = 100
    return t


def tissues():
    return {"box": tissue.box(9, 8, 7), "cable": tissue.box(40, 1, 1), "sheet": tissue.box(12, 9, 1),
            "masked": masked(16, 14, 12), "one": tissue.box(1, 1, 1), "ragged": tissue.box(33, 1, 1),
            "rows": rows(64, 5, 4)}


def run(out):
    res = {}
    for prec in ("fp64", "mixed"):
        for stage in (0, 1, 2, 3):
            # every tissue alone and all of them in one engine (one launch per type)
            ts = tissues()
            with engine.Engine(DT, precision=prec) as e:
                rx, _ = engine.transmural_setup(e, ts["box"], DT)
                e.set_tuning(stage, 0)
                ids = {k: e.add_tissue(t, np.asarray(rx if k == "box" else (t.cell_type - 100), np.uint8))
                       for k, t in ts.items()}
                e.set_ecg(ids["box"], np.array([[3.0, 2.0, 1.5], [0.1, 0.2, 0.3]]), 5)
                e.step(60)
                e.sync()
                for k, tid in ids.items():
                    res["%s_s%d_%s_vm" % (prec, stage, k)] = e.read_vm(tid)
                    res["%s_s%d_%s_act" % (prec, stage, k)] = e.read_activation(tid)
                loops, ecg = e.read_ecg(ids["box"])
                res["%s_s%d_ecg" % (prec, stage)] = ecg
        # the chunked host step
        t = tissue.box(64, 64, 40)
        with engine.Engine(DT, precision=prec) as e:
            rx, _ = engine.transmural_setup(e, t, DT)
            tid = e.add_tissue(t, rx)
            vm = np.ascontiguousarray(t.vm0)
            o = np.empty_like(vm)
            for _ in range(20):
                e.step_host(tid, vm, o)
                vm, o = o, vm
            e.sync()
            res["%s_host" % prec] = vm
    np.savez(out, **res)


if __name__ == "__main__":
    run(sys.argv[1])
