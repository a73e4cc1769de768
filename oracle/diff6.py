"""TEST INFRASTRUCTURE: a numpy restatement of the reference's "cuda"
6-face diffusion (CUDADiffusion), the checker for cdb_diff6_*.  Only tests
use it.

  face conductivities   elec/CUDADiffusion.cc:73-122
  flux and its order    elec/CUDADiffusion_ker.cu:16-140 (diff_6face_v1)

The face conductivities are pinned: tests/test_diff6.py checks face_sigma
bit for bit against the table the reference's own CUDADiffusion
constructor builds on the host (run by the oracle build, oracle/_ref).
calc follows the kernel's code line by line.  The flux is pinned on the
GPU (tests/test_diff6.py): the reference's kernel returns from threads
before __syncthreads unless the local grid's y and z sizes are 30 k + 2,
and on tissues of that shape the reference's own CUDADiffusion runs
(oracle/_ref/ref_gpu_diff6) and both calc and the plugin match it.
"""
import numpy as np


def face_sigma(tissue, scale):
    """[n, 3, 3]: the - face of axis i, component j, of every cell."""
    nx, ny, nz = tissue.nx, tissue.ny, tissue.nz
    present = np.zeros((nz + 2, ny + 2, nx + 2), bool)
    x, y, z = tissue.tuples()
    present[z + 1, y + 1, x + 1] = True
    h = (tissue.dx, tissue.dy, tissue.dz)
    area = (h[1] * h[2], h[0] * h[2], h[0] * h[1])
    vol = h[0] * h[1] * h[2]
    s = tissue.sigma
    sig = np.stack([s[:, [0, 1, 2]], s[:, [1, 3, 4]], s[:, [2, 4, 5]]], axis=1)
    unit = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]      # (dx, dy, dz) of each axis
    P = lambda dx, dy, dz: present[z + 1 + dz, y + 1 + dy, x + 1 + dx]
    out = np.zeros((tissue.n, 3, 3))
    for a in range(3):
        ea = unit[a]
        left = P(-ea[0], -ea[1], -ea[2])
        for b in range(3):
            val = sig[:, a, b] * area[a] / h[b] * scale / vol
            if a != b:
                eb = unit[b]
                ok = (P(-eb[0], -eb[1], -eb[2]) & P(eb[0], eb[1], eb[2]) &
                      P(-ea[0] - eb[0], -ea[1] - eb[1], -ea[2] - eb[2]) & P(-ea[0] + eb[0], -ea[1] + eb[1], -ea[2] + eb[2]))
                val = np.where(ok, val, 0.0)
            out[:, a, b] = np.where(left, val, 0.0)
    return out


def calc(tissue, vm, scale):
    """dVm of every cell (diff_6face_v1 on the padded block)."""
    nx, ny, nz = tissue.nx, tissue.ny, tissue.nz
    V = np.zeros((nz + 2, ny + 2, nx + 2))
    F = np.zeros((3, 3, nz + 2, ny + 2, nx + 2))
    x, y, z = tissue.tuples()
    V[z + 1, y + 1, x + 1] = vm
    fs = face_sigma(tissue, scale)
    for a in range(3):
        for b in range(3):
            F[a, b, z + 1, y + 1, x + 1] = fs[:, a, b]

    def v(cx, cy, cz):
        return V[cz, cy, cx]

    def flux(A, cx, cy, cz):
        # face between a = c - e_A and b = c
        ax, ay, az = cx - (A == 0), cy - (A == 1), cz - (A == 2)
        bx, by, bz = cx, cy, cz
        if A == 0:
            d0 = -v(ax, ay, az) + v(bx, by, bz)
            d1 = (-v(ax, ay - 1, az) + v(ax, ay + 1, az) - v(bx, by - 1, bz) + v(bx, by + 1, bz)) / 4.
            d2 = (-v(ax, ay, az - 1) + v(ax, ay, az + 1) - v(bx, by, bz - 1) + v(bx, by, bz + 1)) / 4.
        elif A == 1:
            d0 = (-v(ax - 1, ay, az) - v(bx - 1, by, bz) + v(ax + 1, ay, az) + v(bx + 1, by, bz)) / 4.
            d1 = -v(ax, ay, az) + v(bx, by, bz)
            d2 = (-v(ax, ay, az - 1) + v(ax, ay, az + 1) - v(bx, by, bz - 1) + v(bx, by, bz + 1)) / 4.
        else:
            d0 = (-v(ax - 1, ay, az) - v(bx - 1, by, bz) + v(ax + 1, ay, az) + v(bx + 1, by, bz)) / 4.
            d1 = (-v(ax, ay - 1, az) - v(bx, by - 1, bz) + v(ax, ay + 1, az) + v(bx, by + 1, bz)) / 4.
            d2 = -v(ax, ay, az) + v(bx, by, bz)
        f = F[A][:, cz, cy, cx]
        return f[0] * d0 + f[1] * d1 + f[2] * d2

    cx, cy, cz = x + 1, y + 1, z + 1
    dV = -flux(0, cx, cy, cz)
    dV = dV + flux(1, cx, cy + 1, cz)
    dV = dV - flux(1, cx, cy, cz)
    dV = dV + flux(2, cx, cy, cz + 1)
    dV = dV - flux(2, cx, cy, cz)
    dV = dV + flux(0, cx + 1, cy, cz)
    return dV
