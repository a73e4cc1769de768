"""Irregular anatomy: a truncated prolate-ellipsoid shell (a left-ventricle-
like cup), voxelised on a regular grid, as a sparse Tissue (gid list with
8-byte gids; voxels outside the wall are not tissue, so the FGR mask gives
them no-flux boundaries, elec/FGRUtils.cc:10-76).

Geometry (millimetres, long axis along z, apex at z = -a):
  outer surface  x^2/b^2 + y^2/c^2 + z^2/a^2 = 1, semi-axes b = c = 25, a = 45;
  inner surface  the same with every semi-axis reduced by the wall (10 mm);
  truncated at `cut` of the long axis from the apex (z <= -a + 2 a cut).
Normalised wall depth t in [0, 1] (0 on the endocardium, 1 on the
epicardium) is the t whose ellipsoid, semi-axes inner + t * wall, passes
through the voxel centre.  Cell types by depth: endo t < 0.30 (anatomy
cellType 100), mid t < 0.65 (101), epi (102).  Fibres are helical: angle
+60 deg at t = 0 to -60 deg at t = 1, measured in the wall's tangent plane
from the circumferential direction towards the meridian; conductivity
sigma = sigma_t I + (sigma_l - sigma_t) f f^T (elec/FibreConductivity.cc:28-66
with a general fibre vector).

Pacing: `n_sites` seeded endocardial sites (tissue voxels with t below one
voxel of depth), each a small box stimulus of (2 half + 1)^3 voxels centred
on the site.  A single-voxel PointStimulus (tissue.point_stim) cannot start
propagation at these voxel sizes: the diffusive sink of its neighbours
drains it before it reaches threshold.
"""
import math

import numpy as np

from .tissue import SIGMA_L, SIGMA_T, BoxStim, Tissue, noisy_vm

OUTER = (25.0, 25.0, 45.0)      # semi-axes b (x), c (y), a (z), mm
WALL = 10.0                     # mm
CUT = 0.6                       # kept fraction of the long axis, from the apex


def grid_shape(dx, outer=OUTER, cut=CUT):
    b, c, a = outer
    return (int(math.ceil(2 * b / dx)), int(math.ceil(2 * c / dx)), int(math.ceil(2 * a * cut / dx)))


def _depth(x, y, z, inner, wall, iters=48):
    """Normalised depth t of points known to lie between the two surfaces
    (bisection on the monotone ellipsoid family)."""
    lo = np.zeros_like(x)
    hi = np.ones_like(x)
    bi, ci, ai = inner
    for _ in range(iters):
        t = 0.5 * (lo + hi)
        g = (x / (bi + t * wall)) ** 2 + (y / (ci + t * wall)) ** 2 + (z / (ai + t * wall)) ** 2
        outside = g > 1.0
        lo = np.where(outside, t, lo)
        hi = np.where(outside, hi, t)
    return 0.5 * (lo + hi)


def _fibre_sigma(x, y, z, t, inner, wall, sigma_l, sigma_t):
    bi, ci, ai = inner
    B, C, A = bi + t * wall, ci + t * wall, ai + t * wall
    n = np.stack([x / B ** 2, y / C ** 2, z / A ** 2], axis=-1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    r = np.hypot(x, y)
    ec = np.stack([-y, x, np.zeros_like(x)], axis=-1)
    on_axis = r < 1e-9
    ec[on_axis] = (1.0, 0.0, 0.0)
    ec /= np.linalg.norm(ec, axis=-1, keepdims=True)
    el = np.cross(n, ec)
    el /= np.linalg.norm(el, axis=-1, keepdims=True)
    ang = np.deg2rad(60.0 - 120.0 * t)[:, None]
    f = np.cos(ang) * ec + np.sin(ang) * el
    d = sigma_l - sigma_t
    out = np.empty(x.shape + (6,))
    out[:, 0] = sigma_t + d * f[:, 0] * f[:, 0]
    out[:, 1] = d * f[:, 0] * f[:, 1]
    out[:, 2] = d * f[:, 0] * f[:, 2]
    out[:, 3] = sigma_t + d * f[:, 1] * f[:, 1]
    out[:, 4] = d * f[:, 1] * f[:, 2]
    out[:, 5] = sigma_t + d * f[:, 2] * f[:, 2]
    return out


def prolate_shell(dx=0.25, outer=OUTER, wall=WALL, cut=CUT, seed=20240611, n_sites=20, site_half=2,
                  vstim=-52.0, duration=2.0, period=1000.0, sigma_l=SIGMA_L, sigma_t=SIGMA_T,
                  chunk_voxels=1 << 22):
    """The shell as a Tissue in gid order (gid = x + nx (y + ny z)).  Built
    slab by slab along z, so memory stays near chunk_voxels times a few
    dozen bytes beyond the tissue arrays themselves."""
    b, c, a = outer
    inner = (b - wall, c - wall, a - wall)
    nx, ny, nz = grid_shape(dx, outer, cut)
    xs = -b + (np.arange(nx) + 0.5) * dx
    ys = -c + (np.arange(ny) + 0.5) * dx
    zs = -a + (np.arange(nz) + 0.5) * dx
    gids, types, sigmas, depths = [], [], [], []
    plane = nx * ny
    zstep = max(1, chunk_voxels // plane)
    X, Y = np.meshgrid(xs, ys, indexing="xy")         # [ny, nx], x fastest
    X, Y = X.ravel(), Y.ravel()
    for z0 in range(0, nz, zstep):
        z1 = min(nz, z0 + zstep)
        zz = np.repeat(zs[z0:z1], plane)
        xx = np.tile(X, z1 - z0)
        yy = np.tile(Y, z1 - z0)
        fo = (xx / b) ** 2 + (yy / c) ** 2 + (zz / a) ** 2
        fi = (xx / inner[0]) ** 2 + (yy / inner[1]) ** 2 + (zz / inner[2]) ** 2
        keep = np.flatnonzero((fo <= 1.0) & (fi > 1.0))
        if keep.size == 0:
            continue
        x, y, z = xx[keep], yy[keep], zz[keep]
        t = _depth(x, y, z, inner, wall)
        ct = np.full(keep.size, 102, np.int32)
        ct[t < 0.65] = 101
        ct[t < 0.30] = 100
        gids.append(keep.astype(np.int64) + z0 * plane)
        types.append(ct)
        depths.append(t)
        sigmas.append(_fibre_sigma(x, y, z, t, inner, wall, sigma_l, sigma_t))
    gid = np.concatenate(gids)
    ct = np.concatenate(types)
    depth = np.concatenate(depths)
    sigma = np.concatenate(sigmas)
    # pacing sites: seeded endocardial voxels (depth below one voxel)
    endo = np.flatnonzero(depth < dx / wall)
    rng = np.random.default_rng(seed)
    sites = np.sort(rng.choice(endo, size=min(n_sites, endo.size), replace=False))
    stims = []
    h = site_half
    for s in sites:
        g = int(gid[s])
        x, y, z = g % nx, (g // nx) % ny, g // plane
        stims.append(BoxStim(xMin=x - h - 1, xMax=x + h + 1, yMin=y - h - 1, yMax=y + h + 1, zMin=z - h - 1,
                             zMax=z + h + 1, vStim=vstim, tStart=0.0, duration=duration, period=period))
    t = Tissue(nx, ny, nz, dx, dx, dx, gid, ct, sigma, noisy_vm(gid, seed), stims)
    t.depth = depth
    t.sites = gid[sites]
    return t


def shell_volume_mm3(outer=OUTER, wall=WALL, cut=CUT):
    """Exact wall volume of the truncated shell (difference of the two
    truncated ellipsoids), for checking a voxelisation's cell count."""
    def cap(b, c, a, zc):
        lo = -a
        hi = min(zc, a)
        f = lambda z: z - z ** 3 / (3 * a * a)
        return math.pi * b * c * (f(hi) - f(lo))
    b, c, a = outer
    zc = -a + 2 * a * cut
    return cap(b, c, a, zc) - cap(b - wall, c - wall, a - wall, zc)
