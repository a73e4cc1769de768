"""Anatomies from the reference's pio anatomy files (snapshot.initial/
anatomy#): gid, cellType and either the conductivity tensor (sigma11 ..
sigma33) or fibre angles (theta, phi), as initializeAnatomy and
setConductivity read them (elec/initializeAnatomy.cc:42-140,
elec/setConductivity.cc:50-205).

Conductivity methods:
  pio    sigma11 sigma12 sigma13 sigma22 sigma23 sigma33 from the file,
         converted from their units to S/mm (the reference's internal
         conductivity unit);
  fibre  sigma = IBT tensor of the fibre angles (FibreConductivity,
         elec/FibreConductivity.cc:25-66) with sigmaLi / sigmaTi (S/mm,
         defaults 0.3e-3 and 0.0315e-3); integer angles are in units of
         pi/256, float angles in radians;
  uniform one tensor for every cell (defaults 0.1e-3 on the diagonal);
  JHU    the rule-based wedge tensor of JHUConductivity (jhu_sigma).
Only tissue cells (cellType > 0) are kept.
"""
import math

import numpy as np

from . import pio
from .tissue import DIFFUSION_SCALE, Tissue, noisy_vm

# conductivity units -> S/mm
_SIGMA_UNITS = {"S/mm": 1.0, "mS/mm": 1e-3, "S/m": 1e-3, "mS/m": 1e-6, "S/cm": 1e-1, "mS/cm": 1e-4}


def ibt_sigma(theta, phi, sigma_l, sigma_t):
    """calcConductivityMatrixIBT (elec/FibreConductivity.cc:25-66): the
    fibre direction (cos phi sin theta, sin phi sin theta, cos theta)."""
    sp, cp, st, ct = np.sin(phi), np.cos(phi), np.sin(theta), np.cos(theta)
    sp2, cp2, st2, ct2 = sp * sp, cp * cp, st * st, ct * ct
    out = np.empty(np.shape(theta) + (6,))
    out[..., 0] = sigma_l * cp2 * st2 + sigma_t * (cp2 * ct2 + sp2)
    out[..., 3] = sigma_l * sp2 * st2 + sigma_t * (cp2 + sp2 * ct2)
    out[..., 5] = sigma_l * ct2 + sigma_t * st2
    out[..., 1] = (sigma_l - sigma_t) * cp * st2 * sp
    out[..., 2] = (sigma_l - sigma_t) * ct * cp * st
    out[..., 4] = (sigma_l - sigma_t) * sp * ct * st
    return out


def jhu_sigma(gid, nx, ny, nz, sigma_l=0.3e-3, sigma_t=0.0315e-3, sheet_angle=45.0, rotation_matrix=1,
              homogeneous_fiber=False):
    """JHUConductivity::compute (elec/JHUConductivity.cc:26-120) for cells
    of an nx x ny x nz grid: sigma = R diag(G_L, G_T, G_N) R^T with G_L =
    sigma_l, G_T = G_N = sigma_t and R = [E1 E2 E3] built from the fibre
    angle (fixed -60 deg when homogeneous, else twisting linearly from
    +60 deg by 120 / (ny - 2) deg per cell along y: 60 - twist (y + 1)),
    the sheet angle and an imbrication angle of 0, in one of the
    reference's two rotation conventions; entries below 1e-12 G_T become
    0.  Arguments as setConductivity's JHU object keys (sigmaLi, sigmaTi,
    sheetAngle, rotatationMatrix, homogeneousFiber;
    elec/setConductivity.cc:207-226).  R must be a rotation: convention 0
    is a reflection, on which the reference's assert aborts and this
    raises ValueError.

    The reference's own setConductivity passes the cell array to its JHU
    branch by value (elec/setConductivity.cc:207-209), so there the tensors
    are computed and then dropped; this reader applies them.  Angles go
    through the C library's sin and cos (math), as the reference's do."""
    gid = np.asarray(gid, dtype=np.int64)
    y = (gid // nx) % ny
    twist = (60.0 - (-60.0)) / (ny - 2)
    if rotation_matrix not in (0, 1):
        raise ValueError("rotatationMatrix must be 0 or 1")
    sh = sheet_angle * math.pi / 180.0
    cs, ss = math.cos(sh), math.sin(sh)
    gl, gt, gn = sigma_l, sigma_t, sigma_t
    out = np.empty((len(gid), 6))
    table = {}
    for yy in np.unique(y):
        fib = -60.0 if homogeneous_fiber else 60.0 - twist * (int(yy) + 1)
        fa = fib * math.pi / 180.0
        cf, sf = math.cos(fa), math.sin(fa)
        if rotation_matrix == 0:
            e1, e2, e3 = (cf, 0.0, sf), (-sf * ss, cs, cf * ss), (sf * cs, ss, -cf * cs)
        else:
            e1, e2, e3 = (cf, 0.0, -sf), (sf * ss, cs, cf * ss), (sf * cs, -ss, cf * cs)
        # the reference asserts that R is a rotation (elec/JHUConductivity.cc:80-83);
        # its convention 0 is a reflection (determinant -1), so that path aborts there
        det = (e1[0] * e2[1] * e3[2] + e2[0] * e3[1] * e1[2] + e3[0] * e1[1] * e2[2] -
               e1[0] * e2[2] * e3[1] - e2[0] * e1[1] * e3[2] - e3[0] * e2[1] * e1[2])
        if not abs(det - 1) < 1e-10:
            raise ValueError("JHU conductivity: the rotation matrix of convention %d has determinant %g, not 1"
                             % (rotation_matrix, det))
        d = [[0.0] * 3 for _ in range(3)]
        # the reference's operand order: squares by pow, off-diagonal terms
        # G E[i] E[j] with the lower index first
        for i in range(3):
            d[i][i] = gl * e1[i] ** 2 + gt * e2[i] ** 2 + gn * e3[i] ** 2
            for j in range(i + 1, 3):
                d[i][j] = d[j][i] = gl * e1[i] * e1[j] + gt * e2[i] * e2[j] + gn * e3[i] * e3[j]
        for i in range(3):
            for j in range(3):
                if abs(d[i][j]) < 1e-12 * gt:
                    d[i][j] = 0.0
        # a12 = D[1][0], a13 = D[2][0], a23 = D[1][2]
        table[int(yy)] = (d[0][0], d[1][0], d[2][0], d[1][1], d[1][2], d[2][2])
    for yy, row in table.items():
        out[y == yy] = row
    return out


def read_anatomy(name, dx=0.2, dy=0.2, dz=0.2, conductivity="pio", sigma_l=0.3e-3, sigma_t=0.0315e-3,
                 sigma_uniform=(0.1e-3, 0.0, 0.0, 0.1e-3, 0.0, 0.1e-3), diffusion_scale=DIFFUSION_SCALE,
                 stimuli=(), vm0=None, seed=20240611, jhu=None):
    """A Tissue (cells in gid order) from a pio anatomy file."""
    f = pio.read(name)
    h = f.header
    nx, ny, nz = int(h["nx"]), int(h["ny"]), int(h["nz"])
    gid = f.fields["gid"]
    ct = f.fields["cellType"].astype(np.int32)
    keep = ct > 0
    order = np.argsort(gid[keep], kind="stable")
    idx = np.flatnonzero(keep)[order]
    gid = gid[idx]
    if np.any(gid < 0) or np.any(gid >= nx * ny * nz) or np.any(np.diff(gid) <= 0):
        raise ValueError("gids must be distinct and inside the %dx%dx%d grid" % (nx, ny, nz))
    if conductivity == "pio":
        names = ["sigma11", "sigma12", "sigma13", "sigma22", "sigma23", "sigma33"]
        sigma = np.stack([f.fields[k][idx] * _SIGMA_UNITS[f.units.get(k, "S/mm")] for k in names], axis=1)
    elif conductivity in ("fibre", "fiber"):
        if "theta" in f.fields:
            th, ph = f.fields["theta"][idx], f.fields["phi"][idx]
            if h["field_types"].split()[f.names.index("theta")] in ("u", "i", "u4", "i4", "u8", "i8"):
                th, ph = th * (np.pi / 256), ph * (np.pi / 256)
        else:
            th = ph = np.zeros(len(idx))
        sigma = ibt_sigma(th.astype(np.float64), ph.astype(np.float64), sigma_l, sigma_t)
    elif conductivity == "uniform":
        sigma = np.tile(np.asarray(sigma_uniform, dtype=np.float64), (len(idx), 1))
    elif conductivity == "JHU":
        sigma = jhu_sigma(gid, nx, ny, nz, sigma_l, sigma_t, **(jhu or {}))
    else:
        raise ValueError("unknown conductivity method " + conductivity)
    vm = noisy_vm(gid, seed) if vm0 is None else np.full(len(idx), float(vm0))
    return Tissue(nx, ny, nz, dx, dy, dz, gid.astype(np.int64), ct[idx], sigma, vm, list(stimuli), diffusion_scale)
