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
  uniform one tensor for every cell (defaults 0.1e-3 on the diagonal).
Only tissue cells (cellType > 0) are kept.
"""
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


def read_anatomy(name, dx=0.2, dy=0.2, dz=0.2, conductivity="pio", sigma_l=0.3e-3, sigma_t=0.0315e-3,
                 sigma_uniform=(0.1e-3, 0.0, 0.0, 0.1e-3, 0.0, 0.1e-3), diffusion_scale=DIFFUSION_SCALE,
                 stimuli=(), vm0=None, seed=20240611):
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
    else:
        raise ValueError("unknown conductivity method " + conductivity)
    vm = noisy_vm(gid, seed) if vm0 is None else np.full(len(idx), float(vm0))
    return Tissue(nx, ny, nz, dx, dy, dz, gid.astype(np.int64), ct[idx], sigma, vm, list(stimuli), diffusion_scale)
