"""Synthetic tissues for the monodomain engine: boxes, sheets and cables
with transmural cell-type slabs, rotating fibres and box stimuli.

Conventions (shared by the engine and the oracle, so both see identical
inputs):
  - cells are stored in gid order, gid = x + nx*(y + ny*z) (the reference's
    IndexToTuple, elec/IndexToTuple.hh);
  - anatomy cellType 100/101/102 = endo/mid/epi, mapped to BetterTT06
    celltype 0/1/2 by one REACTION object each (as in the reference's
    multipleReaction test);
  - conductivity sigma = sigma_t I + (sigma_l - sigma_t) f f^T with the fibre
    f = (cos a, sin a, 0) in the xy-plane (the reference's fibre tensor,
    elec/FibreConductivity.cc:28-66, with its polar angle fixed at 90 deg);
    the angle a rotates linearly across z;
  - initial Vm = -83 mV + U(-0.1, 0.1) from a counter-based generator
    (splitmix64 of seed ^ gid), so any device reproduces it bit for bit.
"""
from dataclasses import dataclass, field
from typing import List

import numpy as np

SIGMA_L = 1.33e-4       # S/mm  (0.133 S/m)
SIGMA_T = 1.76e-5       # S/mm  (0.0176 S/m)
BETA = 140.0            # 1/mm  (1400 /cm)
CM = 1.0e-5             # mF/mm^2 (1 uF/cm^2)
DIFFUSION_SCALE = 1.0 / (BETA * CM)   # mm^3/mF, 714.2857...


@dataclass
class BoxStim:
    """A BoxStimulus with a PeriodicPulse (elec/BoxStimulus.cc:11-70,
    elec/PeriodicPulse.cc:22-28, elec/stimulusFactory.cc:27-118):
    on while t0 < time < tf and phase <= time mod period < phase + duration;
    cells strictly inside the box on the global tuple get iStim = -vStim."""
    xMin: float = -1
    xMax: float = 1e9
    yMin: float = -1
    yMax: float = 1e9
    zMin: float = -1
    zMax: float = 1e9
    vStim: float = -52.0
    tStart: float = 0.0
    duration: float = 1.0
    period: float = 1000.0
    t0: float = -1000.0
    tf: float = 1e30
    mode: int = 0           # 0: box (assigns), 1: point (adds; see point_stim)
    cell: int = -1          # point stimuli: the target gid

    @property
    def amplitude(self):
        return -self.vStim

    def value(self, time):
        if not (time > self.t0 and time < self.tf):
            return 0.0
        t = time - np.floor(time / self.period) * self.period
        if t >= self.tStart and t < self.tStart + self.duration:
            return self.amplitude
        return 0.0

    def as_array(self):
        return np.array([self.t0, self.tf, self.period, self.duration, self.amplitude, self.tStart,
                         self.xMin, self.xMax, self.yMin, self.yMax, self.zMin, self.zMax], dtype=np.float64)


def point_stim(gid, nx, ny, **pulse):
    """A PointStimulus (elec/PointStimulus.cc:6-36) at cell gid: adds the
    pulse to that cell's iStim.  Expressed as the strict box around the
    cell's tuple, which holds that cell alone."""
    x, y, z = gid % nx, (gid // nx) % ny, gid // (nx * ny)
    return BoxStim(xMin=x - 1, xMax=x + 1, yMin=y - 1, yMax=y + 1, zMin=z - 1, zMax=z + 1, mode=1, cell=int(gid),
                   **pulse)


@dataclass
class Tissue:
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    gid: np.ndarray            # int64 [n]
    cell_type: np.ndarray      # int32 [n], anatomy cellType (>0 is tissue)
    sigma: np.ndarray          # float64 [n, 6]: a11 a12 a13 a22 a23 a33
    vm0: np.ndarray            # float64 [n]
    stimuli: List[BoxStim] = field(default_factory=list)
    diffusion_scale: float = DIFFUSION_SCALE

    @property
    def n(self):
        return int(self.gid.shape[0])

    def tuples(self):
        x = self.gid % self.nx
        y = (self.gid // self.nx) % self.ny
        z = self.gid // (self.nx * self.ny)
        return x, y, z


def splitmix64(x):
    """splitmix64 finaliser on uint64 arrays."""
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    return x


def noisy_vm(gid, seed, v0=-83.0, amp=0.1):
    """Vm = v0 + U(-amp, amp), U from the top 53 bits of splitmix64(seed ^ gid)."""
    r = splitmix64(np.uint64(seed) ^ np.asarray(gid, dtype=np.uint64))
    u = (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return v0 + (2.0 * u - 1.0) * amp


def fibre_sigma(angle, sigma_l=SIGMA_L, sigma_t=SIGMA_T):
    """sigma = sigma_t I + (sigma_l - sigma_t) f f^T, f = (cos a, sin a, 0)."""
    c, s = np.cos(angle), np.sin(angle)
    d = sigma_l - sigma_t
    out = np.zeros(np.shape(angle) + (6,))
    out[..., 0] = sigma_t + d * c * c
    out[..., 1] = d * c * s
    out[..., 3] = sigma_t + d * s * s
    out[..., 5] = sigma_t
    return out


def transmural_types(x, nx, endo_frac=0.25, mid_frac=0.35):
    """Slabs along x: endo for x < round(endo_frac*nx), mid below
    round((endo_frac+mid_frac)*nx), epi after (anatomy cellType 100/101/102).
    Python's round() is round-half-even; 64 -> 16 / 38."""
    e = int(round(endo_frac * nx))
    m = int(round((endo_frac + mid_frac) * nx))
    t = np.full(np.shape(x), 102, dtype=np.int32)
    t[x < m] = 101
    t[x < e] = 100
    return t


def box(nx, ny, nz, dx=0.2, seed=20240611, period=1000.0, duration=1.0, vstim=-52.0,
        angle_min_deg=-60.0, angle_max_deg=60.0, stim_face=True, zrange=None):
    """A dense box of tissue, the workload of the reference's Niederer-style
    runs restated on our conventions (cell types by x-slab, fibre angle
    rotating linearly across z, a pacing stimulus on the x = 0 face).

    zrange = (z0, z1) keeps only the cells with z0 <= z < z1 (one rank's
    slab of the box, as a z-decomposition over processes gives it): the same
    gids, fibres, types, initial Vm and stimulus as in the whole box; the
    slab's faces at z0 and z1 - 1 have no neighbours (no-flux)."""
    z0, z1 = zrange if zrange is not None else (0, nz)
    if not (0 <= z0 < z1 <= nz):
        raise ValueError("zrange outside the box")
    gid = np.arange(z0 * nx * ny, z1 * nx * ny, dtype=np.int64)
    n = gid.shape[0]
    x = gid % nx
    z = gid // (nx * ny)
    ct = transmural_types(x, nx)
    frac = z / (nz - 1) if nz > 1 else np.zeros(n)
    ang = np.deg2rad(angle_min_deg + (angle_max_deg - angle_min_deg) * frac)
    sigma = fibre_sigma(ang)
    stims = []
    if stim_face:
        stims.append(BoxStim(xMin=-1, xMax=1, yMin=-1, yMax=ny, zMin=-1, zMax=nz, vStim=vstim,
                             tStart=0.0, duration=duration, period=period))
    return Tissue(nx, ny, nz, dx, dx, dx, gid, ct, sigma, noisy_vm(gid, seed), stims)


def reaction_objects_text(fit_names=None):
    """REACTION objects for the three transmural types (anatomy cellType
    100/101/102 -> BetterTT06 celltype 0/1/2), optionally naming FIT objects."""
    out = []
    for ct, (name, celltype) in zip((100, 101, 102), (("tt06Endo", 0), ("tt06Mid", 1), ("tt06Epi", 2))):
        fit = "" if not fit_names else " fit = %s;" % fit_names[celltype]
        out.append("%s REACTION { method = BetterTT06; cellTypes = %d; celltype = %d;%s }" % (name, ct, celltype, fit))
    return "\n".join(out) + "\n"


def stimulus_objects_text(stims, prefix="stim"):
    """STIMULUS objects (method = box or point) for the reference's
    stimulusFactory."""
    out = []
    for i, s in enumerate(stims):
        if s.mode == 1:
            out.append("%s%d STIMULUS { method = point; cell = %d; vStim = %r; tStart = %r; duration = %r; "
                       "period = %r; t0 = %r; tf = %r; }" % (prefix, i, s.cell, s.vStim, s.tStart, s.duration,
                                                             s.period, s.t0, s.tf))
            continue
        out.append("%s%d STIMULUS { method = box; xMin = %r; xMax = %r; yMin = %r; yMax = %r; zMin = %r; zMax = %r; "
                   "vStim = %r; tStart = %r; duration = %r; period = %r; t0 = %r; tf = %r; }" % (
                       prefix, i, s.xMin, s.xMax, s.yMin, s.yMax, s.zMin, s.zMax, s.vStim, s.tStart,
                       s.duration, s.period, s.t0, s.tf))
    return "\n".join(out) + "\n"
