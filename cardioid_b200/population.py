"""Populations of independent tissue instances: the many-small-tissues
workload (virtual cohorts, parameter sweeps) that one engine steps together,
one launch per time step and reaction type.

An instance is a cable (nx x 1 x 1), a sheet (side x side x 1) or a box
(side^3) of one BetterTT06 cell type, with its own g_Kr / g_CaL / g_Na
scales (multiplying the BetterTT06 defaults 0.153, 3.98e-5, 14.838) and
its own pacing cycle length: a 1 ms, 52 mV/ms S1 pulse every CL ms on the
three layers x = 0, 1, 2 (elec/BoxStimulus.cc, elec/PeriodicPulse.cc; one
layer does not excite a cable or sheet whose fibres run along x, since the
longitudinal conductivity drains it).  Sizes are
log-uniform in their ranges; every draw comes from one seeded generator, so
a population is reproducible from its seed.
"""
import math
from dataclasses import dataclass

import numpy as np

from .tissue import BoxStim, Tissue, fibre_sigma, noisy_vm

KINDS = ("cable", "sheet", "box")


@dataclass
class Instance:
    index: int
    kind: str
    dims: tuple            # (nx, ny, nz)
    celltype: int          # BetterTT06 celltype 0/1/2 (anatomy cellType 100 + celltype)
    scales: tuple          # (g_Kr, g_CaL, g_Na) multipliers
    cl: float              # pacing cycle length, ms

    @property
    def cells(self):
        return self.dims[0] * self.dims[1] * self.dims[2]


@dataclass
class PopulationSpec:
    """Defaults: 4096 instances, 50 % cables L in [100, 5000], 40 % sheets
    side in [64, 512], 10 % boxes side in [32, 96], scales U[0, 1],
    CL U[400, 2000] ms."""
    n: int = 4096
    fractions: tuple = (0.5, 0.4, 0.1)
    cable: tuple = (100, 5000)
    sheet: tuple = (64, 512)
    box: tuple = (32, 96)
    scale: tuple = (0.0, 1.0)
    cl: tuple = (400.0, 2000.0)


def _log_uniform_int(rng, lo, hi):
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))


def draw(spec=None, seed=20240611):
    """The instances of a population, in index order."""
    spec = spec or PopulationSpec()
    rng = np.random.default_rng(seed)
    counts = [int(round(f * spec.n)) for f in spec.fractions]
    counts[0] += spec.n - sum(counts)
    kinds = np.repeat(np.arange(3), counts)
    rng.shuffle(kinds)
    out = []
    for i, k in enumerate(kinds):
        kind = KINDS[k]
        if kind == "cable":
            dims = (_log_uniform_int(rng, *spec.cable), 1, 1)
        elif kind == "sheet":
            s = _log_uniform_int(rng, *spec.sheet)
            dims = (s, s, 1)
        else:
            s = _log_uniform_int(rng, *spec.box)
            dims = (s, s, s)
        celltype = int(rng.integers(0, 3))
        scales = tuple(float(v) for v in rng.uniform(spec.scale[0], spec.scale[1], size=3))
        cl = float(rng.uniform(*spec.cl))
        out.append(Instance(i, kind, dims, celltype, scales, cl))
    return out


def build(inst, dx=0.2, seed=20240611):
    """The Tissue of one instance: fibres along x for cables and sheets,
    rotating -60..+60 deg across z for boxes; Vm0 = -83 + U(-0.1, 0.1)."""
    nx, ny, nz = inst.dims
    n = nx * ny * nz
    gid = np.arange(n, dtype=np.int64)
    if nz > 1:
        z = gid // (nx * ny)
        ang = np.deg2rad(-60.0 + 120.0 * z / (nz - 1))
    else:
        ang = np.zeros(n)
    ct = np.full(n, 100 + inst.celltype, np.int32)
    stim = BoxStim(xMin=-1, xMax=3, yMin=-1, yMax=ny, zMin=-1, zMax=nz, vStim=-52.0, tStart=0.0, duration=1.0,
                   period=inst.cl)
    return Tissue(nx, ny, nz, dx, dx, dx, gid, ct, fibre_sigma(ang), noisy_vm(gid, seed ^ inst.index), [stim])


def total_cells(instances):
    return sum(i.cells for i in instances)
