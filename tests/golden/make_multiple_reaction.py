"""Builds tests/golden/multiple_reaction.npz from the reference's
multipleReaction test (test/tests/multipleReaction: the pio anatomy, the
three BetterTT06 REACTION objects with their dt 0.01 fit files and
SINGLECELL initial states, the box stimulus) and its expected output
(test/results/osx/seq/multipleReaction/traces: Vm of cells 487, 500 and
513 every 200 steps for 30 000 steps).

The inputs go through this package's own readers (pio anatomy, object
database, fit reuse rule, initial-state rule), so the fixture is the
reference's data as the engine sees it.  Run from the repository root:
    python tests/golden/make_multiple_reaction.py [reference checkout]
(default: CARDIOID_REF, else the checkout the oracle build recorded).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from cardioid_b200 import anatomy, objectdb, tt06  # noqa: E402


def main(ref):
    case = os.path.join(ref, "test", "tests", "multipleReaction")
    db = objectdb.ObjectDB()
    for f in ("object.data", "tt06Endo.fit.data", "tt06Mid.fit.data", "tt06Epi.fit.data", "tt06Endo.sv",
              "tt06Mid.sv", "tt06Epi.sv"):
        db.compile_file(os.path.join(case, f))
    sim = db.find("simulate", "SIMULATE")
    dt = objectdb.get_float(sim, "dt")
    rnames = objectdb.get_list(sim, "reaction")
    t = anatomy.read_anatomy(os.path.join(case, "snapshot.initial", "anatomy#"))
    params, cell_types, states, vm0 = [], [], [], []
    for rn in rnames:
        p = tt06.params_from_object(db, rn, dt)
        params.append(p)
        cell_types.append(int(objectdb.get_float(db.find(rn, "REACTION"), "cellTypes")))
        v, st = tt06.initial_state_from_object(db, rn)
        vm0.append(v)
        states.append([st[k] for k in tt06.STATE_NAMES])
    stim = db.find(objectdb.get_str(sim, "stimulus"), "STIMULUS")
    g = lambda k, d: objectdb.get_float(stim, k, d)
    traces = np.loadtxt(os.path.join(ref, "test", "results", "osx", "seq", "multipleReaction", "traces"))
    sensor = np.loadtxt(os.path.join(case, "sensor.txt"), dtype=np.int64)
    fits = np.zeros((len(params), 30, 66))
    for r, p in enumerate(params):
        for k, f in enumerate(p.fits):
            fits[r, k, 0], fits[r, k, 1] = f.numer, f.denom
            fits[r, k, 2:2 + len(f.coeff)] = f.coeff
    np.savez_compressed(
        os.path.join(HERE, "multiple_reaction.npz"),
        nx=t.nx, ny=t.ny, nz=t.nz, dx=t.dx, gid=t.gid, cell_type=t.cell_type, sigma=t.sigma,
        dt=dt, steps=int(objectdb.get_float(sim, "maxLoop")),
        diffusion_scale=objectdb.get_float(db.find(objectdb.get_str(sim, "diffusion"), "DIFFUSION"), "diffusionScale"),
        reaction_cell_types=np.array(cell_types), params=np.array([p.as_array() for p in params]), fits=fits,
        states=np.array(states), vm0=np.array(vm0),
        stim=np.array([g("xMin", -1), g("xMax", t.nx), g("yMin", -1), g("yMax", t.ny), g("zMin", -1), g("zMax", t.nz),
                       g("vStim", -52), g("tStart", 0), g("duration", 1), g("period", 1000), g("t0", -1000),
                       g("tf", 1e30)]),
        sensor=sensor, traces=traces)


if __name__ == "__main__":
    sys.path.insert(0, os.path.join(HERE, ".."))
    from conftest import reference_root
    main(sys.argv[1] if len(sys.argv) > 1 else reference_root())
