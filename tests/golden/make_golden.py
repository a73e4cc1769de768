"""Generates the committed golden fixtures by running the reference's own CPU
code (oracle/_ref, compiled from the Cardioid sources by oracle/ref/Makefile).

    python tests/golden/make_golden.py

ref_box_dt002.npz: a 10x8x6 box with the three transmural BetterTT06 types,
fibre-rotated FGR diffusion and a box stimulus on the x = 0 face, dt = 0.02
with the shipped fit files, run through ReactionManager + FGRDiffusionOMP +
BoxStimulus + the omp-loop integrator; Vm after 25/50/100 steps, every state
and the activation times after 100 steps, and the last step's dVm terms.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cardioid_b200 import engine, tissue  # noqa: E402
from oracle import refsim  # noqa: E402

DT = 0.02
BOX = (10, 8, 6)


def box_case():
    return tissue.box(*BOX, dx=0.2, seed=7)


def reference_sim(t, dt=DT):
    """A RefSim of tissue t with the three transmural BetterTT06 types on the
    shipped fits (compiled into the reference's object database once) and
    t's stimuli (under fresh names)."""
    text = ""
    for ct in (0, 1, 2):
        with open(engine.shipped_fit_path(dt, ct)) as f:
            text += f.read()
    text += tissue.reaction_objects_text(["tt06Endo_fit", "tt06Mid_fit", "tt06Epi_fit"])
    refsim.compile_once("tt06-transmural-dt%g" % dt, text)
    prefix = refsim.unique_prefix()
    refsim.compile_objects(tissue.stimulus_objects_text(t.stimuli, prefix=prefix))
    return refsim.RefSim(["tt06Endo", "tt06Mid", "tt06Epi"], ["%s%d" % (prefix, i) for i in range(len(t.stimuli))],
                         (t.nx, t.ny, t.nz), (t.dx, t.dy, t.dz), t.gid, t.cell_type, t.sigma, dt,
                         t.diffusion_scale)


def run_reference(t, steps=(25, 50, 100)):
    sim = reference_sim(t)
    sim.set_vm(t.vm0)
    out = {}
    done = 0
    for s in steps:
        sim.step(s - done)
        done = s
        out["vm_%d" % s] = sim.vm()
    names = sim.field_names()
    out["field_names"] = np.array(names)
    out["states"] = np.stack([sim.state(n) for n in names])
    out["activation"] = sim.activation()
    r, d, i = sim.dvm()
    out["dvmR"], out["dvmD"], out["iStim"] = r, d, i
    out["time"] = np.array(sim.time)
    return out


def main():
    t = box_case()
    out = run_reference(t)
    path = os.path.join(HERE, "ref_box_dt002.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main()
