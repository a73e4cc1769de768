"""Generates tests/golden/ref_fits/: the fits the reference's own generator
makes for BetterTT06 at the shipped time step, by running the reference
code built here (oracle/_ref, with the Householder DGELS of
oracle/ref/ref_dgels.c in place of LAPACK).

A REACTION object without a reusable FIT makes the reference's factory
(reactionFactoryForBetterTT06, elec/BetterTT06.cc:69-200) call
createInterpolants (elec/BetterTT06.cc:206-1002) -> Interpolation::create
(elec/Interpolation.cc:115-423) and write `<name>.fit.data` into the working
directory; each celltype runs in its own process and scratch directory (the
reference's object database is global).

    python tests/golden/make_ref_fits.py [dt]          (default 0.02)
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "ref_fits")


def generate(dt, celltype, workdir):
    """Runs the reference's fit generator for one celltype in `workdir`;
    returns the path of the FIT file it wrote."""
    name = "refGen%d" % celltype
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "from oracle import refsim\n"
        "refsim.compile_objects('%s REACTION { method = BetterTT06; cellTypes = 100; celltype = %d; }\\n')\n"
        "refsim.RefSim(['%s'], [], (1, 1, 1), (0.2, 0.2, 0.2), np.array([0]), np.array([100], np.int32),\n"
        "              np.array([[1e-4, 0, 0, 1e-4, 0, 1e-4]]), %r, 714.0, diffusion=False).close()\n"
        % (ROOT, name, celltype, name, dt))
    subprocess.run([sys.executable, "-c", code], cwd=workdir, check=True, stdout=subprocess.DEVNULL)
    return os.path.join(workdir, name + ".fit.data")


def main(dt=0.02):
    os.makedirs(OUT, exist_ok=True)
    procs = []
    for ct in (0, 1, 2):
        d = tempfile.mkdtemp()
        name = "refGen%d" % ct
        code = [sys.executable, os.path.abspath(__file__), "--one", repr(dt), str(ct), d]
        procs.append((ct, d, name, subprocess.Popen(code)))
    for ct, d, name, p in procs:
        if p.wait() != 0:
            raise RuntimeError("celltype %d failed" % ct)
        dst = os.path.join(OUT, "ref_dt%g_celltype%d.fit.data" % (dt, ct))
        shutil.copy(os.path.join(d, name + ".fit.data"), dst)
        shutil.rmtree(d, ignore_errors=True)
        print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--one":
        generate(float(sys.argv[2]), int(sys.argv[3]), sys.argv[4])
    else:
        main(float(sys.argv[1]) if len(sys.argv) > 1 else 0.02)
