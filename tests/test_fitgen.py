"""Pins of the BetterTT06 fit generator (cardioid_b200.fitgen) and of the
shipped dt = 0.02 fit files against the reference's own generator.

The reference fits its 30 lookup functions at start-up
(ThisReaction::createInterpolants, elec/BetterTT06.cc:206-1002, through
Interpolation::create, elec/Interpolation.cc:115-423, which calls LAPACK's
DGELS).  The oracle build runs that code with our own Householder DGELS
(oracle/ref/ref_dgels.c); tests/golden/make_ref_fits.py saved its output for
dt = 0.02 as tests/golden/ref_fits/.  Checked here:
  - with our DGELS the reference generator reproduces the fit files the
    reference ships, made with LAPACK (dt = 0.01, test/tests/multipleReaction);
  - fitgen.sample computes the reference's functions: every fit the
    reference generator made meets its tolerance on fitgen's samples;
  - fitgen picks the reference generator's shapes (numerator and
    denominator term counts) and its fits agree with the reference's;
  - the shipped fit files have the reference generator's shapes and agree
    with its fits, and the reference's factory reuses them (its reuse rule,
    elec/BetterTT06.cc:124-149) instead of refitting.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from cardioid_b200 import engine, fitgen, objectdb, tt06
from cardioid_b200.data import make_fit_shapes as mfs
from conftest import REFERENCE, ROOT

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF_FITS = os.path.join(GOLDEN, "ref_fits")
# The reference's LAPACK-made fit files (dt = 0.01, default g_K1), by celltype.
LAPACK_FITS = {0: ("multipleReaction", "tt06Endo.fit.data"), 1: ("multipleReaction", "tt06Mid.fit.data"),
               2: ("Niederer", "tt06.fit.data")}


def _ref_built():
    from oracle import refsim
    return refsim.available()


def fits_of(path):
    db = objectdb.ObjectDB().compile_file(path)
    fobj = db.find(db.names("FIT")[0], "FIT")
    return tt06.fits_from_fit_object(db, db.names("FIT")[0]), objectdb.get_float(fobj, "celltype"), \
        objectdb.get_float(fobj, "dt"), objectdb.get_float(fobj, "g_K1")


def eval_diff(a, b, slot):
    """Largest difference of two fits of one function over its domain,
    relative to the function's largest magnitude."""
    x = mfs.domain(slot)
    va = a.eval(x)
    return float(np.abs(va - b.eval(x)).max() / np.abs(va).max())


def windowed_error(fit, x, y, window):
    """Interpolation::create's error measure: RMS of the error divided by the
    moving-window range of the sampled function (elec/Interpolation.cc:160-270)."""
    rng = fitgen._moving_range(y, window)
    return float(np.sqrt(np.mean(((y - fit.eval(x)) / rng) ** 2)))


def lapack_fit_path(celltype):
    case, name = LAPACK_FITS[celltype]
    return os.path.join(REFERENCE, "test", "tests", case, name)


def reference_fit_sets():
    """(label, fits, params) of every reference-generated fit set present:
    the committed dt = 0.02 fixture and the reference's own dt = 0.01 files."""
    out = []
    for ct in (0, 1, 2):
        fits, fct, fdt, gk1 = fits_of(os.path.join(REF_FITS, "ref_dt0.02_celltype%d.fit.data" % ct))
        p = tt06.TT06Params.defaults(fct)
        p.g_K1 = gk1
        out.append(("generator dt %g celltype %d" % (fdt, ct), fits, p, fdt))
        if REFERENCE and os.path.exists(lapack_fit_path(ct)):
            fits, fct, fdt, gk1 = fits_of(lapack_fit_path(ct))
            p = tt06.TT06Params.defaults(fct)
            p.g_K1 = gk1
            out.append(("LAPACK file dt %g celltype %d" % (fdt, fct), fits, p, fdt))
    return out


def test_samples_are_the_reference_functions():
    """Each of the reference generator's fits (and the reference's shipped
    LAPACK fits) meets its fitting tolerance against fitgen.sample: the 30
    sampled functions, grids and windows are the reference's."""
    for label, fits, p, dt in reference_fit_sets():
        for i, f in enumerate(fits):
            x, y, tol, window = fitgen.sample(i, dt, p)
            err = windowed_error(f, x, y, window)
            assert err <= tol, (label, i, err, tol)


@pytest.mark.parametrize("celltype", [0, 1, 2])
def test_shipped_fits_have_the_reference_generators_shapes(celltype):
    ref, _, _, _ = fits_of(os.path.join(REF_FITS, "ref_dt0.02_celltype%d.fit.data" % celltype))
    p = engine.default_params(celltype, 0.02)
    for i, (a, b) in enumerate(zip(ref, p.fits)):
        assert (a.numer, a.denom) == (b.numer, b.denom), i
        assert eval_diff(a, b, i) <= 1e-4, (i, eval_diff(a, b, i))


def test_fitgen_picks_the_reference_generators_shapes():
    """fitgen's cost search (Householder QR least squares, as DGELS) stops
    at the reference generator's shapes, including h_RLA (slot 13), whose
    error sits near the tolerance at the deciding cost."""
    ref, _, _, _ = fits_of(os.path.join(REF_FITS, "ref_dt0.02_celltype1.fit.data"))
    p = tt06.TT06Params.defaults(1)
    for i in (0, 2, 13, 21, 28, 29):
        x, y, tol, window = fitgen.sample(i, 0.02, p)
        f, err = fitgen.fit_samples(x, y, tol, window)
        assert err < tol
        assert (f.numer, f.denom) == (ref[i].numer, ref[i].denom), i
        assert eval_diff(ref[i], f, i) <= 1e-4, (i, eval_diff(ref[i], f, i))


@pytest.mark.skipif(not (_ref_built() and REFERENCE and os.path.exists(lapack_fit_path(0))),
                    reason="needs the reference build and checkout")
def test_our_dgels_reproduces_the_lapack_fits():
    """The reference generator linked with oracle/ref/ref_dgels.c writes the
    fits the reference ships for dt = 0.01, celltype 0 (made with LAPACK):
    the same 30 shapes and functions within 5e-5 of their range (the
    least-squares solutions differ in rounding only)."""
    sys.path.insert(0, GOLDEN)
    import make_ref_fits
    with tempfile.TemporaryDirectory() as d:
        ours, _, _, _ = fits_of(make_ref_fits.generate(0.01, 0, d))
    lapack, _, _, _ = fits_of(lapack_fit_path(0))
    for i, (a, b) in enumerate(zip(lapack, ours)):
        assert (a.numer, a.denom) == (b.numer, b.denom), i
        assert eval_diff(a, b, i) <= 5e-5, (i, eval_diff(a, b, i))


@pytest.mark.skipif(not _ref_built(), reason="needs the reference build")
def test_reference_factory_reuses_the_shipped_fits():
    """The reference's factory, given the shipped FIT objects for the three
    celltypes at dt = 0.02, reuses them: it writes no refitted
    `<name>.fit.data` (which it does whenever it regenerates)."""
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r); sys.path.insert(0, %r)\n"
        "from oracle import refsim\n"
        "from cardioid_b200 import engine, tissue\n"
        "text = ''.join(open(engine.shipped_fit_path(0.02, c)).read() for c in (0, 1, 2))\n"
        "text += tissue.reaction_objects_text(['tt06Endo_fit', 'tt06Mid_fit', 'tt06Epi_fit'])\n"
        "refsim.compile_objects(text)\n"
        "refsim.RefSim(['tt06Endo', 'tt06Mid', 'tt06Epi'], [], (3, 1, 1), (0.2, 0.2, 0.2), np.arange(3),\n"
        "              np.array([100, 101, 102], np.int32), np.tile([1e-4, 0, 0, 1e-4, 0, 1e-4], (3, 1)),\n"
        "              0.02, 714.0, diffusion=False).close()\n" % (ROOT, os.path.join(ROOT, "tests")))
    with tempfile.TemporaryDirectory() as d:
        subprocess.run([sys.executable, "-c", code], cwd=d, check=True, capture_output=True)
        assert [f for f in os.listdir(d) if f.endswith(".fit.data")] == []
