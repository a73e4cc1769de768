"""Writes the shipped BetterTT06 fit files: dt = 0.02 ms, celltype 0/1/2,
default g_K1, in the reference's FIT/FUNCTION object format.

    python -m cardioid_b200.data.make_fits
"""
import os

from cardioid_b200 import fitgen, tt06

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = {0: "tt06Endo", 1: "tt06Mid", 2: "tt06Epi"}


def fit_path(dt, celltype):
    return os.path.join(HERE, "tt06_dt%g_celltype%d.fit.data" % (dt, celltype))


def main(dt=0.02):
    for ct, name in NAMES.items():
        p = tt06.TT06Params.defaults(ct)
        p.fits = fitgen.generate(dt, p, verbose=True)
        with open(fit_path(dt, ct), "w") as f:
            f.write(tt06.fit_file_text(name, dt, p))
        print("wrote", fit_path(dt, ct))


if __name__ == "__main__":
    main()
