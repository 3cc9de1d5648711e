"""Loader for the committed golden fixtures (made by tests/golden/make_golden.py)."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: z[k] for k in z.files}
    for k in ("kt", "np_", "ptsmax", "maxlevel", "rootlvl"):
        d[k] = int(d[k])
    d["ref_relerr"] = float(d["ref_relerr"])
    return d


def options(d, precision=None):
    o = {"-fmm3d_np": str(d["np_"]), "-fmm3d_let3d_ptsmax": str(d["ptsmax"]),
         "-fmm3d_let3d_maxlevel": str(d["maxlevel"])}
    if precision:
        o["-fmm3d_precision"] = precision
    return o
