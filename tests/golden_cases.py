"""Loaders for the committed golden fixtures.

* ``<name>.npz``      small cases with full inputs, outputs, tree and lists
                      (made by tests/golden/make_golden.py);
* ``batched_stokes_ref.npz``  the reference's own errors on the batched
                      workload's Stokes instances (tests/golden/make_batched_golden.py);
* ``cfg_<name>.npz``  the benchmark configurations at full size: reference
                      output and direct sum at the check targets only; the
                      inputs are regenerated from their seeds by workloads.py
                      (made by tests/golden/make_config_golden.py).
"""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith(("cfg_", "batched_")))


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


def config_names():
    return sorted(os.path.basename(p)[4:-4] for p in glob.glob(os.path.join(GOLDEN, "cfg_*.npz")))


def load_config(name):
    z = np.load(os.path.join(GOLDEN, "cfg_" + name + ".npz"))
    d = {k: z[k] for k in z.files}
    for k in ("kt", "np_", "ptsmax", "maxlevel", "n"):
        d[k] = int(d[k])
    d["workload"] = str(d["workload"])
    for k in ("ref_relerr", "ref_setup_s", "ref_first_eval_s", "ref_direct_s"):
        d[k] = float(d[k])
    return d
