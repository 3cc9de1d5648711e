"""Reference pins for the batched workload's Stokes instances.

The batched workload (workloads.batched_instances: 64 instances, np=6,
ptsmax 64, 8 density vectors each) is checked per instance against the
FP64 direct sum at 256 targets, for density vectors 0 and 7.  Its Stokes
single-layer instances (kernel 311) sit at the FMM truncation error of
np=6, around 1e-5.  This script runs the unmodified reference
(oracle/_ref/libkifmm_ref.so) on each Stokes instance for the same two
density vectors and stores the reference's own error there,
||fmm - direct|| / ||fmm|| (fmm3d/fmm3d_check.cpp:61-69), in
tests/golden/batched_stokes_ref.npz, so that the batched results can be held
to max(1e-5, 10 x the reference's error) instance by instance.

Usage:  python tests/golden/make_batched_golden.py [index ...]
        (about 10 minutes on one core for all 16 instances; indices given
        on the command line are computed and merged into the file)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "kernel-independent-fast-multipole-method_b200"))

import oracle  # noqa: E402
import workloads as W  # noqa: E402

RHS = 8
NCHK = 256
OUT = os.path.join(HERE, "batched_stokes_ref.npz")


def instance_errors(inst):
    n, sd = inst["n"], 3
    p, _ = W.GEOMETRIES[inst["geometry"]](n, inst["seed"])
    den = W.densities(n * RHS, sd, "uniform", inst["seed"] + 1)
    chk = W.check_indices(n, NCHK, inst["seed"] + 2)
    errs = []
    for r in (0, RHS - 1):
        dr = den[r * n * sd:(r + 1) * n * sd]
        val, _ = oracle.ref_fmm(inst["kt"], list(inst["coefs"]), 6, 64, 10, np.zeros(3), 0, p, p, p, dr)
        direct = oracle.ref_direct(inst["kt"], list(inst["coefs"]), p, p, dr, p[chk]).reshape(-1, 3)
        errs.append(oracle.relerr(val.reshape(-1, 3)[chk], direct))
    return errs


def main():
    if not oracle.ref_available():
        oracle.build(ref=True)
    insts = W.batched_instances()
    want = [int(a) for a in sys.argv[1:]] or [i["index"] for i in insts if i["kt"] == 311]
    have = {}
    if os.path.exists(OUT):
        z = np.load(OUT)
        have = {int(i): list(e) for i, e in zip(z["index"], z["ref_relerr"])}
    for i in want:
        have[i] = instance_errors(insts[i])
        print(f"instance {i}: n={insts[i]['n']} {insts[i]['geometry']} reference relerr rhs0 {have[i][0]:.3e} "
              f"rhs7 {have[i][1]:.3e}", flush=True)
    idx = sorted(have)
    np.savez_compressed(OUT, index=np.array(idx), ref_relerr=np.array([have[i] for i in idx]))


if __name__ == "__main__":
    main()
