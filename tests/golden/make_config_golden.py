"""Reference pins for the benchmark configurations at their full sizes.

Runs the unmodified reference KIFMM (oracle/_ref/libkifmm_ref.so, compiled
from the reference's own sources by oracle/Makefile) once per configuration,
on the seeded point clouds of workloads.py, and stores in
tests/golden/cfg_<name>.npz only what a parity test needs at that size:

  * the check-target indices (1,000 or 4,096, seed 2, workloads.check_indices);
  * the reference's FMM3d::eval output at those targets;
  * the reference's Dense3d direct sum there and the reference's own
    relative error, ||fmm - direct|| / ||fmm|| (fmm3d/fmm3d_check.cpp:61-69);
  * checksums of the generated inputs, so that a test regenerating the cloud
    on another machine can tell that it has the same input;
  * the reference's setup time and its first eval time (lazy operator
    build included) on the host that made the fixture, for information.

The full point clouds (up to 1M points) are not stored: workloads.py
regenerates them bit for bit from their seeds (numpy PCG64).

Usage:  python tests/golden/make_config_golden.py [name ...]
        (needs oracle/_ref/libkifmm_ref.so; the Navier np=8 case takes
        about 6 minutes on one core, the Stokes double-layer case about 1)
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "kernel-independent-fast-multipole-method_b200"))

import oracle  # noqa: E402
import workloads as W  # noqa: E402

# name: (workload key in workloads.WORKLOADS, number of points)
CASES = {
    "laplace_sphere_np4": ("laplace_sphere_np4", 32768),
    "stokes_dl_ellipsoid_np6": ("stokes_dl_ellipsoid_np6", 262144),
    "navier_sphere_np8": ("navier_sphere_np8", 1048576),
    # the mixed-precision configuration's cloud at 1/16 of its size
    "laplace_cube_plummer_np6_262k": ("laplace_cube_plummer_np6", 262144),
}


def input_checksums(p, nor, den):
    """Order-sensitive checksums of the generated inputs."""
    w = np.arange(1, len(p) + 1, dtype=np.float64)
    return np.array([p.sum(), (p[:, 0] * w).sum(), nor.sum(), (nor[:, 2] * w).sum(), den.sum(),
                     (den * np.arange(1, den.size + 1)).sum()])


def build_case(name):
    key, n = CASES[name]
    wl = W.WORKLOADS[key]
    p, nor = wl.points(n)
    den = wl.density(n)
    chk = W.check_indices(n, wl.nchk, 2)
    val, times = oracle.ref_fmm(wl.kt, list(wl.coefs), wl.np_, wl.ptsmax, wl.maxlevel, np.zeros(3), 0, p, nor, p,
                                den, neval=1)
    td = wl.tdof
    t0 = time.perf_counter()
    direct = oracle.ref_direct(wl.kt, list(wl.coefs), p, nor, den, p[chk])
    t_direct = time.perf_counter() - t0
    ref_chk = val.reshape(-1, td)[chk]
    rel = oracle.relerr(ref_chk, direct)
    np.savez_compressed(os.path.join(HERE, "cfg_" + name + ".npz"), workload=key, n=n, kt=wl.kt,
                        coefs=np.asarray(wl.coefs, float), np_=wl.np_, ptsmax=wl.ptsmax, maxlevel=wl.maxlevel,
                        chk=chk, ref_val_chk=ref_chk, ref_direct=direct.reshape(-1, td), ref_relerr=rel,
                        checksums=input_checksums(p, nor, den), ref_setup_s=times[0], ref_first_eval_s=times[1],
                        ref_direct_s=t_direct)
    return rel, times


def main():
    if not oracle.ref_available():
        oracle.build(ref=True)
    names = sys.argv[1:] or list(CASES)
    for name in names:
        rel, times = build_case(name)
        print(f"{name}: reference relerr {rel:.3e}, setup {times[0]:.2f} s, first eval {times[1]:.2f} s", flush=True)


if __name__ == "__main__":
    main()
