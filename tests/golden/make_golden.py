"""Generates the golden fixtures in tests/golden/ from the reference itself.

Runs the unmodified reference KIFMM (oracle/_ref/libkifmm_ref.so, compiled
from the reference's own sources by oracle/Makefile) on small seeded inputs
and stores, per case:
  * the inputs (positions, normals, densities, options);
  * the reference's FMM3d::eval output for every target;
  * the reference's Dense3d direct sum at seeded check targets, and the
    reference's own relative error there (FMM3d::check's metric);
  * the reference's Let3d tree (depth, path, parent, child, tag, leaf
    counts) and its U/V/W/X lists.
The reference ships no fixtures or known-answer tests of its own, so these
are the pins for both the C restatement and the GPU engine.

Usage:  python tests/golden/make_golden.py      (needs the reference library oracle/_ref/libkifmm_ref.so,
                                               built by oracle/Makefile from the reference sources)
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

# name: (kt, coefs, np, ptsmax, maxlevel, geometry, n_src, n_trg, density, ctr, rootlvl)
CASES = {
    "lap_s_np4_sphere": (111, (1.0, 0.25), 4, 40, 10, "sphere", 2000, None, "uniform", (0, 0, 0), 0),
    "lap_d_np4_cube": (121, (1.0, 0.25), 4, 30, 10, "cube", 1500, None, "uniform", (0, 0, 0), 0),
    "stk_s_np6_cube": (311, (1.0, 0.25), 6, 30, 10, "cube", 1200, None, "uniform", (0, 0, 0), 0),
    "stk_d_np6_ellipsoid": (321, (1.0, 0.25), 6, 30, 10, "ellipsoid", 1200, None, "uniform", (0, 0, 0), 0),
    "stk_sp_np4_cube": (312, (1.0, 0.25), 4, 30, 10, "cube", 1000, None, "uniform", (0, 0, 0), 0),
    "stk_dp_np4_sphere": (322, (1.0, 0.25), 4, 30, 10, "sphere", 1000, None, "uniform", (0, 0, 0), 0),
    "nav_s_np6_sphere": (511, (1.0, 0.3), 6, 40, 10, "sphere", 1200, None, "normal", (0, 0, 0), 0),
    "nav_d_np4_cube": (521, (1.0, 0.3), 4, 30, 10, "cube", 1000, None, "normal", (0, 0, 0), 0),
    "lap_s_np8_plummer": (111, (1.0, 0.25), 8, 20, 10, "cube_plummer", 1500, None, "uniform", (0, 0, 0), 0),
    # separate source / target sets, as the reference's own tt driver uses (fmm3d/options_0)
    "lap_s_np6_tt_style": (111, (1.0, 0.25), 6, 30, 10, "cube", 1000, 2000, "uniform01", (0, 0, 0), 0),
    # shifted and shrunk root box
    "lap_s_np4_rootlvl1": (111, (1.0, 0.25), 4, 20, 8, "cube", 1000, None, "uniform", (0.25, -0.25, 0.5), 1),
}

NCHK = 200


def make_points(geom, n, seed, ctr, rootlvl):
    p, nor = getattr(W, geom)(n, seed)
    r = 2.0 ** (-rootlvl)
    p = np.asarray(ctr) + p * r * 0.999
    return np.ascontiguousarray(p), np.ascontiguousarray(nor)


def build_case(name, spec):
    kt, coefs, np_, pm, ml, geom, ns, ntrg, dens, ctr, rl = spec
    sd, td = W.KERNEL_DOFS[kt]
    src, nor = make_points(geom, ns, 0, ctr, rl)
    trg = src if ntrg is None else make_points(geom, ntrg, 4, ctr, rl)[0]
    den = W.densities(ns, sd, dens, 1)
    val, _ = oracle.ref_fmm(kt, coefs, np_, pm, ml, np.asarray(ctr, float), rl, src, nor, trg, den)
    chk = W.check_indices(len(trg), NCHK, 2)
    direct = oracle.ref_direct(kt, coefs, src, nor, den, trg[chk])
    tree = oracle.ref_tree(pm, ml, np.asarray(ctr, float), rl, src, trg)
    out = dict(kt=kt, coefs=np.asarray(coefs, float), np_=np_, ptsmax=pm, maxlevel=ml, ctr=np.asarray(ctr, float),
               rootlvl=rl, src=src, nor=nor, trg=trg, den=den, ref_val=val, chk=chk, ref_direct=direct,
               ref_relerr=oracle.relerr(val.reshape(-1, td)[chk], direct))
    for k in ("depth", "par", "chd", "tag", "snum", "tnum", "path"):
        out["tree_" + k] = tree[k]
    for L in "UVWX":
        out["list_" + L] = tree[L]
        out["list_" + L + "_ptr"] = tree[L + "_ptr"]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return out["ref_relerr"]


def main():
    if not oracle.ref_available():
        oracle.build(ref=True)
    for name, spec in CASES.items():
        e = build_case(name, spec)
        print(f"{name}: reference relerr {e:.3e}")


if __name__ == "__main__":
    main()
