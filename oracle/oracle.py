"""Test infrastructure (oracle only): ctypes access to the two CPU checkers.

* ``libkifmm_oracle.so`` -- the plain-C restatement in kifmm_oracle.c
  (kernels, Dense3d direct sum, Let3d tree and U/V/W/X lists);
* ``libkifmm_ref.so``    -- the unmodified reference compiled from its own
  sources by oracle/Makefile (present only where the reference tree was
  available at build time).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module, and only as the checker.  Positions and normals are
(n, 3) arrays, i.e. the reference's 3 x n column-major DblNumMat.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)
_LP = ctypes.POINTER(ctypes.c_long)

LIST_NAMES = ("U", "V", "W", "X")


def build(ref: bool = True) -> None:
    """Builds the oracle libraries (the reference one only if its sources exist)."""
    target = "all" if ref else "oracle"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_DP)


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        path = os.path.join(OUT, "libkifmm_oracle.so")
        if not os.path.exists(path):
            build(ref=False)
        lib = ctypes.CDLL(path)
        lib.ko_tree_build.restype = ctypes.c_void_p
        lib.ko_tree_list_total.restype = ctypes.c_long
        for f in ("ko_tree_nnodes", "ko_tree_nodes", "ko_tree_list_total", "ko_tree_lists", "ko_tree_free"):
            getattr(lib, f).argtypes = None
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(os.path.join(OUT, "libkifmm_ref.so"))


def ref_lib():
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(os.path.join(OUT, "libkifmm_ref.so"))
        lib.kref_tree_build.restype = ctypes.c_void_p
        lib.kref_tree_list_total.restype = ctypes.c_long
        _ref = lib
    return _ref


def kernel_dofs(kt: int):
    sd, td = ctypes.c_int(), ctypes.c_int()
    if oracle_lib().ko_kernel_dofs(kt, ctypes.byref(sd), ctypes.byref(td)) != 0:
        raise ValueError(f"unknown kernel {kt}")
    return sd.value, td.value


def direct(kt, coefs, srcpos, srcnor, srcden, trgpos, nthreads: int = 0):
    """FP64 direct sum (Dense3d::eval restated).  Returns td*nt values."""
    srcpos = np.ascontiguousarray(srcpos, np.float64)
    srcnor = np.ascontiguousarray(srcnor, np.float64)
    trgpos = np.ascontiguousarray(trgpos, np.float64)
    srcden = np.ascontiguousarray(srcden, np.float64)
    coefs = np.ascontiguousarray(coefs, np.float64)
    _, td = kernel_dofs(kt)
    out = np.zeros(td * len(trgpos))
    rc = oracle_lib().ko_direct(kt, len(coefs), _d(coefs), len(srcpos), _d(srcpos), _d(srcnor),
                                _d(srcden), len(trgpos), _d(trgpos), out.ctypes.data_as(_DP), nthreads)
    if rc != 0:
        raise ValueError("ko_direct failed")
    return out


def relerr(fmm_vals, direct_vals) -> float:
    """FMM3d::check's metric: ||fmm - direct|| / ||fmm|| (fmm3d/fmm3d_check.cpp:61-71)."""
    fmm_vals = np.asarray(fmm_vals, np.float64).ravel()
    direct_vals = np.asarray(direct_vals, np.float64).ravel()
    return float(np.linalg.norm(direct_vals - fmm_vals) / np.linalg.norm(fmm_vals))


def _tree_dict(lib, prefix, h):
    n = getattr(lib, prefix + "tree_nnodes")(ctypes.c_void_p(h))
    arrs = {k: np.zeros(n, np.int32) for k in ("depth", "par", "chd", "tag", "sbeg", "snum", "tbeg", "tnum")}
    path = np.zeros((n, 3), np.int32)
    ip = lambda a: a.ctypes.data_as(_IP)
    getattr(lib, prefix + "tree_nodes")(ctypes.c_void_p(h), ip(arrs["depth"]), ip(path), ip(arrs["par"]),
                                       ip(arrs["chd"]), ip(arrs["tag"]), ip(arrs["sbeg"]), ip(arrs["snum"]),
                                       ip(arrs["tbeg"]), ip(arrs["tnum"]))
    arrs["path"] = path
    total = getattr(lib, prefix + "tree_list_total")
    total.restype = ctypes.c_long
    for w, name in enumerate(LIST_NAMES + ("sownvis", "townvis")):
        tot = total(ctypes.c_void_p(h), w)
        ptr = np.zeros(n + 1, np.int64)
        idx = np.zeros(max(tot, 1), np.int32)
        getattr(lib, prefix + "tree_lists")(ctypes.c_void_p(h), w, ptr.ctypes.data_as(_LP), ip(idx))
        arrs[name + "_ptr"] = ptr
        arrs[name] = idx[:tot]
    getattr(lib, prefix + "tree_free")(ctypes.c_void_p(h))
    return arrs


def tree(ptsmax, maxlevel, ctr, rootlvl, srcpos, trgpos):
    """Octree + lists from the C restatement, in the reference's BFS numbering."""
    lib = oracle_lib()
    srcpos = np.ascontiguousarray(srcpos, np.float64)
    trgpos = np.ascontiguousarray(trgpos, np.float64)
    ctr = np.ascontiguousarray(ctr, np.float64)
    st = ctypes.c_int()
    h = lib.ko_tree_build(ptsmax, maxlevel, _d(ctr), rootlvl, len(srcpos), _d(srcpos), len(trgpos), _d(trgpos),
                          ctypes.byref(st))
    if st.value != 0:
        lib.ko_tree_free(ctypes.c_void_p(h))
        raise ValueError("point outside the root box")
    return _tree_dict(lib, "ko_", h)


def ref_tree(ptsmax, maxlevel, ctr, rootlvl, srcpos, trgpos):
    """Octree + lists from the reference's own Let3d (needs libkifmm_ref.so)."""
    lib = ref_lib()
    srcpos = np.ascontiguousarray(srcpos, np.float64)
    trgpos = np.ascontiguousarray(trgpos, np.float64)
    ctr = np.ascontiguousarray(ctr, np.float64)
    h = lib.kref_tree_build(ptsmax, maxlevel, _d(ctr), rootlvl, len(srcpos), _d(srcpos), len(trgpos), _d(trgpos))
    return _tree_dict(lib, "kref_", h)


def ref_fmm(kt, coefs, np_, ptsmax, maxlevel, ctr, rootlvl, srcpos, srcnor, trgpos, srcden, neval: int = 1):
    """Runs the reference FMM3d setup + neval evals.  Returns (trgval, times)."""
    lib = ref_lib()
    srcpos = np.ascontiguousarray(srcpos, np.float64)
    srcnor = np.ascontiguousarray(srcnor, np.float64)
    trgpos = np.ascontiguousarray(trgpos, np.float64)
    srcden = np.ascontiguousarray(srcden, np.float64)
    coefs = np.ascontiguousarray(coefs, np.float64)
    ctr = np.ascontiguousarray(ctr, np.float64)
    _, td = kernel_dofs(kt)
    out = np.zeros(td * len(trgpos))
    times = np.zeros(1 + neval)
    rc = lib.kref_fmm(kt, len(coefs), _d(coefs), np_, ptsmax, maxlevel, _d(ctr), rootlvl, len(srcpos), _d(srcpos),
                      _d(srcnor), len(trgpos), _d(trgpos), _d(srcden), out.ctypes.data_as(_DP), neval,
                      times.ctypes.data_as(_DP))
    if rc != 0:
        raise RuntimeError("reference FMM failed")
    return out, times


def ref_direct(kt, coefs, srcpos, srcnor, srcden, trgpos):
    lib = ref_lib()
    _, td = kernel_dofs(kt)
    out = np.zeros(td * len(trgpos))
    coefs = np.ascontiguousarray(coefs, np.float64)
    srcpos = np.ascontiguousarray(srcpos, np.float64)
    srcnor = np.ascontiguousarray(srcnor, np.float64)
    trgpos = np.ascontiguousarray(trgpos, np.float64)
    srcden = np.ascontiguousarray(srcden, np.float64)
    lib.kref_direct(kt, len(coefs), _d(coefs), len(srcpos), _d(srcpos), _d(srcnor), _d(srcden), len(trgpos),
                    _d(trgpos), out.ctypes.data_as(_DP))
    return out
