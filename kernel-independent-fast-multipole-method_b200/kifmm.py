"""Python mirror of the reference's FMM3d interface over libkifmm_b200.so.

Same object model as the reference (fmm3d/fmm3d.hpp:27-115,
fmm3d/knlmat3d.hpp:26-49, fmm3d/tt.cpp:85-106)::

    fmm = FMM3d("fmm3d_")
    fmm.srcpos = srcpos; fmm.srcnor = srcnor; fmm.trgpos = trgpos   # (n, 3) = DblNumMat(3, n)
    fmm.ctr = (0, 0, 0); fmm.rootlvl = 0
    fmm.knl = Kernel3d(111, [1.0, 0.25])
    fmm.setup({"-fmm3d_np": "6", "-fmm3d_let3d_ptsmax": "150", "-fmm3d_let3d_maxlevel": "10"})
    fmm.eval(srcden, trgval)        # trgval is overwritten in place
    fmm.check(srcden, trgval, 20)   # relative error against the direct sum

Every failure raises KifmmError carrying the library's status code; the
reference's silent assert paths (common/commoninc.hpp:59-60) become
exceptions.  There is no CPU fallback: without a CUDA device setup()
raises KifmmError(KIFMM_ERR_NO_DEVICE) after building the tree.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libkifmm_b200.so")

STATUS = {0: "KIFMM_OK", 1: "KIFMM_ERR_ARG", 2: "KIFMM_ERR_KERNEL", 3: "KIFMM_ERR_OUT_OF_BOX",
          4: "KIFMM_ERR_STATE", 5: "KIFMM_ERR_OPTION", 6: "KIFMM_ERR_CUDA", 7: "KIFMM_ERR_ALLOC",
          8: "KIFMM_ERR_NUMERIC", 9: "KIFMM_ERR_NO_DEVICE", 10: "KIFMM_ERR_CAPACITY"}
for _c, _n in STATUS.items():
    globals()[_n] = _c

_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)
_LP = ctypes.POINTER(ctypes.c_int64)
_H = ctypes.c_void_p

# (name, argtypes) of every entry point declared in include/kifmm.h
SIGNATURES = {
    "kifmm_create": [ctypes.c_char_p, ctypes.POINTER(_H)],
    "kifmm_destroy": [_H],
    "kifmm_set_geometry": [_H, ctypes.c_int, _DP, _DP, ctypes.c_int, _DP],
    "kifmm_set_kernel": [_H, ctypes.c_int, ctypes.c_int, _DP],
    "kifmm_set_box": [_H, _DP, ctypes.c_int],
    "kifmm_set_option": [_H, ctypes.c_char_p, ctypes.c_char_p],
    "kifmm_setup": [_H],
    "kifmm_eval": [_H, _DP, _DP],
    "kifmm_eval_multi": [_H, ctypes.c_int, _DP, _DP],
    "kifmm_eval_device": [_H, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int],
    "kifmm_check": [_H, _DP, _DP, ctypes.c_int, ctypes.c_uint64, _DP],
    "kifmm_direct": [_H, _DP, ctypes.c_int, _DP, _DP],
    "kifmm_direct_noalloc": [ctypes.c_int, ctypes.c_int, _DP, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                             ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "kifmm_tree_size": [_H, _IP, _IP],
    "kifmm_tree_nodes": [_H, _IP, _IP, _IP, _IP, _IP, _IP, _IP],
    "kifmm_tree_lists": [_H, ctypes.c_int, _LP, _LP, _IP],
    "kifmm_tree_points": [_H, ctypes.c_int, _LP, _IP],
    "kifmm_dofs": [_H, _IP, _IP],
    "kifmm_phase_times": [_H, _DP, _IP],
    "kifmm_set_profiling": [_H, ctypes.c_int],
    "kifmm_setup_times": [_H, _DP, _IP],
    "kifmm_schedule": [_H, _DP, _IP],
    "kifmm_work_counters": [_H, _DP, _IP],
    "kifmm_last_launch_count": [_H, _IP],
    "kifmm_batch_create": [ctypes.c_int, ctypes.POINTER(_H), ctypes.POINTER(ctypes.c_void_p)],
    "kifmm_batch_create_opts": [ctypes.c_int, ctypes.POINTER(_H), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    "kifmm_batch_info": [ctypes.c_void_p, _IP, _IP, _IP],
    "kifmm_batch_destroy": [ctypes.c_void_p],
    "kifmm_batch_eval_device": [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_int],
    "kifmm_batch_last_error": [ctypes.c_void_p],
    "kifmm_batch_poll_status": [ctypes.c_void_p],
    "kifmm_poll_status": [_H],
    "kifmm_status_string": [ctypes.c_int],
    "kifmm_last_error": [_H],
}

_lib = None


def lib():
    """Loads the in-tree CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run __graft_entry__.build() (make -C the package dir)")
        L = ctypes.CDLL(LIB_PATH)
        for name, argt in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = argt
            f.restype = (ctypes.c_char_p if name in ("kifmm_status_string", "kifmm_last_error", "kifmm_batch_last_error")
                         else ctypes.c_int)
        _lib = L
    return _lib


class KifmmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Kernel3d:
    """Kernel3d(kt, coefs) of fmm3d/kernel3d.hpp:56-80 (coefs[0]=mu, coefs[1]=nu)."""

    DOFS = {111: (1, 1), 121: (1, 1), 311: (3, 3), 312: (3, 1), 321: (3, 3), 322: (3, 1), 511: (3, 3), 521: (3, 3)}

    def __init__(self, kt: int, coefs=(1.0, 0.25)):
        self.kt = int(kt)
        self.coefs = [float(c) for c in coefs]

    def sdof(self):
        return self.DOFS[self.kt][0]

    def tdof(self):
        return self.DOFS[self.kt][1]


def _dptr(a):
    return a.ctypes.data_as(_DP)


def _as3(a, name):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.ndim != 2 or a.shape[1] != 3:
        raise ValueError(f"{name} must have shape (n, 3)")
    return a


class FMM3d:
    """FMM3d (fmm3d/fmm3d.hpp:27) evaluated on the GPU."""

    def __init__(self, prefix: str = "fmm3d_"):
        self._h = _H()
        self._check(lib().kifmm_create(prefix.encode(), ctypes.byref(self._h)))
        self.prefix = prefix
        self.srcpos = None
        self.srcnor = None
        self.trgpos = None
        self.ctr = (0.0, 0.0, 0.0)
        self.rootlvl = 0
        self.knl = None
        self.np = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.kifmm_destroy(h)
            self._h = None

    def _check(self, st):
        if st != 0:
            msg = lib().kifmm_last_error(self._h).decode() if getattr(self, "_h", None) else ""
            raise KifmmError(st, msg or lib().kifmm_status_string(st).decode())
        return 0

    # -- FMM3d::setup (fmm3d/fmm3d_setup.cpp:26-63)
    def setup(self, opts: dict) -> int:
        if self.srcpos is None or self.trgpos is None or self.knl is None:
            raise KifmmError(KIFMM_ERR_STATE, "srcpos, trgpos and knl must be set before setup")
        sp = _as3(self.srcpos, "srcpos")
        sn = _as3(self.srcnor if self.srcnor is not None else self.srcpos, "srcnor")
        tp = _as3(self.trgpos, "trgpos")
        if len(sn) != len(sp):
            raise KifmmError(KIFMM_ERR_ARG, "srcnor and srcpos differ in length")
        self._keep = (sp, sn, tp)
        L = lib()
        self._check(L.kifmm_set_geometry(self._h, len(sp), _dptr(sp), _dptr(sn), len(tp), _dptr(tp)))
        cf = np.ascontiguousarray(self.knl.coefs, np.float64)
        self._check(L.kifmm_set_kernel(self._h, self.knl.kt, len(cf), _dptr(cf)))
        ctr = np.ascontiguousarray(self.ctr, np.float64)
        self._check(L.kifmm_set_box(self._h, _dptr(ctr), int(self.rootlvl)))
        for k, v in opts.items():
            self._check(L.kifmm_set_option(self._h, str(k).encode(), str(v).encode()))
        self._check(L.kifmm_setup(self._h))
        self.ns, self.nt = len(sp), len(tp)
        return 0

    def sdof(self):
        return self.knl.sdof()

    def tdof(self):
        return self.knl.tdof()

    # -- FMM3d::eval (fmm3d/fmm3d_eval.cpp:24-243)
    def eval(self, srcden, trgval) -> int:
        srcden = np.ascontiguousarray(srcden, np.float64)
        if srcden.size != self.sdof() * self.ns:
            raise KifmmError(KIFMM_ERR_ARG, "srcden must have sdof*ns entries")
        if not (isinstance(trgval, np.ndarray) and trgval.dtype == np.float64 and trgval.flags.c_contiguous
                and trgval.size == self.tdof() * self.nt):
            raise KifmmError(KIFMM_ERR_ARG, "trgval must be a contiguous float64 array of tdof*nt entries")
        return self._check(lib().kifmm_eval(self._h, _dptr(srcden), _dptr(trgval)))

    def eval_multi(self, srcden, trgval) -> int:
        """nrhs density vectors per call: srcden (nrhs, sdof*ns), trgval (nrhs, tdof*nt)."""
        srcden = np.ascontiguousarray(srcden, np.float64)
        nrhs = srcden.shape[0]
        if srcden.shape[1] != self.sdof() * self.ns or trgval.shape != (nrhs, self.tdof() * self.nt):
            raise KifmmError(KIFMM_ERR_ARG, "bad eval_multi shapes")
        return self._check(lib().kifmm_eval_multi(self._h, nrhs, _dptr(srcden), _dptr(trgval)))

    def eval_device(self, d_srcden: int, d_trgval: int, nrhs: int = 1, stream: int = 0, sync: bool = True) -> int:
        """Device pointers (e.g. torch tensor .data_ptr()) and a cudaStream_t handle."""
        return self._check(lib().kifmm_eval_device(self._h, nrhs, ctypes.c_void_p(d_srcden),
                                                   ctypes.c_void_p(d_trgval), ctypes.c_void_p(stream),
                                                   1 if sync else 0))

    def poll_status(self) -> int:
        """Raises KifmmError(KIFMM_ERR_CUDA) if a device-side wait of an eval
        that has completed since the last poll timed out (synchronise the
        stream of an asynchronous eval_device first)."""
        return self._check(lib().kifmm_poll_status(self._h))

    # -- FMM3d::check (fmm3d/fmm3d_check.cpp:25-73)
    def check(self, srcden, trgval, numchk: int = 20, seed: int = 0) -> float:
        srcden = np.ascontiguousarray(srcden, np.float64)
        trgval = np.ascontiguousarray(trgval, np.float64)
        rel = ctypes.c_double()
        self._check(lib().kifmm_check(self._h, _dptr(srcden), _dptr(trgval), numchk, seed, ctypes.byref(rel)))
        return rel.value

    def direct(self, srcden, trgpos):
        """FP64 direct sum on the device (Dense3d::eval) at arbitrary targets."""
        srcden = np.ascontiguousarray(srcden, np.float64)
        tp = _as3(trgpos, "trgpos")
        out = np.zeros(len(tp) * self.tdof())
        self._check(lib().kifmm_direct(self._h, _dptr(srcden), len(tp), _dptr(tp), _dptr(out)))
        return out

    # -- introspection
    def tree(self) -> dict:
        L = lib()
        nn, md = ctypes.c_int(), ctypes.c_int()
        self._check(L.kifmm_tree_size(self._h, ctypes.byref(nn), ctypes.byref(md)))
        n = nn.value
        out = {k: np.zeros(n, np.int32) for k in ("depth", "par", "chd", "tag", "snum", "tnum")}
        path = np.zeros((n, 3), np.int32)
        ip = lambda a: a.ctypes.data_as(_IP)
        self._check(L.kifmm_tree_nodes(self._h, ip(out["depth"]), ip(path), ip(out["par"]), ip(out["chd"]),
                                       ip(out["tag"]), ip(out["snum"]), ip(out["tnum"])))
        out["path"] = path
        out["maxdepth"] = md.value
        for w, name in enumerate("UVWX"):
            tot = ctypes.c_int64()
            self._check(L.kifmm_tree_lists(self._h, w, ctypes.byref(tot), None, None))
            ptr = np.zeros(n + 1, np.int64)
            idx = np.zeros(max(1, tot.value), np.int32)
            self._check(L.kifmm_tree_lists(self._h, w, None, ptr.ctypes.data_as(_LP), ip(idx)))
            out[name + "_ptr"] = ptr
            out[name] = idx[:tot.value]
        for w, name in enumerate(("sownvis", "townvis")):
            ptr = np.zeros(n + 1, np.int64)
            self._check(L.kifmm_tree_points(self._h, w, ptr.ctypes.data_as(_LP), None))
            idx = np.zeros(max(1, int(ptr[-1])), np.int32)
            self._check(L.kifmm_tree_points(self._h, w, ptr.ctypes.data_as(_LP), ip(idx)))
            out[name + "_ptr"] = ptr
            out[name] = idx[:int(ptr[-1])]
        return out

    def set_profiling(self, on: bool = True):
        self._check(lib().kifmm_set_profiling(self._h, 1 if on else 0))

    def phase_times(self):
        ms = (ctypes.c_double * 16)()
        n = ctypes.c_int()
        self._check(lib().kifmm_phase_times(self._h, ms, ctypes.byref(n)))
        names = ("upward", "vlist", "xlist", "downward", "leaf", "total", "m2l_forward", "m2l_hadamard",
                 "m2l_inverse")
        return {names[i]: ms[i] for i in range(n.value)}

    def setup_times(self):
        """Host wall-clock ms of the last setup: tree + lists, operators, device build."""
        ms = (ctypes.c_double * 8)()
        n = ctypes.c_int()
        self._check(lib().kifmm_setup_times(self._h, ms, ctypes.byref(n)))
        return dict(zip(("tree_lists", "operators", "device_build", "autotune"), ms[:n.value]))

    def schedule(self):
        """kifmm_schedule: the evaluation schedule in use (autotuned at setup
        with -<prefix>autotune 1)."""
        v = (ctypes.c_double * 8)()
        n = ctypes.c_int()
        self._check(lib().kifmm_schedule(self._h, v, ctypes.byref(n)))
        names = ("had_groups", "rhs_chunk", "autotuned", "from_cache", "candidates", "best_ms")
        d = {names[i]: v[i] for i in range(n.value)}
        for k in ("had_groups", "rhs_chunk", "autotuned", "from_cache", "candidates"):
            if k in d:
                d[k] = int(d[k])
        return d

    def work_counters(self):
        c = (ctypes.c_double * 16)()
        n = ctypes.c_int()
        self._check(lib().kifmm_work_counters(self._h, c, ctypes.byref(n)))
        names = ("near_interactions", "v_pairs", "wx_direct", "nodes", "leaves", "gemm_flops", "fwd_spectra",
                 "inv_spectra", "surface_interactions", "tc_hadamard_flops")
        return {names[i]: c[i] for i in range(n.value)}

    def last_launch_count(self) -> int:
        n = ctypes.c_int()
        self._check(lib().kifmm_last_launch_count(self._h, ctypes.byref(n)))
        return n.value


class Batch:
    """Many set-up FMM3d instances evaluated together in one CUDA graph
    (kifmm_batch_*): eval(srcden_ptrs, trgval_ptrs, nrhs, stream) takes one
    device pointer pair per instance."""

    def __init__(self, fmms, concatenate: bool = True):
        self.fmms = list(fmms)
        hs = (_H * len(self.fmms))(*[f._h for f in self.fmms])
        self._b = ctypes.c_void_p()
        st = lib().kifmm_batch_create_opts(len(self.fmms), hs, 1 if concatenate else 0, ctypes.byref(self._b))
        if st != 0:
            raise KifmmError(st, "kifmm_batch_create failed")

    def info(self):
        """kifmm_batch_info: units, forests among them, kernel launches per replay."""
        u, f, l = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        st = lib().kifmm_batch_info(self._b, ctypes.byref(u), ctypes.byref(f), ctypes.byref(l))
        if st != 0:
            raise KifmmError(st, "kifmm_batch_info failed")
        return {"units": u.value, "forests": f.value, "launches": l.value}

    def eval(self, d_srcden, d_trgval, nrhs: int = 1, stream: int = 0, sync: bool = True) -> int:
        n = len(self.fmms)
        src = (ctypes.c_void_p * n)(*d_srcden)
        dst = (ctypes.c_void_p * n)(*d_trgval)
        st = lib().kifmm_batch_eval_device(self._b, nrhs, src, dst, ctypes.c_void_p(stream), 1 if sync else 0)
        if st != 0:
            raise KifmmError(st, lib().kifmm_batch_last_error(self._b).decode())
        return 0

    def poll_status(self) -> int:
        """kifmm_batch_poll_status: raises if an instance's device-side wait timed out."""
        st = lib().kifmm_batch_poll_status(self._b)
        if st != 0:
            raise KifmmError(st, lib().kifmm_batch_last_error(self._b).decode())
        return 0

    def __del__(self):
        b = getattr(self, "_b", None)
        if b is not None and b.value and _lib is not None:
            _lib.kifmm_batch_destroy(b)
            self._b = None


def fmm3d_mex(srcpos, srcnor, trgpos, ctr, rootlvl, knl, np_, srcden, numchk: int = 20, precision: str = "fp64",
              return_check: bool = False):
    """The reference's MATLAB entry point (fmm3d/fmm3d_mex.cpp:13-64) with its
    8 arguments, over the same engine:

        trgval = fmm3d_mex(srcpos, srcnor, trgpos, ctr, rootlvl, knl, np, srcden)

    srcpos, srcnor: 3 x ns, trgpos: 3 x nt (MATLAB's column-major DblNumMat);
    ctr: 3 values; rootlvl: int; knl: (kt, coefs) like the 2 x 1 cell
    {kt; coefs} (or a Kernel3d); np in {4, 6, 8}; srcden: sdof * ns values.
    Options as the MEX file sets them: ptsmax 150, maxlevel 10 (:32-46).
    Returns trgval (tdof * nt values); the check against the direct sum at
    numchk targets (:59) is returned beside it when return_check is true.

    Differences from the MEX file, whose own code does not do what its
    arguments say: it passes srcpos as the normals and ignores ctr and rootlvl
    (:51-52); here srcnor, ctr and rootlvl are used.  Its iA asserts (np, the
    density size) raise ValueError."""
    if int(np_) not in (4, 6, 8):
        raise ValueError("np must be 4, 6 or 8")
    k = knl if isinstance(knl, Kernel3d) else Kernel3d(int(knl[0]), knl[1])

    def cols(a, name):
        a = np.asarray(a, dtype=np.float64)
        if a.ndim != 2 or a.shape[0] != 3:
            raise ValueError(f"{name} must be 3 x n")
        return np.ascontiguousarray(a.T)

    sp, sn, tp = cols(srcpos, "srcpos"), cols(srcnor, "srcnor"), cols(trgpos, "trgpos")
    if sn.shape != sp.shape:
        raise ValueError("srcnor must have the shape of srcpos")
    den = np.ascontiguousarray(srcden, dtype=np.float64).ravel()
    if den.size != k.sdof() * len(sp):
        raise ValueError("srcden must have sdof * ns values")
    c = np.asarray(ctr, dtype=np.float64).ravel()
    if c.size != 3:
        raise ValueError("ctr must have 3 values")
    fmm = FMM3d("fmm3d_")
    fmm.srcpos, fmm.srcnor, fmm.trgpos = sp, sn, tp
    fmm.ctr, fmm.rootlvl = (float(c[0]), float(c[1]), float(c[2])), int(rootlvl)
    fmm.knl = k
    fmm.setup({"-fmm3d_np": str(int(np_)), "-fmm3d_let3d_ptsmax": "150", "-fmm3d_let3d_maxlevel": "10",
               "-fmm3d_precision": precision})
    trgval = np.zeros(k.tdof() * len(tp))
    fmm.eval(den, trgval)
    rel = fmm.check(den, trgval, numchk) if numchk > 0 else None
    return (trgval, rel) if return_check else trgval


def header_symbols(header_path: str | None = None):
    """Entry points declared in include/kifmm.h (for the ABI test)."""
    import re
    if header_path is None:
        header_path = os.path.join(os.path.dirname(HERE), "include", "kifmm.h")
    txt = open(header_path).read()
    return sorted(set(re.findall(r"\b(kifmm_[a-z_]+)\s*\(", txt)))
