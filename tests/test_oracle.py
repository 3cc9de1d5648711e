"""The oracle (C restatement of the reference) against the golden fixtures
made by the reference itself, and -- where the reference was compiled into
oracle/_ref -- against the reference directly on extra seeded inputs."""
import numpy as np
import pytest

import golden_cases as G
import oracle
import workloads as W

TREE_KEYS = ("depth", "par", "chd", "tag", "path")


@pytest.mark.parametrize("name", G.names())
def test_tree_and_lists_match_reference_fixture(name):
    d = G.load(name)
    t = oracle.tree(d["ptsmax"], d["maxlevel"], d["ctr"], d["rootlvl"], d["src"], d["trg"])
    for k in TREE_KEYS:
        assert np.array_equal(t[k], d["tree_" + k]), k
    assert np.array_equal(t["snum"], d["tree_snum"]) and np.array_equal(t["tnum"], d["tree_tnum"])
    for L in "UVWX":
        assert np.array_equal(t[L + "_ptr"], d["list_" + L + "_ptr"]), L
        assert np.array_equal(t[L], d["list_" + L]), L


@pytest.mark.parametrize("name", G.names())
def test_direct_sum_matches_reference_fixture(name):
    d = G.load(name)
    v = oracle.direct(d["kt"], d["coefs"], d["src"], d["nor"], d["den"], d["trg"][d["chk"]])
    ref = d["ref_direct"]
    assert np.linalg.norm(v - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("name", G.names())
def test_fixture_reference_error_is_the_checked_metric(name):
    d = G.load(name)
    td = W.KERNEL_DOFS[d["kt"]][1]
    e = oracle.relerr(d["ref_val"].reshape(-1, td)[d["chk"]], d["ref_direct"])
    assert abs(e - d["ref_relerr"]) <= 1e-12 + 1e-9 * d["ref_relerr"]


def test_relerr_metric_uses_fmm_norm():
    # FMM3d::check divides by the FMM solution norm (fmm3d/fmm3d_check.cpp:61-71)
    assert oracle.relerr([2.0, 0.0], [1.0, 0.0]) == pytest.approx(0.5)


def test_tree_rejects_points_outside_box():
    p = np.array([[0.0, 0.0, 0.0], [1.5, 0.0, 0.0]])
    with pytest.raises(ValueError):
        oracle.tree(1, 4, np.zeros(3), 0, p, p)


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference not compiled here")


@needs_ref
@pytest.mark.parametrize("geom,n,pm,ml", [("cube", 4000, 25, 10), ("sphere", 6000, 30, 10),
                                          ("cube_plummer", 8000, 16, 7), ("ellipsoid", 3000, 8, 5)])
def test_tree_matches_reference_library(geom, n, pm, ml):
    p, _ = getattr(W, geom)(n, 11)
    a = oracle.tree(pm, ml, np.zeros(3), 0, p, p)
    b = oracle.ref_tree(pm, ml, np.zeros(3), 0, p, p)
    for k in TREE_KEYS + ("U", "V", "W", "X", "sownvis", "townvis", "U_ptr", "V_ptr"):
        assert np.array_equal(a[k], b[k]), k


@needs_ref
@pytest.mark.parametrize("kt", [111, 121, 311, 312, 321, 322, 511, 521])
def test_direct_matches_reference_library(kt):
    rng = np.random.default_rng(kt)
    s = rng.uniform(-1, 1, (300, 3))
    nor = rng.standard_normal((300, 3))
    t = rng.uniform(-1, 1, (50, 3))
    t[0] = s[3]  # coincident point: the r < 1e-8 cut-off
    sd, _ = W.KERNEL_DOFS[kt]
    den = rng.standard_normal(300 * sd)
    a = oracle.direct(kt, [1.3, 0.3], s, nor, den, t)
    b = oracle.ref_direct(kt, [1.3, 0.3], s, nor, den, t)
    assert np.allclose(a, b, rtol=1e-12, atol=1e-12 * np.abs(b).max())


@needs_ref
def test_fft_shim_matches_numpy():
    # The FFTW2-interface shim the reference is built with must be a true DFT.
    import ctypes
    L = oracle.ref_lib()
    L.rfftw3d_create_plan.restype = ctypes.c_void_p
    n0, n1, n2 = 6, 12, 10
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2, n0, n1, n2))
    xi = np.ascontiguousarray(np.moveaxis(x, 0, -1))  # howmany=2 interleaved (stride 2, dist 1)
    out = np.zeros((n0, n1, n2 // 2 + 1, 2, 2))
    plan = L.rfftw3d_create_plan(n0, n1, n2, -1, 0)
    dp = ctypes.POINTER(ctypes.c_double)
    L.rfftwnd_real_to_complex(ctypes.c_void_p(plan), 2, xi.ctypes.data_as(dp), 2, 1, out.ctypes.data_as(dp), 2, 1)
    got = out[..., 0] + 1j * out[..., 1]
    for h in range(2):
        assert np.allclose(got[..., h], np.fft.rfftn(x[h]), atol=1e-10)
    back = np.zeros((n0, n1, n2, 2))
    plan_b = L.rfftw3d_create_plan(n0, n1, n2, 1, 0)
    L.rfftwnd_complex_to_real(ctypes.c_void_p(plan_b), 2, out.ctypes.data_as(dp), 2, 1, back.ctypes.data_as(dp), 2, 1)
    for h in range(2):
        assert np.allclose(back[..., h] / (n0 * n1 * n2), x[h], atol=1e-10)
    L.rfftwnd_destroy_plan(ctypes.c_void_p(plan))
    L.rfftwnd_destroy_plan(ctypes.c_void_p(plan_b))
