"""The engine's octree and U/V/W/X lists (built on the host inside
kifmm_setup) against the reference: bit-exact node arrays and lists in the
reference's breadth-first numbering, and the same point sets per leaf."""
import numpy as np
import pytest

import golden_cases as G
import kifmm
import oracle
import workloads as W
from test_abi import setup_ok


def engine_tree(kt, coefs, np_, pm, ml, ctr, rl, src, nor, trg):
    f = kifmm.FMM3d()
    f.srcpos, f.srcnor, f.trgpos = src, nor, trg
    f.ctr, f.rootlvl = tuple(ctr), rl
    f.knl = kifmm.Kernel3d(kt, coefs)
    setup_ok(f, {"-fmm3d_np": str(np_), "-fmm3d_let3d_ptsmax": str(pm), "-fmm3d_let3d_maxlevel": str(ml)})
    return f.tree()


def assert_same_tree(a, depth, par, chd, tag, path, snum, tnum, lists):
    assert np.array_equal(a["depth"], depth)
    assert np.array_equal(a["par"], par)
    assert np.array_equal(a["chd"], chd)
    assert np.array_equal(a["tag"], tag)
    assert np.array_equal(a["path"], path)
    assert np.array_equal(a["snum"], snum)
    assert np.array_equal(a["tnum"], tnum)
    for L, (ptr, idx) in lists.items():
        assert np.array_equal(a[L + "_ptr"], ptr), L
        assert np.array_equal(a[L], idx), L


@pytest.mark.parametrize("name", G.names())
def test_lists_bit_exact_against_reference_fixture(name):
    d = G.load(name)
    a = engine_tree(d["kt"], d["coefs"], d["np_"], d["ptsmax"], d["maxlevel"], d["ctr"], d["rootlvl"], d["src"],
                    d["nor"], d["trg"])
    assert_same_tree(a, d["tree_depth"], d["tree_par"], d["tree_chd"], d["tree_tag"], d["tree_path"],
                     d["tree_snum"], d["tree_tnum"],
                     {L: (d["list_" + L + "_ptr"], d["list_" + L]) for L in "UVWX"})


@pytest.mark.parametrize("geom,n,pm,ml,seed", [("cube", 20000, 30, 10, 1), ("sphere", 40000, 40, 10, 2),
                                               ("cube_plummer", 60000, 20, 8, 3), ("ellipsoid", 30000, 10, 6, 4),
                                               ("cube", 5000, 1, 4, 5), ("sphere", 3000, 3000, 10, 6)])
def test_lists_bit_exact_against_oracle(geom, n, pm, ml, seed):
    p, nor = getattr(W, geom)(n, seed)
    a = engine_tree(111, (1.0,), 4, pm, ml, (0, 0, 0), 0, p, nor, p)
    b = oracle.tree(pm, ml, np.zeros(3), 0, p, p)
    assert_same_tree(a, b["depth"], b["par"], b["chd"], b["tag"], b["path"], b["snum"], b["tnum"],
                     {L: (b[L + "_ptr"], b[L]) for L in "UVWX"})
    # same point set in every leaf (the order inside a leaf is the engine's own)
    leaves = np.nonzero(b["chd"] == -1)[0]
    for nm in ("sownvis", "townvis"):
        for g in leaves:
            x = np.sort(a[nm][a[nm + "_ptr"][g]:a[nm + "_ptr"][g + 1]])
            y = np.sort(b[nm][b[nm + "_ptr"][g]:b[nm + "_ptr"][g + 1]])
            assert np.array_equal(x, y)


def test_distinct_sources_and_targets_and_shifted_box():
    rng = np.random.default_rng(9)
    s = rng.uniform(-0.5, 1.5, (7000, 3))
    t = rng.uniform(-0.5, 1.5, (11000, 3))
    ctr = np.array([0.5, 0.5, 0.5])
    a = engine_tree(111, (1.0,), 4, 25, 9, ctr, 0, s, s, t)
    b = oracle.tree(25, 9, ctr, 0, s, t)
    assert_same_tree(a, b["depth"], b["par"], b["chd"], b["tag"], b["path"], b["snum"], b["tnum"],
                     {L: (b[L + "_ptr"], b[L]) for L in "UVWX"})


def test_v_lists_bounded_and_offsets_in_range():
    p, _ = W.cube_plummer(30000, 7)
    a = engine_tree(111, (1.0,), 4, 16, 10, (0, 0, 0), 0, p, p, p)
    cnt = np.diff(a["V_ptr"])
    assert cnt.max() <= 189
    for g in np.nonzero(cnt)[0][:500]:
        v = a["V"][a["V_ptr"][g]:a["V_ptr"][g + 1]]
        off = a["path"][v] - a["path"][g]
        assert np.abs(off).max() <= 3 and (np.abs(off).max(axis=1) >= 2).all()
        assert (a["depth"][v] == a["depth"][g]).all()
