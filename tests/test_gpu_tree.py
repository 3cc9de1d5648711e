"""The octree and U/V/W/X lists built on the GPU (tree_gpu.cu, the default
of kifmm_setup on a GPU) against the reference: bit-exact node arrays and
lists in the reference's breadth-first numbering for every golden fixture
(made by the reference itself), against the oracle's restatement of Let3d
on larger clouds, and identical to the host builder (tree.cpp) including
the order of the points inside every leaf (both sorts are stable, so equal
keys keep the original point order the reference inserts them in)."""
import numpy as np
import pytest

import golden_cases as G
import kifmm
import oracle
import workloads as W

pytestmark = pytest.mark.gpu

KEYS = ("depth", "par", "chd", "tag", "path", "snum", "tnum")


def tree_of(src, nor, trg, pm, ml, ctr=(0, 0, 0), rl=0, where="device", kt=111, coefs=(1.0,)):
    f = kifmm.FMM3d()
    f.srcpos, f.srcnor, f.trgpos = src, nor, trg
    f.ctr, f.rootlvl = tuple(ctr), rl
    f.knl = kifmm.Kernel3d(kt, coefs)
    f.setup({"-fmm3d_np": "4", "-fmm3d_let3d_ptsmax": str(pm), "-fmm3d_let3d_maxlevel": str(ml),
             "-fmm3d_tree": where})
    return f.tree()


def same(a, b):
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k
    for L in "UVWX":
        assert np.array_equal(a[L + "_ptr"], b[L + "_ptr"]), L
        assert np.array_equal(a[L], b[L]), L


@pytest.mark.parametrize("name", G.names())
def test_device_lists_bit_exact_against_reference_fixture(gpu, name):
    d = G.load(name)
    a = tree_of(d["src"], d["nor"], d["trg"], d["ptsmax"], d["maxlevel"], d["ctr"], d["rootlvl"], kt=d["kt"],
                coefs=d["coefs"])
    same(a, {"depth": d["tree_depth"], "par": d["tree_par"], "chd": d["tree_chd"], "tag": d["tree_tag"],
             "path": d["tree_path"], "snum": d["tree_snum"], "tnum": d["tree_tnum"],
             **{L + "_ptr": d["list_" + L + "_ptr"] for L in "UVWX"}, **{L: d["list_" + L] for L in "UVWX"}})


@pytest.mark.parametrize("geom,n,pm,ml,seed", [("cube", 20000, 30, 10, 1), ("sphere", 40000, 40, 10, 2),
                                               ("cube_plummer", 60000, 20, 8, 3), ("ellipsoid", 30000, 10, 6, 4),
                                               ("cube", 5000, 1, 4, 5), ("sphere", 3000, 3000, 10, 6)])
def test_device_lists_bit_exact_against_oracle(gpu, geom, n, pm, ml, seed):
    p, nor = getattr(W, geom)(n, seed)
    a = tree_of(p, nor, p, pm, ml)
    b = oracle.tree(pm, ml, np.zeros(3), 0, p, p)
    same(a, b)


@pytest.mark.parametrize("geom,n,pm,ml,seed", [("cube_plummer", 200000, 64, 10, 7), ("sphere", 100000, 1, 12, 8),
                                               ("ellipsoid", 150000, 100, 21, 9), ("cube", 1, 1, 10, 10)])
def test_device_tree_equals_host_tree_with_leaf_point_order(gpu, geom, n, pm, ml, seed):
    p, nor = getattr(W, geom)(n, seed)
    a = tree_of(p, nor, p, pm, ml, where="device")
    b = tree_of(p, nor, p, pm, ml, where="host")
    same(a, b)
    for k in ("sownvis", "townvis", "sownvis_ptr", "townvis_ptr"):
        assert np.array_equal(a[k], b[k]), k


def test_device_tree_separate_targets_and_shifted_box(gpu):
    rng = np.random.default_rng(9)
    s = rng.uniform(-0.5, 1.5, (7000, 3))
    t = rng.uniform(-0.5, 1.5, (11000, 3))
    ctr = np.array([0.5, 0.5, 0.5])
    a = tree_of(s, s, t, 25, 9, ctr)
    same(a, oracle.tree(25, 9, ctr, 0, s, t))
    c = tree_of(s, s, t, 25, 9, ctr, where="host")
    for k in ("sownvis", "townvis"):
        assert np.array_equal(a[k], c[k]), k


def test_device_tree_rejects_points_outside_the_box(gpu):
    p = np.array([[0.0, 0.0, 0.0], [1.5, 0.0, 0.0]])
    f = kifmm.FMM3d()
    f.srcpos = f.srcnor = f.trgpos = p
    f.knl = kifmm.Kernel3d(111, [1.0])
    with pytest.raises(kifmm.KifmmError) as e:
        f.setup({"-fmm3d_np": "4", "-fmm3d_let3d_ptsmax": "1", "-fmm3d_let3d_maxlevel": "4"})
    assert e.value.status == kifmm.KIFMM_ERR_OUT_OF_BOX
