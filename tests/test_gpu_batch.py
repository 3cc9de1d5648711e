"""Batched evaluation (kifmm_batch_*): several set-up instances, of different
kernels and precisions, evaluated in one captured CUDA graph.

Without concatenation the graph replays exactly the passes a single
eval_device enqueues, so each instance's output must be bit-identical to its
own eval_device call; a new set of buffers or rhs count recaptures the
graph.  Instances that share kernel, np, precision, V-list form and root level
are concatenated into one forest engine (one launch per pass for all of
them): equal to their single evals to rounding (1e-12 relative in FP64, 1e-6
in mixed precision, whose FP16 spectra scale the forest shares).
"""
import numpy as np
import pytest

import golden_cases as G
import kifmm
import workloads as W

pytestmark = pytest.mark.gpu


def _engine(d, precision):
    f = kifmm.FMM3d("fmm3d_")
    f.srcpos, f.srcnor, f.trgpos = d["src"], d["nor"], d["trg"]
    f.ctr, f.rootlvl = tuple(d["ctr"]), d["rootlvl"]
    f.knl = kifmm.Kernel3d(d["kt"], d["coefs"])
    f.setup(G.options(d, precision))
    return f


def test_batch_matches_single_instance_evals(gpu):
    torch = pytest.importorskip("torch")
    cases = [("lap_s_np6_tt_style", "mixed"), ("stk_s_np6_cube", "mixed"), ("lap_s_np4_sphere", "fp64"),
             ("nav_s_np6_sphere", "fp64")]
    nrhs = 2
    fmms, srcs, outs, want = [], [], [], []
    rng = np.random.default_rng(11)
    for name, prec in cases:
        d = G.load(name)
        f = _engine(d, prec)
        sd, td = W.KERNEL_DOFS[d["kt"]]
        den = rng.standard_normal(nrhs * sd * len(d["src"]))
        s = torch.tensor(den, device="cuda", dtype=torch.float64)
        o = torch.zeros(nrhs * td * len(d["trg"]), device="cuda", dtype=torch.float64)
        ref = torch.zeros_like(o)
        f.eval_device(s.data_ptr(), ref.data_ptr(), nrhs, 0, sync=True)
        fmms.append(f)
        srcs.append(s)
        outs.append(o)
        want.append(ref.cpu().numpy())
    b = kifmm.Batch(fmms, concatenate=False)
    for _ in range(2):  # capture, then replay
        for o in outs:
            o.zero_()
        torch.cuda.synchronize()
        b.eval([s.data_ptr() for s in srcs], [o.data_ptr() for o in outs], nrhs, 0, sync=True)
        for o, w in zip(outs, want):
            assert np.array_equal(o.cpu().numpy(), w)
    # other buffers and a single rhs: recaptured.  One density vector alone
    # runs the surface contractions over half the columns of the two-vector
    # pass, so the split-K schedule (and the FP32 summation order) may differ:
    # equal to rounding, 1e-13 relative in FP64 and 1e-6 in mixed precision
    outs1 = [torch.zeros(o.numel() // nrhs, device="cuda", dtype=torch.float64) for o in outs]
    b.eval([s.data_ptr() for s in srcs], [o.data_ptr() for o in outs1], 1, 0, sync=True)
    for (name, prec), o, w in zip(cases, outs1, want):
        got, ref = o.cpu().numpy(), w[: o.numel()]
        tol = 1e-13 if prec == "fp64" else 1e-6
        assert np.linalg.norm(got - ref) <= tol * np.linalg.norm(ref), name


def test_batch_rejects_bad_arguments(gpu):
    d = G.load("lap_s_np4_sphere")
    f = _engine(d, "fp64")
    b = kifmm.Batch([f])
    with pytest.raises(kifmm.KifmmError):
        b.eval([0], [0], 0)
    unset = kifmm.FMM3d("fmm3d_")
    with pytest.raises(kifmm.KifmmError):
        kifmm.Batch([unset])


def _cloud_engine(kt, n, geometry, seed, precision):
    p, _ = W.GEOMETRIES[geometry](n, seed)
    f = kifmm.FMM3d("fmm3d_")
    f.srcpos = f.srcnor = f.trgpos = p
    f.knl = kifmm.Kernel3d(kt, [1.0, 0.25])
    f.setup({"-fmm3d_np": "6", "-fmm3d_let3d_ptsmax": "64", "-fmm3d_let3d_maxlevel": "10",
             "-fmm3d_precision": precision})
    return f


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_concatenated_instances_match_single_instance_evals(gpu, precision, tol):
    """Five Laplace instances (one with separate source and target sets and
    its own root box) and two Stokes instances: two forests, each one launch
    per pass; every instance's potentials equal its own eval to rounding."""
    torch = pytest.importorskip("torch")
    nrhs = 3
    fmms = [_cloud_engine(111, 4000, "sphere", 1, precision), _cloud_engine(111, 9000, "cube", 2, precision),
            _cloud_engine(111, 6000, "plummer_ball", 3, precision), _cloud_engine(111, 2500, "cube", 4, precision),
            _cloud_engine(311, 5000, "cube", 5, precision), _cloud_engine(311, 3000, "sphere", 6, precision)]
    d = G.load("lap_s_np6_tt_style")
    t = _engine(d, precision)
    fmms.insert(2, t)
    rng = np.random.default_rng(5)
    srcs, outs, want, single_launches = [], [], [], 0
    for f in fmms:
        den = rng.uniform(-1, 1, nrhs * f.sdof() * f.ns)
        s = torch.tensor(den, device="cuda", dtype=torch.float64)
        ref = torch.zeros(nrhs * f.tdof() * f.nt, device="cuda", dtype=torch.float64)
        f.eval_device(s.data_ptr(), ref.data_ptr(), nrhs, 0, sync=True)
        single_launches += f.last_launch_count()
        srcs.append(s)
        outs.append(torch.zeros_like(ref))
        want.append(ref.cpu().numpy())
    b = kifmm.Batch(fmms)
    for _ in range(2):  # capture, then replay
        for o in outs:
            o.zero_()
        b.eval([s.data_ptr() for s in srcs], [o.data_ptr() for o in outs], nrhs, 0, sync=True)
        for f, o, w in zip(fmms, outs, want):
            got = o.cpu().numpy()
            assert np.linalg.norm(got - w) <= tol * np.linalg.norm(w), (f.knl.kt, np.linalg.norm(got - w) / np.linalg.norm(w))
    info = b.info()
    assert info["forests"] == 2 and info["units"] == 2
    assert 0 < info["launches"] < single_launches / 2


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_concatenated_double_layer_instances(gpu, precision, tol):
    """Double-layer instances (Stokes 321 and Navier 521, with normals) in
    forests: in mixed precision their U lists run in FP64 through the
    forest's own FP64 near-field pass."""
    torch = pytest.importorskip("torch")
    fmms = []
    for kt, n, geo, seed in ((321, 3000, "sphere", 7), (321, 5000, "ellipsoid", 8), (521, 2500, "sphere", 9),
                             (521, 4000, "sphere", 10)):
        p, nor = W.GEOMETRIES[geo](n, seed)
        f = kifmm.FMM3d("fmm3d_")
        f.srcpos, f.srcnor, f.trgpos = p, nor, p
        f.knl = kifmm.Kernel3d(kt, [1.0, 0.3])
        f.setup({"-fmm3d_np": "4", "-fmm3d_let3d_ptsmax": "60", "-fmm3d_let3d_maxlevel": "10",
                 "-fmm3d_precision": precision})
        fmms.append(f)
    rng = np.random.default_rng(9)
    srcs, outs, want = [], [], []
    for f in fmms:
        s = torch.tensor(rng.uniform(-1, 1, 2 * f.sdof() * f.ns), device="cuda", dtype=torch.float64)
        ref = torch.zeros(2 * f.tdof() * f.nt, device="cuda", dtype=torch.float64)
        f.eval_device(s.data_ptr(), ref.data_ptr(), 2, 0, sync=True)
        srcs.append(s)
        outs.append(torch.zeros_like(ref))
        want.append(ref.cpu().numpy())
    b = kifmm.Batch(fmms)
    b.eval([s.data_ptr() for s in srcs], [o.data_ptr() for o in outs], 2, 0, sync=True)
    assert b.info()["forests"] == 2
    for f, o, w in zip(fmms, outs, want):
        got = o.cpu().numpy()
        assert np.linalg.norm(got - w) <= tol * np.linalg.norm(w), (f.knl.kt, np.linalg.norm(got - w) / np.linalg.norm(w))
