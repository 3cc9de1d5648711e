"""The benchmark configurations at full size against the reference's own
results on the same inputs (fixtures tests/golden/cfg_*.npz, made by
tests/golden/make_config_golden.py from the reference compiled here):

  laplace_sphere_np4               32,768 points on the unit sphere, kernel 111, np=4, ptsmax 100
  stokes_dl_ellipsoid_np6         262,144 points on the (1, .5, .25) ellipsoid, kernel 321, np=6
  navier_sphere_np8             1,048,576 points on the unit sphere, kernel 511 (nu=.3), np=8, ptsmax 150
  laplace_cube_plummer_np6_262k   262,144 points, 70 % cube + 30 % Plummer, kernel 111, np=6, ptsmax 64

Tolerances (the acceptance rule for this path, stated per test):
  * FP64 engine: error against the reference's direct sum at the check
    targets <= 10 x the reference's own error there, and distance to the
    reference's eval output at the same targets <= the same bound;
  * mixed engine: error <= max(10 x the reference's error, 1e-5).
The CPU tests check that the regenerated inputs are the fixture's inputs
(checksums) and that the oracle's direct sum reproduces the reference's at
the check targets to 1e-12.
"""
import os

import numpy as np
import pytest

import golden_cases as G
import oracle
import workloads as W

CONFIGS = G.config_names()
FP64_FACTOR = 10.0
MIXED_FLOOR = 1e-5


def inputs(d):
    wl = W.WORKLOADS[d["workload"]]
    p, nor = wl.points(d["n"])
    den = wl.density(d["n"])
    return wl, p, nor, den


def checksums(p, nor, den):
    w = np.arange(1, len(p) + 1, dtype=np.float64)
    return np.array([p.sum(), (p[:, 0] * w).sum(), nor.sum(), (nor[:, 2] * w).sum(), den.sum(),
                     (den * np.arange(1, den.size + 1)).sum()])


def test_every_benchmark_configuration_is_pinned():
    assert set(CONFIGS) >= {"laplace_sphere_np4", "stokes_dl_ellipsoid_np6", "navier_sphere_np8",
                            "laplace_cube_plummer_np6_262k"}


@pytest.mark.parametrize("name", CONFIGS)
def test_regenerated_inputs_are_the_fixture_inputs(name):
    d = G.load_config(name)
    _, p, nor, den = inputs(d)
    assert np.allclose(checksums(p, nor, den), d["checksums"], rtol=1e-13, atol=1e-9)


@pytest.mark.parametrize("name", ["laplace_sphere_np4", "stokes_dl_ellipsoid_np6", "laplace_cube_plummer_np6_262k"])
def test_oracle_direct_sum_matches_reference_at_size(name):
    d = G.load_config(name)
    _, p, nor, den = inputs(d)
    chk = d["chk"][:200]
    v = oracle.direct(d["kt"], d["coefs"], p, nor, den, p[chk]).reshape(-1, d["ref_direct"].shape[1])
    ref = d["ref_direct"][:200]
    assert np.linalg.norm(v - ref) <= 1e-12 * np.linalg.norm(ref)


def run_engine(d, precision):
    import kifmm
    _, p, nor, den = inputs(d)
    f = kifmm.FMM3d("fmm3d_")
    f.srcpos, f.srcnor, f.trgpos = p, nor, p
    f.knl = kifmm.Kernel3d(d["kt"], list(d["coefs"]))
    f.setup({"-fmm3d_np": str(d["np_"]), "-fmm3d_let3d_ptsmax": str(d["ptsmax"]),
             "-fmm3d_let3d_maxlevel": str(d["maxlevel"]), "-fmm3d_precision": precision})
    td = W.KERNEL_DOFS[d["kt"]][1]
    out = np.zeros(td * d["n"])
    f.eval(den, out)
    return out.reshape(-1, td)[d["chk"]]


@pytest.mark.gpu
@pytest.mark.parametrize("name", CONFIGS)
def test_fp64_engine_matches_reference_at_size(gpu, name):
    d = G.load_config(name)
    got = run_engine(d, "fp64")
    bound = FP64_FACTOR * d["ref_relerr"]
    err = oracle.relerr(got, d["ref_direct"])
    assert err <= bound, (err, d["ref_relerr"])
    diff = float(np.linalg.norm(got - d["ref_val_chk"]) / np.linalg.norm(d["ref_val_chk"]))
    assert diff <= bound, (diff, d["ref_relerr"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", CONFIGS)
def test_mixed_engine_matches_reference_at_size(gpu, name):
    d = G.load_config(name)
    got = run_engine(d, "mixed")
    err = oracle.relerr(got, d["ref_direct"])
    assert err <= max(FP64_FACTOR * d["ref_relerr"], MIXED_FLOOR), (err, d["ref_relerr"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_stokes_instance_matches_reference_error(gpu, precision):
    """The batched workload's largest-error Stokes instance (index 11: 75,496
    points of the Plummer ball, kernel 311, np=6, 8 density vectors in one
    pass) against the reference's own error on it, for density vectors 0 and
    7 (tests/golden/batched_stokes_ref.npz): within 10x, and the bench's
    per-instance bound max(1e-5, 10 x the reference)."""
    import kifmm
    z = np.load(os.path.join(G.GOLDEN, "batched_stokes_ref.npz"))
    ref = dict(zip(z["index"].tolist(), z["ref_relerr"].tolist()))
    inst = W.batched_instances()[11]
    n, rhs = inst["n"], 8
    p, _ = W.GEOMETRIES[inst["geometry"]](n, inst["seed"])
    den = W.densities(n * rhs, 3, "uniform", inst["seed"] + 1)
    f = kifmm.FMM3d("fmm3d_")
    f.srcpos = f.srcnor = f.trgpos = p
    f.knl = kifmm.Kernel3d(inst["kt"], list(inst["coefs"]))
    f.setup({"-fmm3d_np": "6", "-fmm3d_let3d_ptsmax": "64", "-fmm3d_let3d_maxlevel": "10",
             "-fmm3d_precision": precision})
    out = np.zeros((rhs, 3 * n))
    f.eval_multi(den.reshape(rhs, 3 * n), out)
    chk = W.check_indices(n, 256, inst["seed"] + 2)
    for k, r in enumerate((0, rhs - 1)):
        dr = den[r * n * 3:(r + 1) * n * 3]
        direct = f.direct(dr, p[chk]).reshape(-1, 3)
        got = out[r].reshape(-1, 3)[chk]
        err = oracle.relerr(got, direct)
        assert err <= 10 * ref[11][k], (r, err, ref[11][k])
