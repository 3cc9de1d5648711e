"""The non-homogeneous operator path (-fmm3d_operators per_level).

The reference builds its translation operators once at level 0 and rescales
them by 2^(+-l deg) when the kernel is homogeneous, and otherwise builds
them at every level's radius R = 2^-l with no rescaling
(fmm3d/matmgnt3d.cpp:93-361, the _hom == false branches).  Every kernel the
reference's FMM3d accepts is homogeneous, so the second branch only runs
here when asked for.  The two forms compute the same sums:

  * Laplace (degree 1) and Navier (degree 1 in every dof) scale all singular
    values of a level's surface-to-surface matrices alike, so the truncated
    pseudo-inverses keep the same ranks and the results agree to rounding
    (1e-10 relative, FP64);
  * Stokes (degrees 1, 1, 1, 2) rescales its pressure dof differently, so
    the truncation at 0.1^(np+1) keeps slightly different spectra per
    level: both results stay within 10 x the reference's own error against
    the direct sum.
"""
import numpy as np
import pytest

import golden_cases as G
import kifmm
import oracle
import workloads as W

pytestmark = pytest.mark.gpu


def run(d, precision, operators):
    f = kifmm.FMM3d("fmm3d_")
    f.srcpos, f.srcnor, f.trgpos = d["src"], d["nor"], d["trg"]
    f.ctr, f.rootlvl = tuple(d["ctr"]), d["rootlvl"]
    f.knl = kifmm.Kernel3d(d["kt"], d["coefs"])
    o = G.options(d, precision)
    o["-fmm3d_operators"] = operators
    f.setup(o)
    td = W.KERNEL_DOFS[d["kt"]][1]
    out = np.zeros(td * len(d["trg"]))
    f.eval(d["den"], out)
    return out.reshape(-1, td)


@pytest.mark.parametrize("name,tol", [("lap_s_np6_tt_style", 1e-10), ("lap_s_np4_rootlvl1", 1e-10),
                                      ("lap_s_np8_plummer", 1e-10), ("lap_d_np4_cube", 1e-10),
                                      ("nav_s_np6_sphere", 1e-10), ("stk_s_np6_cube", None),
                                      ("stk_d_np6_ellipsoid", None)])
def test_per_level_operators_match_the_scaled_ones(gpu, name, tol):
    d = G.load(name)
    scaled = run(d, "fp64", "scaled")
    lev = run(d, "fp64", "per_level")
    bound = 10 * d["ref_relerr"] + 1e-13
    for out in (scaled, lev):
        err = oracle.relerr(out[d["chk"]], d["ref_direct"])
        assert err <= bound, (err, d["ref_relerr"])
    diff = np.linalg.norm(lev - scaled) / np.linalg.norm(scaled)
    assert diff <= (tol if tol is not None else bound), diff


@pytest.mark.parametrize("name", ["lap_s_np6_tt_style", "stk_s_np6_cube"])
def test_per_level_operators_in_mixed_precision(gpu, name):
    d = G.load(name)
    out = run(d, "mixed", "per_level")
    err = oracle.relerr(out[d["chk"]], d["ref_direct"])
    assert err <= max(10 * d["ref_relerr"], 1e-5), (err, d["ref_relerr"])
