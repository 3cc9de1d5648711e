"""The setup-time autotuner (-fmm3d_autotune 1, kifmm_schedule).

It times the candidate schedules -- the FP16 tensor-core Hadamard's producer
warp groups (2 or 3) and the density vectors one pass of the surface
contractions carries (1, 2, 4, ... up to the tuned vector count) -- on the
engine itself and keeps the fastest.  None of these knobs changes what is
computed, only its order on the device, so every schedule must give the
same potentials as the default one to FP32 rounding.
"""
import numpy as np
import pytest

import golden_cases as G
import kifmm
import oracle

pytestmark = pytest.mark.gpu


def engine(d, precision, extra=None):
    f = kifmm.FMM3d("fmm3d_")
    f.srcpos, f.srcnor, f.trgpos = d["src"], d["nor"], d["trg"]
    f.ctr, f.rootlvl = tuple(d["ctr"]), d["rootlvl"]
    f.knl = kifmm.Kernel3d(d["kt"], d["coefs"])
    o = G.options(d, precision)
    o.update(extra or {})
    f.setup(o)
    return f


def multi(f, d, rhs):
    den = np.stack([d["den"] * (1.0 + 0.25 * r) + 0.01 * r for r in range(rhs)])
    out = np.zeros((rhs, f.tdof() * len(d["trg"])))
    f.eval_multi(den, out)
    return out


@pytest.mark.parametrize("name,precision", [("lap_s_np6_tt_style", "mixed"), ("lap_s_np6_tt_style", "fp64"),
                                            ("stk_s_np6_cube", "mixed")])
def test_autotuner_picks_a_schedule_with_the_same_results(gpu, name, precision):
    d = G.load(name)
    rhs = 4
    base = engine(d, precision)
    sb = base.schedule()
    assert sb["autotuned"] == 0 and sb["had_groups"] == 3 and sb["rhs_chunk"] == 0
    want = multi(base, d, rhs)
    f = engine(d, precision, {"-fmm3d_autotune": "1", "-fmm3d_autotune_rhs": str(rhs)})
    s = f.schedule()
    assert s["autotuned"] == 1 and s["candidates"] >= 3 and s["best_ms"] > 0
    assert s["had_groups"] in (2, 3) and s["rhs_chunk"] in (1, 2, 4)
    assert f.setup_times()["autotune"] > 0
    got = multi(f, d, rhs)
    tol = 1e-12 if precision == "fp64" else 1e-6
    assert np.linalg.norm(got - want) <= tol * np.linalg.norm(want)
    # a second setup with the same key takes the cached choice
    g = engine(d, precision, {"-fmm3d_autotune": "1", "-fmm3d_autotune_rhs": str(rhs)})
    sg = g.schedule()
    assert sg["from_cache"] == 1 and (sg["had_groups"], sg["rhs_chunk"]) == (s["had_groups"], s["rhs_chunk"])
    # a knob given as an option is kept, the other one tuned
    h = engine(d, precision, {"-fmm3d_autotune": "1", "-fmm3d_autotune_rhs": "2", "-fmm3d_rhs_chunk": "1",
                              "-fmm3d_had_groups": "2"})
    sh = h.schedule()
    assert sh["rhs_chunk"] == 1 and sh["had_groups"] == 2


@pytest.mark.parametrize("chunk", [1, 2, 3])
def test_every_rhs_chunk_gives_the_reference_accuracy(gpu, chunk):
    d = G.load("lap_s_np6_tt_style")
    f = engine(d, "mixed", {"-fmm3d_rhs_chunk": str(chunk)})
    out = multi(f, d, 3)
    for r in range(3):
        den = d["den"] * (1.0 + 0.25 * r) + 0.01 * r
        direct = oracle.direct(d["kt"], d["coefs"], d["src"], d["nor"], den, d["trg"][d["chk"]])
        assert oracle.relerr(out[r][d["chk"]], direct) <= max(10 * d["ref_relerr"], 1e-5)
