"""The C-ABI boundary (include/kifmm.h): the library loads, exports every
declared entry point, and turns the reference's assert paths into status
codes.  No compute is launched here; on a machine without a GPU, setup
stops with KIFMM_ERR_NO_DEVICE after building the host tree."""
import ctypes
import os

import numpy as np
import pytest

import kifmm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_header_symbol():
    L = kifmm.lib()
    declared = kifmm.header_symbols(os.path.join(ROOT, "include", "kifmm.h"))
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    assert set(declared) == set(kifmm.SIGNATURES), set(declared) ^ set(kifmm.SIGNATURES)


def test_status_strings():
    L = kifmm.lib()
    for code in kifmm.STATUS:
        assert L.kifmm_status_string(code).decode()
    assert L.kifmm_status_string(0).decode() == "ok"


def make(kt=111, n=500, coefs=(1.0, 0.25), seed=0):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-1, 1, (n, 3))
    f = kifmm.FMM3d("fmm3d_")
    f.srcpos = p
    f.srcnor = p
    f.trgpos = p
    f.knl = kifmm.Kernel3d(kt, coefs)
    return f


OPTS = {"-fmm3d_np": "4", "-fmm3d_let3d_ptsmax": "50", "-fmm3d_let3d_maxlevel": "10"}


def setup_ok(f, opts=OPTS):
    """setup() must succeed on a GPU box and stop at the device stage elsewhere."""
    try:
        f.setup(opts)
        return True
    except kifmm.KifmmError as e:
        assert e.status == kifmm.KIFMM_ERR_NO_DEVICE, e
        return False


def test_missing_options_are_errors():
    for drop in OPTS:
        o = dict(OPTS)
        del o[drop]
        with pytest.raises(kifmm.KifmmError) as ei:
            make().setup(o)
        assert ei.value.status == kifmm.KIFMM_ERR_OPTION


def test_option_values_parse_like_the_reference():
    # option files carry trailing %comments (fmm3d/options_0); only the first token counts
    o = dict(OPTS)
    o["-fmm3d_np"] = "4\t\t%np=4 low accuracy"
    setup_ok(make(), o)
    o["-fmm3d_np"] = "abc"
    with pytest.raises(kifmm.KifmmError) as ei:
        make().setup(o)
    assert ei.value.status == kifmm.KIFMM_ERR_OPTION


def test_unsupported_np_and_precision():
    for key, val in (("-fmm3d_np", "9"), ("-fmm3d_np", "1"), ("-fmm3d_precision", "bf16")):
        o = dict(OPTS)
        o[key] = val
        with pytest.raises(kifmm.KifmmError) as ei:
            make().setup(o)
        assert ei.value.status == kifmm.KIFMM_ERR_OPTION


def test_engine_option_ranges():
    # the engine's own keys: out-of-range values are option errors before any device work
    for key, val in (("-fmm3d_had_groups", "4"), ("-fmm3d_rhs_chunk", "9"), ("-fmm3d_rhs_chunk", "-1"),
                     ("-fmm3d_autotune", "2"), ("-fmm3d_autotune_rhs", "0"), ("-fmm3d_autotune_rhs", "65"),
                     ("-fmm3d_wait_limit", "-1"), ("-fmm3d_m2l_form", "fft"), ("-fmm3d_tree", "gpu"),
                     ("-fmm3d_operators", "homogeneous")):
        o = dict(OPTS)
        o[key] = val
        with pytest.raises(kifmm.KifmmError) as ei:
            make().setup(o)
        assert ei.value.status == kifmm.KIFMM_ERR_OPTION, (key, val)
    o = dict(OPTS, **{"-fmm3d_rhs_chunk": "4", "-fmm3d_autotune": "1", "-fmm3d_autotune_rhs": "8",
                      "-fmm3d_had_groups": "2"})
    setup_ok(make(), o)
    # the per-level (non-homogeneous) operators run with the direct V-list form, np 4, 6 or 8
    for extra in ({"-fmm3d_m2l_form": "toeplitz"}, {"-fmm3d_np": "5"}):
        o = dict(OPTS, **{"-fmm3d_operators": "per_level"}, **extra)
        with pytest.raises(kifmm.KifmmError) as ei:
            make().setup(o)
        assert ei.value.status == kifmm.KIFMM_ERR_OPTION, extra
    setup_ok(make(), dict(OPTS, **{"-fmm3d_operators": "per_level", "-fmm3d_m2l_form": "direct"}))


@pytest.mark.parametrize("kt", [191, 331, 391, 392, 531, 591, 592, 301, 0, -1])
def test_kernels_rejected_by_fmm3d_setup(kt):
    # fmm3d/fmm3d_setup.cpp:53 rejects every kernel without an equivalent kernel
    with pytest.raises(kifmm.KifmmError) as ei:
        make(kt=kt).setup(OPTS)
    assert ei.value.status == kifmm.KIFMM_ERR_KERNEL


def test_missing_coefficients_rejected():
    with pytest.raises(kifmm.KifmmError) as ei:
        make(kt=511, coefs=(1.0,)).setup(OPTS)
    assert ei.value.status == kifmm.KIFMM_ERR_KERNEL


def test_point_outside_root_box():
    f = make()
    p = f.srcpos.copy()
    p[7, 1] = 1.0000001
    f.srcpos = p
    f.srcnor = p
    f.trgpos = p
    with pytest.raises(kifmm.KifmmError) as ei:
        f.setup(OPTS)
    assert ei.value.status == kifmm.KIFMM_ERR_OUT_OF_BOX


def test_box_boundary_is_inside():
    f = make()
    p = f.srcpos.copy()
    p[3] = (1.0, -1.0, 1.0)  # the reference's box test is inclusive (fmm3d/let3d.cpp:73)
    f.srcpos = p
    f.srcnor = p
    f.trgpos = p
    setup_ok(f)


def test_eval_before_setup_is_a_state_error():
    L = kifmm.lib()
    h = ctypes.c_void_p()
    assert L.kifmm_create(b"fmm3d_", ctypes.byref(h)) == 0
    x = np.zeros(4)
    dp = ctypes.POINTER(ctypes.c_double)
    assert L.kifmm_eval(h, x.ctypes.data_as(dp), x.ctypes.data_as(dp)) == kifmm.KIFMM_ERR_STATE
    assert L.kifmm_setup(h) == kifmm.KIFMM_ERR_STATE  # no geometry, no kernel
    assert L.kifmm_destroy(h) == 0


def test_null_arguments():
    L = kifmm.lib()
    assert L.kifmm_create(b"x", None) == kifmm.KIFMM_ERR_ARG
    assert L.kifmm_setup(None) == kifmm.KIFMM_ERR_ARG
    assert L.kifmm_destroy(None) == kifmm.KIFMM_ERR_ARG
    h = ctypes.c_void_p()
    L.kifmm_create(b"fmm3d_", ctypes.byref(h))
    assert L.kifmm_set_geometry(h, -1, None, None, 0, None) == kifmm.KIFMM_ERR_ARG
    assert L.kifmm_set_geometry(h, 3, None, None, 0, None) == kifmm.KIFMM_ERR_ARG
    L.kifmm_destroy(h)


def test_custom_prefix():
    f = make()
    g = kifmm.FMM3d("myfmm_")
    g.srcpos, g.srcnor, g.trgpos, g.knl = f.srcpos, f.srcnor, f.trgpos, f.knl
    with pytest.raises(kifmm.KifmmError):
        g.setup(OPTS)  # keys carry the wrong prefix
    setup_ok(g, {k.replace("fmm3d_", "myfmm_"): v for k, v in OPTS.items()})


def test_empty_target_and_source_sets():
    f = make(n=0)
    assert setup_ok(f) in (True, False)
    assert f.tree()["depth"].tolist() == [0]


def test_mex_front_end_checks_its_arguments():
    """fmm3d_mex mirrors fmm3d/fmm3d_mex.cpp's 8 arguments; its asserts
    (np in {4, 6, 8}, srcden size, 3 x n matrices) raise before any device
    work, and valid arguments reach setup (KIFMM_ERR_NO_DEVICE without a GPU)."""
    rng = np.random.default_rng(3)
    p = rng.uniform(-1, 1, (3, 200))
    den = rng.uniform(-1, 1, 200)
    with pytest.raises(ValueError):
        kifmm.fmm3d_mex(p, p, p, (0, 0, 0), 0, (111, [1.0]), 5, den)
    with pytest.raises(ValueError):
        kifmm.fmm3d_mex(p, p, p, (0, 0, 0), 0, (111, [1.0]), 4, den[:-1])
    with pytest.raises(ValueError):
        kifmm.fmm3d_mex(p.T, p.T, p.T, (0, 0, 0), 0, (111, [1.0]), 4, den)
    with pytest.raises(ValueError):
        kifmm.fmm3d_mex(p, p, p, (0, 0), 0, (111, [1.0]), 4, den)
    try:
        out = kifmm.fmm3d_mex(p, p, p, (0, 0, 0), 0, (111, [1.0]), 4, den)
        assert out.shape == (200,)
    except kifmm.KifmmError as e:
        assert e.status == kifmm.KIFMM_ERR_NO_DEVICE, e
