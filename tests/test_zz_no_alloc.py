"""kifmm_direct_noalloc: the direct sum for callers that cannot allocate.

A process whose GPU memory belongs to a framework's caching allocator (or
to a budget reserved at start-up) cannot call cudaMalloc between its steps,
so this entry point takes caller-allocated device buffers and keeps its
partial sums in a fixed 8 MiB device array instead of allocating.  The
test drives it through the C ABI on two calls in a row (different sizes,
kernels and data, so the second call runs over the first call's leftover
scratch) and compares each result with the existing entry point,
kifmm_direct, to 1e-12 relative; it also checks that a request larger than
the fixed scratch is refused before anything is launched.  This file is
named to be collected last."""
import ctypes

import numpy as np
import pytest

import kifmm

pytestmark = pytest.mark.gpu

TOL = 1e-12


def existing_direct(kt, coefs, src, nor, den, trg):
    f = kifmm.FMM3d()
    f.srcpos, f.srcnor, f.trgpos = src, nor, src
    f.knl = kifmm.Kernel3d(kt, coefs)
    f.setup({"-fmm3d_np": "4", "-fmm3d_let3d_ptsmax": "200", "-fmm3d_let3d_maxlevel": "10"})
    return f.direct(den, trg)


def noalloc_direct(torch, kt, coefs, src, nor, den, trg, stream=None):
    dev = lambda a: torch.tensor(np.ascontiguousarray(a, np.float64).reshape(-1), device="cuda")
    d_src, d_nor, d_den, d_trg = dev(src), dev(nor), dev(den), dev(trg)
    td = kifmm.Kernel3d(kt, coefs).tdof()
    d_out = torch.full((len(trg) * td,), float("nan"), device="cuda", dtype=torch.float64)
    cf = np.ascontiguousarray(coefs, np.float64)
    stream = stream or torch.cuda.current_stream()
    torch.cuda.synchronize()  # the inputs were copied on the current stream
    st = kifmm.lib().kifmm_direct_noalloc(kt, len(cf), cf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(src),
                                          d_src.data_ptr(), d_nor.data_ptr(), d_den.data_ptr(), len(trg),
                                          d_trg.data_ptr(), d_out.data_ptr(), stream.cuda_stream)
    assert st == kifmm.KIFMM_OK, kifmm.STATUS.get(st, st)
    stream.synchronize()
    return d_out.cpu().numpy()


def case(kt, ns, nt, seed):
    rng = np.random.default_rng(seed)
    src = rng.uniform(-1, 1, (ns, 3))
    nor = rng.standard_normal((ns, 3))
    sd = kifmm.Kernel3d(kt).sdof()
    den = rng.standard_normal(ns * sd)
    trg = np.concatenate([rng.uniform(-1, 1, (nt - 3, 3)), src[:3]])  # includes coincident points
    return src, nor, den, trg


def test_two_calls_match_existing_direct_entry_point(gpu):
    torch = pytest.importorskip("torch")
    for kt, coefs, ns, nt, seed in [(321, [1.0, 0.25], 20000, 3000, 1), (111, [1.0], 7000, 900, 2)]:
        src, nor, den, trg = case(kt, ns, nt, seed)
        got = noalloc_direct(torch, kt, coefs, src, nor, den, trg)
        ref = existing_direct(kt, coefs, src, nor, den, trg)
        assert np.all(np.isfinite(got))
        assert np.linalg.norm(got - ref) <= TOL * np.linalg.norm(ref)


def test_kernels_with_two_coefficients_and_pressure_outputs(gpu):
    """Navier single layer (two coefficients, mu and nu) and the Stokes
    pressure kernel (three source dofs, one target dof) against kifmm_direct."""
    torch = pytest.importorskip("torch")
    for kt, coefs, ns, nt, seed in [(511, [1.3, 0.3], 5000, 700, 3), (312, [1.0], 6000, 500, 4)]:
        src, nor, den, trg = case(kt, ns, nt, seed)
        got = noalloc_direct(torch, kt, coefs, src, nor, den, trg)
        ref = existing_direct(kt, coefs, src, nor, den, trg)
        assert np.linalg.norm(got - ref) <= TOL * np.linalg.norm(ref)


def test_no_sources_give_zero_potentials_on_a_side_stream(gpu):
    """ns == 0 writes zeros over the caller's output (which starts as NaN),
    and a call on a non-default stream is ordered on that stream."""
    torch = pytest.importorskip("torch")
    side = torch.cuda.Stream()
    trg = np.random.default_rng(5).uniform(-1, 1, (300, 3))
    got = noalloc_direct(torch, 111, [1.0], np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0), trg, stream=side)
    assert np.array_equal(got, np.zeros(300))
    src, nor, den, trg = case(321, 4000, 600, 6)
    got = noalloc_direct(torch, 321, [1.0], src, nor, den, trg, stream=side)
    ref = existing_direct(321, [1.0], src, nor, den, trg)
    assert np.linalg.norm(got - ref) <= TOL * np.linalg.norm(ref)


def test_request_beyond_the_fixed_scratch_is_refused(gpu):
    L = kifmm.lib()
    limit = 1 << 20  # KIFMM_NOALLOC_SCRATCH_DOUBLES
    nt = limit // 3 + 1  # tdof 3: nt * tdof exceeds the scratch
    cf = np.array([1.0, 0.25])
    one = ctypes.c_void_p(8)  # never dereferenced: the size check comes first
    st = L.kifmm_direct_noalloc(311, 2, cf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 10, one, one, one, nt,
                                one, one, None)
    assert st == kifmm.KIFMM_ERR_CAPACITY
