"""Failure detection on the GPU without a GPU fault.

Every pipeline wait inside the tensor-core V-list kernel is bounded; a wait
that runs out sets a bit of the engine's device status word and the kernel
returns after its copies have landed and its MMAs have completed.  With
-fmm3d_wait_limit 0 every such wait gives up at once, so these tests make
the time-out happen (nothing hangs, nothing faults) and check that it is
reported -- on the synchronous host API, on an asynchronous eval_device
after the stream is synchronised (kifmm_poll_status), and at the next call
-- and that the CUDA context stays usable.
"""
import numpy as np
import pytest

import golden_cases as G
import kifmm
import oracle

pytestmark = pytest.mark.gpu


def engine(d, extra=None):
    f = kifmm.FMM3d("fmm3d_")
    f.srcpos, f.srcnor, f.trgpos = d["src"], d["nor"], d["trg"]
    f.ctr, f.rootlvl = tuple(d["ctr"]), d["rootlvl"]
    f.knl = kifmm.Kernel3d(d["kt"], d["coefs"])
    o = G.options(d, "mixed")
    o.update(extra or {})
    f.setup(o)
    return f


def test_timed_out_wait_is_reported_and_the_context_stays_usable(gpu):
    d = G.load("lap_s_np6_tt_style")  # single dof: the tensor-core V-list kernel runs
    f = engine(d, {"-fmm3d_wait_limit": "0"})
    out = np.zeros(len(d["trg"]))
    with pytest.raises(kifmm.KifmmError) as e:
        f.eval(d["den"], out)
    assert e.value.status == kifmm.KIFMM_ERR_CUDA and "timed out" in str(e.value)
    f.poll_status()  # the synchronous call has read and cleared the word
    # a fresh engine on the same context evaluates correctly
    g = engine(d)
    good = np.zeros(len(d["trg"]))
    g.eval(d["den"], good)
    err = oracle.relerr(good[d["chk"]], d["ref_direct"])
    assert err <= max(10 * d["ref_relerr"], 1e-5), err


def test_asynchronous_time_out_surfaces_at_poll_and_next_call(gpu):
    torch = pytest.importorskip("torch")
    d = G.load("lap_s_np6_tt_style")
    f = engine(d, {"-fmm3d_wait_limit": "0"})
    sden = torch.tensor(d["den"], device="cuda", dtype=torch.float64)
    tval = torch.zeros(len(d["trg"]), device="cuda", dtype=torch.float64)
    st = torch.cuda.Stream()
    f.eval_device(sden.data_ptr(), tval.data_ptr(), 1, st.cuda_stream, sync=False)  # returns before the kernels ran
    st.synchronize()
    with pytest.raises(kifmm.KifmmError) as e:
        f.poll_status()
    assert e.value.status == kifmm.KIFMM_ERR_CUDA
    f.poll_status()  # read and cleared
    f.eval_device(sden.data_ptr(), tval.data_ptr(), 1, st.cuda_stream, sync=False)
    st.synchronize()
    with pytest.raises(kifmm.KifmmError):  # the next asynchronous call reports the earlier time-out
        f.eval_device(sden.data_ptr(), tval.data_ptr(), 1, st.cuda_stream, sync=False)
    st.synchronize()


def test_batch_replay_reports_an_instance_time_out(gpu):
    torch = pytest.importorskip("torch")
    d = G.load("lap_s_np6_tt_style")
    good, bad = engine(d), engine(d, {"-fmm3d_wait_limit": "0"})
    n = len(d["trg"])
    src = [torch.tensor(d["den"], device="cuda", dtype=torch.float64) for _ in range(2)]
    dst = [torch.zeros(n, device="cuda", dtype=torch.float64) for _ in range(2)]
    b = kifmm.Batch([good, bad])
    st = torch.cuda.Stream()
    with pytest.raises(kifmm.KifmmError) as e:
        b.eval([x.data_ptr() for x in src], [x.data_ptr() for x in dst], 1, st.cuda_stream, sync=True)
    assert "instance 1" in str(e.value)
    ref = np.zeros(n)
    good.eval(d["den"], ref)
    assert np.array_equal(dst[0].cpu().numpy(), ref)  # the healthy instance's result is complete
