"""KIFMM evaluation benchmark (one JSON line on rank 0).

Workload: Laplace single-layer (kernel 111), np=6, ptsmax=64, maxlevel=10,
N = 4,194,304 points, 70% uniform in [-1,1]^3 and 30% from a Plummer ball
(scale 0.1, centre (0.3, 0.2, -0.4)), sources = targets, densities U[-1,1],
seeded synthetic data (no dataset is involved).  A step is one FMM3d::eval
(device-resident densities in, device-resident potentials out) of that whole
point cloud; setup (tree, lists, operators) is done once, outside timing.

  value      Mpoints/s of the mixed-precision engine (FP32 point sums and
             spectra, V-list Hadamard and surface contractions in split TF32
             on the tensor cores), all ranks together
  fp64       the plain FP64 GPU engine on the same workload
  batched    64 independent instances (48 Laplace + 16 Stokes single-layer,
             np=6, log-uniform sizes in [1e4, 5e5], sphere / cube / Plummer
             ball), 8 density vectors each, as one captured CUDA graph:
             aggregate point-evaluations/s, mixed and FP64, with per-instance
             errors against the direct sum
  e2e        Mpoints/s through the host-pointer C API (kifmm_eval): H2D of the
             densities and D2H of the potentials inside the timed region
  relerr     ||fmm - direct|| / ||fmm|| at 4096 check targets against the
             FP64 direct sum (the reference's FMM3d::check metric)
  cpu_baseline  the reference's own CPU eval (oracle/_ref, built from the
             reference sources) on a 65,536-point sample of the same cloud,
             one host thread, rank 0 at N=1 only
  roofline   the dominant kernel, k_m2l_had_tc (V-list Hadamard): algorithmic
             flops (8 per V-list pair and stored frequency) over its CUDA-event
             time against the TF32 dense rate (half the measured bf16 rate),
             with the executed tensor rate, the algorithmic HBM rate and the
             DRAM traffic scaled from an ncu capture beside it

--impl reference runs the reference's CPU eval instead, one process per host
core on independent 65,536-point samples, and reports their aggregate.

Multi-GPU (torchrun): every rank evaluates its own replica of the workload
(the single-instance FMM does not shard), so scaling is weak and the value is
the total points of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "kernel-independent-fast-multipole-method_b200")
sys.path.insert(0, PKG)

import workloads as W  # noqa: E402

N_POINTS = 4194304
SAMPLE = 65536
NCHK = 4096
OPTS = {"-fmm3d_np": "6", "-fmm3d_let3d_ptsmax": "64", "-fmm3d_let3d_maxlevel": "10"}
METRIC = "Mpoints/s per FMM eval at rel err <=1e-5: batched FP32 vs plain FP64 GPU"
WORKLOAD = "laplace_cube_plummer_np6"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--n", type=int, default=N_POINTS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ---------------------------------------------------------------------------
# reference arm / CPU baseline
# ---------------------------------------------------------------------------
def _ref_worker(n, steps, warmup, seed):
    """One reference instance: setup + warmup + timed evals.  Prints JSON."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    p, _ = W.cube_plummer(n, seed)
    den = W.densities(n, 1, "uniform", 1 + seed)
    val, times = oracle.ref_fmm(111, [1.0], 6, 64, 10, np.zeros(3), 0, p, p, p, den, neval=warmup + steps)
    print(json.dumps({"setup_s": times[0], "evals_s": list(times[1 + warmup:])}))


def run_reference_procs(nproc, n, steps, warmup):
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
    procs = [subprocess.Popen([sys.executable, os.path.abspath(__file__), "--_ref-worker", str(n), str(steps),
                               str(warmup), str(i)], stdout=subprocess.PIPE, stderr=subprocess.PIPE, env=env, text=True)
             for i in range(nproc)]
    outs = []
    for pr in procs:
        o, e = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError(f"reference worker failed: {e[-500:]}")
        outs.append(json.loads(o.strip().splitlines()[-1]))
    return outs


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_available():
        try:
            oracle.build(ref=True)
        except Exception:
            pass
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref/libkifmm_ref.so not built"}))
        return
    nproc = max(1, min(host_cores(), 64))
    outs = run_reference_procs(nproc, SAMPLE, args.steps, args.warmup)
    # step k = the k-th eval of every process, running concurrently
    step_s = [max(o["evals_s"][k] for o in outs) for k in range(args.steps)]
    ms = 1e3 * statistics.mean(step_s)
    value = nproc * SAMPLE / (ms / 1e3) / 1e6
    line = {"metric": METRIC, "value": value, "unit": "Mpoints/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "n_points_per_instance": SAMPLE, "instances": nproc, "kernel": 111,
                       "np": 6, "ptsmax": 64, "maxlevel": 10, "precision": "fp64 (reference CPU)"},
            "cpu_baseline": {"value": value, "unit": "Mpoints/s", "cores": nproc, "kind": "reference",
                             "sample": f"{nproc} independent {SAMPLE}-point instances of the workload's cloud, "
                                       f"one reference process per core, OPENBLAS_NUM_THREADS=1"},
            "e2e": {"value": value, "unit": "Mpoints/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index: int):
        self.proc = None
        self.rows = []
        self.idx = gpu_index

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.idx)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.th.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower().startswith("active"):
                        reasons.add(nm)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# engine arm
# ---------------------------------------------------------------------------
def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def peak_bf16():
    """Measured dense bf16 TFLOP/s (burst) of this pool's B200s, else None."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"])
    except Exception:
        return None


BATCH_RHS = 8
BATCH_NCHK = 256


def batched_section(torch, kifmm, stream, flush, steps, warmup, precision, pg=None):
    """64 independent instances (48 Laplace + 16 Stokes single-layer, np=6,
    log-uniform sizes in [1e4, 5e5], sphere / cube / Plummer ball), 8 density
    vectors each, evaluated as one captured CUDA graph (kifmm_batch_eval_device).
    Returns the aggregate point-evaluations per second and per-instance errors
    against the FP64 direct sum (first and last density vector, 256 targets)."""
    insts = W.batched_instances()
    fmms, srcs, outs, dens, pts = [], [], [], [], []
    t0 = time.perf_counter()
    for inst in insts:
        p, _ = W.GEOMETRIES[inst["geometry"]](inst["n"], inst["seed"])
        f = kifmm.FMM3d("fmm3d_")
        f.srcpos = f.srcnor = f.trgpos = p
        f.knl = kifmm.Kernel3d(inst["kt"], list(inst["coefs"]))
        o = dict(OPTS)
        o["-fmm3d_precision"] = precision
        f.setup(o)
        sd, td = W.KERNEL_DOFS[inst["kt"]]
        den = W.densities(inst["n"] * BATCH_RHS, sd, "uniform", inst["seed"] + 1)
        fmms.append(f)
        dens.append(den)
        pts.append(p)
        srcs.append(torch.tensor(den, device="cuda", dtype=torch.float64))
        outs.append(torch.zeros(inst["n"] * td * BATCH_RHS, device="cuda", dtype=torch.float64))
    setup_s = time.perf_counter() - t0
    b = kifmm.Batch(fmms)
    sp, op = [s.data_ptr() for s in srcs], [o.data_ptr() for o in outs]
    for _ in range(warmup):
        b.eval(sp, op, BATCH_RHS, stream.cuda_stream, sync=True)
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        b.eval(sp, op, BATCH_RHS, stream.cuda_stream, sync=False)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = statistics.mean(times)
    if pg is not None:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    launches = int(sum(f.last_launch_count() for f in fmms))
    world = pg.get_world_size() if pg is not None else 1
    errs = []
    for inst, f, den, p, out in zip(insts, fmms, dens, pts, outs):
        n = inst["n"]
        sd, td = W.KERNEL_DOFS[inst["kt"]]
        chk = W.check_indices(n, BATCH_NCHK, inst["seed"] + 2)
        val = out.cpu().numpy().reshape(BATCH_RHS, n, td)
        for r in (0, BATCH_RHS - 1):
            direct = f.direct(den[r * n * sd:(r + 1) * n * sd], p[chk]).reshape(-1, td)
            got = val[r][chk]
            errs.append(float(np.linalg.norm(direct - got) / np.linalg.norm(got)))
    npts = sum(i["n"] for i in insts)
    del b
    return {"value": world * npts * BATCH_RHS / (ms / 1e3) / 1e6, "unit": "Mpoints/s", "ms_per_step": ms,
            "relerr_max": max(errs), "relerr_median": statistics.median(errs), "setup_s": setup_s,
            "launches_per_step": launches, "points_per_instance_total": npts}


def engine_arm(args):
    import torch
    import kifmm
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    n = args.n
    p, _ = W.cube_plummer(n, 0)
    den = W.densities(n, 1, "uniform", 1)

    def make(prec):
        f = kifmm.FMM3d("fmm3d_")
        f.srcpos = f.srcnor = f.trgpos = p
        f.knl = kifmm.Kernel3d(111, [1.0])
        o = dict(OPTS)
        o["-fmm3d_precision"] = prec
        t0 = time.perf_counter()
        f.setup(o)
        return f, time.perf_counter() - t0

    stream = torch.cuda.Stream()
    d_den = torch.tensor(den, device="cuda", dtype=torch.float64)
    d_out = torch.zeros(n, device="cuda", dtype=torch.float64)
    flush = torch.empty(256 * 1024 * 1024 // 4, device="cuda", dtype=torch.float32)  # 256 MB > 126 MB L2

    def barrier():
        if pg is not None:
            pg.barrier()

    def timed(f, steps, warmup, profile=False):
        for _ in range(warmup):
            f.eval_device(d_den.data_ptr(), d_out.data_ptr(), 1, stream.cuda_stream, sync=True)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        times = []
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)  # L2 flush, outside the events
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            f.eval_device(d_den.data_ptr(), d_out.data_ptr(), 1, stream.cuda_stream, sync=False)
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
        barrier()
        ms = statistics.mean(times)
        if pg is not None:
            t = torch.tensor([ms], device="cuda", dtype=torch.float64)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms = float(t.item())
        return ms, times

    # ---- mixed (headline)
    fm, setup_mixed = make("mixed")
    clocks = ClockSampler(local)
    clocks.start()
    ms_mixed, _ = timed(fm, args.steps, args.warmup)
    clk = clocks.stop()
    launches = fm.last_launch_count()
    out_mixed = d_out.cpu().numpy()
    # per-kernel device times of one profiled eval (roofline of the dominant kernel)
    fm.set_profiling(True)
    fm.eval_device(d_den.data_ptr(), d_out.data_ptr(), 1, stream.cuda_stream, sync=True)
    phases = fm.phase_times()
    fm.set_profiling(False)
    wc = fm.work_counters()
    # accuracy (FMM3d::check metric) against the FP64 direct sum on the device
    chk = W.check_indices(n, NCHK, 2)
    direct = fm.direct(den, p[chk])
    relerr = float(np.linalg.norm(direct - out_mixed[chk]) / np.linalg.norm(out_mixed[chk]))
    # ---- e2e through the host-pointer API, pinned host buffers
    h_den = torch.from_numpy(den).pin_memory()
    h_out = torch.zeros(n, dtype=torch.float64).pin_memory()
    hd, ho = h_den.numpy(), h_out.numpy()
    for _ in range(max(1, args.warmup)):
        fm.eval(hd, ho)
    barrier()
    e2e_times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        fm.eval(hd, ho)
        e2e_times.append(time.perf_counter() - t0)
    e2e_ms = 1e3 * statistics.mean(e2e_times)
    if pg is not None:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t.item())
    del fm
    # ---- plain FP64 engine on the same workload
    fp64 = None
    if not args.no_fp64:
        f64, setup_fp64 = make("fp64")
        ms64, _ = timed(f64, max(1, min(args.steps, 5)), 1)
        out64 = d_out.cpu().numpy()
        err64 = float(np.linalg.norm(direct - out64[chk]) / np.linalg.norm(out64[chk]))
        fp64 = {"value": world * n / (ms64 / 1e3) / 1e6, "unit": "Mpoints/s", "ms_per_step": ms64,
                "relerr": err64, "setup_s": setup_fp64, "dtype": "f64"}
        del f64
    # ---- batched form: 64 instances x 8 density vectors in one graph
    batched = None
    if not args.no_batched:
        bsteps, bwarm = max(1, min(args.steps, 5)), max(1, min(args.warmup, 3))
        batched = {"workload": "batched_64x8rhs_np6", "instances": 64, "rhs": BATCH_RHS,
                   "kernels": "48 x Laplace SL (111), 16 x Stokes SL (311)",
                   "sizes": "log-uniform in [1e4, 5e5] points", "geometries": "sphere / cube / Plummer ball",
                   "check": f"{BATCH_NCHK} targets per instance, density vectors 0 and {BATCH_RHS - 1}",
                   "mixed": batched_section(torch, kifmm, stream, flush, bsteps, bwarm, "mixed", pg)}
        if not args.no_fp64:
            batched["fp64"] = batched_section(torch, kifmm, stream, flush, bsteps, bwarm, "fp64", pg)
    # ---- CPU baseline: the reference on a bounded sample, rank 0, N=1
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        if oracle.ref_available():
            o = run_reference_procs(1, SAMPLE, 2, 1)[0]
            s = statistics.mean(o["evals_s"])
            cpu = {"value": SAMPLE / s / 1e6, "unit": "Mpoints/s", "cores": 1, "kind": "reference",
                   "sample": f"one {SAMPLE}-point instance of the workload's cloud, mean of 2 evals after 1 warm-up, "
                             f"reference built from its sources (FFTW2-interface shim, scipy OpenBLAS)"}
        else:
            cpu = {"value": None, "unit": "Mpoints/s", "cores": 1, "kind": "reference",
                   "sample": "reference library not built on this host"}
    if rank != 0:
        return
    hbm, peak_kind = peaks()
    bf16 = peak_bf16()
    # dominant kernel: the V-list Hadamard accumulation on the tensor cores
    # (k_m2l_had_tc).  Algorithmic work = one complex multiply-add (8 flops) per
    # V-list pair and stored frequency; algorithmic bytes = source spectra read
    # once + accumulated target spectra written once + the operator images.
    # Executed tensor work adds the split-TF32 products (head*head, head*tail,
    # tail*head) and the adjacent-child zero blocks of every parent pair.
    nf = 4 * 6 ** 3 + 4  # independent (Hermitian-canonical) frequencies at np=6
    cplx = 8  # FP32 complex
    alg_bytes = (wc["fwd_spectra"] + wc["inv_spectra"]) * nf * cplx + 26 * nf * 2048
    had_ms = phases.get("m2l_hadamard") or phases["vlist"]
    had_flops = wc["v_pairs"] * nf * 8
    had_exec_flops = wc.get("tc_hadamard_flops", 0.0)
    achieved = had_flops / (had_ms / 1e3) / 1e12
    tf32_peak = bf16 / 2 if bf16 else 1590.0 / 2  # TF32 dense = half the bf16 rate
    # DRAM traffic per launch: 14,236 B per spectrum node, read + write, from the
    # ncu capture of this kernel on the 1M-point case (profiles/hadamard_tc_*),
    # scaled by the spectra of this workload
    traffic = 14236.0 * wc["fwd_spectra"]
    line = {
        "metric": METRIC, "value": world * n / (ms_mixed / 1e3) / 1e6, "unit": "Mpoints/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_points": n, "kernel": 111, "np": 6, "ptsmax": 64, "maxlevel": 10,
                   "precision": "mixed (FP32 point sums and spectra; V-list Hadamard and surface contractions "
                                "in split TF32 on tcgen05 with FP32 accumulation; FP64 operator SVDs)", "rhs": 1,
                   "l2": "flushed (256 MB write) before every timed step", "parallelism": f"replicas x{world}"},
        "relerr": relerr, "check_targets": NCHK,
        "fp64": fp64,
        "batched": batched,
        "e2e": {"value": world * n / (e2e_ms / 1e3) / 1e6, "unit": "Mpoints/s",
                "h2d_bytes_per_step": int(n * 8), "d2h_bytes_per_step": int(n * 8), "ms_per_step": e2e_ms},
        "gpu_launches": int(launches * args.steps),
        "launches_per_step": launches,
        "phases_ms": phases,
        "work": wc,
        "setup_s": setup_mixed,
        "roofline": {"bound": "tensor", "kernel": "k_m2l_had_tc (V-list Hadamard on tcgen05, split TF32)",
                     "achieved": achieved, "peak": tf32_peak, "unit": "TFLOP/s", "frac": achieved / tf32_peak,
                     "peak_kind": ("measured" if bf16 else "fallback") + " (TF32 dense = half the bf16 burst)",
                     "traffic": traffic, "traffic_unit": "bytes per launch", "kernel_ms": had_ms,
                     "algorithmic": "8 flops per V-list pair and stored frequency",
                     "executed_tensor_tflops": had_exec_flops / (had_ms / 1e3) / 1e12,
                     "hbm_achieved_gbs": alg_bytes / (had_ms / 1e3) / 1e9, "hbm_peak_gbs": hbm,
                     "limiter": "round trip of each producer group's TMEM A stage (gather loads, wait for the "
                                "stage's previous MMAs, split and store, operator images), one third of it per "
                                "step with three stages; neither the tensor pipe (~18 % active) nor DRAM (~8 % "
                                "of peak) is saturated"},
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "--_ref-worker":
        _ref_worker(int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4]), int(sys.argv[5]))
        return
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        engine_arm(args)


if __name__ == "__main__":
    main()
