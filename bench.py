#!/usr/bin/env python
"""Benchmark: forward+backward Sinkhorn iterations/s of the dictionary-learning
objective (evaluate_both) on the batched 128x128 workload.

One step = one evaluate_both over all P histograms of a rank: L forward Bregman
iterations with the iterate store, the loss, and the reverse pass through the
stored iterates for the atom and weight gradients.  Its unit of work is one
histogram-iteration (P*L per step, all K atoms, forward and backward).

Workload (per rank): P=64 seeded blob histograms (2-5 blobs) on 128x128, K=5
atoms, L=100, gamma=1, KL loss.  Under torchrun each rank owns its own 64
histograms (weak scaling); the dictionary gradient and the loss are summed
across ranks with one NCCL all-reduce per step (the path's only exchange).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision split_bf16|tf32|fp32|fp64]
    python bench.py --impl reference      # the reference's own CPU path (oracle/_ref)

The headline line is the batched 128x128 workload.  `--workload dict64`
(64x64, K=4, L=25, gamma=2, quadratic, FP32 kernel domain) and `--workload
log256` (256x256, K=8, L=200, gamma=0.5, TV, FP32 log domain) measure the
other two dictionary-learning configurations the same way; `--workload
images272` measures the grid of the reference's bundled images (272x240, K=4,
L=50, split-BF16 through the tensor-core axis passes).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd Sinkhorn iters/s (128², K=5) vs plain FP32; p50/p99 serve latency"
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of the
# fused split-BF16 kernel on batched128 (P=64, L=100), from one ncu capture.
FUSED_DRAM_BYTES_P64_L100 = 29.82e9
UNIT = "hist-iter/s"
WORKLOADS = {
    "batched128": dict(name="batched128", P=64, W=128, H=128, K=5, L=100, gamma=1.0, loss=4,
                       loss_name="KL", n_blobs=(2, 5), std_frac=(0.03, 0.12), domain="kernel",
                       precision=None, cpu_P=4, cpu_L=100),
    "dict64": dict(name="dict64", P=16, W=64, H=64, K=4, L=25, gamma=2.0, loss=2,
                   loss_name="quadratic", n_blobs=(1, 3), std_frac=(0.03, 0.12), domain="kernel",
                   precision="fp32", cpu_P=16, cpu_L=25),
    "log256": dict(name="log256", P=32, W=256, H=256, K=8, L=200, gamma=0.5, loss=1,
                   loss_name="TV", n_blobs=(1, 3), std_frac=(0.01, 0.04), domain="log",
                   precision="fp32", cpu_P=1, cpu_L=4),
    # the grid of the reference's bundled heart images (272 x 240), synthetic data
    "images272": dict(name="images272", P=8, W=272, H=240, K=4, L=50, gamma=25.0, loss=2,
                      loss_name="quadratic", n_blobs=(1, 3), std_frac=(0.03, 0.12),
                      domain="kernel", precision=None, cpu_P=1, cpu_L=10),
}


def metric_for(wl):
    if wl["name"] == "batched128":
        return METRIC
    return f"fwd+bwd Sinkhorn iters/s ({wl['W']}x{wl['H']}, K={wl['K']}, {wl['domain']} domain)"


def describe(wl):
    return (f"{wl['name']}: P={wl['P']} per GPU, {wl['W']}x{wl['H']}, K={wl['K']}, L={wl['L']}, "
            f"gamma={wl['gamma']:g}, {wl['loss_name']} loss, {wl['domain']} domain")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched128", choices=sorted(WORKLOADS) + ["uneven512"])
    ap.add_argument("--precision", default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-arms", action="store_true")
    ap.add_argument("--no-regress", action="store_true")
    ap.add_argument("--regress-iters", type=int, default=3)
    ap.add_argument("--serve-rates", default="8,50,200,500,2000")
    ap.add_argument("--serve-requests", type=int, default=120)
    # Reduced sizes for profiler captures (the bench line itself uses the workload's).
    ap.add_argument("--P", type=int, default=None)
    ap.add_argument("--L", type=int, default=None)
    return ap.parse_args()


def default_precision():
    return os.environ.get("WDL_BENCH_PRECISION", "split_bf16")


def dtype_name(precision):
    return {"fp32": "f32", "tf32": "tf32+f32", "split_bf16": "bf16x3+f32", "fp64": "f64"}[precision]


# ---------------------------------------------------------------- CPU arms ---------
def cpu_threads():
    return len(os.sched_getaffinity(0))


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def time_cpu_reference(wl, steps=1, warmup=0):
    """The reference's own evaluate_both (GaussianSSE2DKernel, or the
    LogSignArray kernel in the log domain, OpenMP over all host cores) on a
    bounded sample: wl['cpu_P'] histograms at wl['cpu_L'] iterations."""
    from oracle import oracle as orc
    from wassersteindictionarylearning_b200.synthetic import make_problem, to_variables
    w = wl
    P, L = w["cpu_P"], w["cpu_L"]
    log_domain = w["domain"] == "log"
    cfg, obs, atoms, wts = make_problem(None, seed=0, P=P, W=w["W"], H=w["H"], K=w["K"], L=L,
                                        gamma=w["gamma"], loss=w["loss"], n_blobs=w["n_blobs"],
                                        std_frac=w["std_frac"])
    x = to_variables(wts, atoms, cfg["scale_dic"])
    os.environ.setdefault("OMP_NUM_THREADS", str(cpu_threads()))
    if orc.ref_available():
        lib, kind = orc.RefLib(), "reference"

        def run():
            return lib.evaluate_both(w["W"], w["H"], 1, w["gamma"], P, w["K"], L, w["loss"],
                                     cfg["scale_dic"], x, obs, log_domain=log_domain, kind=1)
        cores = lib.omp_threads()
        what = ("LogSignArrayGaussian2DKernel" if log_domain else "GaussianSSE2DKernel") + \
            " evaluate_both (cpp/inverseWasserstein.h:986), OpenMP"
    else:
        lib, kind = orc.OracleLib(), "port"
        cores = cpu_threads()

        def run():
            return lib.evaluate_both(w["W"], w["H"], 1, w["gamma"], P, w["K"], L, w["loss"],
                                     cfg["scale_dic"], x, obs, log_domain=log_domain,
                                     nthreads=cores)
        what = "C restatement evaluate_both, OpenMP over histograms"
    for _ in range(warmup):
        run()
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
    per_step = statistics.median(times)
    units = P * L
    return dict(value=units / per_step, unit=UNIT, cores=cores, kind=kind,
                sample=f"{what}; {P} of {w['P']} histograms, L={L} of {w['L']} ({w['W']}x{w['H']}, "
                       f"K={w['K']}, {w['loss_name']}), {units} hist-iters per step, median of "
                       f"{steps}; CPU: {cpu_model()}"), per_step


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = WORKLOADS[args.workload]
    base, per_step = time_cpu_reference(wl, steps=args.steps, warmup=min(args.warmup, 1))
    line = dict(metric=metric_for(wl), value=base["value"], unit=UNIT, n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=per_step * 1e3, higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="f64", data="synthetic",
                config=dict(workload=describe(wl), P=wl["cpu_P"], W=wl["W"], H=wl["H"], K=wl["K"],
                            L=wl["cpu_L"], gamma=wl["gamma"], loss=wl["loss_name"],
                            note="bounded sample of the workload"),
                impl="reference", cpu_baseline=base,
                e2e=dict(value=base["value"], unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- clocks ------------
class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        except OSError:
            pass
        finally:
            if self.path:
                os.unlink(self.path)
        return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=mx,
                    reasons=sorted(reasons), samples=len(sm))


# ---------------------------------------------------------------- GPU arm -----------
def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    import wassersteindictionarylearning_b200 as w
    from wassersteindictionarylearning_b200 import _lib
    from wassersteindictionarylearning_b200.parallel import allreduce_atoms_and_loss
    from wassersteindictionarylearning_b200.synthetic import make_problem, to_variables

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    wl = dict(WORKLOADS[args.workload])
    precision = args.precision or wl["precision"] or default_precision()
    if args.P:
        wl["P"] = args.P
    if args.L:
        wl["L"] = args.L
    P, W, H, K, L = wl["P"], wl["W"], wl["H"], wl["K"], wl["L"]
    N = W * H
    cfg, obs, atoms, wts = make_problem(None, seed=1000 * rank, P=P, W=W, H=H, K=K, L=L,
                                        gamma=wl["gamma"], loss=wl["loss"], n_blobs=wl["n_blobs"],
                                        std_frac=wl["std_frac"])
    sd = cfg["scale_dic"]
    x = to_variables(wts, atoms, sd)
    n = x.size
    PK = P * K
    if wl["domain"] == "log":
        kern = w.CudaLogSignArrayGaussian2DKernel(wl["gamma"], W, H, precision=precision, device=local)
    else:
        kern = w.CudaGaussian2DKernel(wl["gamma"], W, H, precision=precision, device=local)
    ctx = kern.ctx
    L_ = _lib.lib()
    dev = torch.device("cuda", local)
    x_d = torch.from_numpy(x).to(dev)
    obs_d = torch.from_numpy(obs.reshape(-1)).to(dev)
    g_d = torch.empty(n, dtype=torch.float64, device=dev)
    f_d = torch.empty(1, dtype=torch.float64, device=dev)
    # An explicit stream: the library runs on it and the CUDA events below are
    # recorded on it (handle 0, the legacy default stream, would mean "the
    # context's own stream" to the C ABI).
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    sptr = C.c_void_p(stream.cuda_stream)

    def step():
        rc = L_.wdl_evaluate_both_device(ctx, P, K, L, wl["loss"], sd, C.c_void_p(x_d.data_ptr()),
                                         C.c_void_p(g_d.data_ptr()), n,
                                         C.c_void_p(obs_d.data_ptr()), C.c_void_p(f_d.data_ptr()),
                                         None, None, None, sptr)
        _lib.check(rc, ctx)
        if world > 1:  # the path's one exchange: dictionary gradient + loss
            allreduce_atoms_and_loss(g_d, f_d, PK, dist)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    tape_gb = L_.wdl_eval_bytes(ctx, P, K, L) / 1e9

    launches0 = L_.wdl_launch_count(ctx)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    ms = ev0.elapsed_time(ev1)
    gpu_launches = L_.wdl_launch_count(ctx) - launches0
    clocks = clk.summary()
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    units = P * L * args.steps * world
    value = units / (ms / 1e3)
    fval = float(f_d.item())

    # Dominant kernel (the separable operator): average duration over one profiled
    # step, with CUDA events on the launching stream, outside the timed loop.
    L_.wdl_set_profiling(ctx, 1)
    step()
    torch.cuda.synchronize()
    conv_ms, conv_launches, conv_imgs = C.c_double(), C.c_longlong(), C.c_double()
    L_.wdl_conv_profile(ctx, C.byref(conv_ms), C.byref(conv_launches), C.byref(conv_imgs))
    exps = C.c_double()
    L_.wdl_exp_profile(ctx, C.byref(exps))
    L_.wdl_set_profiling(ctx, 0)
    tuned = []
    key6, choice, tms = (C.c_longlong * 6)(), C.c_int(), C.c_float()
    for i in range(max(L_.wdl_autotune_count(ctx), 0)):
        if L_.wdl_autotune_entry(ctx, i, key6, C.byref(choice), C.byref(tms)) == 0:
            if key6[0] == 2:  # tensor-core axis pass: output tile height
                tuned.append(dict(kind="tc_axis_pass", rows=key6[1], row_len=key6[2], images=key6[3],
                                  tile_rows=choice.value, ms=round(tms.value, 4)))
            else:  # log-domain axis pass: rows per block
                tuned.append(dict(kind="log_axis_pass", rows=key6[1], row_len=key6[2], images=key6[3],
                                  signed=bool(key6[5]), rows_per_block=choice.value,
                                  ms=round(tms.value, 4)))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    flop_per_img = 2.0 * N * (W + H)  # dense separable contraction, both axes
    products = 3 if precision == "split_bf16" else 1
    conv_launch_ms = conv_ms.value / max(conv_launches.value, 1)
    imgs_per_launch = conv_imgs.value / max(conv_launches.value, 1)
    # algorithmic (useful) FLOPs: one dense contraction per operator application;
    # the split-BF16 form executes three tensor products for each
    achieved_tflops = flop_per_img * imgs_per_launch / (conv_launch_ms * 1e-3) / 1e12
    if wl["domain"] == "log":
        # With the negligible-tail cut the log-sum-exp passes execute a few
        # exps per output (counted on the device), so the operator's floor is
        # HBM: each of the two axis passes reads and writes every image once
        # (4 bytes per value in FP32, 8 in FP64, plus a sign byte each way in
        # the signed reverse pass, not counted here).  The reference evaluates
        # one exp per tap (N*(W+H) per image): reference_equivalent_texp_s.
        mhz = peaks.get("sm_max_mhz", 1965.0)
        esz = 8 if precision == "fp64" else 4
        bytes_per_launch = imgs_per_launch * N * esz * 4
        gbs = bytes_per_launch / (conv_launch_ms * 1e-3) / 1e9
        hbm = peaks.get("hbm_gbs", 6650.0)
        ref_rate = N * (W + H) * imgs_per_launch / (conv_launch_ms * 1e-3) / 1e12
        exec_rate = exps.value / max(conv_launches.value, 1) / (conv_launch_ms * 1e-3) / 1e12
        sfu_peak = 148 * 16 * mhz * 1e6 / 1e12
        roofline = dict(bound="hbm", achieved=gbs, peak=hbm, unit="GB/s", frac=gbs / hbm,
                        traffic=None,
                        peak_source="of measured HBM copy bandwidth" if "hbm_gbs" in peaks else "of fallback",
                        kernel=f"log-domain separable operator: one launch = {imgs_per_launch:.0f} images "
                               "(two log-sum-exp axis passes)",
                        algorithmic_bytes_per_launch=bytes_per_launch,
                        executed_texp_s=exec_rate, sfu_peak_texp_s=sfu_peak,
                        reference_equivalent_texp_s=ref_rate,
                        executed_exp_share=exps.value / max(conv_imgs.value * N * (W + H), 1),
                        conv_share_of_step=conv_ms.value / (ms / args.steps))
    elif precision in ("split_bf16", "tf32"):
        peak = peaks.get("bf16_tflops", 1590.0) * (0.5 if precision == "tf32" else 1.0)
        peak_src = "of measured bf16 burst" if peaks else "of fallback"
        bound = "tensor"
    else:
        # CUDA-core FMA peak: 148 SMs x 128 lanes x 2 flop x max SM clock (nominal)
        mhz = peaks.get("sm_max_mhz", 1965.0)
        peak = 148 * 128 * 2 * mhz * 1e6 / 1e12 / (2.0 if precision == "fp64" else 1.0)
        peak_src = "of nominal CUDA-core FMA peak at max clock"
        bound = "fp32-cuda-core" if precision == "fp32" else "fp64-cuda-core"
    if wl["domain"] != "log":
        # DRAM bytes (read + write) of one fused launch at P=64, L=100, from a
        # one-pass ncu capture of this workload, scaled by P*L
        traffic = (FUSED_DRAM_BYTES_P64_L100 * (P * L) / (64 * 100)
                   if wl["name"] == "batched128" and precision == "split_bf16" else None)
        roofline = dict(bound=bound, achieved=achieved_tflops, peak=peak, unit="TFLOP/s",
                        frac=achieved_tflops / peak, traffic=traffic, peak_source=peak_src,
                        algorithmic_bytes_per_launch=8.0 * K * N * 4 * P * L,
                        executed_tflops=achieved_tflops * products,
                        ceiling_frac=1.0 / products,
                        kernel=(f"fused Sinkhorn kernel: one launch = {imgs_per_launch:.0f} separable-operator "
                                "applications (whole forward + reverse pass)"
                                if precision in ("split_bf16", "tf32") and W <= 128 and H <= 128
                                else f"separable Gaussian operator ({'tensor-core axis passes' if precision in ('split_bf16', 'tf32') else 'CUDA cores'}): "
                                     f"one launch = {imgs_per_launch:.0f} images"),
                        conv_share_of_step=conv_ms.value / (ms / args.steps))

    # End to end through the public host-pointer API (pinned host buffers).
    e2e = None
    if not args.no_e2e:
        xh = torch.from_numpy(x).pin_memory()
        oh = torch.from_numpy(obs.reshape(-1)).pin_memory()
        gh = torch.empty(n, dtype=torch.float64).pin_memory()
        fh = torch.empty(1, dtype=torch.float64).pin_memory()
        dp = C.POINTER(C.c_double)

        def host_step():
            rc = L_.wdl_evaluate_both(ctx, P, K, L, wl["loss"], sd,
                                      C.cast(xh.data_ptr(), dp), C.cast(gh.data_ptr(), dp), n,
                                      C.cast(oh.data_ptr(), dp), C.cast(fh.data_ptr(), dp),
                                      None, None, None)
            _lib.check(rc, ctx)
            if world > 1:
                gd_, fd_ = gh.to(dev), fh.to(dev)
                allreduce_atoms_and_loss(gd_, fd_, PK, dist)
                gh[PK:].copy_(gd_[PK:].cpu())
                fh.copy_(fd_.cpu())
        host_step()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            host_step()
        el = time.perf_counter() - t0
        if world > 1:
            t = torch.tensor([el], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        h2d = (n + P * N) * 8 + (K * N * 8 if world > 1 else 0)
        d2h = (n + 1) * 8 + (K * N * 8 if world > 1 else 0)
        e2e = dict(value=units / el, unit=UNIT, h2d_bytes_per_step=h2d, d2h_bytes_per_step=d2h)

    # The other precisions on the same inputs, timed the same way (CUDA events on
    # the same stream, max over ranks): plain FP32 on the CUDA cores is the
    # metric's "vs plain FP32"; FP64 on the GPU is the reference's arithmetic.
    arms, report, regress_fp64 = None, None, None
    if wl["name"] == "batched128" and wl["domain"] == "kernel" and not args.no_arms:
        outs = {precision: run_outputs(L_, ctx, wl, x_d, obs_d, sd, sptr, dev)}
        arms = {}
        for prec in ("fp32", "fp64"):
            if prec == precision:
                continue
            k2 = w.CudaGaussian2DKernel(wl["gamma"], W, H, precision=prec, device=local)
            arms[prec] = time_arm(L_, k2.ctx, wl, x_d, obs_d, sd, sptr, dev, args, world, dist)
            outs[prec] = run_outputs(L_, k2.ctx, wl, x_d, obs_d, sd, sptr, dev)
            if prec == "fp64" and not args.no_regress and world == 1:
                # dictionary learning wholly on the device in the reference's arithmetic
                regress_fp64 = time_regress(L_, k2.ctx, wl, wts, atoms, obs_d, sd, sptr, dev,
                                            iters=args.regress_iters)
            k2.close()
            torch.cuda.synchronize()
        if "fp64" in outs and rank == 0:
            report = precision_report(outs, wl, x, obs, sd)

    # Dictionary learning with the L-BFGS on the device (wdl_regress_both_device):
    # a few iterations of regress_both on the bench inputs, wall clock on the
    # device (CUDA events), to report L-BFGS iterations/s beside the evaluations.
    regress = None
    if wl["domain"] == "kernel" and not args.no_regress and world == 1:
        regress = time_regress(L_, ctx, wl, wts, atoms, obs_d, sd, sptr, dev, iters=args.regress_iters)

    serving = None
    if rank == 0 and not args.no_serving and wl["name"] == "batched128":
        serving = run_serving([float(r) for r in args.serve_rates.split(",") if r], args.serve_requests,
                              local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, _ = time_cpu_reference(wl, steps=1, warmup=0)

    if world > 1:
        torch.cuda.synchronize()
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = dict(metric=metric_for(wl), value=value, unit=UNIT, n_gpus=world, steps=args.steps,
                warmup=args.warmup, ms_per_step=ms / args.steps, higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype=dtype_name(precision),
                data=f"synthetic: seeded anisotropic Gaussian-blob histograms ({wl['n_blobs'][0]}-"
                     f"{wl['n_blobs'][1]} blobs, std {wl['std_frac'][0]}-{wl['std_frac'][1]} of the side), "
                     "uniform+noise atoms, U[0,1] weights",
                config=dict(workload=describe(wl),
                            P_per_gpu=P, W=W, H=H, K=K, L=L, gamma=wl["gamma"], loss=wl["loss_name"],
                            precision=precision, parallelism=f"dp{world} over histograms",
                            l2=f"working set larger than L2: iterate store {tape_gb:.2f} GB per GPU",
                            autotuned=tuned or None,
                            objective=fval),
                roofline=roofline, cpu_baseline=cpu, e2e=e2e, gpu_launches=int(gpu_launches),
                clocks=clocks, serving=serving,
                regress_both_device=dict(headline_precision=regress, fp64=regress_fp64)
                if (regress or regress_fp64) else None)
    if arms:
        for prec, a in arms.items():
            line[f"value_{prec}"] = a["value"]
            line[f"ms_per_step_{prec}"] = a["ms_per_step"]
        if "fp32" in arms:
            # the metric's comparison: this line's precision over plain FP32 on the GPU
            line["vs_fp32"] = value / arms["fp32"]["value"]
        if "fp64" in arms:
            line["vs_fp64"] = value / arms["fp64"]["value"]
        line["arms"] = {p: dict(a, precision=p, dtype=dtype_name(p)) for p, a in arms.items()}
    if report:
        line["precision_report"] = report
    print(json.dumps(line), flush=True)


def time_regress(L_, ctx, wl, wts, atoms, obs_d, sd, sptr, dev, iters=3):
    """regress_both's optimisation on the device for `iters` L-BFGS iterations
    (epsilon 1e-50 as the reference sets it, so every iteration runs)."""
    import numpy as np
    import torch
    from wassersteindictionarylearning_b200 import _lib
    P, K, L = wl["P"], wl["K"], wl["L"]
    sol = torch.from_numpy(np.concatenate([wts.reshape(-1), atoms.reshape(-1)])).to(dev)
    status, fval, evals = C.c_int(), C.c_double(), C.c_int()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    _lib.check(L_.wdl_regress_both_device(ctx, P, K, L, wl["loss"], sd, C.c_void_p(sol.data_ptr()),
                                          C.c_void_p(obs_d.data_ptr()), iters, 1e-50, 0, C.byref(status),
                                          C.byref(fval), C.byref(evals), sptr), ctx)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    # status -1021 (LBFGSERR_CANCELED): a line-search trial's objective was NaN and
    # the run stopped there, as the reference's progress_both stops it; on the FP32
    # forms that is a trial point whose scalings leave the float range
    return dict(iterations=iters, evaluations=evals.value, status=status.value, objective=fval.value,
                ms=ms, lbfgs_iterations_per_s=iters / (ms / 1e3),
                evaluations_per_s=evals.value / (ms / 1e3),
                hist_iter_per_s=evals.value * P * L / (ms / 1e3),
                note="wdl_regress_both_device: every evaluation and L-BFGS step on the device, "
                     "one 4-byte status read per evaluation")


def time_arm(L_, ctx, wl, x_d, obs_d, sd, sptr, dev, args, world, dist):
    """One precision's evaluate_both on the bench inputs: warm-up, then the same
    number of steps as the headline between CUDA events on the same stream."""
    import torch
    from wassersteindictionarylearning_b200 import _lib
    P, K, L = wl["P"], wl["K"], wl["L"]
    n = x_d.numel()
    g_d = torch.empty(n, dtype=torch.float64, device=dev)
    f_d = torch.empty(1, dtype=torch.float64, device=dev)

    def step():
        _lib.check(L_.wdl_evaluate_both_device(ctx, P, K, L, wl["loss"], sd, C.c_void_p(x_d.data_ptr()),
                                               C.c_void_p(g_d.data_ptr()), n, C.c_void_p(obs_d.data_ptr()),
                                               C.c_void_p(f_d.data_ptr()), None, None, None, sptr), ctx)
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    units = P * L * args.steps * world
    return dict(value=units / (ms / 1e3), ms_per_step=ms / args.steps)


def run_outputs(L_, ctx, wl, x_d, obs_d, sd, sptr, dev):
    """Objective, gradient and barycenters of one evaluation (host copies)."""
    import torch
    from wassersteindictionarylearning_b200 import _lib
    P, K, L, N = wl["P"], wl["K"], wl["L"], wl["W"] * wl["H"]
    n = x_d.numel()
    g_d = torch.empty(n, dtype=torch.float64, device=dev)
    f_d = torch.empty(1, dtype=torch.float64, device=dev)
    b_d = torch.empty(P * N, dtype=torch.float64, device=dev)
    _lib.check(L_.wdl_evaluate_both_device(ctx, P, K, L, wl["loss"], sd, C.c_void_p(x_d.data_ptr()),
                                           C.c_void_p(g_d.data_ptr()), n, C.c_void_p(obs_d.data_ptr()),
                                           C.c_void_p(f_d.data_ptr()), None, None,
                                           C.c_void_p(b_d.data_ptr()), sptr), ctx)
    torch.cuda.synchronize()
    return dict(f=float(f_d.item()), g=g_d.cpu().numpy(), bary=b_d.cpu().numpy())


def precision_report(outs, wl, x, obs, sd, n_scale=4):
    """Each output's error against the FP64 arm (the GPU FP64 path, which the
    parity tests hold to the reference within 1e-10): barycenters and the atom
    gradient normwise (max|a-b| / max|b|), the objective relatively, the weight
    gradient both normwise and against its floating-point condition scale (the
    mass of the terms summed into it, from the oracle; computed for the first
    n_scale histograms, whose weight gradients do not depend on the others)."""
    import numpy as np
    P, K, L, W, H = wl["P"], wl["K"], wl["L"], wl["W"], wl["H"]
    N = W * H
    PK = P * K
    ref = outs["fp64"]

    def nrm(a, b):
        return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))
    scale = None
    try:
        from oracle.oracle import OracleLib
        xs = np.concatenate([x[:n_scale * K], x[PK:]])
        scale = OracleLib().weight_gradient_scale(W, H, 1, wl["gamma"], n_scale, K, L, wl["loss"], sd, xs,
                                                  obs.reshape(P, N)[:n_scale].reshape(-1))
    except Exception:  # the oracle's C build is absent: report the normwise errors only
        scale = None
    rep = {}
    for prec, o in outs.items():
        if prec == "fp64":
            continue
        e = dict(barycenter=nrm(o["bary"], ref["bary"]),
                 objective=abs(o["f"] - ref["f"]) / abs(ref["f"]),
                 atom_gradient=nrm(o["g"][PK:], ref["g"][PK:]),
                 weight_gradient_normwise=nrm(o["g"][:PK], ref["g"][:PK]))
        if scale is not None:
            d = np.abs(o["g"][:n_scale * K] - ref["g"][:n_scale * K])
            e["weight_gradient_vs_condition_scale"] = float(np.max(d) / max(float(np.max(scale)), 1e-300))
        rep[prec] = e
    rep["against"] = "fp64 arm (GPU FP64, same inputs)"
    return rep


def run_serving(rates, n, device):
    """p50/p99 latency of Poisson request streams through the serving loop, one
    stream per offered rate on the same running server: half projection (fit 5
    weights of a new histogram, L-BFGS) and half barycenter requests, square
    2-D grids of side uniform in 64..256 and 20 % 48^3 volumes, L = 50,
    gamma = 2, split-BF16 where the tensor-core operator applies.  The server
    starts with the resident dictionaries of every served shape (193 square
    grids and the volume), one warm-up request per operator form and the
    one-request calls of every shape recorded as CUDA graphs; none of that is
    timed."""
    import time as _t

    from wassersteindictionarylearning_b200.serving import (ServingEngine, latency_summary,
                                                            poisson_requests)
    eng = ServingEngine(K=5, L=50, gamma=2.0, loss_type=2, precision="split_bf16",
                        lbfgs_iterations=20, device=device, workers=16, hbm_budget=32e9)
    # server start-up: resident dictionaries, device kernels loaded once, graphs recorded
    eng.preload([(s, s, 1) for s in range(64, 257)] + [(48, 48, 48)])
    eng.warm_up()
    eng.capture_graphs()
    results = []
    for rate in rates:
        arr = poisson_requests(rate, n, seed=11, K=5)
        eng.completed = []
        t0 = _t.perf_counter()
        done = eng.run(arr, timeout=240.0)
        wall = _t.perf_counter() - t0
        out = latency_summary(done)
        out.update(offered_rate_req_s=rate, requests=n, wall_s=wall,
                   throughput_req_s=out["completed"] / wall,
                   mix="50% projection (20 L-BFGS iterations) / 50% barycenter; square 2-D grids, "
                       "side U[64,256], 20% 48^3; L=50, gamma=2, K=5; dictionaries of all 194 shapes "
                       "resident, one-request calls recorded as CUDA graphs at start-up; 16 workers")
        results.append(out)
    eng.close()
    return results


def run_uneven(args):
    """The uneven weight-fitting workload: 512 independent problems (side from
    {32,48,64,96,128,192}, K 3-8, L 25-100, gamma {1,2,4}, quadratic loss, 40
    L-BFGS iterations, split-BF16), fitted by batch.fit_weights.  With the
    workload's random-blob dictionaries (atoms that differ in where their mass
    sits) and gamma of 1-4 pixels^2 the kernel-domain scalings leave the float
    range within ~10 iterations, so every problem ends up fitted in the log
    domain.  `--P n` fits the first n problems only."""
    import numpy as np
    import torch

    from wassersteindictionarylearning_b200.batch import fit_weights, uneven_problems
    n = args.P or 512
    iters = 40
    probs = uneven_problems(n=n, seed=0)
    torch.cuda.set_device(0)
    # warm-up: one small problem per (kind of) path, builds every kernel
    fit_weights(probs[:4], lbfgs_iterations=2)
    torch.cuda.synchronize()
    with ClockSampler(0) as clk:
        t0 = time.perf_counter()
        res = fit_weights(probs, precision="split_bf16", lbfgs_iterations=iters)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
    clocks = clk.summary()
    evals = np.array([r[3] for r in res])
    doms = [r[4] for r in res]
    hist_iters = float(sum(e * pr["L"] for e, pr in zip(evals, probs)))
    statuses = {}
    for r in res:
        statuses[str(r[2])] = statuses.get(str(r[2]), 0) + 1
    line = dict(metric="weight fits/s (uneven 512-problem batch)", value=n / el, unit="fits/s",
                n_gpus=1, steps=1, warmup=1, ms_per_step=el * 1e3, higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="bf16x3+f32 (kernel domain), f32 (log domain)",
                data="synthetic: per problem a seeded random-blob dictionary and one blob histogram",
                config=dict(workload=args.workload, problems=n, sides=[32, 48, 64, 96, 128, 192],
                            K="3-8", L="25-100", gamma=[1, 2, 4], loss="quadratic",
                            lbfgs_iterations=iters, timing="wall clock around the whole fit "
                            "(kernel-domain device fits per gamma, then one persistent log-domain "
                            "launch per gamma)"),
                hist_iter_per_s=hist_iters / el,
                evaluations=dict(total=int(evals.sum()), mean=float(evals.mean())),
                domains=dict(kernel=doms.count("kernel"), log=doms.count("log")),
                lbfgs_status=statuses, clocks=clocks)
    print(json.dumps(line), flush=True)


def run_uneven_reference(args):
    """The reference's own CPU path on the uneven workload: it fits one problem
    at a time, each L-BFGS evaluation one evaluate_both (log domain, the
    domain the workload needs; LogSignArrayGaussian2DKernel, OpenMP over all
    host cores).  Bounded sample: one evaluation of each of the two problems
    of median operator work (K L N (W + H)); the whole workload's time is that
    rate times the workload's total work, times the 57.1 evaluations per fit
    our run of the same problems used (regress_both's L-BFGS settings: each fit
    runs its 40 iterations unless the line search stops it)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import numpy as np

    from oracle import oracle as orc
    from wassersteindictionarylearning_b200.batch import uneven_problems
    from wassersteindictionarylearning_b200.synthetic import to_variables
    os.environ.setdefault("OMP_NUM_THREADS", str(cpu_threads()))
    lib = orc.RefLib()
    probs = uneven_problems(n=512, seed=0)
    work = [pr["K"] * pr["L"] * pr["W"] * pr["H"] * (pr["W"] + pr["H"]) for pr in probs]
    order = sorted(range(len(probs)), key=lambda i: work[i])
    sample = [order[len(order) // 2 - 1], order[len(order) // 2]]
    t_sample, w_sample = 0.0, 0.0
    for i in sample:
        pr = probs[i]
        W, H, K, L, g = pr["W"], pr["H"], pr["K"], pr["L"], pr["gamma"]
        a = pr["atoms"].reshape(K, -1)
        x = to_variables(np.ones((1, K)) / K, a / a.sum(axis=1, keepdims=True), 1.0)
        t0 = time.perf_counter()
        lib.evaluate_both(W, H, 1, g, 1, K, L, pr.get("loss_type", 2), 1.0, x, pr["observed"],
                          log_domain=True)
        t_sample += time.perf_counter() - t0
        w_sample += work[i]
    evals_per_fit = 57.1
    total = sum(work) / w_sample * t_sample * evals_per_fit
    value = len(probs) / total
    desc = ", ".join(f"{probs[i]['W']}x{probs[i]['H']} K={probs[i]['K']} L={probs[i]['L']}" for i in sample)
    line = dict(metric="weight fits/s (uneven 512-problem batch)", value=value, unit="fits/s",
                n_gpus=args.gpus, steps=1, warmup=0, ms_per_step=total * 1e3, higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="f64", data="synthetic",
                config=dict(workload="uneven512", note="bounded sample of the workload, scaled by work"),
                impl="reference",
                cpu_baseline=dict(value=value, unit="fits/s", cores=lib.omp_threads(), kind="reference",
                                  sample=f"LogSignArrayGaussian2DKernel evaluate_both "
                                         f"(cpp/inverseWasserstein.h:986), OpenMP; one evaluation each "
                                         f"of the 2 median-work problems ({desc}), {t_sample:.2f} s, "
                                         f"scaled to the 512 problems' work x {evals_per_fit} "
                                         f"evaluations per fit; CPU: {cpu_model()}"),
                e2e=dict(value=value, unit="fits/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "uneven512":
        if args.impl == "reference":
            run_uneven_reference(args)
        else:
            run_uneven(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
