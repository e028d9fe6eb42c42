#!/usr/bin/env python
"""Benchmark of the B200 Cholesky-vector MP2 path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
    python bench.py --impl reference ...   # the reference CPU path

Default workload: CD-MP2 energy plus the exact orbital gradient (dE/dC,
dE/deps) of a closed-shell system with N=2000 basis functions, o=200
occupied orbitals and M=8000 Cholesky vectors, synthetic inputs of the seeded
recipe (mshqc_b200/synthetic.py) at the scaled magnitude |E_corr| ~ 0.05 o Eh.
Its FP64 AO vectors would take 256 GB, so the library generates them on the
device chunk by chunk (mshqc_cd_gen_vectors) wherever they are read.

One step = one mp2_gradient call in the mixed precision: AO->MO half
transform, integral tiles of the unique pairs (the energy comes out of them),
element-wise amplitude pass, Gamma GEMM, transposed transforms.  The FP64
path is timed once on the same inputs for the mixed-vs-FP64 comparison and
the energy / gradient errors.

`value` = FP64-equivalent algorithmic TFLOP/s of the work the step performs
(split products not counted), over all ranks, inputs resident in HBM:
F_T + F_E + F_G + F_Tt with F_T = 2 M N o (N + v) (half transform),
F_E = v^2 M o (o + 1) (integral tiles of the unique pairs i <= j),
F_G = 2 v^2 M o^2 (Gamma), F_Tt = 2 M N o (N + 2 v) (transposed transforms);
an energy-only step is F_T + F_E.  `e2e` = the same metric through the C ABI
from host buffers, copies inside the timed region.  With --gpus N > 1 the
ranks share one gradient (mshqc_cd_set_partition: block pairs of the
backward; mshqc_cd_set_collectives: the half and transposed transforms over
occupied orbitals with an NCCL all-gather of B and reduce-scatter of Gamma;
an NCCL all-reduce of the shares); --parallelism replicas runs N
independent copies instead.

The reference arm (--impl reference) runs the reference's own CPU code
(oracle/_ref, compiled from its sources) on a bounded sample of the workload:
the same synthetic recipe at the same ratios v/o and M/N with fewer occupied
orbitals, timed inside the reference, and extrapolated to the workload as
o^5 (the operation count of the reference's loops at fixed ratios) from the
sample's own rate; same-size workloads that fit (N <= 400) run in full.
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
sys.path.insert(0, ROOT)

METRIC = "CD-MP2 energy+OMP2 grad s & TFLOP/s: mixed vs FP64 on B200 at ≤1 µEh"

WORKLOADS = {
    # the north-star size: energy + exact gradient, vectors generated on the
    # device (their FP64 AO form, 256 GB, does not fit)
    "cdmp2_grad_n2000_o200_m8000": dict(N=2000, o=200, M=8000, gradient=True, precision="fp16x3",
                                        gen=True),
    # energy + exact gradient, mixed vs FP64, stored vectors
    "cdmp2_grad_n1000_o100_m4000": dict(N=1000, o=100, M=4000, gradient=True, precision="fp16x3"),
    # smaller variants of the same step
    "cdmp2_grad_n400_o40_m1600": dict(N=400, o=40, M=1600, gradient=True, precision="fp16x3"),
    "cdmp2_grad_n600_o60_m2400": dict(N=600, o=60, M=2400, gradient=True, precision="fp16x3"),
    # energy only (the CD-RMP2 drop-in), N=400, o=40, M=1600 and N=1000, o=100, M=4000
    "cdrmp2_energy_n400_o40_m1600": dict(N=400, o=40, M=1600, gradient=False, precision="fp16x3"),
    "cdrmp2_energy_n1000_o100_m4000": dict(N=1000, o=100, M=4000, gradient=False, precision="fp16x3"),
    # differentiated CD-UMP2 (the OMP2 step): separate alpha / beta orbitals
    "cdump2_grad_n600_o60_58_m2400": dict(N=600, o=60, ob=58, M=2400, gradient=True, precision="fp16x3",
                                          kind="unrestricted"),
}
DEFAULT_WORKLOAD = "cdmp2_grad_n2000_o200_m8000"


# ---------------------------------------------------------------------------
# algorithmic work (FP64-equivalent flops; split products not counted)
# ---------------------------------------------------------------------------
def flops_transform(N, o, M):
    """AO->MO half transform of one spin: 2 M N o (N + v)."""
    return 2.0 * M * N * o * (N + (N - o))


def flops_transposed(N, o, M):
    """dE/dC of one spin from Gamma: dC_vir (2 M N o v), W = Gamma C_vir^T
    (2 M N o v), dC_occ (2 M N^2 o)."""
    return 2.0 * M * N * o * (N + 2 * (N - o))


def flops_energy(N, o, M):
    """(ia|jb) of the unique pairs i <= j: 2 v^2 M o (o + 1) / 2."""
    v = N - o
    return 1.0 * v * v * M * o * (o + 1)


def flops_gamma(N, o, M):
    v = N - o
    return 2.0 * v * v * M * o * o


def workload_parts(w):
    """{stage: flops} of the work one step performs."""
    N, o, M = w["N"], w["o"], w["M"]
    if w.get("kind") == "unrestricted":
        ob = w["ob"]
        va, vb = N - o, N - ob
        tiles = 2.0 * M * (va * va * o * (o + 1) / 2 + vb * vb * ob * (ob + 1) / 2 + va * vb * o * ob)
        parts = {"transform": flops_transform(N, o, M) + flops_transform(N, ob, M), "tiles": tiles}
        if w["gradient"]:
            parts["gamma"] = 2.0 * M * (va * va * o * o + vb * vb * ob * ob + 2.0 * va * vb * o * ob)
            parts["transposed"] = flops_transposed(N, o, M) + flops_transposed(N, ob, M)
        return parts
    parts = {"transform": flops_transform(N, o, M), "tiles": flops_energy(N, o, M)}
    if w["gradient"]:
        parts["gamma"] = flops_gamma(N, o, M)
        parts["transposed"] = flops_transposed(N, o, M)
    return parts


def workload_flops_w(w):
    return sum(workload_parts(w).values())


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self._t = None
        self.t_begin = 0.0
        self.t_end = float("inf")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        window = [ln for (t, ln) in self.lines if self.t_begin - 0.25 <= t <= self.t_end + 0.25]
        for ln in window:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def max_over_ranks(value: float, device) -> float:
    """The largest value over the ranks (every timing is the max over ranks)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def measure_fp64_peak(torch, device):
    """cuBLAS FP64 GEMM rate (torch float64 matmul 8192^3, best of 5)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


# ---------------------------------------------------------------------------
# reference CPU path (oracle/_ref: the reference's own code, compiled here)
# ---------------------------------------------------------------------------
REF_FULL_MAX_N = 400        # workloads up to this size run in full on the CPU
REF_SAMPLE_O = 12           # occupied orbitals of a scaled sample
REF_CALIBRATION_O = (8, 12, 16)


def sample_shape(w, o_s):
    """The workload's shape scaled to o_s occupied orbitals at its own ratios
    v/o and M/N (the beta count keeps its offset from alpha)."""
    N, o, M = w["N"], w["o"], w["M"]
    if o_s >= o:
        return N, o, w.get("ob", o), M
    N_s = max(o_s + 2, int(round(N * o_s / o)))
    M_s = max(4, int(round(M * N_s / N)))
    ob_s = max(1, o_s - (o - w.get("ob", o)))
    return N_s, o_s, ob_s, M_s


def run_reference_sample(w, o_s, seed, nthreads):
    """The reference's own CPU code on the workload scaled to o_s occupied
    orbitals (in full when o_s >= o): CholeskyOMP2's MP2 part of one gradient
    evaluation (both spins' transforms and t2, the energy, the OPDM blocks;
    src/mp2/cholesky_omp2.cc:445-449) for gradient workloads, with separate
    beta orbitals for the unrestricted one, CholeskyRMP2::compute for energy
    workloads.  Returns (seconds inside the reference, description)."""
    from mshqc_b200 import synthetic as syn
    from oracle import ref
    N, o, ob, M = sample_shape(w, o_s)
    unres = w.get("kind") == "unrestricted"
    base = syn.make_inputs(N, o, M, seed=seed)
    sig = syn.twin_sigma(N, o, M, base.alpha.eps)
    inp = syn.make_inputs(N, o, M, seed=seed, sigma=sig, nocc_beta=ob if unres else None)
    a = inp.alpha
    b = inp.beta if unres else a
    if w["gradient"]:
        r = ref.omp2_mp2_part(inp.L, a.C, b.C, a.eps, b.eps, o, ob, nthreads=nthreads)
        what = "CholeskyOMP2 t2 + energy + OPDM"
    else:
        r = ref.rmp2(inp.L, a.C, a.eps, o, nthreads=nthreads)
        what = "CholeskyRMP2::compute"
    shape = f"N={N}, o={o}{'/%d' % ob if unres else ''}, M={M}"
    return r["seconds"], f"{what} at {shape}"


def ref_extrapolation(w, o_s):
    """Factor from the sample's time to the workload's: (o / o_s)^5."""
    return (w["o"] / float(o_s)) ** 5


def calibrate_reference(w, nthreads, seed=7):
    """Times of the reference on samples of the workload at REF_CALIBRATION_O
    occupied orbitals and the slope of log t against log o (reported; the
    extrapolation itself uses o^5 from the sample's own rate)."""
    ts = []
    for o_s in REF_CALIBRATION_O:
        t, _ = run_reference_sample(w, o_s, seed, nthreads)
        ts.append(t)
    x = np.log(np.asarray(REF_CALIBRATION_O, dtype=float))
    y = np.log(np.asarray(ts))
    slope = float(np.polyfit(x, y, 1)[0])
    return ts, slope


REF_FULL_MAX_O_GRADIENT = 16   # the reference's CD-OMP2 scales ~o^6 (16: ~10 s on 8 cores)


def reference_plan(w):
    """(o of the sample, whether the sample is the whole workload): energy
    workloads up to N = 400 run in full (CholeskyRMP2, ~14 s at N = 400),
    gradient workloads only up to o = 16."""
    if not w["gradient"] and w["N"] <= REF_FULL_MAX_N:
        return w["o"], True
    if w["gradient"] and w["o"] <= REF_FULL_MAX_O_GRADIENT:
        return w["o"], True
    return REF_SAMPLE_O, False


def bench_reference(args, w, rank, world):
    """The reference arm: rank 0 alone times the reference's CPU path on all
    host cores; the other ranks exit without work."""
    if rank != 0:
        return
    from oracle import ref
    nthreads = os.cpu_count() or 1
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmshqc_ref.so not built"}))
        return
    flops = workload_flops_w(w)
    o_s, full = reference_plan(w)
    calib = None
    if not full:
        calib = calibrate_reference(w, nthreads)
    for s in range(args.warmup):
        run_reference_sample(w, o_s, s, nthreads)
    times, sample = [], ""
    for s in range(args.steps):
        t, sample = run_reference_sample(w, o_s, 100 + s, nthreads)
        times.append(t)
    t_sample = sum(times) / len(times)
    t_step = t_sample if full else t_sample * ref_extrapolation(w, o_s)
    value = flops / t_step / 1e12
    note = ("the workload itself" if full else
            f"{sample}, extrapolated to the workload as (o/{o_s})^5 from the sample's rate; "
            f"calibration o={list(REF_CALIBRATION_O)}: {[round(float(t), 3) for t in calib[0]]} s, "
            f"measured slope {calib[1]:.2f}")
    cpu = {"value": value, "unit": "TFLOP/s", "cores": nthreads, "kind": "reference",
           "sample": sample if full else note, "sample_seconds": t_sample,
           "extrapolated": not full}
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_step, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded recipe, scaled twin)",
        "config": {"workload": args.workload, "same_config": full,
                   "sample": sample if full else note},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def cpu_baseline_line(w):
    """cpu_baseline of the GPU arm: the calibration samples of the reference
    (about 10-30 s of CPU work), extrapolated like the reference arm."""
    from oracle import ref
    if not ref.available():
        return {"value": None, "error": "oracle/_ref/libmshqc_ref.so not built"}
    nthreads = os.cpu_count() or 1
    flops = workload_flops_w(w)
    o_s, full = reference_plan(w)
    if full:
        t, sample = run_reference_sample(w, o_s, 7, nthreads)
        return {"value": flops / t / 1e12, "unit": "TFLOP/s", "cores": nthreads, "kind": "reference",
                "sample": sample, "seconds": t, "extrapolated": False}
    ts, slope = calibrate_reference(w, nthreads)
    t_step = ts[REF_CALIBRATION_O.index(REF_SAMPLE_O)] * ref_extrapolation(w, REF_SAMPLE_O)
    N_s, _, ob_s, M_s = sample_shape(w, REF_SAMPLE_O)
    return {"value": flops / t_step / 1e12, "unit": "TFLOP/s", "cores": nthreads, "kind": "reference",
            "sample": (f"reference at o={list(REF_CALIBRATION_O)} (ratios of the workload), "
                       f"{[round(float(t), 3) for t in ts]} s, slope {slope:.2f}; "
                       f"o={REF_SAMPLE_O} (N={N_s}, M={M_s}) extrapolated as (o/{REF_SAMPLE_O})^5"),
            "seconds": sum(ts), "extrapolated_step_s": t_step, "extrapolated": True}


# ---------------------------------------------------------------------------
# the GPU arm
# ---------------------------------------------------------------------------
STAGE_KEYS = ("transform", "split", "pair_energy", "amplitude", "gamma", "transposed", "other", "amp_elem")


def bench_gpu(args, w, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from mshqc_b200 import capi
    from mshqc_b200 import shard
    from mshqc_b200 import synthetic as syn

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    N, o, M = w["N"], w["o"], w["M"]
    gradient = w["gradient"]
    prec = capi.PRECISIONS[w["precision"]]
    unres = w.get("kind") == "unrestricted"
    kind = capi.UNRESTRICTED if unres else capi.RESTRICTED
    ob = w.get("ob", o)
    shared = world > 1 and args.parallelism == "shared" and gradient
    # shared: every rank holds the same inputs; replicas: independent ones
    seed = 1000 + (0 if shared else rank)

    orb = syn.make_orbitals(N, o, seed)
    orb_b = syn.make_orbitals(N, ob, seed + 7919) if unres else orb
    sigma = syn.twin_sigma(N, o, M, orb.eps)
    gen = bool(w.get("gen"))
    L_dev = None if gen else syn.make_vectors_device(N, M, seed, sigma, dev)
    C_dev = torch.from_numpy(orb.C).to(dev)
    e_dev = torch.from_numpy(orb.eps).to(dev)
    Cb_dev = torch.from_numpy(orb_b.C).to(dev)
    eb_dev = torch.from_numpy(orb_b.eps).to(dev)

    stream = torch.cuda.Stream(device=dev)
    ctx = capi.Context(local_rank)
    ctx.set_stream(stream.cuda_stream)
    if gen:
        ctx.gen_vectors(N, M, seed, sigma)
    else:
        ctx.set_vectors(L_dev)
    if shared:
        ctx.set_partition(rank, world)
        ctx.set_collectives(*shard.nccl_collectives(dev))   # transforms shared over occupied orbitals

    def step(context, precision, C, eps):
        context.set_orbitals(capi.ALPHA, C, eps, o)            # new orbitals: full recompute
        if unres:
            context.set_orbitals(capi.BETA, Cb_dev, eb_dev, ob)
        if gradient:
            if shared:
                g = context.mp2_gradient_torch(kind, precision, device=dev)
                torch.cuda.current_stream(dev).synchronize()
                return shard.allreduce_gradient(g)
            return context.mp2_gradient(kind, precision)
        return context.mp2_energy(kind, precision)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        r = step(ctx, prec, C_dev, e_dev)
    torch.cuda.synchronize()

    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(1.0)                                  # nvidia-smi start-up
    barrier()
    torch.cuda.synchronize()
    clocks.t_begin = time.time()
    l0 = ctx.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    stages = []
    for _ in range(args.steps):
        r = step(ctx, prec, C_dev, e_dev)
        stages.append(ctx.stage_times())
    stage_n = ctx.stage_counts()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = ctx.launch_count() - l0
    clocks.t_end = time.time()
    elapsed = ev0.elapsed_time(ev1) / 1e3
    time.sleep(0.3)
    clk = clocks.stop()
    exact = ctx.mixed_exact() if prec != capi.FP64 else True

    elapsed = max_over_ranks(elapsed, dev)
    parts = workload_parts(w)
    flops = sum(parts.values())
    jobs = 1 if shared else world
    value = jobs * flops * args.steps / elapsed / 1e12
    mixed_res = r
    st = {k: statistics.median(s[k] for s in stages) for k in stages[0]}

    def host(x):
        return x.detach().cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)

    # ---- FP64 path on the same inputs (comparison and error) ---------------
    fp64 = {}
    if prec != capi.FP64 and not args.no_fp64:
        # one FP64 step, warmed up by one untimed step when the steps are
        # short (first-call allocations and module loads weigh there); a
        # long step (the default workload's FP64 step takes minutes) is timed
        # once cold
        if elapsed / args.steps < 2.0:
            step(ctx, capi.FP64, C_dev, e_dev)
        torch.cuda.synchronize()
        barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        r64 = step(ctx, capi.FP64, C_dev, e_dev)
        t1.record(stream)
        torch.cuda.synchronize()
        ms64 = max_over_ranks(t0.elapsed_time(t1), dev)
        st64 = ctx.stage_times()
        dgemm = measure_fp64_peak(torch, dev)
        fp64 = {"fp64_ms_per_step": ms64, "fp64_tflops": jobs * flops / (ms64 / 1e3) / 1e12,
                "fp64_stage_ms": st64, "fp64_dgemm_tflops": dgemm,
                "fp64_frac_of_dgemm": (flops / (ms64 / 1e3) / 1e12) / dgemm,
                "speedup_mixed_vs_fp64": ms64 / (1e3 * elapsed / args.steps)}
        if gradient:
            e3, e64 = mixed_res.energy["total"], r64.energy["total"]
            pairs = [(host(mixed_res.dC_a), host(r64.dC_a), host(mixed_res.deps_a), host(r64.deps_a))]
            if unres:
                pairs.append((host(mixed_res.dC_b), host(r64.dC_b), host(mixed_res.deps_b), host(r64.deps_b)))
            fp64.update({"energy_fp64": e64, "energy_mixed": e3,
                         "energy_error_uEh": abs(e3 - e64) * 1e6,
                         "max_abs_dC_error": max(float(np.max(np.abs(x - y))) for x, y, _, _ in pairs),
                         "max_abs_deps_error": max(float(np.max(np.abs(x - y))) for _, _, x, y in pairs),
                         "max_abs_dC": max(float(np.max(np.abs(y))) for _, y, _, _ in pairs)})
        else:
            fp64.update({"energy_fp64": r64["total"], "energy_mixed": mixed_res["total"],
                         "energy_error_uEh": abs(mixed_res["total"] - r64["total"]) * 1e6})

    # ---- end to end through the C ABI from pinned host buffers ------------
    e2e = None
    if not args.no_e2e:
        if not gen:
            L_host = torch.empty(L_dev.shape, dtype=torch.float64, pin_memory=True)
            L_host.copy_(L_dev)
        C_host = np.asfortranarray(orb.C)
        e_host = orb.eps.copy()
        Cb_host = np.asfortranarray(orb_b.C)
        eb_host = orb_b.eps.copy()
        del L_dev
        ctx.close()
        torch.cuda.empty_cache()
        ctx_h = capi.Context(local_rank)
        ctx_h.set_stream(stream.cuda_stream)
        if shared:
            ctx_h.set_partition(rank, world)
            ctx_h.set_collectives(*shard.nccl_collectives(dev))
        L_np = None if gen else L_host.numpy()

        def step_e2e():
            if gen:
                ctx_h.gen_vectors(N, M, seed, sigma)
            else:
                ctx_h.set_vectors(L_np, nbf=N)
            ctx_h.set_orbitals(capi.ALPHA, C_host, e_host, o)
            if unres:
                ctx_h.set_orbitals(capi.BETA, Cb_host, eb_host, ob)
            if gradient:
                g = ctx_h.mp2_gradient(kind, prec)       # results copied to host
                return shard.allreduce_gradient(g, device=dev) if shared else g
            return ctx_h.mp2_energy(kind, prec)

        step_e2e()
        barrier()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for _ in range(args.steps):
            step_e2e()
        torch.cuda.synchronize()
        e2e_elapsed = time.perf_counter() - w0
        e2e_elapsed = max_over_ranks(e2e_elapsed, dev)
        nspin = 2 if unres else 1
        h2d = (0 if gen else L_np.nbytes) + nspin * (C_host.nbytes + e_host.nbytes)
        d2h = 8 * 7 + (nspin * (N * N + N) * 8 if gradient else 0)
        e2e = {"value": jobs * flops * args.steps / e2e_elapsed / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": 1e3 * e2e_elapsed / args.steps}
        ctx_h.close()
    else:
        ctx.close()

    # ---- roofline of the dominant kernel ----------------------------------
    peaks, peak_src = measured_peaks()
    if gradient:
        cand = {"amplitude": ("vtile_tc_kernel", parts["tiles"]), "gamma": ("gamma_tc_kernel", parts["gamma"])}
    else:
        cand = {"pair_energy": ("pair_energy_tc_kernel", parts["tiles"])}
    dom = max(cand, key=lambda k: st.get(k, 0.0))
    kname, kflops = cand[dom]
    if shared:
        kflops /= world                     # this rank's share of the units
    kms = st[dom]
    achieved = kflops / (kms / 1e3) / 1e12 if kms > 0 else None
    if prec == capi.FP64:
        peak = measure_fp64_peak(torch, dev)
        peak_note = "FP64 cuBLAS DGEMM 8192^3 measured in this run"
    else:
        peak = peaks["bf16_tflops_sustained"] / 3.0
        peak_note = (f"dense 16-bit tensor peak ({peak_src}, sustained "
                     f"{peaks['bf16_tflops_sustained']}) / 3: three products per useful product")
    traffic = roofline_traffic(kname, w, stage_n.get(dom, 0), world if shared else 1)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "strong" if shared else "weak", "vs_baseline": None,
            "dtype": ("f64" if prec == capi.FP64 else
                      "fp16x3 (integer hi/lo fixed point on the tensor cores, f32 accumulate; bf16x3 Gamma; "
                      "int8-slice transforms; f64 denominators and sums)"),
            "data": "synthetic (seeded recipe, scaled twin, device Philox stream for L)",
            "config": {"workload": args.workload, "N": N, "o": o, "v": N - o, "M": M,
                       **({"o_beta": ob} if unres else {}),
                       "kind": "unrestricted" if unres else "restricted",
                       "precision": w["precision"], "gradient": gradient,
                       "sigma": sigma,
                       "parallelism": (f"shared{world}" if shared else f"replicas{world}"),
                       "vectors": "generated on the device per chunk" if gen else "stored",
                       "l2": "inputs larger than L2 (AO vectors %.1f GB%s, MO vectors %.2f GB)" % (
                           N * N * M * 8 / 1e9, ", regenerated, never stored" if gen else "",
                           o * (N - o) * M * 8 / 1e9),
                       "work_tflop": {k: v / 1e12 for k, v in parts.items()},
                       "stage_ms": st, "mixed_exact_accumulation": exact, **fp64},
            "clocks": clk,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "roofline": {"bound": "tensor", "kernel": kname, "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic.get("bytes") if traffic else None,
                         "algorithmic_bytes": traffic.get("algorithmic_bytes") if traffic else None,
                         "traffic_note": traffic.get("note") if traffic else "no capture for this kernel",
                         "peak_source": peak_note, "kernel_ms_per_step": kms,
                         "kernel_launches_per_step": stage_n.get(dom, 0)},
        }
        if not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline_line(w)
            except Exception as ex:   # a reported baseline, not the product
                line["cpu_baseline"] = {"value": None, "error": str(ex)}
        print(json.dumps(line))


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one captured
# launch of the dominant kernel, with the extent of that launch: the Gamma
# GEMM of the first block pair of the default step (R = K = 25 occupied
# orbitals x 1920 padded virtuals, Q = 8192, 25 x 1800 rows of Gamma
# read-modified-written), captured in one ncu pass with wave pacing and
# 16-row-block tile groups (profiles/gamma_tc_kernel_cdmp2_grad_n2000_o200_m8000.md).
# A wave of Gamma tiles reads its operand rows once per K step and a launch
# has R / 128 * Q / 256 / 148 waves, so the operand traffic of a launch grows
# as R * K; the read-modify-write of Gamma adds 16 bytes per written element.
CAPTURED_TRAFFIC = {
    "gamma_tc_kernel": {"bytes": 83795767808 + 2927466240, "R": 48000, "K": 48000,
                        "rmw": 16 * 25 * 1800 * 8000},
}


def roofline_traffic(kname, w, launches, share):
    """DRAM bytes per launch of the dominant kernel: the captured launch
    (CAPTURED_TRAFFIC) scaled to this step by the operand extent its
    launches process, averaged over them; None where there is no capture.
    The restricted backward over nb occupied blocks makes nb^2 Gamma
    launches (nb diagonal, two per off-diagonal block pair) whose R * K add
    up to (o * VR)^2 and whose Gamma rows add up to nb * o * v; a rank of a
    shared gradient makes about nb^2 / share of them."""
    cap = CAPTURED_TRAFFIC.get(kname)
    if cap is None or not w.get("gradient") or w.get("kind") == "unrestricted" or launches <= 0:
        return None
    N, o, M = w["N"], w["o"], w["M"]
    v = N - o
    VR = 128 * ((v + 127) // 128)
    nb = max(1, round((launches * share) ** 0.5))
    per_rk = (cap["bytes"] - cap["rmw"]) / (cap["R"] * cap["K"])
    step_bytes = per_rk * float(o * VR) ** 2 + 16.0 * v * M * o * nb
    per_launch = step_bytes / (nb * nb)
    # algorithmic: amplitudes (BF16 hi/lo) and B^T (hi/lo) once, Gamma rows once
    Q = 256 * ((M + 255) // 256)
    algo = (4.0 * float(o * VR) ** 2 + 4.0 * Q * nb * o * VR + 16.0 * v * M * o * nb) / (nb * nb)
    return {"bytes": per_launch, "algorithmic_bytes": algo,
            "note": (f"ncu capture of one launch (R=K={cap['R']}: {cap['bytes'] / 1e9:.1f} GB) scaled by "
                     f"the operand extent to this step's {nb * nb} launches "
                     f"({step_bytes / 1e12:.2f} TB per step, {per_launch / 1e9:.1f} GB per launch; "
                     f"algorithmic {algo / 1e9:.1f} GB per launch)")}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--parallelism", default="shared", choices=["shared", "replicas"],
                    help="N > 1: share one gradient (NCCL all-reduce) or run N replicas")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison step")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    w = WORKLOADS[args.workload]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        bench_reference(args, w, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    try:
        bench_gpu(args, w, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
