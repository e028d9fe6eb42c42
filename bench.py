#!/usr/bin/env python
"""Benchmark of the B200 Cholesky-vector MP2 path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
    python bench.py --impl reference ...   # the reference CPU path

One step = one pass of the hot path over one synthetic input (seeded recipe
of mshqc_b200/synthetic.py): AO->MO half transforms plus the fused pair
kernels (plus the backward for gradient workloads).  `value` is FP64-
equivalent algorithmic TFLOP/s over all ranks with the inputs resident in
HBM; `e2e` is the same metric through the C ABI from pinned host buffers,
host<->device copies inside the timed region.  Multi-GPU runs are replicas
(independent inputs per rank, weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# workload name -> (N, o, M, kind, precision, gradient)
WORKLOADS = {
    "cdrmp2_fp64_n400_o40_m1600": dict(N=400, o=40, M=1600, kind="restricted",
                                       precision="fp64", gradient=False),
    "cdrmp2_fp16x3_n400_o40_m1600": dict(N=400, o=40, M=1600, kind="restricted",
                                         precision="fp16x3", gradient=False),
}
DEFAULT_WORKLOAD = "cdrmp2_fp64_n400_o40_m1600"


# ---------------------------------------------------------------------------
# algorithmic work (FP64-equivalent flops; split products not counted)
# ---------------------------------------------------------------------------
def flops_transform(N, o, M):
    return 2.0 * M * N * o * (N + (N - o))


def flops_energy(N, o, M, restricted=True, ob=None):
    v = N - o
    if restricted:
        pairs = o * (o + 1) / 2
        return 2.0 * v * v * M * pairs
    vb = N - ob
    return 2.0 * M * (v * v * o * (o - 1) / 2 + vb * vb * ob * (ob - 1) / 2 + v * vb * o * ob)


def workload_flops(w):
    N, o, M = w["N"], w["o"], w["M"]
    f = flops_transform(N, o, M) + flops_energy(N, o, M)
    return f


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

    def mark(self, name):
        setattr(self, name, time.time())

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
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # samples inside the timed window (widened by one sampling period on
        # each side so that short windows still get the neighbouring samples)
        t0 = getattr(self, "t_begin", 0.0) - 0.25
        t1 = getattr(self, "t_end", float("inf")) + 0.25
        window = [ln for (t, ln) in self.lines if t0 <= t <= t1]
        for ln in window:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def measure_fp64_peak(torch, device):
    """cuBLAS FP64 GEMM throughput (torch float64 matmul 8192^3, best of 5):
    the denominator of the FP64 roofline (MEASURED_PEAKS.json has none)."""
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
def reference_sample(w, seed=0):
    """A bounded sample of the workload for the reference CPU path: same N
    and M, fewer occupied orbitals, so one run takes seconds."""
    N, o, M = w["N"], w["o"], w["M"]
    o_s = max(2, min(o, int(os.environ.get("MSHQC_REF_SAMPLE_OCC", "12"))))
    return N, o_s, M


def run_reference_once(w, seed, nthreads):
    from mshqc_b200 import synthetic as syn
    from oracle import ref
    N, o_s, M = reference_sample(w, seed)
    inp = syn.make_inputs(N, o_s, M, seed=seed)
    a = inp.alpha
    r = ref.rmp2(inp.L, a.C, a.eps, o_s, nthreads=nthreads)
    flops = flops_transform(N, o_s, M) + flops_energy(N, o_s, M)
    return r["seconds"], flops, f"N={N}, o={o_s}, M={M} CD-RMP2 (reference CholeskyRMP2::compute)"


def bench_reference(args, w, rank, world):
    if rank != 0:
        return
    from oracle import ref
    nthreads = os.cpu_count() or 1
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmshqc_ref.so not built"}))
        return
    for s in range(args.warmup):
        run_reference_once(w, s, nthreads)
    times, flops, sample = [], 0.0, ""
    for s in range(args.steps):
        t, f, sample = run_reference_once(w, 100 + s, nthreads)
        times.append(t)
        flops = f
    tot = sum(times)
    value = flops * args.steps / tot / 1e12
    line = {
        "impl": "reference", "metric": metric_name(w), "value": value, "unit": "TFLOP/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "sample": sample},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": nthreads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def metric_name(w):
    return "CD-MP2 energy+OMP2 grad s & TFLOP/s: mixed vs FP64 on B200 at ≤1 µEh"


# ---------------------------------------------------------------------------
# the GPU arm
# ---------------------------------------------------------------------------
def bench_gpu(args, w, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from mshqc_b200 import capi
    from mshqc_b200 import synthetic as syn

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    N, o, M = w["N"], w["o"], w["M"]
    prec = capi.PRECISIONS[w["precision"]]
    kind = capi.RESTRICTED if w["kind"] == "restricted" else capi.UNRESTRICTED

    inp = syn.make_inputs(N, o, M, seed=1000 + rank)
    a = inp.alpha
    # pinned host copies for the end-to-end leg
    L_host = torch.from_numpy(inp.L).pin_memory()
    C_host = torch.from_numpy(np.asfortranarray(a.C)).pin_memory()
    e_host = torch.from_numpy(a.eps.copy()).pin_memory()
    # device-resident inputs for the kernel leg
    L_dev = L_host.to(dev)
    C_dev = torch.from_numpy(a.C).to(dev)
    e_dev = torch.from_numpy(a.eps).to(dev)

    stream = torch.cuda.Stream(device=dev)
    ctx = capi.Context(local_rank)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_vectors(L_dev)

    def step_device():
        ctx.set_orbitals(capi.ALPHA, C_dev, e_dev, o)     # new orbitals: full recompute
        return ctx.mp2_energy(kind, prec)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(max(3, args.warmup)):
        step_device()
    torch.cuda.synchronize()

    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(1.0)                      # nvidia-smi start-up
    barrier()
    torch.cuda.synchronize()
    clocks.mark("t_begin")
    l0 = ctx.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    energy_ms = []
    for _ in range(args.steps):
        r = step_device()
        energy_ms.append(r["ms_energy"])
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = ctx.launch_count() - l0
    clocks.mark("t_end")
    elapsed = ev0.elapsed_time(ev1) / 1e3
    time.sleep(0.3)
    clk = clocks.stop()

    t = torch.tensor([elapsed], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    elapsed = float(t.item())
    flops = workload_flops(w)
    value = world * flops * args.steps / elapsed / 1e12

    # ---- end to end through the C ABI from pinned host buffers ------------
    ctx_h = capi.Context(local_rank)
    ctx_h.set_stream(stream.cuda_stream)

    def step_e2e():
        ctx_h.set_vectors(L_host.numpy())
        ctx_h.set_orbitals(capi.ALPHA, C_host.numpy(), e_host.numpy(), o)
        return ctx_h.mp2_energy(kind, prec)

    step_e2e()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step_e2e()
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    e2e_elapsed = max(wall, e0.elapsed_time(e1) / 1e3)
    t = torch.tensor([e2e_elapsed], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_elapsed = float(t.item())
    e2e_value = world * flops * args.steps / e2e_elapsed / 1e12
    h2d = L_host.numel() * 8 + C_host.numel() * 8 + e_host.numel() * 8
    d2h = 8 * 7   # the energy record

    # ---- roofline of the dominant kernel (pair energy) --------------------
    peaks, peak_src = measured_peaks()
    if w["precision"] == "fp64":
        fp64_peak = measure_fp64_peak(torch, dev)
        peak, peak_note = fp64_peak, "FP64 cuBLAS DGEMM 8192^3 measured in this run"
    else:
        peak = peaks["bf16_tflops"] / 3.0
        peak_note = f"bf16 dense {peak_src} / 3 (three split products)"
    ke = flops_energy(N, o, M)
    kms = statistics.median(energy_ms)
    achieved = ke / (kms / 1e3) / 1e12
    energy_check = r["total"]

    ctx_h.close()
    ctx.close()

    if rank == 0:
        line = {
            "metric": metric_name(w), "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if w["precision"] == "fp64" else "fp16x3 (scaled fixed point, exact f32 accumulate; f64 denominators, sums)",
            "data": "synthetic",
            "config": {"workload": args.workload, "N": N, "o": o, "v": N - o, "M": M,
                       "kind": w["kind"], "precision": w["precision"],
                       "gradient": w["gradient"], "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (L %.1f GB, B %.2f GB)" % (
                           N * N * M * 8 / 1e9, o * (N - o) * M * 8 / 1e9),
                       "e_corr": energy_check},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "TFLOP/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": d2h, "ms_per_step": 1e3 * e2e_elapsed / args.steps},
            "gpu_launches": int(launches),
            "roofline": {"bound": "tensor",
                         "kernel": ("pair_energy_f64_kernel<RESTRICTED>" if w["precision"] == "fp64"
                                    else "pair_energy_tc_kernel<RESTRICTED>"),
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None, "peak_source": peak_note,
                         "kernel_ms": kms},
        }
        if not args.no_cpu_baseline:
            try:
                from oracle import ref
                if ref.available():
                    nthreads = os.cpu_count() or 1
                    ts, fs, sample = run_reference_once(w, 7, nthreads)
                    line["cpu_baseline"] = {"value": fs / ts / 1e12, "unit": "TFLOP/s",
                                            "cores": nthreads, "kind": "reference",
                                            "sample": sample, "seconds": ts}
            except Exception as ex:  # the baseline is a report, not the product
                line["cpu_baseline"] = {"value": None, "error": str(ex)}
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        bench_gpu(args, w, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
