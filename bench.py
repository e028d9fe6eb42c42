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

One step = AO->MO half transform + integral tiles + amplitude pass + Gamma
GEMM + transposed transforms, i.e. one mp2_gradient call, in the mixed
precision (scaled FP16x3 on the tensor cores).  The FP64 path is timed once on
the same inputs for the mixed-vs-FP64 comparison and the energy / gradient
errors.

`value` = FP64-equivalent algorithmic TFLOP/s over all ranks with the inputs
resident in HBM (work 2 F_T + 2 F_E + 2 v^2 M o^2; F_T = 2 M N o (N+v),
F_E = v^2 M o (o+1)); `e2e` = the same metric through the C ABI from host
buffers, copies inside the timed region.  Multi-GPU runs are replicas
(independent inputs per rank, weak scaling, no data-path collective).
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
    return 2.0 * M * N * o * (N + (N - o))


def flops_energy(N, o, M):
    v = N - o
    return 1.0 * v * v * M * o * (o + 1)


def flops_gamma(N, o, M):
    v = N - o
    return 2.0 * v * v * M * o * o


def workload_flops(N, o, M, gradient):
    if not gradient:
        return flops_transform(N, o, M) + flops_energy(N, o, M)
    return 2 * flops_transform(N, o, M) + 2 * flops_energy(N, o, M) + flops_gamma(N, o, M)


def unrestricted_parts(N, oa, ob, M):
    """(transforms, integral tiles, Gamma) of the unrestricted energy +
    gradient: both spins transformed forward and back; the backward forms
    every same-spin (unique pairs i <= j) and opposite-spin (ia|jb) once and
    Gamma_alpha, Gamma_beta (two products for the opposite-spin block)."""
    va, vb = N - oa, N - ob
    tr = 2 * (flops_transform(N, oa, M) + flops_transform(N, ob, M))
    tiles = 2.0 * M * (va * va * oa * (oa + 1) / 2 + vb * vb * ob * (ob + 1) / 2 + va * vb * oa * ob)
    gam = 2.0 * M * (va * va * oa * oa + vb * vb * ob * ob + 2.0 * va * vb * oa * ob)
    return tr, tiles, gam


def workload_flops_w(w):
    if w.get("kind") == "unrestricted":
        return sum(unrestricted_parts(w["N"], w["o"], w["ob"], w["M"]))
    return workload_flops(w["N"], w["o"], w["M"], w["gradient"])


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
REF_SAMPLE = dict(N=300, o=10, M=1200)


def run_reference_once(w, seed, nthreads):
    """One bounded sample of the workload on the reference's own CPU code:
    CholeskyOMP2's energy + orbital-gradient evaluation (t2, E, OPDM,
    generalized Fock, w_ai; src/mp2/cholesky_omp2.cc:441-466) for gradient
    workloads (separate alpha / beta orbitals for the unrestricted one),
    CholeskyRMP2::compute for energy workloads."""
    from mshqc_b200 import synthetic as syn
    from oracle import ref
    N, o, M = REF_SAMPLE["N"], REF_SAMPLE["o"], REF_SAMPLE["M"]
    unres = w.get("kind") == "unrestricted"
    ob = o - 1 if unres else o
    base = syn.make_inputs(N, o, M, seed=seed)
    sig = syn.twin_sigma(N, o, M, base.alpha.eps)
    inp = syn.make_inputs(N, o, M, seed=seed, sigma=sig, nocc_beta=ob if unres else None)
    a = inp.alpha
    b = inp.beta if unres else a
    if w["gradient"]:
        H = np.eye(N)   # the cost of the Fock build does not depend on H
        r = ref.omp2_pieces(inp.L, a.C, b.C, a.eps, b.eps, o, ob, H, nthreads=nthreads)
        what = "CholeskyOMP2 energy + w_ai"
    else:
        r = ref.rmp2(inp.L, a.C, a.eps, o, nthreads=nthreads)
        what = "CholeskyRMP2::compute"
    if unres:
        flops = sum(unrestricted_parts(N, o, ob, M))
    else:
        flops = workload_flops(N, o, M, w["gradient"])
    return r["seconds"], flops, f"N={N}, o={o}{'/%d' % ob if unres else ''}, M={M} {what}"


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
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "sample": sample},
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": nthreads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


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
    gradient = w["gradient"]
    prec = capi.PRECISIONS[w["precision"]]
    unres = w.get("kind") == "unrestricted"
    kind = capi.UNRESTRICTED if unres else capi.RESTRICTED
    ob = w.get("ob", o)
    seed = 1000 + rank

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

    def step(context, precision, C, eps):
        context.set_orbitals(capi.ALPHA, C, eps, o)            # new orbitals: full recompute
        if unres:
            context.set_orbitals(capi.BETA, Cb_dev, eb_dev, ob)
        if gradient:
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
    flops = workload_flops_w(w)
    value = world * flops * args.steps / elapsed / 1e12
    mixed_res = r

    # ---- FP64 path on the same inputs (comparison and error) ---------------
    fp64 = {}
    if prec != capi.FP64 and not args.no_fp64:
        # one FP64 step, not warmed up: the same transforms ran above and the
        # FP64 kernels' first-launch cost is negligible next to the step
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        r64 = step(ctx, capi.FP64, C_dev, e_dev)
        t1.record(stream)
        torch.cuda.synchronize()
        ms64 = t0.elapsed_time(t1)
        if gradient:
            e3, e64 = mixed_res.energy["total"], r64.energy["total"]
            pairs = [(mixed_res.dC_a, r64.dC_a, mixed_res.deps_a, r64.deps_a)]
            if unres:
                pairs.append((mixed_res.dC_b, r64.dC_b, mixed_res.deps_b, r64.deps_b))
            fp64 = {"fp64_ms_per_step": ms64, "fp64_tflops": flops / (ms64 / 1e3) / 1e12,
                    "speedup_mixed_vs_fp64": ms64 / (1e3 * elapsed / args.steps),
                    "energy_fp64": e64, "energy_mixed": e3,
                    "energy_error_uEh": abs(e3 - e64) * 1e6,
                    "max_abs_dC_error": max(float(np.max(np.abs(x - y))) for x, y, _, _ in pairs),
                    "max_abs_deps_error": max(float(np.max(np.abs(x - y))) for _, _, x, y in pairs),
                    "max_abs_dC": max(float(np.max(np.abs(y))) for _, y, _, _ in pairs)}
        else:
            fp64 = {"fp64_ms_per_step": ms64,
                    "speedup_mixed_vs_fp64": ms64 / (1e3 * elapsed / args.steps),
                    "energy_error_uEh": abs(mixed_res["total"] - r64["total"]) * 1e6}

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
                return ctx_h.mp2_gradient(kind, prec)       # results copied to host
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
        e2e = {"value": world * flops * args.steps / e2e_elapsed / 1e12, "unit": "TFLOP/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": 1e3 * e2e_elapsed / args.steps}
        ctx_h.close()
    else:
        ctx.close()

    # ---- roofline of the dominant kernel ----------------------------------
    peaks, peak_src = measured_peaks()
    st = {k: statistics.median(s[k] for s in stages) for k in stages[0]}
    if gradient and unres:
        _, ftiles, fgam = unrestricted_parts(N, o, ob, M)
        cand = {"amplitude": ("vtile_tc_kernel", ftiles), "gamma": ("gamma_tc_kernel", fgam)}
    elif gradient:
        cand = {"amplitude": ("vtile_tc_kernel", flops_energy(N, o, M)),   # unique pairs i <= j
                "gamma": ("gamma_tc_kernel", flops_gamma(N, o, M))}
    else:
        cand = {"pair_energy": ("pair_energy_tc_kernel<RESTRICTED>", flops_energy(N, o, M))}
    dom = max(cand, key=lambda k: st.get(k, 0.0))
    kname, kflops = cand[dom]
    kms = st[dom]
    achieved = kflops / (kms / 1e3) / 1e12 if kms > 0 else None
    if prec == capi.FP64:
        peak = measure_fp64_peak(torch, dev)
        peak_note = "FP64 cuBLAS DGEMM 8192^3 measured in this run"
    else:
        peak = peaks["bf16_tflops_sustained"] / 3.0
        peak_note = (f"dense 16-bit tensor peak ({peak_src}, sustained "
                     f"{peaks['bf16_tflops_sustained']}) / 3: three products per useful product")

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": ("f64" if prec == capi.FP64 else
                      "fp16x3 (scaled fixed point, exact f32 accumulate; f64 denominators, sums)"),
            "data": "synthetic (seeded recipe, scaled twin, device Philox stream for L)",
            "config": {"workload": args.workload, "N": N, "o": o, "v": N - o, "M": M,
                       **({"o_beta": ob} if unres else {}),
                       "kind": "unrestricted" if unres else "restricted",
                       "precision": w["precision"], "gradient": gradient,
                       "sigma": sigma, "parallelism": f"replicas{world}",
                       "vectors": "generated on the device per chunk" if gen else "stored",
                       "l2": "inputs larger than L2 (AO vectors %.1f GB%s, MO vectors %.2f GB)" % (
                           N * N * M * 8 / 1e9, ", regenerated, never stored" if gen else "",
                           o * (N - o) * M * 8 / 1e9),
                       "stage_ms": st, "mixed_exact_accumulation": exact, **fp64},
            "clocks": clk,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "roofline": {"bound": "tensor", "kernel": kname, "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": (achieved / peak) if achieved else None,
                         "traffic": None,
                         "traffic_note": "not captured at this size; small-case DRAM traffic does not scale "
                                         "in proportion (profiles/launches_cdmp2_grad_n2000_o200_m8000.md)",
                         "peak_source": peak_note, "kernel_ms_per_step": kms},
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
            except Exception as ex:   # a reported baseline, not the product
                line["cpu_baseline"] = {"value": None, "error": str(ex)}
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
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
