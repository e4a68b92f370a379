#!/usr/bin/env python
"""Benchmark of the TensorBLAS hot path on B200 (one JSON line on rank 0).

Step = one plain SYRK (lower, C = A A^T, n = k = 16384, nb = 256, A i.i.d.
U[-1,1]) + one plain TRSM (left/lower/no-trans/non-unit, m = n = 16384,
nb = 512, A off-diagonal U[-1,1]/sqrt(n), diagonal U[1,2], B U[-1,1]).
Metric: effective TFLOP/s = (n^2 k + m^2 n) / device time (reference flop
conventions, testing/testing_syrk.cu:100 and testing_trsm.cu:61). The chosen
(split, FP32-accurate) form is timed the same way and reported beside it,
each with its error against an FP64 evaluation on the host.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]

N > 1 runs independent replicas, one per GPU (the path has no exchange step);
value = all ranks' flops / max-over-ranks device time.

--impl reference runs the reference library (built from its sources into
oracle/_ref by oracle/Makefile) on the same seeded inputs and prints its line
with the same config; it also records sampled entries of its SYRK and TRSM
outputs in .bench_reference_samples.npz, from which a later run of this arm on
the same machine reports its agreement with the reference
(agreement_vs_reference).
"""
import argparse
import datetime
import json
import os
import subprocess
import sys
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tensor-blas_b200", "python"))
METRIC = "SYRK/TRSM n=16384 eff. TFLOP/s at stated FP64-oracle error, chosen vs plain"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["mine", "reference"], default="mine")
    p.add_argument("--n", type=int, default=16384)
    p.add_argument("--nb-syrk", type=int, default=256)
    p.add_argument("--nb-trsm", type=int, default=512)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    p.add_argument("--no-extra", action="store_true", help="skip the other configurations")
    p.add_argument("--profile-step", action="store_true",
                   help="run one untimed step (plain, then split) and exit: the command profiled with ncu")
    p.add_argument("--plain-only", action="store_true", help="--profile-step: the plain step alone")
    p.add_argument("--profile-aux", action="store_true",
                   help="run the non-GEMM kernels once each (conversions, TRSM leaf inverses, Ozaki slicing, FP8 "
                        "quantisation) at bench sizes and exit: the command their ncu summaries come from")
    p.add_argument("--profile-gemm", type=int, default=0, metavar="N",
                   help="run three plain N x N x N SGEMMs and exit (the GEMM-engine ncu captures)")
    p.add_argument("--profile-syrk", type=int, default=0, metavar="N",
                   help="run two plain SYRKs n = k = N and exit (the SYRK captures)")
    p.add_argument("--split", action="store_true", help="--profile-syrk: split precision")
    p.add_argument("--profile-ozaki", type=int, default=0, metavar="N",
                   help="run two FP64 Ozaki DSYRKs n = k = N with 8 slices and exit (the Ozaki-engine ncu captures)")
    return p.parse_args()


# ------------------------------------------------------------------ process / ranks
def dist_setup(args):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE): NCCL
    on GPUs, gloo where no GPU is visible (the CPU tests of this plumbing)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    gpu = torch.cuda.is_available()
    if gpu:
        torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist

        if gpu:
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    """The largest of the ranks' values (device times: the job's time is the
    slowest rank's)."""
    if world == 1:
        return x
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_tflops(world, steps, flops_step, ms_max):
    """Whole-job throughput of N replicas: every rank runs `steps` steps of
    `flops_step`, the job takes the slowest rank's `ms_max`."""
    return world * steps * flops_step / (ms_max * 1e-3) / 1e12


def physical_gpu(local):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local < len(ids) and ids[local].isdigit():
            return int(ids[local])
    return local


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


SAMPLES = os.path.join(ROOT, ".bench_reference_samples.npz")


def workload(n, nb_syrk, nb_trsm):
    """The config both arms report: the same matrices, shapes and flops."""
    return {"workload": f"plain SYRK n=k={n} nb={nb_syrk} + plain TRSM m=n={n} nb={nb_trsm} (lower, non-unit, "
                        f"{n} right-hand sides) per step", "n": n, "precision": "plain",
            "l2": "inputs larger than L2 (1 GiB per matrix)",
            "parallelism": "replicas: one process per GPU, each running this step (n_gpus gives the count)"}


def sample_indices(n):
    """Entries compared with the reference: 4096 lower SYRK entries and 32
    rows of the right-side TRSM solution X (X A^T = B)."""
    g = np.random.Generator(np.random.PCG64(7))
    i, j = g.integers(0, n, 4096), g.integers(0, n, 4096)
    rows = np.random.Generator(np.random.PCG64(8)).integers(0, n, 32)
    return np.maximum(i, j), np.minimum(i, j), rows


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d.get("bf16_tflops"), d.get("bf16_tflops_sustained"), "measured"
    except (OSError, ValueError):
        return 1590.0, 1400.0, "fallback"


def measured_hbm():
    """HBM copy bandwidth (GB/s) and its source."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError, TypeError):
        return 6650.0, "fallback"


def traffic_summary():
    """DRAM bytes per algorithmic flop of the GEMM kernels, from a committed
    small-case ncu summary (scaled here to a launch by its flops)."""
    try:
        with open(os.path.join(ROOT, "profiles", "gemm_engine_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


# ------------------------------------------------------------------ inputs
def make_inputs(n, seed=1234):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    A = torch.rand(n, n, device="cuda", generator=g) * 2 - 1            # SYRK A (column-major storage)
    L = torch.rand(n, n, device="cuda", generator=g) * 2 - 1
    L = torch.tril(L, -1) / n ** 0.5 + torch.diag(torch.rand(n, device="cuda", generator=g) + 1)
    T = L.t().contiguous()                                             # column-major lower triangle
    del L
    B0 = torch.rand(n, n, device="cuda", generator=g) * 2 - 1           # column-major B
    return A, T, B0


# ------------------------------------------------------------------ error vs FP64 (sampled)
def fp64_errors(n, A, C, T, B0, X, seed=7):
    """Sampled errors against FP64 evaluation on the host.

    SYRK: 4096 random lower entries C_ij = sum_p a_ip a_jp in FP64.
    TRSM: 32 random columns x_j = A^{-1} b_j by FP64 forward substitution.
    Returns max elementwise relative and normwise relative error of each.
    """
    from scipy.linalg import solve_triangular

    g = np.random.Generator(np.random.PCG64(seed))
    # element (i, p) of the column-major n x k matrix A is Ah[p, i]
    Ah = A.cpu().numpy().astype(np.float64)
    i = g.integers(0, n, 4096)
    j = g.integers(0, n, 4096)
    lo, hi = np.maximum(i, j), np.minimum(i, j)
    ref = np.einsum("pk,pk->k", Ah[:, lo], Ah[:, hi])
    Cs = C.cpu().numpy()
    got = Cs[hi, lo].astype(np.float64)              # element (lo, hi) of column-major C at storage [hi, lo]
    d = np.abs(got - ref)
    syrk = {"max_rel": float(np.max(d / np.maximum(np.abs(ref), 1e-300))),
            "norm_rel": float(np.linalg.norm(d) / np.linalg.norm(ref)), "sample": "4096 entries"}
    cols = g.integers(0, n, 32)
    Lh = T.cpu().numpy().T.astype(np.float64)        # logical lower-triangular A
    Bh = B0.cpu().numpy().T.astype(np.float64)       # logical B (m x n)
    Xh = X.cpu().numpy().T.astype(np.float64)
    xr = solve_triangular(Lh, Bh[:, cols], lower=True)
    dx = np.abs(Xh[:, cols] - xr)
    trsm = {"max_rel": float(np.max(dx / np.maximum(np.abs(xr), 1e-300))),
            "norm_rel": float(np.linalg.norm(dx) / np.linalg.norm(xr)), "sample": "32 columns"}
    return {"syrk": syrk, "trsm": trsm}


# ------------------------------------------------------------------ arms
def run_mine(args, world, rank, local):
    import TensorBLAS as TB

    n = args.n
    flops_step = 2.0 * float(n) ** 3
    A, T, B0 = make_inputs(n)
    C = torch.zeros(n, n, device="cuda")
    Bw = torch.empty_like(B0)
    stream = torch.cuda.current_stream()

    def step(prec):
        TB.ssyrk(A, C, n, n, n, n, 1.0, 0.0, "N", args.nb_syrk, prec)
        TB.strsm("L", T, Bw, n, n, n, n, args.nb_trsm, prec)

    def timed(prec, steps, warmup):
        for _ in range(warmup):
            Bw.copy_(B0)
            step(prec)
        TB.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        l0 = TB.lib.tb_launch_count()
        for e0, e1 in evs:
            Bw.copy_(B0)                     # restore B (TRSM overwrites it); outside the event window
            e0.record(stream)
            step(prec)
            e1.record(stream)
        torch.cuda.synchronize()
        launches = TB.lib.tb_launch_count() - l0
        barrier(world)
        TB.synchronize()
        ms_total = sum(e0.elapsed_time(e1) for e0, e1 in evs)
        return ms_total, launches


    # ---- plain (headline), then chosen (split); clocks sampled over both timed regions
    sampler = Clocks(physical_gpu(local))
    ms_plain, launches = timed(TB.PLAIN, args.steps, args.warmup)
    ms_split, _ = timed(TB.SPLIT, args.steps, args.warmup)
    clk = sampler.stop()
    ms_plain = max_over_ranks(ms_plain, world)
    ms_split = max_over_ranks(ms_split, world)
    Bw.copy_(B0)
    step(TB.PLAIN)
    TB.synchronize()
    err_plain = fp64_errors(n, A, C, T, B0, Bw) if rank == 0 else None
    Bw.copy_(B0)
    step(TB.SPLIT)
    TB.synchronize()
    err_split = fp64_errors(n, A, C, T, B0, Bw) if rank == 0 else None
    # ---- TRSM alone in each precision, with the refinement sweep (plain
    # solve + split-product residual + plain correction) beside plain / split
    trsm_only = {}
    for prec, name in ((TB.PLAIN, "plain"), (TB.SPLIT, "split"), (TB.REFINE, "refine")):
        ms_t = _median_ms(lambda: TB.strsm("L", T, Bw, n, n, n, n, args.nb_trsm, prec), 5,  # noqa: B023
                          lambda: Bw.copy_(B0))
        Bw.copy_(B0)
        TB.strsm("L", T, Bw, n, n, n, n, args.nb_trsm, prec)
        TB.synchronize()
        e = fp64_errors(n, A, C, T, B0, Bw)["trsm"] if rank == 0 else None
        trsm_only[name] = {"ms": ms_t, "tflops": float(n) ** 3 / (ms_t * 1e-3) / 1e12, "errors_vs_fp64": e}

    ms_syrk = _median_ms(lambda: TB.ssyrk(A, C, n, n, n, n, 1.0, 0.0, "N", args.nb_syrk, TB.PLAIN), 5)
    # per-kernel rooflines: 5 plain steps (SYRK + TRSM) with every GEMM-engine
    # launch event-timed on its own stream (tb_profile_begin / end), split by
    # kernel (tb_profile_kernel): launch durations, algorithmic flops and
    # DRAM bytes, launches
    TB.lib.tb_profile_begin()
    for _ in range(5):
        Bw.copy_(B0)
        step(TB.PLAIN)
    torch.cuda.synchronize()
    ms, fl, cnt = TB.ctypes.c_double(), TB.ctypes.c_double(), TB.ctypes.c_long()
    TB.lib.tb_profile_end(TB.ctypes.byref(ms), TB.ctypes.byref(fl), TB.ctypes.byref(cnt))
    prof = (ms.value / 5, fl.value / 5, cnt.value / 5)
    kernels, kernel_bytes = {}, {}
    by = TB.ctypes.c_double()
    for kind in range(4):
        TB.lib.tb_profile_kernel(kind, TB.ctypes.byref(ms), TB.ctypes.byref(fl), TB.ctypes.byref(by),
                                 TB.ctypes.byref(cnt))
        if cnt.value:
            kernels[kind] = (ms.value / 5, fl.value / 5, cnt.value / 5)
            kernel_bytes[kind] = by.value / 5

    value = job_tflops(world, args.steps, flops_step, ms_plain)
    value_split = job_tflops(world, args.steps, flops_step, ms_split)
    agreement = agreement_vs_reference(TB, args, A, C, T, B0, Bw) if rank == 0 else None

    # ---- end to end through the public host-memory API (page-locked buffers):
    # every byte of the step's inputs crosses PCIe inside the timed region
    # and its results come back to host memory (tb_ssyrk_host / tb_strsm_host
    # stream them in panels and overlap the copies with the kernels)
    pin = lambda t: t.cpu().pin_memory()  # noqa: E731
    hA, hT, hB0 = pin(A), pin(T), pin(B0)
    hB = torch.empty_like(hB0).pin_memory()
    hC = torch.zeros(n, n, dtype=torch.float32).pin_memory()

    def e2e_step(em):
        TB.ssyrk_host(hA, hC, n, n, n, n, 1.0, 0.0, args.nb_syrk, TB.PLAIN)
        em.record(stream)
        TB.strsm_host("L", hT, hB, n, n, n, n, args.nb_trsm, TB.PLAIN)

    ms_e2e, ms_e2e_syrk = 0.0, 0.0
    for i in range(max(1, args.warmup) + args.e2e_steps):
        hB.copy_(hB0)                        # TRSM overwrites B in host memory; restored outside the timing
        torch.cuda.synchronize()
        barrier(world)
        e0, em, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        e2e_step(em)
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= max(1, args.warmup):
            ms_e2e += e0.elapsed_time(e1)
            ms_e2e_syrk += e0.elapsed_time(em)
    ms_e2e = max_over_ranks(ms_e2e, world)
    barrier(world)
    e2e_value = job_tflops(world, args.e2e_steps, flops_step, ms_e2e)
    if rank == 0:
        # the host copies must reproduce the device results
        Bw.copy_(B0)
        step(TB.PLAIN)
        TB.synchronize()
        ok = torch.equal(hB, Bw.cpu()) and torch.equal(torch.triu(hC), torch.triu(C.cpu()))
    W = 1024
    tri = sum((n - c0) * min(W, n - c0) for c0 in range(0, n, W)) * 4    # A's lower triangle / C's row panels
    diag = sum(min(W, n - r0) ** 2 for r0 in range(0, n, W)) * 4          # C's diagonal blocks (kept intact)
    h2d_bytes = n * n * 4 + tri + n * n * 4 + diag
    d2h_bytes = tri + n * n * 4

    if rank != 0:
        return None
    burst, sustained, peak_src = measured_peaks()
    gemm_ms, gemm_flops, gemm_launches = prof
    tr = traffic_summary() or {}
    names = {0: "tb::gemm_kernel (single-CTA tiles: TRSM leaf products and K <= 1024 updates)",
             1: "tb::gemm_pair_kernel (CTA-pair 256 x 256 tiles: SYRK bands and long-K TRSM updates)",
             2: "tb::trsm_dag_kernel (persistent TRSM solve)",
             3: "tb::oz_* (Ozaki INT8 engine)"}
    keys = {0: "gemm_kernel", 1: "gemm_pair_kernel", 2: "trsm_dag_kernel", 3: "ozaki"}
    per_kernel = {}
    for kind, (ms, fl, cnt) in kernels.items():
        ach = fl / (ms * 1e-3) / 1e12 if ms > 0 else None
        t = tr.get(keys[kind], {})
        per_kernel[keys[kind]] = {
            "bound": "tensor", "kernel": names[kind], "achieved": ach, "peak": burst, "unit": "TFLOP/s",
            "frac": (ach / burst) if ach and burst else None, "launches_per_step": cnt,
            "ms_per_step": ms, "flops_per_launch": fl / cnt if cnt else None,
            "share_of_step_gemm_time": ms / sum(v[0] for v in kernels.values()),
            "traffic": t["bytes_per_flop"] * fl / cnt if ("bytes_per_flop" in t and cnt) else None,
            "traffic_note": t.get("note")}
        if kind == 0 and ms > 0:
            # the short launches move more bytes than their MMAs take time:
            # their bound is HBM (algorithmic bytes: operands once, C read
            # and written, FP16 side copies)
            hbm, hbm_src = measured_hbm()
            gbs = kernel_bytes[kind] / (ms * 1e-3) / 1e9
            per_kernel[keys[kind]]["hbm"] = {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s",
                                             "frac": gbs / hbm, "bytes_per_launch": kernel_bytes[kind] / cnt,
                                             "peak_source": f"{hbm_src} hbm_gbs"}
    dominant = keys[max(kernels, key=lambda k: kernels[k][0])]
    roof = dict(per_kernel[dominant])
    roof.update({"peak_source": f"{peak_src} bf16_tflops (burst: each launch timed alone; sustained {sustained})",
                 "achieved_note": "algorithmic flops of the kernel's launches in one plain step (nominal BLAS3 "
                                  "counts of the tiles' products) / the device time during which at least one "
                                  "of them ran (union of their CUDA-event intervals; the SYRK row bands and the "
                                  "TRSM's two streams overlap launches), 5 steps",
                 "step_gemm": {"achieved": gemm_flops / (gemm_ms * 1e-3) / 1e12 if gemm_ms > 0 else None,
                               "launches_per_step": gemm_launches,
                               "note": "all GEMM launches of the step: flops / union of their intervals"},
                 "other_kernels": {k: v for k, v in per_kernel.items() if k != dominant}})
    line = {
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_plain / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f16 operands, f32 accumulate", "data": "synthetic (seeded)",
        "config": workload(n, args.nb_syrk, args.nb_trsm),
        "detail": {"syrk_ms": ms_syrk, "trsm_ms": trsm_only["plain"]["ms"],
                   "timing": "median per call, CUDA events, device-resident", "trsm_side": "left (A X = B)"},
        "errors_vs_fp64": err_plain,
        "agreement_vs_reference": agreement,
        "chosen": {"precision": "split (FP16 hi + scaled lo, 3 products, RN folds)", "value": value_split,
                   "ms_per_step": ms_split / args.steps, "ratio_vs_plain": value_split / value,
                   "errors_vs_fp64": err_split},
        "trsm_16384_by_precision": trsm_only,
        "e2e": {"value": e2e_value, "unit": "TFLOP/s", "steps": args.e2e_steps, "ms_per_step": ms_e2e / args.e2e_steps,
                "ms_syrk_host": ms_e2e_syrk / args.e2e_steps,
                "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
                "api": "TensorBLAS.ssyrk_host / TensorBLAS.strsm_host (tb_ssyrk_host / tb_strsm_host) on page-locked "
                       "host buffers",
                "matches_device_results": bool(ok)},
        "roofline": roof,
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import tb_cpu

        nc = 4096
        fl, reps, el = tb_cpu.time_step(nc, min_seconds=10.0)
        line["cpu_baseline"] = {"value": fl / 1e12, "unit": "TFLOP/s", "cores": tb_cpu.threads(), "kind": "port",
                                "sample": f"{reps} x (SYRK n=k={nc} + TRSM m=n={nc}, FP16-rounded operands, "
                                          f"FP32 OpenBLAS) in {el:.1f} s"}
        line["host_blas"] = {"unit": "TFLOP/s", "n": 4096, "cores": tb_cpu.threads(),
                             "library": "OpenBLAS (SciPy BLAS wrappers)",
                             "rates": tb_cpu.host_blas_rates(4096, 2.0)}
    if world == 1 and not args.no_extra:
        line["other_configs"] = other_configs(TB)
    return line


def agreement_vs_reference(TB, args, A, C, T, B0, Bw):
    """Normwise and largest elementwise relative difference between this
    library's plain outputs and the reference's own tc_syrk / tc_trsm outputs
    on the same seeded inputs (sampled entries the reference arm recorded in
    .bench_reference_samples.npz). TRSM is compared in the reference's form,
    X A^T = B, solved here with tb_strsm('R')."""
    n = args.n
    if not os.path.exists(SAMPLES):
        return {"status": "no reference samples: run bench.py --impl reference first on this machine"}
    z = np.load(SAMPLES)
    if int(z["n"]) != n or int(z["nb_syrk"]) != args.nb_syrk or int(z["nb_trsm"]) != args.nb_trsm:
        return {"status": "reference samples are for another configuration"}
    lo, hi, rows = sample_indices(n)
    Bw.copy_(B0)
    TB.ssyrk(A, C, n, n, n, n, 1.0, 0.0, "N", args.nb_syrk, TB.PLAIN)
    TB.strsm("R", T, Bw, n, n, n, n, args.nb_trsm, TB.PLAIN)
    TB.synchronize()
    mine_s = C.cpu().numpy()[hi, lo].astype(np.float64)
    mine_t = Bw[:, torch.from_numpy(rows).cuda()].cpu().numpy().T.astype(np.float64)   # rows of X
    out = {"sample": "4096 lower SYRK entries; 32 rows of X (X A^T = B)",
           "reference": "tc_syrk / tc_trsm built from the reference's sources (oracle/_ref)"}
    for name, mine, ref in (("syrk", mine_s, z["syrk"]), ("trsm", mine_t, z["trsm_rows"])):
        d = np.abs(mine - ref)
        out[name] = {"norm_rel": float(np.linalg.norm(d) / np.linalg.norm(ref)),
                     "max_rel": float(np.max(d / np.maximum(np.abs(ref), 1e-30)))}
    out["reference_errors_vs_fp64"] = {"syrk": float(z["err_syrk"]), "trsm": float(z["err_trsm"])}
    return out


def _median_ms(fn, reps, prep=None):
    fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        if prep:
            prep()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return float(np.median(out))


def blas3_config(TB):
    """SYR2K n=16384 k=4096, TRMM left/upper m=n=16384 and SYMM left/lower
    m=n=16384 with entries N(0,1) * 2^U(-8,8): plain, split and FP8-e4m3
    (per-128x128-block scaled), each with a sampled FP64 error (the
    reference's tc_syr2k / tc_trmm / tc_symm are timed by the reference arm
    on inputs of the same shape). Flop conventions: SYR2K 2 n^2 k, TRMM m^2 n, SYMM 2 m^2 n."""
    lib = TB.lib
    gen = torch.Generator(device="cuda")
    gen.manual_seed(99)
    rng = np.random.Generator(np.random.PCG64(99))

    def draw(r, c):  # torch (r, c) = column-major c x r matrix
        x = torch.randn(r, c, device="cuda", generator=gen)
        return x * torch.exp2(torch.rand(r, c, device="cuda", generator=gen) * 16 - 8)

    def err(got, ref):
        d = np.abs(got - ref)
        return {"norm_rel": float(np.linalg.norm(d) / np.linalg.norm(ref)),
                "max_rel": float(np.max(d / np.maximum(np.abs(ref), 1e-300)))}

    out = {}
    n, k = 16384, 4096
    # SYR2K: A, B n x k column-major (torch (k, n)); C lower
    A, B = draw(k, n), draw(k, n)
    C = torch.zeros(n, n, device="cuda")
    Ah, Bh = A.cpu().numpy().astype(np.float64), B.cpu().numpy().astype(np.float64)
    i = rng.integers(0, n, 256)
    j = rng.integers(0, n, 256)
    lo, hi = np.maximum(i, j), np.minimum(i, j)
    ref = np.einsum("pk,pk->k", Ah[:, lo], Bh[:, hi]) + np.einsum("pk,pk->k", Bh[:, lo], Ah[:, hi])
    entry = {"n": n, "k": k, "flops": 2.0 * n * n * k}
    for prec, name in ((TB.PLAIN, "plain"), (TB.SPLIT, "split"), (TB.FP8, "fp8")):
        run = lambda: TB._check(lib.tb_ssyr2k(b"L", b"N", n, k, 1.0, A.data_ptr(), n, B.data_ptr(), n,  # noqa: E731
                                              0.0, C.data_ptr(), n, 256, prec))
        ms = _median_ms(run, 5)
        got = C.cpu().numpy()[hi, lo].astype(np.float64)
        entry[name] = {"ms": ms, "tflops": entry["flops"] / (ms * 1e-3) / 1e12, "errors_vs_fp64": err(got, ref)}
    out["syr2k"] = entry
    del A, B, C, Ah, Bh
    torch.cuda.empty_cache()

    m = n = 16384
    A, B = draw(m, m), draw(n, m)  # A m x m (upper part read), B m x n, column-major
    C = torch.zeros(n, m, device="cuda")
    An, Bn = A.cpu().numpy(), B.cpu().numpy()  # An[p, i] = A(i, p); Bn[j, p] = B(p, j)
    i = rng.integers(0, m, 128)
    j = rng.integers(0, n, 128)
    # TRMM upper: C(i, j) = sum_{p >= i} A(i, p) B(p, j)
    ref = np.array([np.dot(An[ii:, ii].astype(np.float64), Bn[jj, ii:].astype(np.float64)) for ii, jj in zip(i, j)])
    entry = {"m": m, "n": n, "uplo": "U", "flops": float(m) * m * n}
    for prec, name in ((TB.PLAIN, "plain"), (TB.SPLIT, "split"), (TB.FP8, "fp8")):
        run = lambda: TB._check(lib.tb_strmm(b"U", m, n, 1.0, A.data_ptr(), m, B.data_ptr(), m,  # noqa: E731
                                             C.data_ptr(), m, 256, prec))
        ms = _median_ms(run, 5)
        got = C.cpu().numpy()[j, i].astype(np.float64)
        entry[name] = {"ms": ms, "tflops": entry["flops"] / (ms * 1e-3) / 1e12, "errors_vs_fp64": err(got, ref)}
    out["trmm"] = entry
    # SYMM lower: C(i, j) = sum_p A(i, p) B(p, j), A(i, p) = A(max, min) from the lower triangle
    ref = []
    for ii, jj in zip(i, j):
        row = np.concatenate([An[:ii + 1, ii], An[ii, ii + 1:]]).astype(np.float64)
        ref.append(np.dot(row, Bn[jj, :].astype(np.float64)))
    ref = np.array(ref)
    entry = {"m": m, "n": n, "uplo": "L", "flops": 2.0 * m * m * n}
    for prec, name in ((TB.PLAIN, "plain"), (TB.SPLIT, "split"), (TB.FP8, "fp8")):
        run = lambda: TB._check(lib.tb_ssymm(b"L", m, n, 1.0, A.data_ptr(), m, B.data_ptr(), m, 0.0,  # noqa: E731
                                             C.data_ptr(), m, prec))
        ms = _median_ms(run, 5)
        got = C.cpu().numpy()[j, i].astype(np.float64)
        entry[name] = {"ms": ms, "tflops": entry["flops"] / (ms * 1e-3) / 1e12, "errors_vs_fp64": err(got, ref)}
    out["symm"] = entry
    del A, B, C
    torch.cuda.empty_cache()
    return out


def other_configs(TB):
    """The other configurations of the hot path, one measurement each (the
    reference library's timings of the same configurations are in the
    reference arm's line): SYRK n=k=4096 (plain, the CPU-runnable case), FP64
    DSYRK n=k=8192 on the INT8 Ozaki engine with the automatic slice count,
    SYR2K / TRMM / SYMM at 16384, and 512 uneven SYRK/TRSM instances as one
    grouped batch vs a per-instance loop, in both precisions."""
    import ctypes

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import tb_oracle as orc

    res = {}
    # ---- SYRK n = k = 4096 (plain)
    n = 4096
    A = torch.rand(n, n, device="cuda") * 2 - 1
    C = torch.zeros(n, n, device="cuda")
    ms = _median_ms(lambda: TB.ssyrk(A, C, n, n, n, n, 1.0, 0.0, "N", 256, TB.PLAIN), 20)
    res["syrk_4096_plain"] = {"ms": ms, "tflops": float(n) ** 3 / (ms * 1e-3) / 1e12}
    del A, C
    # ---- Ozaki DSYRK n = k = 8192, slices chosen by the library
    lib = TB.lib
    P, L = ctypes.c_void_p, ctypes.c_long
    lib.tb_dsyrk_ozaki.argtypes = [ctypes.c_char, ctypes.c_char, L, L, ctypes.c_double, P, L, ctypes.c_double, P, L,
                                   ctypes.c_int]
    n = k = 8192
    oz = {}
    for phi in (0.5, 2.0):
        g = np.random.Generator(np.random.PCG64(17))
        Ah = g.standard_normal((n, k)) * np.exp(phi * g.standard_normal((n, k)))
        dA = torch.from_numpy(np.ascontiguousarray(Ah.T)).cuda()
        dC = torch.zeros(n, n, dtype=torch.float64, device="cuda")
        run = lambda: TB._check(lib.tb_dsyrk_ozaki(b"L", b"N", n, k, 1.0, dA.data_ptr(), n, 0.0,  # noqa: E731
                                                   dC.data_ptr(), n, 0))
        ms = _median_ms(run, 5)
        Ch = dC.cpu().numpy().T
        r = g.integers(0, n, 3000)
        c = g.integers(0, n, 3000)
        lo, hi = np.maximum(r, c), np.minimum(r, c)
        ex = orc.syrk_extended(Ah, lo, hi)
        d = np.abs(Ch[lo, hi] - ex).astype(np.float64)
        oz[f"phi={phi}"] = {"slices": "automatic", "ms": ms, "tflops_eff": float(n) ** 2 * k / (ms * 1e-3) / 1e12,
                            "normwise_err_vs_long_double": float(np.linalg.norm(d) /
                                                                 np.linalg.norm(ex.astype(np.float64)))}
        del dA, dC
    res["dsyrk_ozaki_8192"] = oz
    torch.cuda.empty_cache()
    res["syr2k_trmm_symm_16384"] = blas3_config(TB)
    res["batched_512_uneven"] = batch_config(TB)
    return res


def batch_config(TB):
    """512 independent instances, n log-uniform in [64, 2048], half SYRK
    (k = n) and half TRSM (X A^T = B, square B): the grouped batch (a few
    launches, replayed as one CUDA graph) against a loop of per-instance
    calls, each in the plain and the split precision, with the worst normwise
    error against FP64 over sampled instances."""
    from scipy.linalg import solve_triangular

    g = np.random.Generator(np.random.PCG64(2025))
    ns = np.round(np.exp(g.uniform(np.log(64), np.log(2048), 512))).astype(int)
    kinds, As, BC, B0 = [], [], [], []
    flops = 0.0
    for i, m in enumerate(ns):
        if i % 2 == 0:
            a = torch.rand(m, m, device="cuda") * 2 - 1
            bc = torch.zeros(m, m, device="cuda")
        else:
            lt = torch.tril(torch.rand(m, m, device="cuda") * 2 - 1, -1) / m ** 0.5
            a = (lt + torch.diag(torch.rand(m, device="cuda") + 1)).t().contiguous()
            bc = torch.rand(m, m, device="cuda") * 2 - 1
        kinds.append(i % 2)
        As.append(a)
        BC.append(bc)
        B0.append(bc.clone())
        flops += float(m) ** 3
    restore = lambda: [b.copy_(b0) for b, b0 in zip(BC, B0)]  # noqa: E731
    check = list(range(0, 512, 16)) + list(range(1, 512, 16))  # 32 SYRK and 32 TRSM instances

    def errors():
        worst = {"syrk": 0.0, "trsm": 0.0}
        for i in check:
            Ai = As[i].cpu().numpy().T.astype(np.float64)
            got = BC[i].cpu().numpy().T.astype(np.float64)
            if kinds[i] == 0:
                ref = Ai @ Ai.T
                low = np.tril(np.ones_like(ref, dtype=bool))
                e = float(np.linalg.norm((got - ref)[low]) / np.linalg.norm(ref[low]))
                worst["syrk"] = max(worst["syrk"], e)
            else:
                b0 = B0[i].cpu().numpy().T.astype(np.float64)
                ref = solve_triangular(Ai, b0.T, lower=True).T
                worst["trsm"] = max(worst["trsm"], float(np.linalg.norm(got - ref) / np.linalg.norm(ref)))
        return worst

    out = {"instances": 512, "flops_sum_n3": flops,
           "timing": "median of CUDA-event-timed replays (graph) / loops; B restored outside the timed region",
           "errors": "worst normwise error vs FP64 over 32 SYRK and 32 TRSM instances"}
    for prec, name in ((TB.PLAIN, "plain"), (TB.SPLIT, "split")):
        batch = TB.Batch(kinds, As, BC, precision=prec)
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            batch.run()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            batch.run()
        ms_graph = _median_ms(graph.replay, 5, restore)
        restore()
        graph.replay()
        torch.cuda.synchronize()
        e_grouped = errors()
        l0 = TB.lib.tb_launch_count()
        batch.run()
        torch.cuda.synchronize()
        launches = TB.lib.tb_launch_count() - l0
        del graph
        batch.close()

        def loop(prec=prec):
            for kind, a, bc, m in zip(kinds, As, BC, ns):
                if kind == 0:
                    TB.ssyrk(a, bc, m, m, m, m, 1.0, 0.0, "N", 256, prec)
                else:
                    TB.strsm("R", a, bc, m, m, m, m, 512, prec)

        ms_loop = _median_ms(loop, 3, restore)
        restore()
        loop()
        torch.cuda.synchronize()
        e_loop = errors()
        out[name] = {"grouped_graph_ms": ms_graph, "grouped_tflops": flops / (ms_graph * 1e-3) / 1e12,
                     "grouped_launches_per_run": int(launches), "grouped_errors_vs_fp64": e_grouped,
                     "per_instance_loop_ms": ms_loop, "per_instance_loop_tflops": flops / (ms_loop * 1e-3) / 1e12,
                     "loop_errors_vs_fp64": e_loop, "speedup_grouped_vs_loop": ms_loop / ms_graph}
    return out


def run_reference(args, world, rank, local):
    """The reference library (built from its sources into oracle/_ref/) on this
    B200, on the same seeded inputs as the library's arm: tc_syrk + tc_trsm
    (its right-side form X A^T = B: same shapes and flops), timed per call;
    its sampled outputs and their FP64 errors, recorded for the other arm's
    agreement check; and its timings of the other configurations."""
    if rank != 0:
        return None
    import ctypes

    so = os.path.join(ROOT, "oracle", "_ref", "libTensorBLAS_ref.so")
    if not os.path.exists(so):
        return {"impl": "reference", "unavailable": "oracle/_ref/libTensorBLAS_ref.so not built (make -C oracle)"}
    lib = ctypes.CDLL(so)
    P, L, I = ctypes.c_void_p, ctypes.c_long, ctypes.c_int
    for name, args_t in (("ref_time_syrk", [L, L, L, P, I, I]), ("ref_time_trsm", [L, L, L, P, P, I, I]),
                         ("ref_time_e2e", [L, L, L, P, P, P, I, I]), ("ref_time_syr2k", [L, L, L, P, P, I, I]),
                         ("ref_time_trmm", [L, L, L, P, P, I, I]), ("ref_time_symm", [L, L, P, P, I, I]),
                         ("ref_time_ozimmu_syrk", [L, L, L, P, I, I]), ("ref_time_cublas_dsyrk", [L, L, P, I, I])):
        getattr(lib, name).argtypes = args_t
        getattr(lib, name).restype = ctypes.c_double
    lib.ref_syrk.argtypes = [L, L, ctypes.c_float, P, ctypes.c_float, P, L]
    lib.ref_trsm.argtypes = [L, L, P, P, L]
    n = args.n
    A, T, B0 = make_inputs(n)
    hA = A.cpu().numpy()
    hT = T.cpu().numpy()                            # column-major lower-triangular A, as tc_trsm takes it
    hB = B0.cpu().numpy()
    del A, T, B0
    torch.cuda.empty_cache()
    sampler = Clocks(physical_gpu(local))
    t_syrk = lib.ref_time_syrk(n, n, args.nb_syrk, hA.ctypes.data_as(P), args.warmup, args.steps)
    t_trsm = lib.ref_time_trsm(n, n, args.nb_trsm, hT.ctypes.data_as(P), hB.ctypes.data_as(P), args.warmup,
                               args.steps)
    clk = sampler.stop()
    if t_syrk <= 0 or t_trsm <= 0:
        return {"impl": "reference", "unavailable": "reference routine failed on this device"}
    # end to end through the reference's public API: the same host <-> device
    # bytes per step as the library's own end-to-end measurement
    t_e2e = lib.ref_time_e2e(n, args.nb_syrk, args.nb_trsm, hA.ctypes.data_as(P), hT.ctypes.data_as(P),
                             hB.ctypes.data_as(P), 1, args.e2e_steps)
    # sampled outputs (for the library arm's agreement check) and their FP64 errors
    lo, hi, rows = sample_indices(n)
    hC = np.zeros((n, n), dtype=np.float32)
    hX = np.ascontiguousarray(hB.copy())
    rc = lib.ref_syrk(n, n, 1.0, hA.ctypes.data_as(P), 0.0, hC.ctypes.data_as(P), args.nb_syrk)
    rc |= lib.ref_trsm(n, n, hT.ctypes.data_as(P), hX.ctypes.data_as(P), args.nb_trsm)
    errors = None
    if rc == 0:
        from scipy.linalg import solve_triangular

        ref_s = hC[hi, lo].astype(np.float64)
        ref_t = hX[:, rows].T.astype(np.float64)      # rows of X (column-major storage)
        Ah = hA.astype(np.float64)
        exact_s = np.einsum("pk,pk->k", Ah[:, lo], Ah[:, hi])
        del Ah
        Lh = hT.T.astype(np.float64)
        exact_t = solve_triangular(Lh, hB[:, rows].astype(np.float64), lower=True).T
        del Lh
        e_s = float(np.linalg.norm(ref_s - exact_s) / np.linalg.norm(exact_s))
        e_t = float(np.linalg.norm(ref_t - exact_t) / np.linalg.norm(exact_t))
        errors = {"syrk": {"norm_rel": e_s, "sample": "4096 lower entries"},
                  "trsm": {"norm_rel": e_t, "sample": "32 rows of X (X A^T = B)"}}
        np.savez(SAMPLES, n=n, nb_syrk=args.nb_syrk, nb_trsm=args.nb_trsm, syrk=ref_s, trsm_rows=ref_t,
                 err_syrk=e_s, err_trsm=e_t)
    del hC, hX
    ms = t_syrk + t_trsm
    value = 2.0 * float(n) ** 3 / (ms * 1e-3) / 1e12
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f16 operands, f32 accumulate (cuBLAS GemmEx) + f32 cublasStrsm leaves", "data": "synthetic (seeded)",
        "config": workload(n, args.nb_syrk, args.nb_trsm),
        "detail": {"syrk_ms": t_syrk, "trsm_ms": t_trsm, "timing": "median per call, CUDA events, device-resident",
                   "trsm_side": "right (X A^T = B, the reference's tc_trsm form)"},
        "errors_vs_fp64": errors,
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": 1, "kind": "reference",
                         "sample": "the reference library itself (oracle/_ref, built from its sources for sm_100a; "
                                   "its path is GPU code on cuBLAS) timed on this B200"},
        "e2e": ({"value": 2.0 * float(n) ** 3 / (t_e2e * 1e-3) / 1e12, "unit": "TFLOP/s",
                 "steps": args.e2e_steps, "h2d_bytes_per_step": 3 * n * n * 4, "d2h_bytes_per_step": 2 * n * n * 4,
                 "api": "tc_syrk / tc_trsm with cudaMemcpyAsync from/to page-locked host buffers"}
                if t_e2e > 0 else {"value": None, "unit": "TFLOP/s", "note": "end-to-end run failed"}),
        "clocks": clk,
    }
    if not args.no_extra:
        line["other_configs"] = reference_other_configs(lib)
    return line


def reference_other_configs(lib):
    """The reference's timings of the other configurations, on inputs drawn
    as in the library arm: tc_syrk n=k=4096 (its one-full-GEMM branch,
    BLAS/tc_syrk.cu:104-110), tc_syr2k n=16384 k=4096, tc_trmm 16384 (lower:
    its only form; same flops as the library's upper case), tc_symm 16384,
    and FP64 SYRK n=k=8192 through tc_ozimmu_syrk (native FP64 cuBLAS
    recursion) and one cuBLAS DSYRK, the native-FP64 baselines of the Ozaki
    engine."""
    P = ctypes_P()
    out = {}
    n = 4096
    hA = (np.random.Generator(np.random.PCG64(1)).random((n, n), dtype=np.float32) * 2 - 1)
    t = lib.ref_time_syrk(n, n, 256, hA.ctypes.data_as(P), 3, 20)
    out["syrk_4096_plain"] = {"ms": t, "tflops": float(n) ** 3 / (t * 1e-3) / 1e12 if t > 0 else None,
                              "note": "n < 8192: the reference computes one full n x n x k GEMM"}
    g = np.random.Generator(np.random.PCG64(99))

    def wide(r, c):
        return np.ascontiguousarray((g.standard_normal((r, c)) * np.exp2(g.uniform(-8, 8, (r, c)))).astype(np.float32))

    n, k = 16384, 4096
    A, B = wide(k, n), wide(k, n)
    t = lib.ref_time_syr2k(n, k, 256, A.ctypes.data_as(P), B.ctypes.data_as(P), 1, 5)
    out["syr2k_16384x4096_plain"] = {"ms": t, "tflops": 2.0 * n * n * k / (t * 1e-3) / 1e12 if t > 0 else None}
    del A, B
    m = 16384
    A, B = wide(m, m), wide(m, m)
    At = np.ascontiguousarray(np.triu(A))   # storage (m, m) row-major = column-major A^T: keep A's lower part
    t = lib.ref_time_trmm(m, m, 256, At.ctypes.data_as(P), B.ctypes.data_as(P), 1, 5)
    out["trmm_16384_plain"] = {"ms": t, "tflops": float(m) ** 3 / (t * 1e-3) / 1e12 if t > 0 else None,
                               "note": "tc_trmm is lower-only"}
    del At
    t = lib.ref_time_symm(m, m, A.ctypes.data_as(P), B.ctypes.data_as(P), 1, 5)
    out["symm_16384_plain"] = {"ms": t, "tflops": 2.0 * float(m) ** 3 / (t * 1e-3) / 1e12 if t > 0 else None}
    del A, B
    n = k = 8192
    fp64 = {}
    for phi in (0.5, 2.0):
        g2 = np.random.Generator(np.random.PCG64(17))
        Ah = np.asfortranarray(g2.standard_normal((n, k)) * np.exp(phi * g2.standard_normal((n, k))))
        t_oz = lib.ref_time_ozimmu_syrk(n, k, 256, Ah.ctypes.data_as(P), 1, 3)
        t_cb = lib.ref_time_cublas_dsyrk(n, k, Ah.ctypes.data_as(P), 1, 3)
        fp64[f"phi={phi}"] = {"tc_ozimmu_syrk_ms": t_oz, "cublas_dsyrk_ms": t_cb}
        del Ah
    out["dsyrk_8192_native_fp64"] = fp64
    return out


def ctypes_P():
    import ctypes

    return ctypes.c_void_p


def profile_step(args):
    """One plain and one split step (plain only with --plain-only) on fresh
    inputs, nothing timed (the command the committed ncu summaries were
    captured from)."""
    import TensorBLAS as TB

    n = args.n
    A, T, B0 = make_inputs(n)
    C = torch.zeros(n, n, device="cuda")
    for prec in (TB.PLAIN,) if args.plain_only else (TB.PLAIN, TB.SPLIT):
        Bw = B0.clone()
        TB.ssyrk(A, C, n, n, n, n, 1.0, 0.0, "N", args.nb_syrk, prec)
        TB.strsm("L", T, Bw, n, n, n, n, args.nb_trsm, prec)
        TB.synchronize()
    print("profile step done", flush=True)


def profile_syrk(args):
    """Two untimed SYRKs n = k = args.profile_syrk (lower, 'N', nb 256; plain,
    or split with --split), nothing timed: the command the SYRK captures come
    from."""
    import TensorBLAS as TB

    n = args.profile_syrk
    A, _, _ = make_inputs(n)
    C = torch.zeros(n, n, device="cuda")
    for _ in range(2):
        TB.ssyrk(A, C, n, n, n, n, 1.0, 0.0, "N", args.nb_syrk, TB.SPLIT if args.split else TB.PLAIN)
    TB.synchronize()
    print("profile syrk done", flush=True)


def profile_gemm(args):
    """Three untimed plain SGEMMs of order args.profile_gemm (NN), nothing
    timed: the command the GEMM-engine ncu summaries were captured from."""
    import TensorBLAS as TB

    n = args.profile_gemm
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    X = torch.rand(n, n, device="cuda", generator=g) - 0.5
    Y = torch.rand(n, n, device="cuda", generator=g) - 0.5
    Z = torch.zeros(n, n, device="cuda")
    for _ in range(3):
        TB.sgemm("N", "N", n, n, n, 1.0, X, n, Y, n, 0.0, Z, n, TB.PLAIN)
    TB.synchronize()
    print("profile gemm done", flush=True)


def profile_ozaki(args):
    """Two untimed Ozaki DSYRKs n = k = args.profile_ozaki, 8 slices (lower,
    'N'): the command the Ozaki-engine ncu summaries were captured from."""
    import ctypes

    import TensorBLAS as TB

    m = args.profile_ozaki
    g = torch.Generator(device="cuda")
    g.manual_seed(9)
    D = torch.randn(m, m, dtype=torch.float64, device="cuda", generator=g)
    E = torch.zeros(m, m, dtype=torch.float64, device="cuda")
    L, P = ctypes.c_long, ctypes.c_void_p
    TB.lib.tb_dsyrk_ozaki.argtypes = [ctypes.c_char, ctypes.c_char, L, L, ctypes.c_double, P, L, ctypes.c_double, P, L,
                                      ctypes.c_int]
    for _ in range(2):
        TB._check(TB.lib.tb_dsyrk_ozaki(b"L", b"N", m, m, 1.0, D.data_ptr(), m, 0.0, E.data_ptr(), m, 8))
    TB.synchronize()
    print("profile ozaki done", flush=True)


def profile_aux(args):
    """One plain SYRK and TRSM at n (FP32->FP16 conversions, 32x32 and leaf
    inverses), one Ozaki DSYRK n=k=n/2 with the slice count chosen by the
    library (range measurement, exponent, slicing and level-fold passes) and
    one FP8 SYR2K n/2 x n/4 (block quantisation);
    nothing timed. At n = 8192 the whole run holds about 2 GB on the device
    (the size the ncu captures of these kernels use)."""
    import ctypes

    import TensorBLAS as TB

    n = args.n
    A, T, B0 = make_inputs(n)
    C = torch.zeros(n, n, device="cuda")
    TB.ssyrk(A, C, n, n, n, n, 1.0, 0.0, "N", args.nb_syrk, TB.PLAIN)
    TB.strsm("L", T, B0, n, n, n, n, args.nb_trsm, TB.PLAIN)
    TB.synchronize()
    del A, T, B0, C
    torch.cuda.empty_cache()
    m = n // 2
    D = torch.randn(m, m, dtype=torch.float64, device="cuda")
    E = torch.zeros(m, m, dtype=torch.float64, device="cuda")
    L, P = ctypes.c_long, ctypes.c_void_p
    TB.lib.tb_dsyrk_ozaki.argtypes = [ctypes.c_char, ctypes.c_char, L, L, ctypes.c_double, P, L, ctypes.c_double, P, L,
                                      ctypes.c_int]
    TB._check(TB.lib.tb_dsyrk_ozaki(b"L", b"N", m, m, 1.0, D.data_ptr(), m, 0.0, E.data_ptr(), m, 0))
    del D, E
    kk = m // 2
    X = torch.randn(kk, m, device="cuda")
    Y = torch.randn(kk, m, device="cuda")
    Z = torch.zeros(m, m, device="cuda")
    TB._check(TB.lib.tb_ssyr2k(b"L", b"N", m, kk, 1.0, X.data_ptr(), m, Y.data_ptr(), m, 0.0, Z.data_ptr(), m, 256,
                               TB.FP8))
    TB.synchronize()
    print("profile aux done", flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.profile_aux:
        profile_aux(args)
        return
    if args.profile_gemm:
        profile_gemm(args)
        return
    if args.profile_ozaki:
        profile_ozaki(args)
        return
    if args.profile_syrk:
        profile_syrk(args)
        return
    if args.profile_step:
        profile_step(args)
        return
    try:
        line = run_mine(args, world, rank, local) if args.impl == "mine" else run_reference(args, world, rank, local)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
