#!/usr/bin/env python
"""Benchmarks on B200.  The default workload is the batched uneven SVD.

Default workload (one "step"): 100,000 square f64 matrices, n ~ U{2..64},
A = Q1 diag(s) Q2^T with Haar Q1, Q2, s_i = 10^(-k i/(n-1)), k ~ U[0, 12],
5% with a repeated-singular-value cluster (seeded synthetic data; the
reference publishes no dataset).  Each matrix takes the exact route the
reference dispatcher takes for it: LieSvdMicro for n <= 4, LieSvdSmall
otherwise (newton_schulz_polar + Jacobi eigensolve + U = QV + repair).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload batched|polar|jade|single] [--precision fp64|tf32|bf16]

Other workloads (each prints its own JSON line):
  polar  : Newton-Schulz polar factor of 16 dense matrices per step, 4096x4096
           and 8192x2048 alternating, A = Q1 diag(s) Q2^T with geometric spectra
           of condition 1e2, 1e5, 1e8 (metric: polar TFLOP/s);
  jade   : Phase-JADE of 512 families of K=64 symmetric 256x256 matrices,
           A_k = Q diag(d_k) Q^T + eps E_k, eps cycling over {0, 1e-8, 1e-4}
           (metric: families/s);
  single : one 64x64 Gaussian through the exact polar/Jacobi route (SVDs/s);
  adjoint: SVD/polar vector-Jacobian products of 4,096 matrices 128x64 (sigma
           uniform in [0.1, 10], gap >= 1e-3, 10% with one 1e-6 gap) from the
           stored rotor streams, cotangents N(0,1) on U, S, V and U V^T (VJPs/s);
  bss    : Phase-BSS (LieSvdBss.separate) of 32 mixed sinusoid-plus-noise
           channels x 2^20 samples from host arrays, lags {1, 2, 3, 5}
           (samples/s, copies inside the step).

Prints ONE JSON line (rank 0).  ``value`` is SVDs/s of the whole job with the
inputs resident in HBM (CUDA events on the launching stream, max over ranks);
``e2e`` is the same metric through the C ABI with host (pinned) buffers, the
host<->device copies inside the timed region.  ``--impl reference`` times the
CPU restatement of the reference (the Rust crate cannot be built here) on the
host cores over a bounded sample of the same workload.
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

METRIC = "SVDs/sec & polar TFLOP/s, mixed+refined vs plain FP64, at 1e-12 sigma rel err"
# dram__bytes_read.sum + dram__bytes_write.sum of one batched_kernel launch on
# 20,000 matrices of this workload (ncu --set full): 655.3 MB, i.e. per matrix
NCU_DRAM_BYTES_PER_MATRIX = 655.3e6 / 20000
WORKLOAD = "batched_uneven_svd_100k_n2-64_kappa1e0-1e12"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--count", type=int, default=100_000)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "tf32", "bf16"])
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision comparisons added to the batched line")
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="batched workload on N GPUs: weak = a full batch per rank; strong = one "
                         "batch split into cost-balanced contiguous shards")
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "polar", "jade", "single", "adjoint", "svd_large", "bss"])
    ap.add_argument("--families", type=int, default=512)
    ap.add_argument("--polar-size", default="full", choices=["full", "small"],
                    help="small: 2048x2048 and 4096x1024 instead of 4096x4096 and 8192x2048")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers --

def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def flops_per_matrix(n, ns_iters, sweeps, rotations, route):
    """FP64 flops of one solve by the reference algorithm (the algorithmic
    count the roofline uses).  Small route: Newton-Schulz iterations x
    (X^T X + X T), the final X^T X, P = Q^T A, U = Q V and U^T U, each 2n^3
    (src/lie_svd_small.rs:158-183, :296-323); per Jacobi sweep the off-norm
    test, n(n-1) (:220-228); per accepted rotation the update of two rows and
    columns of P and two columns of V, 12n (:244-270).  Micro route: per
    rotation 4 two-row/column updates (~24n)."""
    n = n.astype(np.float64)
    small = (4.0 * ns_iters + 8.0) * n ** 3 + sweeps * n * (n - 1) + rotations * 12 * n
    micro = rotations * 24.0 * n + 2 * n ** 3
    return np.where(route == 0, micro, small)


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_for(self, count: int, timeout: float = 2.0):
        """Block until ``count`` samples have arrived (bounded), so that a
        timed region shorter than the 200 ms sampling period still has a
        sample at each end."""
        end = time.perf_counter() + timeout
        while self.proc is not None and len(self.lines) < count and time.perf_counter() < end:
            time.sleep(0.01)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def fp64_peak_tflops(torch, device) -> float:
    """cuBLAS DGEMM throughput on this GPU (best of 5, 8192^3)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    best = 0.0
    for _ in range(6):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def batched_config(args, ws):
    """The ``config`` of the batched workload: one dict for both arms."""
    return {"workload": WORKLOAD,
            "count_per_gpu" if args.scaling == "weak" else "count_total": args.count,
            "n_range": [2, 64],
            "kappa": "10^U[0,12]", "degenerate_fraction": 0.05,
            "precision": args.precision,
            "route": "LieSvdMicro (n<=4) / LieSvdSmall",
            "l2": "inputs 1.1 GB per step, larger than the 126 MB L2",
            "parallelism": f"dp{ws} ({args.scaling} scaling, independent shards)"}


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # noqa: E402  (checker / CPU baseline only)
    O.lib()
    return O


def cpu_sample(ns, a, count: int, seed: int, cores: int):
    """Solves `count` matrices drawn uniformly (without replacement) from the
    batch with the oracle (the C++ restatement of the reference CPU path,
    single-threaded per matrix like the reference) in one threaded call on
    `cores` host threads.  Returns (solved, seconds)."""
    O = _oracle()
    idx = np.random.default_rng(seed).permutation(ns.size)[:count]
    t0 = time.perf_counter()
    got, *_ = O.svd_batch(ns, a, idx, cores)
    return got, time.perf_counter() - t0


def cpu_baseline(ns, a, seconds: float, seed: int):
    """The oracle on all host cores over a bounded random sample of the
    workload sized for about `seconds` of CPU time (calibrated on a small
    sample first)."""
    cores = cpu_cores()
    got, el = cpu_sample(ns, a, min(ns.size, 40 * cores), seed, cores)
    count = int(min(ns.size, max(100, got / max(el, 1e-9) * seconds)))
    got, el = cpu_sample(ns, a, count, seed + 1, cores)
    return {"value": got / el, "unit": "SVDs/s", "cores": cores, "kind": "port",
            "sample": f"{got} matrices drawn uniformly from the same {ns.size} matrices, one threaded "
                      f"call, {el:.2f} s on {cores} host threads (oracle/lsvd_oracle.cpp, -O3)"}


# ---------------------------------------------------------------- reference --

def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    from lie_cliffalg_analog_svd_b200 import profiles as P
    ns, a, _ = P.uneven_batch_workload(args.count, seed=args.seed)
    cores = cpu_cores()
    # per-step sample sized so that the whole run stays within about two minutes
    got, el = cpu_sample(ns, a, min(ns.size, 40 * cores), args.seed - 1, cores)
    per_step_s = max(1.0, min(10.0, 120.0 / max(args.steps + args.warmup, 1)))
    sample = int(min(ns.size, max(100, got / max(el, 1e-9) * per_step_s)))
    times, solved = [], []
    for i in range(args.warmup + args.steps):
        g, t = cpu_sample(ns, a, sample, args.seed + i, cores)
        if i >= args.warmup:
            times.append(t)
            solved.append(g)
    total_t, total_n = float(sum(times)), int(sum(solved))
    v = total_n / total_t
    cb = {"value": v, "unit": "SVDs/s", "cores": cores, "kind": "port",
          "sample": f"{sample} matrices per step drawn uniformly from the {ns.size}-matrix batch (a fresh "
                    f"draw each step), one threaded call per step on {cores} host threads "
                    f"(oracle/lsvd_oracle.cpp, -O3); {args.steps} timed steps, {total_t:.1f} s"}
    line = {"metric": METRIC, "value": v, "unit": "SVDs/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_t / max(args.steps, 1) * 1e3, "higher_is_better": True,
            "scaling": args.scaling, "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": batched_config(args, ws),
            "impl": "reference",
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "SVDs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the Rust crate cannot be compiled in this image (no rustc/cargo); the reference arm "
                    "times its C++ restatement (oracle/) on all host threads; each step solves the "
                    "sample stated in cpu_baseline.sample and ms_per_step is that sample's time"}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------- b200 --

def run_b200(args):
    import torch
    ws, rank, local = dist_setup()
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    from lie_cliffalg_analog_svd_b200 import Context, svd_batched, unpack
    from lie_cliffalg_analog_svd_b200 import _lib as L
    from lie_cliffalg_analog_svd_b200 import profiles as P

    from lie_cliffalg_analog_svd_b200 import dist as D
    if args.scaling == "weak":
        # every rank owns its own full batch
        ns, a, sig = P.uneven_batch_workload(args.count, seed=args.seed + rank)
    else:
        # one batch, cost-balanced contiguous shards (cost n^3)
        ns_all, a_all, sig_all = P.uneven_batch_workload(args.count, seed=args.seed)
        lo, hi = D.shard_bounds(ns_all.astype(np.float64) ** 3, ws, rank)
        ao_all = np.concatenate([[0], np.cumsum(ns_all.astype(np.int64) ** 2)])
        so_all = np.concatenate([[0], np.cumsum(ns_all.astype(np.int64))])
        ns, a, sig = ns_all[lo:hi], a_all[ao_all[lo]:ao_all[hi]], sig_all[so_all[lo]:so_all[hi]]
    local_count = int(ns.size)
    ctx = Context(local)
    stream = torch.cuda.Stream(device)
    ctx.set_stream(stream.cuda_stream)
    ad = torch.from_numpy(a).to(device)
    asz = a.size
    ssz = int(ns.astype(np.int64).sum())
    out = (torch.empty(asz, dtype=torch.float64, device=device),
           torch.empty(ssz, dtype=torch.float64, device=device),
           torch.empty(asz, dtype=torch.float64, device=device),
           torch.empty(local_count * 48, dtype=torch.uint8, device=device))
    fp64_peak = fp64_peak_tflops(torch, device)

    # validation pass (untimed): accuracy against the imposed spectra
    with torch.cuda.stream(stream):
        u, s, vt, dg, st = svd_batched(ns, ad, precision=args.precision, want_diag=True, ctx=ctx,
                                       out=out)
    torch.cuda.synchronize()
    diag = np.frombuffer(dg.cpu().numpy().tobytes(), dtype=L.DIAG_DTYPE)
    s_host = s.cpu().numpy()
    from lie_cliffalg_analog_svd_b200.api import packed_offsets
    _, so = packed_offsets(ns)
    sig_err = 0.0
    for t in range(ns.size):
        x, y = s_host[so[t]:so[t + 1]], sig[so[t]:so[t + 1]]
        sig_err = max(sig_err, float(np.max(np.abs(x - y)) / y[0]))
    acc = {"sigma_err_normwise_max": sig_err,
           "orth_u_max": float(diag["orth_u"].max()), "orth_v_max": float(diag["orth_v"].max()),
           "rel_recon_max": float(diag["rel_recon"].max()),
           "orth_u_max_over_sqrt_n_eps": float((diag["orth_u"] / (np.sqrt(ns) * 2.22e-16)).max()),
           "status": int(st)}
    flops = float(flops_per_matrix(ns, diag["ns_iters"], diag["jacobi_sweeps"],
                                   diag["rotations"], diag["route"]).sum())

    # timed region: inputs resident in HBM (1.1 GB per step > 126 MB L2)
    def step():
        svd_batched(ns, ad, precision=args.precision, ctx=ctx, out=out, device_async=True)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    launches0 = ctx.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        time.sleep(0.4)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        time.sleep(0.2)
    if ws > 1:
        torch.distributed.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    launches = ctx.kernel_launches - launches0
    ms = D.max_over_ranks(ms, device)
    units = ws * args.count if args.scaling == "weak" else args.count
    value = units / (ms * 1e-3)

    # e2e through the C ABI with host (pinned) buffers
    e2e = None
    if not args.no_e2e:
        pin = lambda k: torch.empty(k, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
        a_h = pin(asz)
        a_h[:] = a
        outs_h = (pin(asz), pin(ssz), pin(asz), None)
        for _ in range(max(1, args.warmup // 2)):
            svd_batched(ns, a_h, precision=args.precision, ctx=ctx, out=outs_h)
        if ws > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            svd_batched(ns, a_h, precision=args.precision, ctx=ctx, out=outs_h)
        el = D.max_over_ranks((time.perf_counter() - t0) / args.steps, device)
        e2e = {"value": units / el, "unit": "SVDs/s",
               "h2d_bytes_per_step": int(a_h.nbytes),
               "d2h_bytes_per_step": int(outs_h[0].nbytes + outs_h[1].nbytes + outs_h[2].nbytes),
               "ms_per_step": el * 1e3}

    peaks, peak_src = measured_peaks()
    achieved = flops / (ms * 1e-3) / 1e12
    roof = {"bound": "tensor", "pipe": "fp64", "achieved": achieved, "peak": fp64_peak,
            "unit": "TFLOP/s", "frac": achieved / fp64_peak,
            "traffic": NCU_DRAM_BYTES_PER_MATRIX * local_count,
            "traffic_source": "ncu dram bytes of batched_kernel on 20,000 matrices of this workload, "
                              "scaled by the matrix count (per-matrix traffic: A in, U/S/Vt out)",
            "kernel": "lsvd::batched_kernel",
            "peak_source": "cuBLAS DGEMM 8192^3 (torch.matmul f64) measured in this run; "
                           "MEASURED_PEAKS.json holds no FP64 figure",
            "flops_per_launch": flops,
            "hbm_gbs_peak": peaks.get("hbm_gbs"), "hbm_peak_source": peak_src}
    line = {"metric": METRIC, "value": value, "unit": "SVDs/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": args.scaling, "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else f"{args.precision}+f64",
            "data": "synthetic",
            "config": batched_config(args, ws),
            "accuracy": acc, "roofline": roof, "gpu_launches": launches,
            "clocks": clk.summary(), "e2e": e2e}
    if not args.no_mixed and args.precision == "fp64":
        line["mixed_batched"] = mixed_batched_compare(torch, ctx, stream, ns, ad, sig, out, value / ws, diag, args)
        line["svd_large"] = large_svd_compare(torch, ctx, device, args.seed + 17 + rank)
        pp = line["svd_large"]["per_precision"]
        line["polar_tflops"] = {k: pp[k]["polar_tflops"] for k in ("fp64", "tf32", "bf16")}
    if rank == 0 and ws == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(ns, a, args.cpu_seconds, args.seed)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


KAPPA_BANDS = [(1.0, 1e2), (1e2, 1e5), (1e5, 1e8), (1e8, 1e13)]


def kappa_bands(ns, sig, diag, packed=False):
    """Mean Jacobi sweeps and Newton-Schulz iterations per condition-number
    band (kappa = s_1 / s_n of the imposed spectrum; micro route excluded).
    The mixed kernels pack two counters per field (low precision x 1000 +
    FP64): `packed` splits them."""
    first = np.concatenate([[0], np.cumsum(ns)[:-1]])
    last = first + ns - 1
    kappa = sig[first] / np.maximum(sig[last], 1e-300)
    sw = diag["jacobi_sweeps"].astype(np.int64)
    it = diag["ns_iters"].astype(np.int64)
    out = []
    for lo, hi in KAPPA_BANDS:
        sel = (kappa >= lo) & (kappa < hi) & (ns > 4)
        mean = (lambda x: float(x[sel].mean()) if sel.any() else None)  # noqa: E731
        row = {"kappa": [lo, hi], "matrices": int(sel.sum())}
        if packed:
            row.update({"mean_sweeps_lowp": mean(sw // 1000), "mean_sweeps_fp64": mean(sw % 1000),
                        "mean_ns_iters_lowp": mean(it // 1000), "mean_ns_iters_fp64": mean(it % 1000)})
        else:
            row.update({"mean_sweeps": mean(sw), "mean_ns_iters": mean(it)})
        out.append(row)
    return out


def mixed_batched_compare(torch, ctx, stream, ns, ad, sig, out, fp64_value, fp64_diag, args):
    """The batched workload through the TF32 and BF16 tensor-core paths
    (Newton-Schulz bulk in low precision, FP64 refinement and Jacobi cleanup):
    device-timed SVDs/s, speed-up over the FP64 line, accuracy against the
    imposed spectra, and the FP64 sweeps per condition-number band."""
    from lie_cliffalg_analog_svd_b200 import _lib as L
    from lie_cliffalg_analog_svd_b200 import svd_batched
    from lie_cliffalg_analog_svd_b200.api import packed_offsets
    _, so = packed_offsets(ns)
    res = {"fp64_sweeps_by_kappa": kappa_bands(ns, sig, fp64_diag)}
    steps = max(2, args.steps // 2)
    for prec in ("tf32", "bf16"):
        with torch.cuda.stream(stream):
            u, s, vt, dg, st = svd_batched(ns, ad, precision=prec, want_diag=True, ctx=ctx, out=out)
        torch.cuda.synchronize()
        d = np.frombuffer(dg.cpu().numpy().tobytes(), dtype=L.DIAG_DTYPE)
        sh = s.cpu().numpy()
        err = max(float(np.max(np.abs(sh[so[t]:so[t + 1]] - sig[so[t]:so[t + 1]])) / sig[so[t]])
                  for t in range(ns.size))
        for _ in range(2):
            svd_batched(ns, ad, precision=prec, ctx=ctx, out=out, device_async=True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            svd_batched(ns, ad, precision=prec, ctx=ctx, out=out, device_async=True)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        v = ns.size / (ms * 1e-3)
        res[prec] = {"value": v, "unit": "SVDs/s", "ms_per_step": ms, "speedup_vs_fp64": v / fp64_value,
                     "status": int(st), "sigma_err_normwise_max": err,
                     "orth_u_max": float(d["orth_u"].max()), "orth_v_max": float(d["orth_v"].max()),
                     "rel_recon_max": float(d["rel_recon"].max()),
                     "sweeps_by_kappa": kappa_bands(ns, sig, d, packed=True)}
    return res


# ------------------------------------------------------- other workloads ----

def _base_line(args, metric_unit, value, ms, ws, workload, config, dtype):
    return {"metric": METRIC, "value": value, "unit": metric_unit, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
            "data": "synthetic", "config": {"workload": workload, **config}}


def _init_dist():
    import torch
    ws, rank, local = dist_setup()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    return torch, ws, rank, local, device


def _max_over_ranks(torch, ws, device, x):
    from lie_cliffalg_analog_svd_b200 import dist as D
    return D.max_over_ranks(x, device)


POLAR_SHAPES = [(4096, 4096), (8192, 2048)]
POLAR_KAPPAS = [1e2, 1e5, 1e8]
POLAR_COUNT = 16


def polar_inputs(torch, device, seed, shapes=POLAR_SHAPES):
    """The six distinct polar inputs (2 shapes x 3 condition numbers), built
    on the device from a seeded generator: A = Q1 diag(s) Q2^T with Q1, Q2 from
    QR of Gaussians and s geometric from 1 to 1/kappa.  Returns
    [(shape, kappa, A, exact polar factor Q1 Q2^T)]."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = []
    for (m, n) in shapes:
        for kappa in POLAR_KAPPAS:
            q1 = torch.linalg.qr(torch.randn(m, n, generator=g, device=device, dtype=torch.float64))[0]
            q2 = torch.linalg.qr(torch.randn(n, n, generator=g, device=device, dtype=torch.float64))[0]
            s = kappa ** (-torch.arange(n, device=device, dtype=torch.float64) / (n - 1))
            a = ((q1 * s) @ q2.T).contiguous()
            out.append(((m, n), kappa, a, (q1 @ q2.T).contiguous()))
            del q1, q2
    return out


def run_polar(args):
    torch, ws, rank, local, device = _init_dist()
    from lie_cliffalg_analog_svd_b200 import Context, polar
    ctx = Context(local)
    stream = torch.cuda.Stream(device)
    ctx.set_stream(stream.cuda_stream)
    shapes = POLAR_SHAPES if args.polar_size == "full" else [(2048, 2048), (4096, 1024)]
    with torch.cuda.stream(stream):
        inputs = polar_inputs(torch, device, args.seed + rank, shapes)
    torch.cuda.synchronize()
    order = [inputs[(t % 2) * 3 + (t // 2) % 3] for t in range(POLAR_COUNT)]
    # validation pass (untimed): accuracy per shape / kappa
    acc = []
    for (shape, kappa, a, qex) in inputs:
        r = polar(a, args.precision, ctx=ctx)
        acc.append({"shape": list(shape), "kappa": kappa, "iters_lowp": r.iters_lowp,
                    "iters_fp64": r.iters_fp64, "orth": r.orth,
                    "dist_to_exact_polar": float(torch.linalg.norm(r.q - qex).item()),
                    "converged": r.converged})
    fp64_peak = fp64_peak_tflops(torch, device)

    def step():
        fl, gms, gfl = 0.0, 0.0, 0.0
        for (_, _, a, _) in order:
            r = polar(a, args.precision, ctx=ctx)
            fl += r.flops_lowp + r.flops_fp64
            if args.precision == "fp64":
                gms += r.gemm_ms_fp64; gfl += r.flops_fp64
            else:
                gms += r.gemm_ms_lowp; gfl += r.flops_lowp
        return fl, gms, gfl

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    launches0 = ctx.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    flops = gemm_ms = gemm_flops = 0.0
    with ClockSampler(local) as clk:
        time.sleep(0.4)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            f, gm, gf = step()
            flops += f; gemm_ms += gm; gemm_flops += gf
        e1.record(stream)
        torch.cuda.synchronize()
        time.sleep(0.2)
    ms = _max_over_ranks(torch, ws, device, e0.elapsed_time(e1) / args.steps)
    launches = ctx.kernel_launches - launches0
    value = ws * flops / args.steps / (ms * 1e-3) / 1e12
    # e2e: host (pinned) A in, host Q out, through the C ABI
    pinned = {}
    for (shape, kappa, a, _) in inputs:
        h = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        h.copy_(a)
        pinned[id(a)] = (h.numpy(), torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy())
    from lie_cliffalg_analog_svd_b200 import _lib as L
    import ctypes as C
    info = L.PolarInfo()
    prec = {"fp64": 0, "tf32": 1, "bf16": 2}[args.precision]

    def e2e_step():
        for (_, _, a, _) in order:
            ah, qh = pinned[id(a)]
            m, n = ah.shape
            st = ctx.lib.lsvd_polar_f64(ctx.handle, m, n, ah.ctypes.data, n, qh.ctypes.data, n, prec,
                                        C.byref(info), 0)
            assert st in (0, 1), st
    e2e_step()
    if ws > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    el = _max_over_ranks(torch, ws, device, (time.perf_counter() - t0) / args.steps)
    bytes_io = sum(a.numel() * 8 for (_, _, a, _) in order)
    peaks, peak_src = measured_peaks()
    if args.precision == "fp64":
        peak, psrc, kern = fp64_peak, "cuBLAS DGEMM 8192^3 measured in this run", "cuBLAS DGEMM (FP64 Newton-Schulz products)"
    elif args.precision == "bf16":
        peak, psrc, kern = peaks["bf16_tflops"], f"bf16_tflops ({peak_src})", "lsvd::tc::tc_gemm_kernel<BF16>"
    else:
        peak = peaks["bf16_tflops"] / 2
        psrc, kern = f"bf16_tflops / 2 ({peak_src}; dense TF32 runs at half the BF16 rate)", "lsvd::tc::tc_gemm_kernel<TF32>"
    achieved = gemm_flops / (gemm_ms * 1e-3) / 1e12 if gemm_ms > 0 else None
    wl = "|".join(f"{m}x{n}" for m, n in shapes)
    line = _base_line(args, "TFLOP/s", value, ms, ws, f"polar_newton_schulz_16x({wl})_kappa1e2-1e8",
                      {"matrices_per_step": POLAR_COUNT, "shapes": shapes, "kappas": POLAR_KAPPAS,
                       "precision": args.precision,
                       "flops_model": "4 m n^2 per executed Newton-Schulz iteration",
                       "l2": "inputs of 134 MB (full) / 34 MB (small) each, 6 distinct per step, "
                             "together larger than the 126 MB L2",
                       "parallelism": f"dp{ws} (independent matrices)"},
                      "f64" if args.precision == "fp64" else f"{args.precision}+f64")
    line.update({"polar_per_s": ws * POLAR_COUNT / (ms * 1e-3), "accuracy": acc,
                 "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                              "frac": achieved / peak if achieved else None, "traffic": None,
                              "kernel": kern, "peak_source": psrc,
                              "timing": "summed CUDA-event durations of the GEMM launches on the polar stream"},
                 "gpu_launches": launches, "clocks": clk.summary(),
                 "e2e": {"value": ws * flops / args.steps / el / 1e12, "unit": "TFLOP/s",
                         "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io,
                         "ms_per_step": el * 1e3}})
    if rank == 0 and ws == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_polar(args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def large_inputs(torch, device, seed, shapes, kappas=POLAR_KAPPAS):
    """SVD inputs of the mixed-precision workload, built on the device: A =
    Q1 diag(s) Q2^T with Q1 (m x n), Q2 (n x n) from QR of seeded Gaussians and
    s geometric from 1 to 1/kappa.  Returns [(shape, kappa, A, s)]."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = []
    for (m, n) in shapes:
        for kappa in kappas:
            q1 = torch.linalg.qr(torch.randn(m, n, generator=g, device=device, dtype=torch.float64))[0]
            q2 = torch.linalg.qr(torch.randn(n, n, generator=g, device=device, dtype=torch.float64))[0]
            sv = kappa ** (-torch.arange(n, device=device, dtype=torch.float64) / (n - 1))
            out.append(((m, n), kappa, ((q1 * sv) @ q2.T).contiguous(), sv))
            del q1, q2
    return out


def large_accuracy(r, sv):
    i = r.info
    return {"status": int(r.status), "sigma_err_normwise": float((r.s - sv).abs().max() / sv[0]),
            "orth_u": i.orth_u, "orth_v": i.orth_v, "rel_recon": i.rel_recon,
            "ns_iters_lowp": i.ns_iters_lowp, "ns_iters_fp64": i.ns_iters_fp64,
            "sweeps_precond": i.sweeps_lowp, "sweeps_fp64": i.sweeps_fp64,
            "ms_total": i.ms_total, "ms_polar": i.ms_polar, "ms_eig_precond": i.ms_eig_lowp,
            "ms_eig_fp64": i.ms_eig_fp64, "flops_fp64": i.flops_fp64, "flops_lowp": i.flops_lowp}


def large_svd_compare(torch, ctx, device, seed, shape=(4096, 4096), kappa=1e5):
    """One matrix of the mixed-precision workload through every precision:
    device time (CUDA events inside the call), accuracy against the imposed
    spectrum, the speed-up of each mixed route over the FP64 route, and the
    Newton-Schulz phase's TFLOP/s (4 m n^2 per iteration)."""
    from lie_cliffalg_analog_svd_b200 import svd_large
    (_, _, a, sv), = large_inputs(torch, device, seed, [shape], [kappa])
    res = {}
    for prec in ("fp64", "tf32", "bf16"):
        svd_large(a, prec, want_diag=False, ctx=ctx)  # warm (workspace, graph capture)
        r = svd_large(a, prec, want_diag=True, ctx=ctx)
        res[prec] = large_accuracy(r, sv)
    m, n = shape
    for prec in ("fp64", "tf32", "bf16"):
        r = res[prec]
        it = r["ns_iters_fp64"] if prec == "fp64" else r["ns_iters_lowp"]
        r["polar_tflops"] = 4.0 * m * n * n * it / (r["ms_polar"] * 1e-3) / 1e12 if r["ms_polar"] > 0 else None
        if prec != "fp64":
            r["speedup_vs_fp64"] = res["fp64"]["ms_total"] / r["ms_total"]
    return {"shape": list(shape), "kappa": kappa, "per_precision": res,
            "polar_note": "polar_tflops = 4 m n^2 per Newton-Schulz iteration / polar-phase time; the mixed "
                          "polar phase alone is not FP64-accurate -- at equal accuracy the mixed polar factor "
                          "is U V^T of the mixed SVD, i.e. the mixed SVD's time"}


def run_svd_large(args):
    """Config 3 as SVDs: 16 dense matrices per step, 4096x4096 and 8192x2048
    alternating, kappa cycling over 1e2, 1e5, 1e8, through lsvd_svd_large_f64
    in the requested precision; every input is first solved in FP64, TF32 and
    BF16 (untimed) for the accuracy table and the per-precision speed-ups."""
    torch, ws, rank, local, device = _init_dist()
    from lie_cliffalg_analog_svd_b200 import Context, svd_large
    ctx = Context(local)
    stream = torch.cuda.Stream(device)
    ctx.set_stream(stream.cuda_stream)
    shapes = POLAR_SHAPES if args.polar_size == "full" else [(2048, 2048), (4096, 1024)]
    inputs = large_inputs(torch, device, args.seed + rank, shapes)
    torch.cuda.synchronize()
    table = []
    for (shape, kappa, a, sv) in inputs:
        row = {"shape": list(shape), "kappa": kappa}
        for prec in ("fp64", "tf32", "bf16"):
            r = svd_large(a, prec, want_diag=True, ctx=ctx)
            row[prec] = large_accuracy(r, sv)
        for prec in ("tf32", "bf16"):
            row[prec]["speedup_vs_fp64"] = row["fp64"]["ms_total"] / row[prec]["ms_total"]
        table.append(row)
    fp64_peak = fp64_peak_tflops(torch, device)
    order = [inputs[(t % 2) * 3 + (t // 2) % 3] for t in range(POLAR_COUNT)]

    def step():
        fl = 0.0
        for (_, _, a, _) in order:
            fl += svd_large(a, args.precision, want_diag=False, ctx=ctx).info.flops_fp64
        return fl

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches0 = ctx.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    flops = 0.0
    with ClockSampler(local) as clk:
        time.sleep(0.4)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            flops += step()
        e1.record(stream)
        torch.cuda.synchronize()
        time.sleep(0.2)
    ms = _max_over_ranks(torch, ws, device, e0.elapsed_time(e1) / args.steps)
    launches = ctx.kernel_launches - launches0
    value = ws * POLAR_COUNT / (ms * 1e-3)
    # e2e: host (pinned) A in, host U, S, Vt out, through the C ABI
    import ctypes as C
    from lie_cliffalg_analog_svd_b200 import _lib as L
    prec = {"fp64": 0, "tf32": 1, "bf16": 2}[args.precision]
    pinned = {}
    for (shape, kappa, a, _) in inputs:
        m, n = shape
        h = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        h.copy_(a)
        pinned[id(a)] = (h.numpy(), torch.empty((m, n), dtype=torch.float64, pin_memory=True).numpy(),
                         torch.empty(n, dtype=torch.float64, pin_memory=True).numpy(),
                         torch.empty((n, n), dtype=torch.float64, pin_memory=True).numpy())
    info = L.LargeInfo()

    def e2e_step():
        for (_, _, a, _) in order:
            ah, uh, sh, vh = pinned[id(a)]
            m, n = ah.shape
            st = ctx.lib.lsvd_svd_large_f64(ctx.handle, m, n, ah.ctypes.data, n, uh.ctypes.data, n,
                                            sh.ctypes.data, vh.ctypes.data, n, prec, C.byref(info), 0)
            assert st in (0, 1), st
    e2e_step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    el = _max_over_ranks(torch, ws, device, (time.perf_counter() - t0) / args.steps)
    bin_ = sum(a.numel() * 8 for (_, _, a, _) in order)
    bout = sum((a.shape[0] * a.shape[1] + a.shape[1] + a.shape[1] ** 2) * 8 for (_, _, a, _) in order)
    achieved = flops / args.steps / (ms * 1e-3) / 1e12
    wl = "|".join(f"{m}x{n}" for m, n in shapes)
    line = _base_line(args, "SVDs/s", value, ms, ws, f"svd_large_16x({wl})_kappa1e2-1e8",
                      {"matrices_per_step": POLAR_COUNT, "shapes": shapes, "kappas": POLAR_KAPPAS,
                       "precision": args.precision,
                       "route": "fp64: Newton-Schulz + blocked two-sided Jacobi on P + U = QV; "
                                "tf32/bf16: tensor-core Newton-Schulz bulk, preconditioning eigensolve to "
                                "the low-precision level, FP64 one-sided Jacobi on A V0",
                       "l2": "inputs of 134 MB each, 6 distinct, larger than the 126 MB L2",
                       "parallelism": f"dp{ws} (independent matrices)"},
                      "f64" if args.precision == "fp64" else f"{args.precision}+f64")
    line.update({"accuracy_and_speedup": table,
                 "roofline": {"bound": "tensor", "pipe": "fp64", "achieved": achieved, "peak": fp64_peak,
                              "unit": "TFLOP/s", "frac": achieved / fp64_peak, "traffic": None,
                              "kernel": "whole solve: lsvd::dg::dgemm_kernel and the block-Jacobi kernels",
                              "peak_source": "cuBLAS DGEMM 8192^3 (torch.matmul f64) measured in this run",
                              "flops": "executed FP64 flops counted by the library (info.flops_fp64)"},
                 "gpu_launches": launches, "clocks": clk.summary(),
                 "e2e": {"value": ws * POLAR_COUNT / el, "unit": "SVDs/s", "h2d_bytes_per_step": bin_,
                         "d2h_bytes_per_step": bout, "ms_per_step": el * 1e3}})
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_reference_svd_large(args):
    """The oracle's LieSvdSmall::solve (single-threaded, like the reference)
    on square kappa = 1e5 inputs of growing size for about --cpu-seconds; the
    rate at 4096 x 4096 is extrapolated from the largest size timed by the n^3
    cost of the solve (stated in the sample)."""
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    O = _oracle()
    from lie_cliffalg_analog_svd_b200 import profiles as P
    done, last = [], None
    n, el = 128, 0.0
    while n <= 512 and el < args.cpu_seconds:
        a, _ = P.conditioned_matrix(n, n, 1e5, seed=n)
        t0 = time.perf_counter()
        O.LieSvdSmall.solve(a)
        dt = time.perf_counter() - t0
        el += dt
        done.append(f"{n}^2 {dt:.2f} s")
        last = (n, dt)
        n *= 2
    n0, dt0 = last
    t4096 = dt0 * (4096 / n0) ** 3
    v = 1.0 / t4096
    shapes = POLAR_SHAPES if args.polar_size == "full" else [(2048, 2048), (4096, 1024)]
    wl = "|".join(f"{m}x{n}" for m, n in shapes)
    line = _base_line(args, "SVDs/s", v, t4096 * 1e3, 1, f"svd_large_16x({wl})_kappa1e2-1e8",
                      {"matrices_per_step": POLAR_COUNT, "shapes": shapes, "kappas": POLAR_KAPPAS,
                       "precision": args.precision, "parallelism": "dp1 (independent matrices)"}, "f64")
    line.update({"impl": "reference",
                 "cpu_baseline": {"value": v, "unit": "SVDs/s", "cores": 1, "kind": "port",
                                  "sample": "oracle LieSvdSmall::solve on kappa=1e5 matrices " + ", ".join(done)
                                            + f"; 4096^2 extrapolated as {dt0:.2f} s x (4096/{n0})^3"},
                 "e2e": {"value": v, "unit": "SVDs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                 "note": "a 4096^2 solve of the single-threaded CPU restatement takes hours: timed at the "
                         "sizes listed and scaled by n^3"})
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_polar(seconds: float):
    """The oracle's newton_schulz_polar (src/lie_svd_small.rs:158-183, single
    thread like the reference) on square matrices of growing size until the
    time budget is spent; the rate is reported in TFLOP/s (4 n^3 per
    iteration), so it compares with the GPU's per-flop rate."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # noqa: E402  (CPU baseline only)
    from lie_cliffalg_analog_svd_b200 import profiles as P
    fl, el, done = 0.0, 0.0, []
    n = 128
    while el < seconds and n <= 1024:
        a, _ = P.conditioned_matrix(n, n, 1e5, seed=n)
        t0 = time.perf_counter()
        _, ok, it = O.ns_polar(a)
        dt = time.perf_counter() - t0
        fl += 4.0 * n ** 3 * it; el += dt; done.append(f"{n}^2 ({it} it, {dt:.1f} s)")
        n *= 2
    return {"value": fl / el / 1e12, "unit": "TFLOP/s", "cores": 1, "kind": "port",
            "sample": "oracle newton_schulz_polar on kappa=1e5 matrices " + ", ".join(done)}


def run_reference_polar(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    vals = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline_polar(max(2.0, 60.0 / max(args.steps + args.warmup, 1)))
        if i >= args.warmup:
            vals.append(cb["value"])
    v = float(statistics.median(vals))
    cb["value"] = v
    line = _base_line(args, "TFLOP/s", v, None, args.gpus, "polar_newton_schulz (reference CPU, square proxies)",
                      {"precision": "fp64", "l2": "n/a (CPU)"}, "f64")
    line.update({"impl": "reference", "cpu_baseline": cb,
                 "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)
    return 0


JADE_EPS = [0.0, 1e-8, 1e-4]


def jade_inputs(torch, device, families, K, n, seed):
    """Phase-JADE families on the device from a seeded generator:
    A_k = Q diag(d_k) Q^T + eps E_k (Q from QR of a Gaussian, d_k ~ N(0,1),
    E_k = (G + G^T)/2), eps cycling over {0, 1e-8, 1e-4} by family."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    m = torch.empty(families, K, n, n, dtype=torch.float64, device=device)
    for f0 in range(0, families, 32):
        f1 = min(families, f0 + 32)
        q = torch.linalg.qr(torch.randn(f1 - f0, n, n, generator=g, device=device, dtype=torch.float64))[0]
        d = torch.randn(f1 - f0, K, n, generator=g, device=device, dtype=torch.float64)
        blk = (q[:, None] * d[:, :, None, :]) @ q.transpose(1, 2)[:, None]
        eps = torch.tensor([JADE_EPS[f % 3] for f in range(f0, f1)], dtype=torch.float64, device=device)
        e = torch.randn(f1 - f0, K, n, n, generator=g, device=device, dtype=torch.float64)
        blk += eps[:, None, None, None] * 0.5 * (e + e.transpose(2, 3))
        m[f0:f1] = blk
        del q, d, blk, e
    return m


def run_jade(args):
    torch, ws, rank, local, device = _init_dist()
    import ctypes as C
    from lie_cliffalg_analog_svd_b200 import Context
    from lie_cliffalg_analog_svd_b200 import _lib as L
    F, K, n = args.families, 64, 256
    ctx = Context(local)
    stream = torch.cuda.Stream(device)
    ctx.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        m = jade_inputs(torch, device, F, K, n, args.seed + rank)
        v = torch.empty(F, n, n, dtype=torch.float64, device=device)
        d = torch.empty(F, K, n, dtype=torch.float64, device=device)
    torch.cuda.synchronize()
    traces = (L.JointTrace * F)()

    def step():
        st = ctx.lib.lsvd_jade_sym_f64(ctx.handle, F, K, n, C.c_void_p(m.data_ptr()), None,
                                       C.c_void_p(v.data_ptr()), C.c_void_p(d.data_ptr()), traces,
                                       L.DEVICE_POINTERS)
        if st != 0:
            raise L.LsvdError(st, ctx.lib.lsvd_context_last_error(ctx.handle).decode())

    step()
    sweeps = np.array([t.sweeps for t in traces]); rots = np.array([t.rotations for t in traces])
    ratio = np.array([t.final_offdiag / max(t.initial_offdiag, 1e-300) for t in traces])
    vv = v[:8]
    orth = float(torch.linalg.norm(vv.transpose(1, 2) @ vv - torch.eye(n, device=device, dtype=torch.float64),
                                   dim=(1, 2)).max().item())
    acc = {"sweeps_mean": float(sweeps.mean()), "sweeps_max": int(sweeps.max()),
           "rotations_mean": float(rots.mean()),
           "final_over_initial_offdiag_by_eps": {str(e): float(ratio[[f for f in range(F) if JADE_EPS[f % 3] == e]].max())
                                                 for e in JADE_EPS},
           "orth_v_max_first8": orth}
    for _ in range(args.warmup - 1):
        step()
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    launches0 = ctx.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        time.sleep(0.4)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        time.sleep(0.2)
    ms = _max_over_ranks(torch, ws, device, e0.elapsed_time(e1) / args.steps)
    launches = ctx.kernel_launches - launches0
    peaks, peak_src = measured_peaks()
    # algorithmic bytes: every layer reads and writes each matrix of every
    # live family once (rotations of block rows and columns), plus V
    nb = n // 8
    layers = nb - 1
    bytes_step = float(sweeps.sum()) * layers * 2 * (K + 1) * n * n * 8
    achieved = bytes_step / (ms * 1e-3) / 1e9
    line = _base_line(args, "families/s", ws * F / (ms * 1e-3), ms, ws,
                      f"phase_jade_{F}x(K=64,256x256)_eps(0,1e-8,1e-4)",
                      {"families_per_gpu": F, "K": K, "n": n, "eps": JADE_EPS,
                       "l2": "17 GB of matrices per step, larger than the 126 MB L2",
                       "parallelism": f"dp{ws} (independent families)"}, "f64")
    line.update({"accuracy": acc,
                 "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                              "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                              "kernel": "jade_apply_kernel (+ jade_solve_kernel)",
                              "peak_source": f"hbm_gbs ({peak_src})",
                              "timing": "whole step (all JADE launches) on the launching stream"},
                 "gpu_launches": launches, "clocks": clk.summary(), "e2e": None})
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_reference_jade(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # noqa: E402
    from lie_cliffalg_analog_svd_b200 import profiles as P
    fam = P.jade_family_workload(1, 64, 256, 1e-8, seed=args.seed)[0]
    t0 = time.perf_counter()
    O.LieSvdJoint.diagonalize_symmetric(list(fam))
    el = time.perf_counter() - t0
    v = 1.0 / el
    line = _base_line(args, "families/s", v, el * 1e3, args.gpus, "phase_jade (reference CPU, 1 family K=64 256x256)",
                      {"l2": "n/a (CPU)"}, "f64")
    line.update({"impl": "reference",
                 "cpu_baseline": {"value": v, "unit": "families/s", "cores": 1, "kind": "port",
                                  "sample": f"1 family (K=64, n=256, eps=1e-8), {el:.1f} s, 1 thread"},
                 "e2e": {"value": v, "unit": "families/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)
    return 0


def run_single(args):
    torch, ws, rank, local, device = _init_dist()
    from lie_cliffalg_analog_svd_b200 import Context, LieSvdSmall
    from lie_cliffalg_analog_svd_b200 import profiles as P
    ctx = Context(local)
    a = P.generate(64, "uniform_random", args.seed + rank)[0]
    for _ in range(args.warmup):
        LieSvdSmall.solve(a, ctx=ctx)
    reps = 200
    t0 = time.perf_counter()
    for _ in range(reps * args.steps):
        LieSvdSmall.solve(a, ctx=ctx)
    el = _max_over_ranks(torch, ws, device, (time.perf_counter() - t0) / (reps * args.steps))
    line = _base_line(args, "SVDs/s", ws / el, el * 1e3, ws, "single_64x64_gaussian_exact_route",
                      {"n": 64, "calls_per_step": reps, "l2": "one 32 KB matrix (latency-bound)"}, "f64")
    line.update({"e2e": {"value": ws / el, "unit": "SVDs/s", "h2d_bytes_per_step": 64 * 64 * 8,
                         "d2h_bytes_per_step": 2 * 64 * 64 * 8 + 64 * 8, "ms_per_step": el * 1e3},
                 "gpu_launches": None})
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_reference_single(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # noqa: E402
    from lie_cliffalg_analog_svd_b200 import profiles as P
    a = P.generate(64, "uniform_random", args.seed)[0]
    t0 = time.perf_counter(); k = 0
    while time.perf_counter() - t0 < 5.0:
        O.LieSvdSmall.solve(a); k += 1
    el = (time.perf_counter() - t0) / k
    line = _base_line(args, "SVDs/s", 1 / el, el * 1e3, args.gpus, "single_64x64_gaussian_exact_route (reference CPU)",
                      {"n": 64, "l2": "n/a (CPU)"}, "f64")
    line.update({"impl": "reference",
                 "cpu_baseline": {"value": 1 / el, "unit": "SVDs/s", "cores": 1, "kind": "port",
                                  "sample": f"{k} solves of one 64x64 Gaussian, 1 thread"},
                 "e2e": {"value": 1 / el, "unit": "SVDs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)
    return 0


BSS_CHANNELS, BSS_SAMPLES, BSS_LAGS = 32, 1 << 20, [1, 2, 3, 5]


def bss_flops(ch, s, lags):
    """FP64 flops of the products of one separation: channel means and the
    centring update (inner dimension 2), covariance, whitening, one lagged
    covariance per lag, separation."""
    return 8.0 * ch * s + 2.0 * ch * ch * (3 * s + sum(s - g for g in lags if 0 < g < s))


def run_bss(args):
    torch, ws, rank, local, device = _init_dist()
    from lie_cliffalg_analog_svd_b200 import Context, LieSvdBss, PhaseBssParams
    from lie_cliffalg_analog_svd_b200 import profiles as P
    from lie_cliffalg_analog_svd_b200.consumers import estimate_sir_db
    ctx = Context(local)
    ch, s = BSS_CHANNELS, BSS_SAMPLES
    src, _, obs = P.bss_workload(ch, s, args.seed + rank)
    params = PhaseBssParams.for_channels(ch)
    params.lags = list(BSS_LAGS)
    r = LieSvdBss.separate(obs, params, ctx=ctx)  # validation (untimed)
    sir_before, sir_after = estimate_sir_db(src, obs), estimate_sir_db(src, r.separated)
    for _ in range(args.warmup):
        LieSvdBss.separate(obs, params, ctx=ctx)
    torch.cuda.synchronize()
    l0 = ctx.kernel_launches
    with ClockSampler(local) as clk:
        clk.wait_for(1)  # a separation takes tens of ms: sample at both ends of the timed region
        t0 = time.perf_counter()
        for _ in range(args.steps):
            LieSvdBss.separate(obs, params, ctx=ctx)
        torch.cuda.synchronize()
        el = _max_over_ranks(torch, ws, device, (time.perf_counter() - t0) / args.steps)
        clk.wait_for(len(clk.lines) + 1, 0.5)
    launches = (ctx.kernel_launches - l0) // max(args.steps, 1)
    h2d, d2h = obs.nbytes, obs.nbytes + ch * ch * 8 * (len(BSS_LAGS) + 2)
    line = _base_line(args, "samples/s", ws * s / el, el * 1e3, ws, f"phase_bss_{ch}ch_{s}samples",
                      {"channels": ch, "samples": s, "lags": BSS_LAGS,
                       "l2": f"observations {obs.nbytes / 1e6:.0f} MB per step, larger than the 126 MB L2"}, "f64")
    fl = bss_flops(ch, s, BSS_LAGS)
    line.update({
        "e2e": {"value": ws * s / el, "unit": "samples/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": el * 1e3},
        "note": "value = e2e: LieSvdBss.separate takes host arrays (the reference's API), so the copies are "
                "inside every step; the products are 2C^2T-sized GEMMs on the FP64 product kernel",
        "products_gflop_per_step": fl / 1e9,
        "copy_gbs": (h2d + d2h) / el / 1e9,
        "accuracy": {"sir_db_before": sir_before, "sir_db_after": sir_after,
                     "joint_initial_offdiag": r.trace.joint_initial_offdiag,
                     "joint_final_offdiag": r.trace.joint_final_offdiag},
        "gpu_launches": int(launches), "clocks": clk.summary()})
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = _bss_cpu_sample(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def _bss_cpu_sample(args, samples=1 << 17):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_consumers as OC  # noqa: E402
    from lie_cliffalg_analog_svd_b200 import profiles as P
    _, _, obs = P.bss_workload(BSS_CHANNELS, samples, args.seed)
    p = OC.PhaseBssParams.for_channels(BSS_CHANNELS)
    p.lags = list(BSS_LAGS)
    t0 = time.perf_counter()
    OC.bss_separate(obs, p)
    el = time.perf_counter() - t0
    return {"value": samples / el, "unit": "samples/s", "cores": 1, "kind": "port",
            "sample": f"one separation of {BSS_CHANNELS} channels x {samples} samples of the same generator, "
                      f"{el:.2f} s (oracle/oracle_consumers.py: the reference's per-sample lagged-covariance "
                      "loop compiled in oracle/lsvd_oracle.cpp, products in ndarray order, 1 thread as the "
                      "reference runs it)"}


def run_reference_bss(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    cb = _bss_cpu_sample(args)
    el = BSS_SAMPLES / cb["value"]
    line = _base_line(args, "samples/s", cb["value"], el * 1e3, args.gpus,
                      f"phase_bss_{BSS_CHANNELS}ch_{BSS_SAMPLES}samples (reference CPU, bounded sample)",
                      {"channels": BSS_CHANNELS, "samples": BSS_SAMPLES, "lags": BSS_LAGS, "l2": "n/a (CPU)"},
                      "f64")
    line.update({"impl": "reference", "cpu_baseline": cb,
                 "e2e": {"value": cb["value"], "unit": "samples/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)
    return 0


ADJ_COUNT, ADJ_M, ADJ_N = 4096, 128, 64


def numpy_svd_adjoint(u, s, v, ub, sb, vb, qb, gap_tol=0.0):
    """The analytic thin-SVD + polar adjoint in numpy (the CPU comparison)."""
    den = s[None, :] ** 2 - s[:, None] ** 2
    close = np.abs(s[None, :] - s[:, None]) <= gap_tol * s.max()
    f = np.where((den == 0) | close, 0.0, 1.0 / np.where(den == 0, 1.0, den))
    np.fill_diagonal(f, 0.0)
    g = u.T @ ub
    h = v.T @ vb
    mm = u.T @ qb @ v
    core = (f * (g - g.T)) * s[None, :] + s[:, None] * (f * (h - h.T)) \
        + (mm - mm.T) / (s[:, None] + s[None, :]) + np.diag(sb)
    proj = (ub + qb @ v) - u @ (u.T @ (ub + qb @ v))
    return u @ core @ v.T + (proj / s[None, :]) @ v.T


def vjp_flops(m, n, rotations):
    """FP64 flops of one adjoint: A^T Ubar, A^T Qbar and the three m x n
    products of Abar (10 m n^2), seven n x n products (14 n^3), and the
    replay (6 n flops per rotation)."""
    return 10.0 * m * n * n + 14.0 * n ** 3 + 6.0 * n * rotations


def run_adjoint(args):
    torch, ws, rank, local, device = _init_dist()
    from lie_cliffalg_analog_svd_b200 import Context, svd_batched_stream, svd_vjp
    from lie_cliffalg_analog_svd_b200 import profiles as P
    cnt, m, n = ADJ_COUNT, ADJ_M, ADJ_N
    ctx = Context(local)
    stream = torch.cuda.Stream(device)
    ctx.set_stream(stream.cuda_stream)
    a, sig = P.adjoint_workload(cnt, m, n, seed=args.seed + rank)
    rng = np.random.default_rng(args.seed + 1 + rank)
    cot = {k: rng.standard_normal(shape) for k, shape in
           (("ub", (cnt, m, n)), ("sb", (cnt, n)), ("vb", (cnt, n, n)), ("qb", (cnt, m, n)))}
    ad = torch.from_numpy(a).to(device)
    cd = {k: torch.from_numpy(v).to(device) for k, v in cot.items()}
    torch.cuda.synchronize()
    # forward with the stream (and U, V for the accuracy check and the stored-V path)
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fwd = svd_batched_stream(ad, ctx=ctx)
    e1.record(stream); torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    fwd_uv = svd_batched_stream(ad, want_uv=True, ctx=ctx)
    counts = fwd.counts.cpu().numpy()
    stream_bytes = fwd.stream_bytes()
    uv_bytes = fwd.uv_bytes()
    flops = float(sum(vjp_flops(m, n, int(c)) for c in counts))

    def step(stored=False):
        return svd_vjp(fwd, ubar=cd["ub"], sbar=cd["sb"], vbar=cd["vb"], qbar=cd["qb"], ctx=ctx,
                       stored_vt=fwd_uv.vt if stored else None)

    ab = step()
    # accuracy on a subset: the analytic formula on the forward's own U, V
    ab_h = ab[:32].cpu().numpy()
    u_h = fwd_uv.u[:32].cpu().numpy(); vt_h = fwd_uv.vt[:32].cpu().numpy(); s_h = fwd_uv.s[:32].cpu().numpy()
    gaps = np.min(-np.diff(sig, axis=1), axis=1)
    errs = []
    for t in range(32):
        if gaps[t] < 1e-4:
            continue
        ref = numpy_svd_adjoint(u_h[t], s_h[t], vt_h[t].T, cot["ub"][t], cot["sb"][t], cot["vb"][t], cot["qb"][t])
        errs.append(float(np.linalg.norm(ab_h[t] - ref) / np.linalg.norm(ref)))
    fwd_sig_err = float(np.max(np.abs(fwd.s.cpu().numpy() - sig) / sig[:, :1]))
    fp64_peak = fp64_peak_tflops(torch, device)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        l0 = ctx.kernel_launches
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return _max_over_ranks(torch, ws, device, e0.elapsed_time(e1) / args.steps), ctx.kernel_launches - l0

    with ClockSampler(local) as clk:
        time.sleep(0.4)
        ms, launches = timed(step)
        time.sleep(0.2)
    ms_stored, _ = timed(lambda: step(True))
    # e2e: host arrays through the C ABI (A, S, perm, stream, cotangents in; Abar out)
    fwd_h = svd_batched_stream(a, ctx=ctx)

    def e2e_step():
        return svd_vjp(fwd_h, ubar=cot["ub"], sbar=cot["sb"], vbar=cot["vb"], qbar=cot["qb"], ctx=ctx)
    e2e_step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    el = _max_over_ranks(torch, ws, device, (time.perf_counter() - t0) / args.steps)
    h2d = a.nbytes + sum(v.nbytes for v in cot.values()) + fwd_h.s.nbytes + fwd_h.perm.nbytes \
        + fwd_h.rotors.nbytes + fwd_h.counts.nbytes
    achieved = flops / (ms * 1e-3) / 1e12
    line = _base_line(args, "VJPs/s", ws * cnt / (ms * 1e-3), ms, ws,
                      f"svd_polar_vjp_rotor_replay_{cnt}x{m}x{n}",
                      {"count_per_gpu": cnt, "m": m, "n": n, "sigma": "U[0.1, 10], gap >= 1e-3, 10% one 1e-6 gap",
                       "cotangents": "N(0,1) on U, S, V and the polar factor",
                       "l2": "A and cotangents 0.8 GB + streams per step, larger than the 126 MB L2",
                       "parallelism": f"dp{ws} (independent matrices)"}, "f64")
    line.update({
        "accuracy": {"vs_analytic_fp64_rel_max": max(errs) if errs else None, "checked": len(errs),
                     "forward_sigma_err_max": fwd_sig_err},
        "memory": {"stream_bytes": stream_bytes, "stored_uv_bytes": uv_bytes,
                   "rotations_mean": float(counts.mean()), "ratio_stream_over_uv": stream_bytes / uv_bytes},
        "time": {"vjp_replay_ms": ms, "vjp_stored_v_ms": ms_stored, "forward_stream_ms": fwd_ms},
        "roofline": {"bound": "tensor", "pipe": "fp64", "achieved": achieved, "peak": fp64_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp64_peak, "traffic": None,
                     "kernel": "svd_vjp_kernel", "flops_per_launch": flops,
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run"},
        "gpu_launches": launches, "clocks": clk.summary(),
        "e2e": {"value": ws * cnt / el, "unit": "VJPs/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(a.nbytes), "ms_per_step": el * 1e3}})
    if rank == 0 and ws == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_adjoint(a[:256], {k: v[:256] for k, v in cot.items()},
                                                    args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def cpu_baseline_adjoint(a, cot, seconds):
    """Per matrix on the host cores: the oracle's solve_rectangular (the
    reference's forward) and the analytic adjoint in numpy."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # noqa: E402  (CPU baseline only)
    from concurrent.futures import ThreadPoolExecutor
    cores = cpu_cores()
    stop = time.perf_counter() + seconds
    done = [0]
    lock = threading.Lock()

    def work(idx):
        c = 0
        while time.perf_counter() < stop:  # passes over the sample until the budget is spent
            for t in idx:
                if time.perf_counter() > stop:
                    break
                u, s, vt = O.LieSvdSmall.solve_rectangular(a[t])
                numpy_svd_adjoint(u, s, vt.T, cot["ub"][t], cot["sb"][t], cot["vb"][t], cot["qb"][t])
                c += 1
        with lock:
            done[0] += c

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=cores) as ex:
        list(ex.map(work, np.array_split(np.arange(a.shape[0]), cores)))
    el = time.perf_counter() - t0
    return {"value": done[0] / el, "unit": "VJPs/s", "cores": cores, "kind": "port",
            "sample": f"{done[0]} solves (passes over {a.shape[0]} of the 128x64 matrices): oracle "
                      f"solve_rectangular + numpy analytic adjoint, {el:.1f} s on {cores} host threads"}


def run_reference_adjoint(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    from lie_cliffalg_analog_svd_b200 import profiles as P
    a, _ = P.adjoint_workload(256, ADJ_M, ADJ_N, seed=args.seed)
    rng = np.random.default_rng(args.seed + 1)
    cot = {"ub": rng.standard_normal(a.shape), "sb": rng.standard_normal((256, ADJ_N)),
           "vb": rng.standard_normal((256, ADJ_N, ADJ_N)), "qb": rng.standard_normal(a.shape)}
    vals = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline_adjoint(a, cot, max(2.0, 60.0 / max(args.steps + args.warmup, 1)))
        if i >= args.warmup:
            vals.append(cb["value"])
    v = float(statistics.median(vals))
    cb["value"] = v
    line = _base_line(args, "VJPs/s", v, ADJ_COUNT / v * 1e3, args.gpus,
                      f"svd_polar_vjp (reference CPU forward + numpy adjoint) {ADJ_M}x{ADJ_N}",
                      {"l2": "n/a (CPU)"}, "f64")
    line.update({"impl": "reference", "cpu_baseline": cb,
                 "e2e": {"value": v, "unit": "VJPs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return {"batched": run_reference, "polar": run_reference_polar,
                "jade": run_reference_jade, "single": run_reference_single,
                "adjoint": run_reference_adjoint, "svd_large": run_reference_svd_large,
                "bss": run_reference_bss}[args.workload](args)
    return {"batched": run_b200, "polar": run_polar, "jade": run_jade,
            "single": run_single, "adjoint": run_adjoint, "svd_large": run_svd_large,
            "bss": run_bss}[args.workload](args)


if __name__ == "__main__":
    sys.exit(main())
