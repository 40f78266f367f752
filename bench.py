"""Benchmark: seconds from device-resident X to relative duality gap 1e-6 for the TensorSVM
training path (kernel factor + SMW interior point), on the n=1M, d=18, k=256 two-Gaussian
workload (gamma 0.05, C 32, 10% label noise), synthetic data.

One step = one full training solve: GPU sketch, two fused kernel-block passes, CholeskyQR,
projection, Jacobi eigen-factor, then the IPM until rel_gap = (pobj-dobj)/max(1,|pobj|) <= 1e-6
with ||rd||/(1+sqrt n) and |rp|/(1+sqrt n) <= 1e-6.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp16|bf16|fp32]
    python bench.py --impl reference ...     # the reference trainer's own build, host cores

Multi-GPU (torchrun): replicas only -- every rank trains an independent problem of the same
size (a different data seed), there is no collective on the data path; the line reports the
max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s to rel. gap 1e-6, mixed/TC vs FP32 form (n=1M,d=18,k=256); % of roofline"
WORKLOAD = "two_gaussians_rbf"
N_DEFAULT, D, K, GAMMA, CPEN, NOISE = 1_000_000, 18, 256, 0.05, 32.0, 0.10


def workload_config(n: int, world: int) -> dict:
    """The benchmark workload, named the same way by both arms."""
    return {"workload": WORKLOAD, "n": n, "d": D, "k": K, "gamma": GAMMA, "C": CPEN,
            "stop": "rel_gap<=1e-6 and ||rd||,|rp|/(1+sqrt n)<=1e-6",
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (Z 1 GiB fp32, kernel operand 0.5 GiB)"}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index, self.proc, self.samples = index, None, []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for s in self.samples for j in range(4) if s[3 + j] == "Active"})
        pw = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "power_w": statistics.median(pw) if pw else None,
                "samples": len(self.samples)}


def dist_setup():
    """One process per GPU (torchrun env vars); NCCL on GPUs, gloo when there is no CUDA."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def replica_seed(rank: int) -> int:
    """Data seed of a replica: every rank trains an independent problem of the same size."""
    return 2 + rank


def dist_max(values, world):
    """Element-wise max over ranks (the timing of a replica job is its slowest rank)."""
    if world == 1:
        return values
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(values, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.cpu().tolist()


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------

# DRAM bytes (read + write) per 128 x 64 tile of the two tensor-core kernel-block launches of
# the split form at k = 256, from one ncu capture at n = 262144: the range finder (every tile,
# 2.747 GB read + 0.260 GB written over 8,388,608 tiles) and the projection half product (W as
# hi + lo, 2.186 GB + 0.226 GB over 4,196,352 tiles).  The J-side operands are re-read once per
# round of 148 row blocks, so traffic grows with the tiles.
TC_BYTES_PER_TILE = {"range_finder": (2.747472e9 + 0.260303e9) / 8388608,
                     "projection_half": (2.185915e9 + 0.225879e9) / 4196352}


def tc_traffic(n: int) -> dict:
    nrb = -(-n // 128)
    full, half = nrb * 2 * nrb, nrb * (nrb + 1)   # tiles of the full pass and of the half product
    return {"range_finder": round(TC_BYTES_PER_TILE["range_finder"] * full, -6),
            "projection_half": round(TC_BYTES_PER_TILE["projection_half"] * half, -6)}


def tc_executed(n: int, k: int, d: int, split: bool) -> dict:
    """Tensor-core flops the two kernel-block launches execute (128 x 64 tiles; Gram K of
    3 d + 6 rounded up to 64; the split forms run two P A products per tile), against the
    algorithmic 2 n^2 k + 2 n^2 d per product: the range-finder pass takes every tile, the
    projection pass (half product) the tiles from the diagonal on."""
    nrb, ntl = -(-n // 128), 2 * -(-n // 128)
    kp = -(-k // 64) * 64
    kg = 64 if 3 * d + 6 <= 64 else 128 if 3 * d + 6 <= 128 else 192
    per_tile = 2.0 * 128 * 64 * kg + (2 if split else 1) * 2.0 * 128 * 64 * kp
    full = nrb * ntl
    half = sum(ntl - 2 * rb for rb in range(nrb))
    return {"pass1_tiles": full, "pass2_tiles": half, "pass1_flops": full * per_tile,
            "pass2_flops": half * per_tile}


def run_ours(args, world, rank, local):
    import torch
    from tensorsvm_b200 import _lib, api, synth
    torch.cuda.set_device(local)
    n = args.n
    X, y = synth.two_gaussians(n, D, seed=replica_seed(rank), noise=NOISE)
    Xd, yd = torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()
    ctx = _lib.Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    prec = args.precision

    last = {}

    def step(precision):
        Z, finfo = api.factor(ctx, Xd, yd, GAMMA, K, precision)
        alpha, _, _, st = api.ipm(ctx, Z, yd, K, CPEN, rel_gap_tol=1e-6,
                                  precision=_lib.PREC_FP32 if precision == "fp32" else _lib.PREC_BF16)
        last[precision] = (Z, alpha)
        return finfo, st

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step(prec)
        barrier(world)
        torch.cuda.synchronize()
        launches0 = ctx.launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        finfos, stats, per_step = [], [], []
        with ClockSampler(local) as clk:
            e0.record(stream)
            for _ in range(args.steps):
                s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s0.record(stream)
                fi, st = step(prec)
                s1.record(stream)
                finfos.append(fi)
                stats.append(st)
                per_step.append((s0, s1))
            e1.record(stream)
            torch.cuda.synchronize()
        barrier(world)
        launches = ctx.launches - launches0
        total_ms = e0.elapsed_time(e1)
        step_ms = [a.elapsed_time(b) for a, b in per_step]
        # end to end through the public host-buffer API (tsvm_train), H2D/D2H inside
        Xh = torch.from_numpy(X).pin_memory()
        yh = torch.from_numpy(y).pin_memory()
        e2e_ms = []
        for _ in range(args.e2e_steps):
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            m = api.train(ctx, Xh.numpy(), yh.numpy(), _lib.KERNEL_RBF, GAMMA, CPEN, K, prec,
                          rel_gap_tol=1e-6)
            t1.record(stream)
            torch.cuda.synchronize()
            e2e_ms.append(t0.elapsed_time(t1))
        fp32_s = None
        if args.fp32_form and prec != "fp32":
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            fi32, st32 = step("fp32")
            f1.record(stream)
            torch.cuda.synchronize()
            fp32_s = f0.elapsed_time(f1) / 1e3
            # full-size agreement of the two models' decision values (each through its own factor)
            fm = decision_values(ctx, *last[prec], yd, K, CPEN)
            f32 = decision_values(ctx, *last["fp32"], yd, K, CPEN)
            sign_agree = float((torch.sign(fm) == torch.sign(f32)).double().mean())
            dec_rel = float((fm - f32).abs().max() / f32.abs().max())
            del last["fp32"]
        fast = None
        if args.fp32_form and prec in ("fp16", "bf16"):
            # the one-product form of the same precision (no hi + lo operand splits), one warm-up
            fp = prec + "_fast"
            step(fp)
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            q0.record(stream)
            fif, stf = step(fp)
            q1.record(stream)
            torch.cuda.synchronize()
            ff = decision_values(ctx, *last[fp], yd, K, CPEN)
            fm = decision_values(ctx, *last[prec], yd, K, CPEN)
            fast = {"precision": fp, "value": round(q0.elapsed_time(q1) / 1e3, 4), "unit": "s",
                    "ms_kermatmul_per_launch": round(fif["ms_kermatmul_kernel"] / 2, 2),
                    "pobj_rel_diff": abs(stf["pobj"] - stats[-1]["pobj"]) / abs(stats[-1]["pobj"]),
                    "decision_sign_agreement_with_split":
                        float((torch.sign(ff) == torch.sign(fm)).double().mean())}
            del last[fp]
    sec = total_ms / 1e3 / args.steps
    sec, e2e_s = dist_max([sec, (sum(e2e_ms) / max(1, len(e2e_ms))) / 1e3], world)
    if rank != 0:
        ctx.close()
        return None
    pk, pk_kind = peaks()
    fi = finfos[-1]
    km_ms = fi["ms_kermatmul_kernel"] / 2.0          # per launch (two launches per step)
    km_flops = fi["flops_kermatmul"] / 2.0
    tensor = prec != "fp32"
    if tensor:
        peak, unit, pname = pk["bf16_tflops_sustained"], "TFLOP/s", "bf16_tflops_sustained"
    else:
        # FP32 SIMT FMA peak: 148 SMs x 128 lanes x 2 flops x 1.965 GHz (nominal, no measured copy)
        peak, unit, pname, pk_kind = 148 * 128 * 2 * 1.965e9 / 1e12, "TFLOP/s", "fp32_simt_nominal", "nominal"
    achieved = km_flops / (km_ms / 1e3) / 1e12
    passes = None
    if tensor:
        ex = tc_executed(n, K, D, prec in ("fp16", "bf16"))
        passes = {}
        for name, key, tiles, fl in (("range_finder", "ms_pass1", ex["pass1_tiles"], ex["pass1_flops"]),
                                      ("projection_half", "ms_pass2", ex["pass2_tiles"], ex["pass2_flops"])):
            ms = fi[key]
            passes[name] = {"phase_ms": round(ms, 2), "tiles": tiles,
                            "traffic": tc_traffic(n)[name],
                            "algorithmic_tflops": round(km_flops / (ms / 1e3) / 1e12, 1),
                            "executed_flops": fl,
                            "executed_tflops": round(fl / (ms / 1e3) / 1e12, 1),
                            "executed_frac": round(fl / (ms / 1e3) / 1e12 / peak, 4)}
    st = stats[-1]
    line = {
        "metric": METRIC,
        "value": round(sec, 4),
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 2),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"fp16": "f16 (fp32 accum)", "bf16": "bf16 (fp32 accum)", "fp32": "f32"}[prec]
                 + " contractions, f64 k x k + IPM vectors",
        "data": "synthetic (seeded two-Gaussian mixture, 10% label noise)",
        "precision": prec,
        "config": workload_config(n, world),
        "phases_ms": {"sketch": round(fi["ms_sketch"], 2), "pass1": round(fi["ms_pass1"], 2),
                      "ortho": round(fi["ms_ortho"], 2), "pass2": round(fi["ms_pass2"], 2),
                      "project": round(fi["ms_project"], 2), "factor_total": round(fi["ms_total"], 2),
                      "ipm": round(st["ms_total"], 2), "ipm_syrk": round(st["ms_syrk"], 2),
                      "ipm_chol": round(st["ms_factor"], 2), "ipm_iters": st["iters"]},
        "solution": {"rel_gap": st["rel_gap"], "pobj": st["pobj"], "dobj": st["dobj"],
                     "iters": st["iters"]},
        "step_s": [round(t / 1e3, 4) for t in step_ms],
        "roofline": {"bound": "tensor" if tensor else "fp32-simt", "kernel": "kermatmul (fused kernel-block product)",
                     "achieved": round(achieved, 2), "peak": round(peak, 1), "unit": unit,
                     "frac": round(achieved / peak, 4), "peak_source": f"{pk_kind} {pname}",
                     "traffic": (round(sum(tc_traffic(n).values()) / 2, -6) if tensor else None),
                     "traffic_source": ("dram__bytes_read.sum + dram__bytes_write.sum per launch "
                                        "(mean of the two launches), from one ncu capture at "
                                        "n=262144 scaled by the tile count" if tensor else None),
                     "flops_per_launch": km_flops, "ms_per_launch": round(km_ms, 3),
                     "passes": passes},
        "e2e": {"value": round(e2e_s, 4), "unit": "s",
                "h2d_bytes_per_step": int(X.nbytes + y.nbytes), "d2h_bytes_per_step": int(8 * n + 8)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if fast is not None:
        line["fast_form"] = fast
    if fp32_s is not None:
        line["fp32_form"] = {"value": round(fp32_s, 3), "unit": "s", "speedup_mixed_vs_fp32": round(fp32_s / sec, 2),
                             "decision_sign_agreement": sign_agree,
                             "decision_max_rel_diff": dec_rel}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    ctx.close()
    return line


def decision_values(ctx, Z, alpha, y, k, C):
    """Training-set decision values f = Z_k Z_k^T (alpha o y) + b of a solved model, in FP64."""
    from tensorsvm_b200 import api
    b = api.bias(ctx, Z, y, alpha, k, C)[0]
    Zk = Z[:, :k].double()
    return Zk @ (Zk.T @ (alpha * y.double())) + b


def cpu_baseline(args):
    """The FP64 oracle (same algorithm, host BLAS/LAPACK, all host cores) on bounded samples of
    the same generator, extrapolated to n: the factor time is fitted as a n^2 + b n + c through
    the samples (its two kernel-block passes are quadratic in n), the IPM is timed on the
    largest sample and scaled by n."""
    from oracle import oracle as orc
    from tensorsvm_b200 import synth
    sizes = [int(v) for v in args.cpu_sample.split(",")]
    cores = os.cpu_count() or 1
    fac, ipm_s, ipm_it = [], 0.0, 0
    for ns in sizes:
        X, y = synth.two_gaussians(ns, D, seed=2, noise=NOISE)
        t0 = time.perf_counter()
        f = orc.lra(X, y, GAMMA, K, threads=cores)
        fac.append(time.perf_counter() - t0)
        if ns == sizes[-1]:
            t1 = time.perf_counter()
            r = orc.mpc(f.U, y, CPEN, kernel="rbf", rel_gap_tol=1e-6)
            ipm_s, ipm_it = time.perf_counter() - t1, r.iters
    A = np.array([[float(ns) ** 2, float(ns), 1.0] for ns in sizes])
    coef = np.linalg.lstsq(A, np.array(fac), rcond=None)[0]
    n = float(args.n)
    est = float(coef @ np.array([n * n, n, 1.0])) + ipm_s * n / sizes[-1]
    return {"value": round(est, 1), "unit": "s", "cores": cores, "kind": "port",
            "sample": (f"FP64 oracle (numpy/OpenBLAS, {cores} threads) on n in {sizes} rows of the "
                       f"same generator: factor {[round(t, 2) for t in fac]} s fitted as "
                       f"a n^2 + b n + c (a={coef[0]:.3e}) and evaluated at n; IPM "
                       f"{ipm_s:.2f} s ({ipm_it} it) at n={sizes[-1]} scaled by n")}


# ------------------------------------------------------------------------------------------
# the other workloads (--workload): wide features, the batched grid, the hypergradient.  Rank 0
# only; each prints its own JSON line.  The default line above is the benchmark contract.
# ------------------------------------------------------------------------------------------

def _timed(stream, fn):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1) / 1e3


def _base_line(args, metric, value, config):
    return {"metric": metric, "value": round(value, 4), "unit": "s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic", "config": config}


def run_wide(args, ctx, stream):
    """n=500,000, d=54 (10 uniform + one-hot groups of 4 and 40), gamma 0.02, C 32, k 400: the
    fp16 tensor-core factor + IPM against the FP32 form, to rel. gap 1e-6."""
    import torch
    from tensorsvm_b200 import _lib, api, synth
    X, y, gamma, C, k = synth.make("c3", n=args.n if args.n != N_DEFAULT else None)
    Xd, yd = torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()
    n = X.shape[0]

    def solve(prec):
        Z, fi = api.factor(ctx, Xd, yd, gamma, k, prec)
        a, _, _, st = api.ipm(ctx, Z, yd, k, C, rel_gap_tol=1e-6,
                              precision=_lib.PREC_FP32 if prec == "fp32" else _lib.PREC_BF16)
        return Z, a, fi, st

    for _ in range(args.warmup):
        solve(args.precision)
    times, res = [], None
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            res = None   # the previous step's factor is released before the next allocates
            res, t = _timed(stream, lambda: solve(args.precision))
            times.append(t)
    Z, a, fi, st = res
    (Z32, a32, fi32, st32), t32 = _timed(stream, lambda: solve("fp32"))
    fm = decision_values(ctx, Z, a, yd, k, C)
    f32 = decision_values(ctx, Z32, a32, yd, k, C)
    sec = statistics.mean(times)
    line = _base_line(args, "s to rel. gap 1e-6, n=500k d=54 k=400 (fp16 TC vs FP32 form)", sec,
                      {"workload": "mixed_onehot_rbf", "n": n, "d": X.shape[1], "k": k,
                       "gamma": gamma, "C": C, "precision": args.precision})
    line.update({
        "dtype": f"{args.precision} contractions (fp32 accum), f64 k x k + IPM vectors",
        "phases_ms": {"factor": round(fi["ms_total"], 1), "kermatmul_per_launch": round(fi["ms_kermatmul_kernel"] / 2, 1),
                      "ipm": round(st["ms_total"], 1), "ipm_iters": st["iters"],
                      "ipm_syrk": round(st["ms_syrk"], 1), "mixed_syrk": st["mixed_syrk"]},
        "tflops_kermatmul": round(fi["flops_kermatmul"] / (fi["ms_kermatmul_kernel"] / 1e3) / 1e12, 1),
        "solution": {"rel_gap": st["rel_gap"], "pobj": st["pobj"], "iters": st["iters"]},
        "fp32_form": {"value": round(t32, 3), "unit": "s", "speedup": round(t32 / sec, 2),
                      "pobj": st32["pobj"], "iters": st32["iters"],
                      "pobj_rel_diff": abs(st["pobj"] - st32["pobj"]) / abs(st32["pobj"]),
                      "decision_sign_agreement": float((torch.sign(fm) == torch.sign(f32)).double().mean()),
                      "decision_max_rel_diff": float((fm - f32).abs().max() / f32.abs().max())},
        "step_s": [round(t, 3) for t in times], "clocks": clk.summary()})
    return line


def run_grid(args, ctx, stream):
    """64 tanh-teacher problems (n log-uniform in [2000, 200000], d=28) on the 8 x 8 (C, gamma)
    grid, k=128: batched tensor-core factors (one eigensolver launch for all 64) + one batched
    IPM, against the same factors solved one by one, the factors on --factor-threads host
    threads, and 64 plain FP32 solves (FP32 factor + FP32 IPM)."""
    import torch
    from tensorsvm_b200 import _lib, api, synth
    probs = synth.grid_problems(count=64)
    k = 128
    Xs = [torch.from_numpy(X).cuda() for X, _, _, _ in probs]
    ys = [torch.from_numpy(y).cuda() for _, y, _, _ in probs]
    gs = [g for _, _, g, _ in probs]
    Cs = [C for _, _, _, C in probs]
    rows = sum(X.shape[0] for X in Xs)

    def factors(prec):
        return [api.factor(ctx, X, y, g, k, prec)[0] for X, y, g in zip(Xs, ys, gs)]

    # the tensor-core factors on `factor_threads` host threads, one context and stream each
    # (contexts are per host thread): the problems are independent and most are small, so one
    # factorisation leaves most SMs idle.  Longest-first assignment by the estimated cost
    # (n^2 for the kernel-block passes plus a fixed part); the main stream waits for all workers.
    from concurrent.futures import ThreadPoolExecutor
    nthreads = max(1, args.factor_threads)
    workers = []
    for _ in range(nthreads):
        wctx, wst = _lib.Context(torch.cuda.current_device()), torch.cuda.Stream()
        wctx.set_stream(wst.cuda_stream)
        workers.append((wctx, wst))
    cost = [float(X.shape[0]) ** 2 + 2.5e9 for X in Xs]
    load = [0.0] * nthreads
    assign = [[] for _ in range(nthreads)]
    for i in sorted(range(len(Xs)), key=lambda i: -cost[i]):
        w = min(range(nthreads), key=lambda w: load[w])
        assign[w].append(i)
        load[w] += cost[i]
    dev_index = torch.cuda.current_device()

    def factors_parallel(prec):
        start = torch.cuda.Event()
        start.record(stream)
        out = [None] * len(Xs)

        def work(w):
            torch.cuda.set_device(dev_index)
            wctx, wst = workers[w]
            wst.wait_event(start)
            with torch.cuda.stream(wst):
                for i in assign[w]:
                    out[i] = api.factor(wctx, Xs[i], ys[i], gs[i], k, prec)[0]
            done = torch.cuda.Event()
            done.record(wst)
            return done

        with ThreadPoolExecutor(nthreads) as ex:
            evs = list(ex.map(work, range(nthreads)))
        for ev in evs:
            stream.wait_event(ev)
        return out

    def batched():
        # every problem's factor through its projection, the 64 eigenproblems in one launch,
        # then the batched IPM
        Zs = api.factor_batched(ctx, Xs, ys, gs, k, args.precision)[0]
        _, t_ipm = _timed(stream, lambda: api.ipm_batched(ctx, Zs, ys, k, Cs, rel_gap_tol=1e-6,
                                                          precision=ipm_prec))
        return Zs, t_ipm

    # the 16-bit forms' mixed-precision capacitance matrices in the batched and the one-by-one
    # solves alike
    ipm_prec = _lib.PREC_FP32 if args.precision == "fp32" else _lib.PREC_BF16

    def sequential(Zs, prec):
        out = []
        for Z, y, C in zip(Zs, ys, Cs):
            out.append(api.ipm(ctx, Z, y, k, C, rel_gap_tol=1e-6, precision=prec)[3])
        return out

    for _ in range(args.warmup):
        batched()
    times, ipm_times = [], []
    Zs = None
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            # the previous step's factors (1.6 GB) are released first, as in a loop over grids;
            # held, they made the next step allocate anew (cudaMalloc inside the timed region)
            Zs = None
            (Zs, t_ipm), t = _timed(stream, batched)
            times.append(t)
            ipm_times.append(t_ipm)
    api.factor_batched(ctx, Xs, ys, gs, k, args.precision)   # a second set, untimed
    _, t_fac = _timed(stream, lambda: api.factor_batched(ctx, Xs, ys, gs, k, args.precision))
    factors_parallel(args.precision)
    _, t_fac_thr = _timed(stream, lambda: factors_parallel(args.precision))
    factors(args.precision)   # the main context's scratch, sized before it is timed
    _, t_fac_seq = _timed(stream, lambda: factors(args.precision))
    (alphas, bstats, info) = api.ipm_batched(ctx, Zs, ys, k, Cs, rel_gap_tol=1e-6,
                                             precision=ipm_prec)
    seq_stats, t_seq_ipm = _timed(stream, lambda: sequential(Zs, ipm_prec))
    del Zs
    t_fac32 = t_ipm32 = None
    if args.fp32_form:
        Z32, t_fac32 = _timed(stream, lambda: factors("fp32"))
        st32, t_ipm32 = _timed(stream, lambda: sequential(Z32, _lib.PREC_FP32))
    sec = statistics.mean(times)
    line = _base_line(args, "s for a 64-problem (C, gamma) grid: factors + batched IPM to rel. gap 1e-6",
                      sec, {"workload": "tanh_teacher_grid", "problems": 64, "rows_total": rows,
                            "n_min": min(X.shape[0] for X in Xs), "n_max": max(X.shape[0] for X in Xs),
                            "d": 28, "k": k, "precision": args.precision,
                            "factor_threads": nthreads})
    line.update({
        "dtype": f"{args.precision} kernel-block product; IPM f64 vectors, capacitance matrices "
                 f"{'bf16 hi+lo tensor-core + exact f64 rows, refined' if ipm_prec != _lib.PREC_FP32 else 'f64'}",
        "phases_s": {"factors": round(t_fac, 3), "factors_one_thread": round(t_fac_seq, 3),
                     "factors_threads": round(t_fac_thr, 3),
                     "batched_ipm": round(statistics.mean(ipm_times), 3),
                     "batched_ms_autotune": round(info["ms_autotune"], 1),
                     "unit_rows": info["unit_rows"], "units": info["units"],
                     "graph_used": info["graph_used"], "iters_max": info["iters_max"]},
        "sequential_same_factors": {"ipm_s": round(t_seq_ipm, 3), "total_s": round(t_fac + t_seq_ipm, 3),
                                    "speedup_batched_ipm": round(t_seq_ipm / statistics.mean(ipm_times), 2)},
        "plain_fp32_sequential": None if t_fac32 is None else
                                 {"factors_s": round(t_fac32, 3), "ipm_s": round(t_ipm32, 3),
                                  "total_s": round(t_fac32 + t_ipm32, 3),
                                  "speedup": round((t_fac32 + t_ipm32) / sec, 2)},
        "iters": {"batched": [s["iters"] for s in bstats], "sequential": [s["iters"] for s in seq_stats]},
        "status_ok": sum(1 for s in bstats if s["status"] == _lib.OK),
        "step_s": [round(t, 3) for t in times], "clocks": clk.summary()})
    for wctx, _ in workers:
        wctx.close()
    return line


def run_hypergrad(args, ctx, stream):
    """Validation squared-hinge hypergradient, n=200,000 train + 50,000 validation, d=28,
    gamma 0.03, C 16, k 256: forward (factor + IPM + bias + loss) and backward (tsvm_hypergrad,
    factor recomputed) times."""
    import torch
    from tensorsvm_b200 import _lib, api, synth
    X, y, gamma, C, k = synth.make("c5")
    Xv, yv, _, _, _ = synth.make("c5_val")
    Xd, yd = torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()
    Xvd, yvd = torch.from_numpy(Xv).cuda(), torch.from_numpy(yv).cuda()
    prec = args.precision

    def forward():
        Z, _ = api.factor(ctx, Xd, yd, gamma, k, prec)
        a, xi, ym, st = api.ipm(ctx, Z, yd, k, C, want_xi=True, tol=1e-9,
                                precision=_lib.PREC_FP32 if prec == "fp32" else _lib.PREC_BF16)
        b = api.bias(ctx, Z, yd, a, k, C)[0]
        del Z
        return a, xi, st["s"], ym, b, st

    def backward(sol):
        a, xi, s, ym, b, _ = sol
        return api.hypergrad(ctx, Xd, yd, Xvd, yvd, gamma, C, k, a, xi, s, ym, b, precision=prec,
                             want_dxv=True)

    # the forward's factor is kept for the backward (memory is not tight at this size: the
    # sketch, R, the unrounded basis and Z, 3 n k_padded floats)
    ctx.set_factor_keep(True)
    for _ in range(args.warmup):
        backward(forward())
    fw, bw, res = [], [], None
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            sol, tf = _timed(stream, forward)
            res, tb = _timed(stream, lambda: backward(sol))
            fw.append(tf)
            bw.append(tb)
    r, dxv = res
    # the backward of a context that kept nothing: the factor recomputed (the memory-tight path)
    sol = forward()
    with _lib.Context(torch.cuda.current_device()) as c2:
        hs = torch.cuda.Stream()
        c2.set_stream(hs.cuda_stream)
        with torch.cuda.stream(hs):
            a, xi, s_, ym, b, _ = sol
            api.hypergrad(c2, Xd, yd, Xvd, yvd, gamma, C, k, a, xi, s_, ym, b, precision=prec)
            _, t_rec = _timed(hs, lambda: api.hypergrad(c2, Xd, yd, Xvd, yvd, gamma, C, k, a, xi,
                                                        s_, ym, b, precision=prec))
    sec = statistics.mean(fw) + statistics.mean(bw)
    line = _base_line(args, "s for forward + backward of the validation-loss hypergradient "
                            "(n=200k + 50k, d=28, k=256)", sec,
                      {"workload": "tanh_teacher_hypergrad", "n": X.shape[0], "n_val": Xv.shape[0],
                       "d": X.shape[1], "k": k, "gamma": gamma, "C": C, "precision": prec})
    line.update({
        "dtype": f"{prec} kernel-block product, f64 IPM and adjoint",
        "forward_s": round(statistics.mean(fw), 3), "backward_s": round(statistics.mean(bw), 3),
        "backward_ms_inside": round(r["ms"], 1), "ipm_iters": sol[5]["iters"],
        "factor_reused": r["factor_reused"], "backward_factor_recomputed_s": round(t_rec, 3),
        "loss": r["loss"], "dloss_dlog_gamma": r["dloss_dlog_gamma"], "dloss_dlog_C": r["dloss_dlog_C"],
        "n_free_bias": r["n_free_bias"], "dxv_norm": float(dxv.double().norm()),
        "clocks": clk.summary()})
    return line


def run_workload(args, world, rank, local):
    if rank != 0:
        return None
    import torch
    from tensorsvm_b200 import _lib
    torch.cuda.set_device(local)
    ctx = _lib.Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    fn = {"wide": run_wide, "grid": run_grid, "hypergrad": run_hypergrad}[args.workload]
    with torch.cuda.stream(stream):
        line = fn(args, ctx, stream)
    line["gpu_launches"] = int(ctx.launches)
    ctx.close()
    return line


def kernel_table(args, local):
    """Per-kernel device time of one step (after one warm-up step) through CUPTI (torch.profiler),
    which also sees the kernels a CUDA graph replays: the two-Gaussian solve (factor + IPM) or the
    grid (batched factors, then the batched IPM).  Prints a table per phase; no JSON line."""
    import collections
    import torch
    from torch.profiler import profile, ProfilerActivity
    from tensorsvm_b200 import _lib, api, synth
    torch.cuda.set_device(local)
    ctx = _lib.Context(local)
    prec = args.precision
    mixed = _lib.PREC_FP32 if prec == "fp32" else _lib.PREC_BF16
    if args.workload == "grid":
        probs = synth.grid_problems(count=64)
        Xs = [torch.from_numpy(X).cuda() for X, _, _, _ in probs]
        ys = [torch.from_numpy(y).cuda() for _, y, _, _ in probs]
        gs = [g for _, _, g, _ in probs]
        Cs = [C for _, _, _, C in probs]
        state = {}
        phases = [("factors", lambda: state.__setitem__(
                      "Z", api.factor_batched(ctx, Xs, ys, gs, 128, prec)[0])),
                  ("batched ipm", lambda: api.ipm_batched(ctx, state["Z"], ys, 128, Cs,
                                                          rel_gap_tol=1e-6, precision=mixed))]
    else:
        X, y = synth.two_gaussians(args.n, D, seed=replica_seed(0), noise=NOISE)
        Xd, yd = torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()
        state = {}
        phases = [("factor", lambda: state.__setitem__(
                      "Z", api.factor(ctx, Xd, yd, GAMMA, K, prec)[0])),
                  ("ipm", lambda: api.ipm(ctx, state["Z"], yd, K, CPEN, rel_gap_tol=1e-6,
                                          precision=mixed))]
    for _, fn in phases:   # warm-up
        fn()
    torch.cuda.synchronize()
    for name, fn in phases:
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize()
        tot, cnt = collections.defaultdict(float), collections.Counter()
        for e in prof.events():
            if e.device_type == torch.autograd.DeviceType.CUDA:
                kn = e.name.replace("(anonymous namespace)::", "").split("(")[0][:110]
                tot[kn] += e.time_range.elapsed_us()
                cnt[kn] += 1
        total = sum(tot.values())
        print(f"== {name}: {total / 1e3:.1f} ms of kernels over {sum(cnt.values())} launches")
        for kn, v in sorted(tot.items(), key=lambda x: -x[1])[:30]:
            print(f"{cnt[kn]:6d} {v / 1e3:9.2f} ms {100 * v / total:6.2f}%  "
                  f"{v / cnt[kn]:9.1f} us  {kn}")
    ctx.close()


def run_other_workloads(args, local):
    """The wide-feature, batched-grid and hypergradient lines (their full-size workloads, three
    warm-up and up to three timed steps each), nested in the default line so that one run
    records all of them; a workload that fails records its error instead."""
    import copy
    out = {}
    for name in ("wide", "grid", "hypergrad"):
        sub = copy.copy(args)
        sub.workload, sub.n, sub.steps, sub.warmup = name, N_DEFAULT, min(args.steps, 3), 3
        try:
            out[name] = run_workload(sub, 1, 0, local)
        except Exception as e:   # keep the headline line whatever happens here
            out[name] = {"error": f"{type(e).__name__}: {e}"}
    return out


# ------------------------------------------------------------------------------------------
# reference arm: the reference trainer built from its own source (oracle/_ref)
# ------------------------------------------------------------------------------------------

def parse_ref_log(text):
    """Phase times and the every-5-iterations IPM log of one reference run (tensorsvm-train.cu):
    file read (line 899), LRA (963) and MPC (987) totals in whole seconds, the model write
    (1022-1024, timed by the END_TIMER macro of line 53), and (iter, normdx, normdy, pobj,
    dobj) per logged iterate (1645)."""
    text = re.sub(r"\x1b\[[0-9;]*m", "", text)
    el = [float(v) for v in re.findall(r"elapsed time = ([0-9.]+) seconds", text)]
    read = float(re.search(r"Reading files took ([0-9.]+) seconds", text).group(1))
    lra = float(re.search(r"LRA elapsed time = ([0-9.]+) seconds", text).group(1))
    mpc = float(re.search(r"MPC elapsed time = ([0-9.]+) seconds", text).group(1))
    write = el[-1]
    iters = [(int(i), float(dx), float(dy), float(p), float(d)) for i, dx, dy, p, d in
             re.findall(r"iter (\d+), mu=\S+, normdx=(\S+), normdy=(\S+) max/min\(D\)=\S+ "
                        r"pobj=(\S+) dobj=(\S+)", text)]
    return read, lra, mpc, write, iters


def ref_time_to_gap(wall, read, mpc, write, iters, n):
    """Seconds from the host-resident training set to the first logged iterate that meets the
    stopping rule of this benchmark (rel_gap <= 1e-6, ||rd||/(1+sqrt n) and |rp|/(1+sqrt n)
    <= 1e-6): the run's wall time less its file read and model write, less the part of its
    MPC phase after that iterate (MPC time prorated by iterations; the reference logs every
    5th iterate, so the first one logged at or after the rule is met is used)."""
    last = iters[-1][0]
    hit = last
    for it, dx, dy, p, d in iters:
        if (p - d) / max(1.0, abs(p)) <= 1e-6 and dx / (1 + n ** 0.5) <= 1e-6 \
                and dy / (1 + n ** 0.5) <= 1e-6:
            hit = it
            break
    after = mpc * (last - hit) / (last + 1)
    return wall - read - write - after, hit


def run_reference(args, world, rank):
    """The reference trainer (oracle/_ref, built from its own source) on the benchmark's full
    n = 1M workload, run as a process per step on the box's host cores and its GPU.  A run
    takes about 100 s, so the arm runs as many full-size steps as fit in --ref-budget seconds
    (at least one, at most --steps) and reports the count it ran."""
    if rank != 0:
        return None
    ref = os.path.join(ROOT, "oracle", "_ref", "tensorsvm-train-ref")
    if not os.path.exists(ref):
        return {"impl": "reference", "unavailable": "oracle/_ref/tensorsvm-train-ref not built"}
    from tensorsvm_b200 import synth
    tmp = tempfile.mkdtemp()
    small = os.path.join(tmp, "small.train")
    X, y = synth.two_gaussians(8192, D, seed=2, noise=NOISE)
    synth.write_libsvm(small, X, y)
    big = os.path.join(tmp, "full.train")
    X, y = synth.two_gaussians(args.n, D, seed=replica_seed(0), noise=NOISE)
    synth.write_libsvm(big, X, y)
    del X, y
    cmd = [ref, "-k", str(K), "-c", str(CPEN), "-g", str(GAMMA), "-t", "2"]
    # warm-up on a small file: the driver JIT-compiles the reference's compute_70 PTX once
    for _ in range(args.warmup):
        subprocess.run(cmd + [small, small + ".model"], capture_output=True, text=True, timeout=600)
    vals, walls, details = [], [], []
    t_start = time.perf_counter()
    while len(vals) < args.steps:
        t0 = time.perf_counter()
        p = subprocess.run(cmd + [big, big + ".model"], capture_output=True, text=True, timeout=1800)
        wall = time.perf_counter() - t0
        if p.returncode != 0:
            return {"impl": "reference", "unavailable": f"reference run exited {p.returncode}"}
        read, lra, mpc, write, iters = parse_ref_log(p.stdout)
        v, hit = ref_time_to_gap(wall, read, mpc, write, iters, args.n)
        vals.append(v)
        walls.append(wall)
        details.append({"wall": round(wall, 2), "read": read, "lra": lra, "mpc": mpc,
                        "writemodel": write, "iters": iters[-1][0], "rule_met_at_iter": hit,
                        "pobj": iters[-1][3], "dobj": iters[-1][4]})
        elapsed = time.perf_counter() - t_start
        if elapsed + statistics.mean(walls) > args.ref_budget:
            break
    value = statistics.mean(vals)
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 2), "unit": "s",
        "n_gpus": world, "steps": len(vals), "steps_requested": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * statistics.mean(walls), 1), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 LRA (cuBLAS) + f64 host IPM (OpenBLAS)",
        "data": "synthetic (seeded two-Gaussian mixture, 10% label noise)",
        "config": workload_config(args.n, 1),
        "cpu_baseline": {"value": round(value, 2), "unit": "s", "cores": os.cpu_count(),
                         "kind": "reference",
                         "sample": f"reference build (oracle/_ref) on the full n={args.n} file, "
                                   f"{len(vals)} runs; value = wall time less file read and "
                                   f"model write and less the MPC iterations after the first "
                                   f"logged iterate meeting the stopping rule"},
        "e2e": {"value": round(value, 2), "unit": "s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "detail": details,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp16", choices=["fp16", "bf16", "fp32"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-fp32-form", dest="fp32_form", action="store_false")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", default="32768,65536,131072",
                    help="row counts of the FP64 oracle samples behind cpu_baseline's fit")
    ap.add_argument("--ref-budget", type=float, default=300.0,
                    help="reference arm: seconds of full-size reference runs (at least one run)")
    ap.add_argument("--factor-threads", type=int, default=4,
                    help="grid workload: host threads (one context each) for the 64 factors")
    ap.add_argument("--kernel-table", action="store_true",
                    help="print per-kernel device times of one step (CUPTI) instead of timing; "
                         "two_gaussians or grid")
    ap.add_argument("--no-workloads", dest="workloads", action="store_false",
                    help="default line at N=1: skip the wide / grid / hypergrad lines that are "
                         "otherwise appended under 'workloads'")
    ap.add_argument("--workload", default="two_gaussians", choices=["two_gaussians", "wide", "grid", "hypergrad"],
                    help="two_gaussians (default): the benchmark line; wide: n=500k d=54 k=400; "
                         "grid: 64-problem batched (C, gamma) grid; hypergrad: validation-loss "
                         "hypergradient at n=200k + 50k")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.kernel_table:
        if rank == 0:
            kernel_table(args, local)
        return
    if args.workload != "two_gaussians" and args.impl == "ours":
        line = run_workload(args, world, rank, local)
    elif args.impl == "reference":
        line = run_reference(args, world, rank)
    else:
        line = run_ours(args, world, rank, local)
        if line is not None and world == 1 and args.workloads:
            line["workloads"] = run_other_workloads(args, local)
    if line is not None and rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
