#!/usr/bin/env python
"""CP-ALS benchmark: iterations/s of the mixed-precision (BF16x3 tensor-core
MTTKRP, FP64 Gram/solve/fit) CP-ALS on a 256^3 rank-64 FP32 tensor, beside
the plain-FP32 GPU path, with the fits of both.

    python bench.py --gpus N --steps K --warmup W [--impl reference]

One step = one CP-ALS call of 10 iterations (tol 0) on the resident tensor.
N > 1 runs one independent CP-ALS replica per GPU (weak scaling; the dense
path has no data exchange between replicas). `--impl reference` times the
CPU restatement of tenrso's own serial cp_als path instead (rank 0 only).
Prints one JSON line on rank 0.
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

METRIC = "CP-ALS iter/s (256^3 R=64; CSF 5e7 nnz) mixed vs FP32 GPU at equal fit"
SHAPE = (256, 256, 256)
RANK = 64
ITERS = 10
SEED = 0xC2
WORKLOAD = "dense CP-ALS 256x256x256 rank 64, 10 iterations, tol 0"
# DRAM read + write bytes of one mode-0 launch of the single-layout BF16x3
# MTTKRP at 256^3 rank 64 (ncu, dram__bytes_read.sum + dram__bytes_write.sum)
MTTKRP3_TRAFFIC = 67_278_592 + 960_256


def measured_peaks() -> dict:
    """The pool's measured peaks (HBM copy GB/s, bf16 TFLOP/s), {} if absent."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def max_over_ranks(x: float, dist, device="cuda") -> float:
    """The largest value of x over all ranks (identity without a process group).
    Every rank must call it at the same point: it is a collective."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def hbm_peak_gbs() -> float:
    """Measured HBM copy bandwidth, else the pool's earlier fallback figure."""
    return float(measured_peaks().get("hbm_gbs", 6650.0))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sparse", action="store_true")
    ap.add_argument("--sparse-nnz", type=int, default=50_000_000)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--case", default=None,
                    help="run one small profiling case instead of the bench: mttkrp, cp_als, "
                         "csf_mttkrp, loss_grad, batched")
    ap.add_argument("--precision", default="bf16x3")
    ap.add_argument("--shape", type=int, nargs="+", default=[256, 256, 256])
    ap.add_argument("--rank", type=int, default=64)
    ap.add_argument("--mode", type=int, default=0)
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--launches", type=int, default=1)
    ap.add_argument("--nnz", type=int, default=20_000_000)
    ap.add_argument("--time", action="store_true", help="--case: also print the kernel time")
    return ap.parse_args()


def c2_fp64_fit():
    """The FP64 oracle's fit on this workload (the committed fixture), or None."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "c2_fp64_fit.json")) as f:
            return float(json.load(f)["fp64_fit"])
    except (OSError, KeyError, ValueError):
        return None


def make_inputs():
    from tenrso_b200 import synth
    X, _ = synth.dense_lowrank(SHAPE, RANK, seed=SEED, dist="uniform", noise=0.005)
    init = synth.init_factors(SHAPE, RANK, SEED)
    return X, init


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi sampled every 200 ms while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1", "yes"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------------------
# Single small cases of the hot-path kernels (`--case NAME`), for ncu captures
# and quick timing: each prepares its inputs on the device, runs --warmup
# untimed launches and then --launches more, and prints a checksum. They print
# no bench line.
def _case_ctx():
    import torch

    import tenrso_b200 as tb
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    return tb.Context(0, stream=stream.cuda_stream)


def case_mttkrp(args):
    import torch

    import tenrso_b200 as tb
    ctx = _case_ctx()
    shape = tuple(args.shape)
    g = torch.Generator(device="cuda").manual_seed(1)
    X = torch.rand(shape, device="cuda", generator=g)
    fs = [torch.rand(n, args.rank, device="cuda", generator=g) for n in shape]
    M = torch.empty(shape[args.mode], args.rank, device="cuda")
    for _ in range(args.warmup + args.launches):
        tb.mttkrp_dev(X.data_ptr(), shape, [f.data_ptr() for f in fs], args.rank, args.mode,
                      M.data_ptr(), args.precision, ctx=ctx)
    torch.cuda.synchronize()
    print("mttkrp", args.precision, shape, "rank", args.rank, "mode", args.mode,
          "checksum", float(M.double().sum()))


def case_cp_als(args):
    import torch

    import tenrso_b200 as tb
    from tenrso_b200 import synth
    ctx = _case_ctx()
    shape = tuple(args.shape)
    X, _ = synth.dense_lowrank(shape, args.rank, seed=0xC2, dist="uniform", noise=0.005)
    init = synth.init_factors(shape, args.rank, 0xC2)
    dX = torch.from_numpy(X).cuda()
    dinit = torch.from_numpy(np.concatenate([f.ravel() for f in init])).cuda()
    dout = torch.empty_like(dinit)
    for _ in range(args.warmup + args.launches):
        fit, it, _ = tb.cp_als_dev(dX.data_ptr(), shape, args.rank, args.iters, 0.0,
                                   dinit.data_ptr(), dout.data_ptr(), args.precision, ctx=ctx)
    torch.cuda.synchronize()
    print("cp_als", args.precision, shape, "rank", args.rank, "fit", fit, "iters", it)


def case_csf_mttkrp(args):
    """CSF MTTKRP on the seeded Zipf(1.2) tensor (device-drawn, merged)."""
    import torch

    import tenrso_b200 as tb
    ctx = _case_ctx()
    shape = tuple(args.shape) if len(args.shape) == 3 and args.shape != [256, 256, 256] \
        else (100000, 80000, 10000)
    cap = 12 * args.nnz
    d_idx = torch.empty(cap * 3, dtype=torch.int64, device="cuda")
    d_val = torch.empty(cap, dtype=torch.float32, device="cuda")
    n_raw = tb.synth_zipf_coo_dev(shape, args.nnz, 0xC3, d_idx.data_ptr(), d_val.data_ptr(), cap,
                                  ctx=ctx)
    n = tb.coo_deduplicate_dev(d_idx.data_ptr(), d_val.data_ptr(), n_raw, shape, ctx=ctx)
    sp = tb.SparseTensor(ctx=ctx, d_indices=d_idx.data_ptr(), d_values=d_val.data_ptr(), nnz=n,
                         shape=shape)
    del d_idx, d_val
    g = torch.Generator(device="cuda").manual_seed(1)
    fs = [torch.rand(m, args.rank, device="cuda", generator=g) for m in shape]
    M = torch.empty(shape[args.mode], args.rank, device="cuda")
    for _ in range(args.warmup + args.launches):
        sp.mttkrp_dev([f.data_ptr() for f in fs], args.rank, args.mode, M.data_ptr())
    torch.cuda.synchronize()
    print("csf_mttkrp", shape, "nnz", n, "rank", args.rank, "mode", args.mode,
          "checksum", float(M.double().sum()), sp.info(args.mode))
    if args.time:
        ms = sp.profile_mttkrp_dev([f.data_ptr() for f in fs], args.rank, args.mode, iters=10,
                                   flush_l2=True)
        print(f"csf_mttkrp kernel {ms:.4f} ms (L2 flushed, mean of 10)")
    sp.close()


def case_loss_grad(args):
    """Gram-form loss/gradient of ||X - [[A,B,C,D]]||^2 + 1e-3 sum ||U||^2 at
    128x96x64x48, rank 32 (seeded N(0,1))."""
    import torch

    import tenrso_b200 as tb
    ctx = _case_ctx()
    shape = (128, 96, 64, 48)
    rng = np.random.default_rng(0xC5)
    X = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda()
    fs = [torch.from_numpy(rng.standard_normal((n, args.rank)).astype(np.float32)).cuda()
          for n in shape]
    gs = [torch.empty_like(f) for f in fs]
    d = tb.DenseTensor(X.data_ptr(), shape, args.precision, ctx=ctx)
    loss = None
    for _ in range(args.warmup + args.launches):
        loss = d.loss_grad_dev([f.data_ptr() for f in fs], args.rank, 1e-3,
                               [g.data_ptr() for g in gs])
    torch.cuda.synchronize()
    print("loss_grad", args.precision, shape, "rank", args.rank, "loss", loss)
    d.close()


def case_batched(args):
    """The 512-instance batched CP-ALS run (sizes U{16..96}, ranks U{4..16})."""
    import torch

    import tenrso_b200 as tb
    from tenrso_b200 import synth
    ctx = _case_ctx()
    inst = synth.batched_instances(512, 0xC4)
    b = tb.BatchedCpAls([X.astype(np.float32) for X, _, _ in inst], [R for _, R, _ in inst],
                        ctx=ctx)
    d_init = torch.from_numpy(b.pack([i for _, _, i in inst])).cuda()
    d_out = torch.empty_like(d_init)
    torch.cuda.synchronize()
    info = None
    for _ in range(args.warmup + args.launches):
        info = b.cp_als_dev(args.iters, 0.0, d_init.data_ptr(), d_out.data_ptr(), want_info=True)
    print("batched", len(inst), "instances", args.iters, "iterations, mean fit",
          float(np.mean([f for f, _, _ in info])), b.config)
    b.close()


CASES = {"mttkrp": case_mttkrp, "cp_als": case_cp_als, "csf_mttkrp": case_csf_mttkrp,
         "loss_grad": case_loss_grad, "batched": case_batched}


# ---------------------------------------------------------------------------
def cpu_cp_als_rate(X, init, iters: int = 1):
    """Iterations/s of the oracle's restated cp_als<f32> (cp/core.rs:59-182) on
    this box's host cores: the full loop (three mode updates with their
    MTTKRPs, Gram Hadamards and solves, then the fit's extra MTTKRP), OpenMP
    over all threads. Returns (iter/s, threads)."""
    from oracle import oracle as orc
    t0 = time.perf_counter()
    orc.cp_als(X, RANK, iters, 0.0, init)
    return iters / (time.perf_counter() - t0), orc.num_threads()


def run_reference(args):
    """The CPU restatement of tenrso's cp_als<f32> (oracle/; the reference's
    loop, solve and fit), on the host cores with every OpenMP thread. One step
    = one full ALS iteration (modes 0..2 + fit) from the seeded init. Also
    reported: the single-thread faithful restatement (unfold copy,
    materialised Khatri-Rao, i/r/j loop) of one mode update, x4."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as orc
    X, init = make_inputs()

    def step():
        orc.cp_als(X, RANK, 1, 0.0, init)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    it_s = 1.0 / dt
    G = orc.gram(init[1]) * orc.gram(init[2])
    t1 = time.perf_counter()
    orc.solve(orc.mttkrp(X, init, 0, faithful=True), G)
    faithful = 1.0 / (4.0 * (time.perf_counter() - t1))
    line = {
        "impl": "reference", "metric": METRIC, "value": it_s, "unit": "iter/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SplitMix64)",
        "config": {"workload": WORKLOAD, "sample": "one full ALS iteration per step"},
        "cpu_baseline": {"value": it_s, "unit": "iter/s", "cores": orc.num_threads(),
                         "kind": "port",
                         "sample": "one full iteration of the restated cp_als<f32> "
                                   "(OpenMP over all host threads) per step"},
        "faithful_serial": {"value": faithful, "unit": "iter/s", "cores": 1,
                            "sample": "one mode-0 update of the faithful single-thread "
                                      "restatement, x4 per iteration"},
        "e2e": {"value": it_s, "unit": "iter/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
SP_SHAPE = (100000, 80000, 10000)
SP_RANK = 32
SP_ITERS = 20
SP_SEED = 0xC3


def run_sparse(tb, torch, ctx, stream, args, world, dist):
    """CSF CP-ALS on the Zipf(1.2) tensor: device-drawn raw COO, merged on the
    device (CooTensor::deduplicate semantics), one CSF per mode, then 20 ALS
    iterations at rank 32. Also times the CSF MTTKRP kernel alone."""
    from tenrso_b200 import synth
    nnz = args.sparse_nnz
    cap = 12 * nnz
    d_idx = torch.empty(cap * 3, dtype=torch.int64, device="cuda")
    d_val = torch.empty(cap, dtype=torch.float32, device="cuda")
    t0 = time.perf_counter()
    n_raw = tb.synth_zipf_coo_dev(SP_SHAPE, nnz, SP_SEED, d_idx.data_ptr(), d_val.data_ptr(),
                                  cap, ctx=ctx)
    t1 = time.perf_counter()
    n = tb.coo_deduplicate_dev(d_idx.data_ptr(), d_val.data_ptr(), n_raw, SP_SHAPE, ctx=ctx)
    t2 = time.perf_counter()
    cpu_sample = None
    if world == 1 and not args.no_cpu_baseline:
        # the CPU baseline's sample: the merged entries of every 20th root
        # (mode-0 index % 20 == 0; the Zipf head sits at permuted indices)
        idx = d_idx[:3 * n].view(n, 3)
        keep = idx[:, 0] % 20 == 0
        cpu_sample = (idx[keep].cpu().numpy(), d_val[:n][keep].cpu().numpy())
    sp = tb.SparseTensor(ctx=ctx, d_indices=d_idx.data_ptr(), d_values=d_val.data_ptr(), nnz=n,
                         shape=SP_SHAPE)
    t3 = time.perf_counter()
    del d_idx, d_val
    torch.cuda.empty_cache()
    init = synth.init_factors(SP_SHAPE, SP_RANK, SP_SEED)
    flat = np.concatenate([f.ravel() for f in init])
    dinit = torch.from_numpy(flat).cuda()
    dout = torch.empty_like(dinit)
    sp.cp_als_dev(SP_RANK, SP_ITERS, 0.0, dinit.data_ptr(), dout.data_ptr())  # warm-up
    steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        fit, iters, _ = sp.cp_als_dev(SP_RANK, SP_ITERS, 0.0, dinit.data_ptr(), dout.data_ptr())
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    ms = max_over_ranks(ms, dist)
    d_factors = [dinit.data_ptr() + 4 * sum(SP_SHAPE[:m]) * SP_RANK for m in range(3)]
    modes = []
    for mode in range(3):
        kms = sp.profile_mttkrp_dev(d_factors, SP_RANK, mode, iters=5, flush_l2=True)
        inf = sp.info(mode)
        others = sum(SP_SHAPE[m] for m in range(3) if m != mode)
        b_min = (8 * n + 8 * inf["fibers"] + 8 * inf["roots"] + 4 * others * SP_RANK
                 + 4 * SP_SHAPE[mode] * SP_RANK)
        modes.append({"mode": mode, "kernel_ms": kms, "roots": inf["roots"],
                      "fibers": inf["fibers"], "bytes_min": b_min,
                      "achieved_gbs": b_min / (kms * 1e-3) / 1e9})
    sp.close()
    cpu = None
    if cpu_sample is not None:
        cpu = csf_cpu_baseline(cpu_sample, n, modes[0]["kernel_ms"])
    return {"workload": f"CSF CP-ALS {SP_SHAPE[0]}x{SP_SHAPE[1]}x{SP_SHAPE[2]}, Zipf(1.2) indices "
                        f"over seeded permutations, rank {SP_RANK}, {SP_ITERS} iterations",
            "nnz": n, "raw_entries": n_raw, "duplicates_merged": n_raw - n,
            "iter_per_s": iters * world / (ms / 1e3), "ms_per_run": ms, "fit": fit,
            "iters": iters, "synth_s": t1 - t0, "dedup_s": t2 - t1, "csf_build_s": t3 - t2,
            "mttkrp": modes,
            "mttkrp_hbm_frac_mean": float(np.mean([m["achieved_gbs"] for m in modes])) / hbm_peak_gbs(),
            "cpu_baseline": cpu}


def csf_cpu_baseline(sample, nnz_total: int, gpu_mode0_ms: float):
    """The restated CSF MTTKRP (no tenrso implementation; oracle/) rooted at
    mode 0 on the sampled entries, serial and OpenMP, as nnz/s, with the
    mode-0 time at the full nnz it implies."""
    from oracle import oracle as orc
    idx, vals = sample
    mo = [0, 2, 1]  # the root, then the other modes by ascending size
    t0 = time.perf_counter()
    fp, fi, v = orc.csf_from_coo(idx, vals, mo)
    build_s = time.perf_counter() - t0
    rng = np.random.default_rng(1)
    fs = [rng.random((m, SP_RANK), dtype=np.float32) for m in SP_SHAPE]
    out = {"kind": "port", "unit": "nnz/s", "sample_nnz": int(len(vals)),
           "sample": "merged entries of every 20th mode-0 root; restated CSF MTTKRP rooted at "
                     "mode 0 (mode order 0, 2, 1), fp32",
           "csf_from_coo_s": build_s}
    for label, threads in (("serial", 1), ("openmp", orc.num_threads())):
        orc.csf_mttkrp(fp, fi, v, mo, SP_SHAPE, fs, threads)  # warm
        t0 = time.perf_counter()
        reps = 3
        for _ in range(reps):
            orc.csf_mttkrp(fp, fi, v, mo, SP_SHAPE, fs, threads)
        dt = (time.perf_counter() - t0) / reps
        rate = len(vals) / dt
        out[label] = {"value": rate, "cores": threads,
                      "mode0_ms_at_full_nnz": nnz_total / rate * 1e3,
                      "gpu_speedup_mode0": nnz_total / rate * 1e3 / gpu_mode0_ms}
    out["value"] = out["openmp"]["value"]
    out["cores"] = out["openmp"]["cores"]
    return out


AD_SHAPE = (128, 96, 64, 48)
AD_RANK = 32
AD_REG = 1e-3
AD_SEED = 0xC5


def run_adjoint(tb, torch, ctx, stream, args, world, dist, rank):
    """Loss + gradient of ||X - [[A,B,C,D]]||^2 + 1e-3 sum ||U||^2 at
    128x96x64x48, R=32 (seeded N(0,1) target and factors): the Gram form on a
    prepared tensor (one MTTKRP of X per mode), in FP32 and BF16x3, and the
    recompute form (GPU residual G = 2(Xhat - X), then the reconstruction
    adjoint on G)."""
    rng = np.random.default_rng(AD_SEED)
    X = rng.standard_normal(AD_SHAPE).astype(np.float32)
    fs = [rng.standard_normal((n, AD_RANK)).astype(np.float32) for n in AD_SHAPE]
    dX = torch.from_numpy(X).cuda()
    dF = [torch.from_numpy(f).cuda() for f in fs]
    dGr = [torch.empty_like(f) for f in dF]
    fptr = [f.data_ptr() for f in dF]
    gptr = [g.data_ptr() for g in dGr]
    steps = max(5, args.steps)
    # algorithmic bytes: fp32, two MTTKRP passes (X and its transposed copy,
    # 2 x 4 B per element); bf16x3, one two-sided read of X's
    # bf16 halves (4 B per element)
    out = {"workload": "CP loss+gradient 128x96x64x48, rank 32, reg 1e-3",
           "bytes_alg_per_eval": {"fp32": 2 * 4 * X.size, "bf16x3": 4 * X.size}}

    def timed(fn):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ctx.launches
        ev0.record(stream)
        for _ in range(steps):
            fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / steps
        ms = max_over_ranks(ms, dist)
        return ms, (ctx.launches - l0) // steps

    for prec in ("fp32", "bf16x3"):
        d = tb.DenseTensor(dX.data_ptr(), AD_SHAPE, prec, ctx=ctx)
        ms, launches = timed(lambda: d.loss_grad_dev(fptr, AD_RANK, AD_REG, gptr,
                                                     want_loss=False))
        loss = d.loss_grad_dev(fptr, AD_RANK, AD_REG, gptr)
        d.close()
        out[f"gram_form_{prec}"] = {
            "evals_per_s": world * 1e3 / ms, "ms_per_eval": ms, "loss": loss,
            "launches_per_eval": launches,
            "achieved_gbs": out["bytes_alg_per_eval"][prec] / (ms * 1e-3) / 1e9}
    dG = torch.empty_like(dX)

    def recompute():
        tb.cp_residual_dev(dX.data_ptr(), AD_SHAPE, fptr, AD_RANK, dG.data_ptr(), 2.0,
                           want_sq=False, ctx=ctx)
        tb.reconstruction_grad_dev(dG.data_ptr(), AD_SHAPE, fptr, AD_RANK, gptr, ctx=ctx)

    ms, launches = timed(recompute)
    out["recompute_form_fp32"] = {"evals_per_s": world * 1e3 / ms, "ms_per_eval": ms,
                                  "launches_per_eval": launches}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        t0 = time.perf_counter()
        orc.cp_loss_grad_vjp(X, fs, AD_REG)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 1.0 / dt, "unit": "evals/s", "cores": orc.num_threads(),
                               "kind": "port",
                               "sample": "one FP64 CPU VJP: restated cp_reconstruct, "
                                         "G = 2(Xhat - X), restated CpReconstructionGrad"}
    return out


BT_COUNT = 512
BT_ITERS = 25
BT_SEED = 0xC4


def run_batched(tb, torch, ctx, stream, args, world, dist, rank):
    """512 independent 3-way CP-ALS instances (sizes U{16..96}, ranks
    U{4..16}, seeded low-rank N(0,1) + 1% noise), 25 iterations each, all in
    one persistent launch per run (a captured CUDA graph), launch
    configuration chosen by the autotuner."""
    import tempfile
    from tenrso_b200 import synth
    t0 = time.perf_counter()
    inst = synth.batched_instances(BT_COUNT, BT_SEED)
    gen_s = time.perf_counter() - t0
    tensors = [X.astype(np.float32) for X, _, _ in inst]
    ranks = [R for _, R, _ in inst]
    b = tb.BatchedCpAls(tensors, ranks, ctx=ctx)
    d_init = torch.from_numpy(b.pack([init for _, _, init in inst])).cuda()
    d_out = torch.empty_like(d_init)
    torch.cuda.synchronize()
    cache = os.path.join(tempfile.gettempdir(), "tenrso_b200_batched_tune.json")
    t1 = time.perf_counter()
    cfg, cached = b.autotune(BT_ITERS, d_init.data_ptr(), cache)
    tune_s = time.perf_counter() - t1
    for _ in range(max(3, args.warmup)):
        b.cp_als_dev(BT_ITERS, 0.0, d_init.data_ptr(), d_out.data_ptr())
    steps = max(3, args.steps)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = ctx.launches
    ev0.record(stream)
    for _ in range(steps):
        b.cp_als_dev(BT_ITERS, 0.0, d_init.data_ptr(), d_out.data_ptr())
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    launches = (ctx.launches - l0) // steps
    ms = max_over_ranks(ms, dist)
    info = b.cp_als_dev(BT_ITERS, 0.0, d_init.data_ptr(), d_out.data_ptr(), want_info=True)
    elems = [X.size for X in tensors]
    # two passes over each tensor per sweep, 4 bytes per element
    bytes_alg = float(sum(8 * e for e in elems)) * BT_ITERS
    flops_alg = float(sum(4 * e * R for e, R in zip(elems, ranks))) * BT_ITERS
    out = {"workload": f"{BT_COUNT} CP-ALS instances, sizes U{{16..96}}^3, ranks U{{4..16}}, "
                       f"{BT_ITERS} iterations each",
           "instance_iter_per_s": world * BT_COUNT * BT_ITERS / (ms / 1e3),
           "ms_per_run": ms, "launches_per_run": launches, "config": cfg,
           "config_from_cache": cached, "autotune_s": tune_s, "generate_s": gen_s,
           "elements_total": int(sum(elems)),
           "fit_mean": float(np.mean([f for f, _, _ in info])),
           "fit_min": float(np.min([f for f, _, _ in info])),
           "achieved_gbs_two_pass_model": bytes_alg / (ms * 1e-3) / 1e9,
           "achieved_tflops": flops_alg / (ms * 1e-3) / 1e12}
    b.close()
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        sample = 6
        t0 = time.perf_counter()
        for X, R, init in inst[:sample]:
            orc.cp_als(X.astype(np.float32), R, BT_ITERS, 0.0, init, faithful=True)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": sample * BT_ITERS / dt, "unit": "instance-iter/s",
                               "cores": 1, "kind": "port",
                               "sample": f"faithful serial f32 cp_als on the first {sample} "
                                         f"instances, {BT_ITERS} iterations each"}
    return out


def run_ours(args):
    import torch
    import tenrso_b200 as tb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = tb.Context(local, stream=stream.cuda_stream)

    X, init = make_inputs()
    dX = torch.from_numpy(X).cuda()
    flat_init = np.concatenate([f.ravel() for f in init])
    dinit = torch.from_numpy(flat_init).cuda()
    dout = torch.empty_like(dinit)
    shape = list(SHAPE)

    def step(prec):
        return tb.cp_als_dev(dX.data_ptr(), shape, RANK, ITERS, 0.0, dinit.data_ptr(),
                             dout.data_ptr(), prec, ctx=ctx)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def timed(prec, steps):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        barrier()
        l0 = ctx.launches
        ev0.record(stream)
        res = None
        for _ in range(steps):
            res = step(prec)
        ev1.record(stream)
        barrier()
        ms = ev0.elapsed_time(ev1)
        ms = max_over_ranks(ms, dist)
        return ms, res, ctx.launches - l0

    for _ in range(args.warmup):
        step("bf16x3")
        step("fp32")
    # clocks are sampled while the timed work runs; if one timed pass is too
    # short for the sampler, the same work repeats untimed until ~1.5 s of
    # load has been sampled
    sampler = ClockSampler(local)
    sampler.start()
    soak_t0 = time.perf_counter()
    ms_mixed, res_mixed, launches = timed("bf16x3", args.steps)
    ms_fp32, res_fp32, _ = timed("fp32", args.steps)
    while time.perf_counter() - soak_t0 < 1.5:
        step("bf16x3")
    torch.cuda.synchronize()
    clocks = sampler.stop()

    fp64_fit = c2_fp64_fit()
    iters_total = ITERS * args.steps * world
    value = iters_total / (ms_mixed / 1e3)
    fp32_value = iters_total / (ms_fp32 / 1e3)
    fit_mixed, fit_fp32 = res_mixed[0], res_fp32[0]

    # roofline: the dense MTTKRP kernel alone (L2 flushed between launches)
    d_factors = [dinit.data_ptr() + 4 * sum(SHAPE[:m]) * RANK for m in range(3)]
    kms = []
    for mode in range(3):
        ms, splits = tb.profile_mttkrp_dev(dX.data_ptr(), shape, d_factors, RANK, mode,
                                           "bf16x3", iters=10, flush_l2=True, ctx=ctx)
        kms.append(ms)
    kernel_ms = sum(kms) / len(kms)
    n = SHAPE[0] * SHAPE[1] * SHAPE[2]
    alg_bytes = 4 * n + 3 * SHAPE[0] * RANK * 4  # fp32 tensor + factors (B_min per MTTKRP)
    peaks = measured_peaks()
    peak = hbm_peak_gbs()
    achieved = alg_bytes / (kernel_ms * 1e-3) / 1e9
    # DRAM bytes (read + write) of one launch of the kernel, mode 0, from an
    # ncu capture of `bench.py --case mttkrp --precision bf16x3 --mode 0`
    traffic = MTTKRP3_TRAFFIC
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "traffic_unit": "bytes",
                "algorithmic_bytes": alg_bytes,
                "kernel": "mttkrp3_kernel", "kernel_ms": kernel_ms,
                "kernel_ms_per_mode": kms,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}

    # e2e through the host API: pinned host tensor in, factors out
    Xp = torch.from_numpy(X).pin_memory().numpy()
    initp = [torch.from_numpy(f).pin_memory().numpy() for f in init]
    tb.cp_als(Xp, RANK, ITERS, 0.0, init=initp, precision="bf16x3", ctx=ctx)
    barrier()
    t0 = time.perf_counter()
    e2e_steps = max(3, min(args.steps, 10))
    for _ in range(e2e_steps):
        tb.cp_als(Xp, RANK, ITERS, 0.0, init=initp, precision="bf16x3", ctx=ctx)
    barrier()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_s = max_over_ranks(e2e_s, dist)
    e2e = {"value": ITERS * world / e2e_s, "unit": "iter/s",
           "h2d_bytes_per_step": int(X.nbytes + flat_init.nbytes),
           "d2h_bytes_per_step": int(flat_init.nbytes + 64),
           "api": "tsr_cp_als_f32 (host pointers)"}

    sparse = None if args.no_sparse else run_sparse(tb, torch, ctx, stream, args, world, dist)
    adjoint = None if args.no_adjoint else run_adjoint(tb, torch, ctx, stream, args, world, dist,
                                                       rank)
    batched = None if args.no_batched else run_batched(tb, torch, ctx, stream, args, world, dist,
                                                       rank)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        rate, threads = cpu_cp_als_rate(X, init, 2)
        cpu = {"value": rate, "unit": "iter/s", "cores": threads, "kind": "port",
               "sample": "two full iterations of the restated cp_als<f32> (OpenMP over all "
                         "host threads) on the same tensor and init"}

    if dist is not None:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3 MTTKRP (fp32 accumulate) + f64 Gram/solve/fit",
            "data": "synthetic: seeded rank-64 U(0,1) factors + 0.5% Gaussian noise, fp32",
            "config": {"workload": WORKLOAD, "shape": list(SHAPE), "rank": RANK,
                       "iterations_per_step": ITERS, "precision": "bf16x3",
                       "parallelism": f"replicas{world}" if world > 1 else "1 GPU",
                       "l2": "working set per step > L2 (X 64 MiB + per-mode unfoldings "
                             "192 MiB re-written every step)"},
            "fp32_path": {"value": fp32_value, "unit": "iter/s", "fit": fit_fp32,
                          "ms_per_step": ms_fp32 / args.steps},
            "speedup_mixed_vs_fp32": value / fp32_value,
            "fit_mixed": fit_mixed, "fit_fp32": fit_fp32,
            "fit_abs_diff": abs(fit_mixed - fit_fp32),
            "fit_fp64_oracle": fp64_fit,
            "fit_err_vs_fp64": {"mixed": None if fp64_fit is None else abs(fit_mixed - fp64_fit),
                                "fp32": None if fp64_fit is None else abs(fit_fp32 - fp64_fit),
                                "source": "tests/golden/c2_fp64_fit.json (FP64 oracle, same "
                                          "seeded tensor and init, 10 iterations)"},
            "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks,
            "gpu_launches": int(launches), "sparse": sparse, "adjoint": adjoint,
            "batched": batched,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()


def main():
    args = parse()
    if args.case is not None:
        if args.case not in CASES:
            raise SystemExit(f"unknown case {args.case!r}; one of {sorted(CASES)}")
        CASES[args.case](args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
