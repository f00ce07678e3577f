"""Small standalone cases of the hot-path kernels, for profiling with ncu and
for quick timing. Each case prepares its inputs on the device, runs a few
warm-up launches and then the measured ones.

    python -m tenrso_b200.profile_cases mttkrp --precision bf16x3 --mode 0
    python -m tenrso_b200.profile_cases cp_als --precision fp32 --iters 2
"""
from __future__ import annotations

import argparse
import sys

import numpy as np


def _ctx():
    import torch

    import tenrso_b200 as tb
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    return tb.Context(0, stream=stream.cuda_stream)


def case_mttkrp(args):
    import torch

    import tenrso_b200 as tb
    ctx = _ctx()
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
    ctx = _ctx()
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
    ctx = _ctx()
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
    ctx = _ctx()
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
    ctx = _ctx()
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


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--precision", default="bf16x3")
    ap.add_argument("--shape", type=int, nargs="+", default=[256, 256, 256])
    ap.add_argument("--rank", type=int, default=64)
    ap.add_argument("--mode", type=int, default=0)
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--launches", type=int, default=1)
    ap.add_argument("--nnz", type=int, default=20_000_000)
    ap.add_argument("--time", action="store_true", help="also print the kernel time")
    args = ap.parse_args(argv)
    CASES[args.case](args)


if __name__ == "__main__":
    sys.exit(main())
