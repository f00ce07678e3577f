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


CASES = {"mttkrp": case_mttkrp, "cp_als": case_cp_als}


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
    args = ap.parse_args(argv)
    CASES[args.case](args)


if __name__ == "__main__":
    sys.exit(main())
