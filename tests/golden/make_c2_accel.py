"""Writes tests/golden/c2_accel_fp64.json: the FP64 oracle's cp_als_accelerated
(cp/advanced.rs:51-213) on the dense 256x256x256 rank-64 workload (seeded
rank-64 U(0,1) factors plus 0.5% Gaussian noise, seed 0xC2; init U(0,1) from
the same seed), 8 iterations, tol 1e-9: the fit history, the line search's
choices per (iteration, mode) and the margin between the best and the
second-best trial fit of each (a choice with a margin near the fp32
evaluation error may differ on the device).

The oracle is the FP64 restatement in oracle/oracle.py; this script only
runs it (about 30 s) and records its output for the GPU tests.

    python tests/golden/make_c2_accel.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SHAPE, RANK, ITERS, TOL, SEED = (256, 256, 256), 64, 8, 1e-9, 0xC2


def compute():
    from oracle import oracle
    from tenrso_b200 import synth
    X, _ = synth.dense_lowrank(SHAPE, RANK, seed=SEED, dist="uniform", noise=0.005)
    init = synth.init_factors(SHAPE, RANK, SEED)
    trace = []
    _, info = oracle.cp_als_accelerated(X.astype(np.float64), RANK, ITERS, TOL,
                                        [f.astype(np.float64) for f in init], trace=trace)
    steps = []
    for it, n, a, fits in trace:
        srt = sorted(fits, reverse=True)
        steps.append({"iter": it, "mode": n, "alpha": a, "fits": [float(v) for v in fits],
                      "margin": float(srt[0] - srt[1])})
    return {
        "workload": "dense cp_als_accelerated 256x256x256 rank 64, 8 iterations, tol 1e-9",
        "generator": "tenrso_b200.synth.dense_lowrank(uniform, noise 0.005, seed 0xC2); "
                     "init tenrso_b200.synth.init_factors(seed 0xC2)",
        "fp64_fit": info["fit"], "fp64_fit_history": [float(v) for v in info["fit_history"]],
        "iters": info["iters"], "reason": info["reason"],
        "oscillation_count": info["oscillation_count"],
        "line_search": steps,
    }


if __name__ == "__main__":
    out = compute()
    with open(os.path.join(HERE, "c2_accel_fp64.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(json.dumps({k: v for k, v in out.items() if k != "line_search"}, indent=1))
    for s in out["line_search"]:
        print(s["iter"], s["mode"], s["alpha"], "%.3e" % s["margin"])
