"""Writes tests/golden/c2_fp64_fit.json: the FP64 oracle's CP-ALS fit history
on the dense 256x256x256 rank-64 workload (seeded rank-64 U(0,1) factors plus
0.5% Gaussian noise, seed 0xC2; init U(0,1) from the same seed; 10
iterations, tol 0), and the oracle's fp32 (fast flavour) history beside it.

The oracle is the C++ restatement of tenrso's cp_als (cp/core.rs:59-182) in
oracle/; this script only runs it and records its output, so GPU tests and
bench.py can compare against the FP64 fit without a ten-second CPU run.

    python tests/golden/make_c2_fit.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SHAPE, RANK, ITERS, SEED = (256, 256, 256), 64, 10, 0xC2


def compute():
    from oracle import oracle
    from tenrso_b200 import synth
    X, _ = synth.dense_lowrank(SHAPE, RANK, seed=SEED, dist="uniform", noise=0.005)
    init = synth.init_factors(SHAPE, RANK, SEED)
    _, i64 = oracle.cp_als(X.astype(np.float64), RANK, ITERS, 0.0,
                           [f.astype(np.float64) for f in init])
    _, i32 = oracle.cp_als(X, RANK, ITERS, 0.0, init)
    return {
        "workload": "dense CP-ALS 256x256x256 rank 64, 10 iterations, tol 0",
        "generator": "tenrso_b200.synth.dense_lowrank(uniform, noise 0.005, seed 0xC2); "
                     "init tenrso_b200.synth.init_factors(seed 0xC2)",
        "fp64_fit": i64["fit"], "fp64_fit_history": [float(v) for v in i64["fit_history"]],
        "fp32_fit": i32["fit"], "fp32_fit_history": [float(v) for v in i32["fit_history"]],
    }


if __name__ == "__main__":
    out = compute()
    with open(os.path.join(HERE, "c2_fp64_fit.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(json.dumps(out, indent=1))
