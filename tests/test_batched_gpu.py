"""Batched CP-ALS on the GPU against the oracle: every instance's fit after
the same iterations from the same injected factors within 1e-4 of the FP64
restatement of tenrso's cp_als (identical iteration counts and stop reasons),
the same results for every launch configuration, and the autotuner's JSON
cache."""
import json

import numpy as np
import pytest

import tenrso_b200 as tb
from tenrso_b200 import synth

pytestmark = pytest.mark.gpu


def small_batch(count=24, seed=0xC4):
    inst = synth.batched_instances(count, seed, nmin=5, nmax=40, rmin=1, rmax=16)
    tensors, ranks, inits = [], [], []
    for X, R, init in inst:
        R = max(1, min(R, min(X.shape) - 1))  # well-conditioned Grams
        tensors.append(X.astype(np.float32))
        ranks.append(R)
        inits.append([f[:, :R] for f in init])
    return tensors, ranks, inits


@pytest.fixture(scope="module")
def batch():
    tensors, ranks, inits = small_batch()
    return tensors, ranks, inits


def test_batched_fits_match_oracle(orc, batch):
    tensors, ranks, inits = batch
    b = tb.BatchedCpAls(tensors, ranks)
    res = b.cp_als(12, 0.0, init=inits)
    for X, R, init, r in zip(tensors, ranks, inits, res):
        _, info = orc.cp_als(X.astype(np.float64), R, 12, 0.0,
                             [f.astype(np.float64) for f in init])
        assert r.iters == info["iters"] == 12
        assert abs(r.fit - info["fit"]) <= 1e-4, (X.shape, R, r.fit, info["fit"])
        assert [f.shape for f in r.factors] == [(n, R) for n in X.shape]
    b.close()


def test_batched_convergence_rules_match_oracle(orc, batch):
    """tol > 0: per-instance early stops (FitTolerance) at the oracle's iteration."""
    tensors, ranks, inits = batch
    b = tb.BatchedCpAls(tensors, ranks)
    res = b.cp_als(30, 1e-4, init=inits)
    agree = 0
    for X, R, init, r in zip(tensors, ranks, inits, res):
        _, info = orc.cp_als(X.astype(np.float64), R, 30, 1e-4,
                             [f.astype(np.float64) for f in init])
        assert abs(r.fit - info["fit"]) <= 1e-4
        agree += (r.iters == info["iters"]) and (r.convergence.reason == info["reason"])
    # fp32 sums may move a stop that sits right at the tolerance by one sweep
    assert agree >= len(tensors) - 2
    b.close()


@pytest.mark.parametrize("threads,spl,cps", [(128, 0, 4), (256, 1, 2), (512, 0, 1),
                                             (256, 5, 1)])
def test_launch_configs_agree(batch, threads, spl, cps):
    tensors, ranks, inits = batch
    b = tb.BatchedCpAls(tensors, ranks)
    ref = b.cp_als(10, 0.0, init=inits)
    b.set_config(threads, spl, cps)
    assert b.config == {"threads": threads, "sweeps_per_launch": spl, "ctas_per_sm": cps}
    res = b.cp_als(10, 0.0, init=inits)
    for a, c in zip(ref, res):
        assert abs(a.fit - c.fit) <= 1e-5
        assert a.iters == c.iters
    b.close()


def test_autotune_cache(tmp_path, batch):
    import torch
    tensors, ranks, inits = batch
    b = tb.BatchedCpAls(tensors, ranks)
    d_init = torch.from_numpy(b.pack(inits)).cuda()
    torch.cuda.synchronize()
    path = tmp_path / "tune.json"
    cfg, cached = b.autotune(5, d_init.data_ptr(), path)
    assert not cached
    data = json.loads(path.read_text())
    assert len(data) == 1
    entry = next(iter(data.values()))
    assert entry["threads"] == cfg["threads"]
    b.set_config(128, 1, 1)
    cfg2, cached2 = b.autotune(5, d_init.data_ptr(), path)
    assert cached2 and cfg2 == cfg
    b.close()


def test_device_run_and_random_init():
    import torch
    tensors, ranks, inits = small_batch(8, seed=3)
    b = tb.BatchedCpAls(tensors, ranks)
    d_init = torch.from_numpy(b.pack(inits)).cuda()
    d_out = torch.empty_like(d_init)
    torch.cuda.synchronize()
    info = b.cp_als_dev(6, 0.0, d_init.data_ptr(), d_out.data_ptr(), want_info=True)
    host = b.cp_als(6, 0.0, init=inits)
    for (fit, iters, _), h in zip(info, host):
        assert iters == 6 and abs(fit - h.fit) <= 1e-5
    r1 = b.cp_als(3, 0.0, init="random", seed=9)
    r2 = b.cp_als(3, 0.0, init="random", seed=9)
    assert [x.fit for x in r1] == pytest.approx([x.fit for x in r2], abs=1e-6)
    b.close()


def test_c4_shape_batch_vs_dense_path():
    """A slice of the 512-instance workload (16..96 sizes, ranks 4..16): each
    instance's fit after 25 iterations equals the single-instance FP32 GPU
    cp_als within 1e-4."""
    inst = synth.batched_instances(16, 0xC4)
    tensors = [X.astype(np.float32) for X, _, _ in inst]
    ranks = [R for _, R, _ in inst]
    inits = [init for _, _, init in inst]
    b = tb.BatchedCpAls(tensors, ranks)
    res = b.cp_als(25, 0.0, init=inits)
    for X, R, init, r in zip(tensors, ranks, inits, res):
        d = tb.cp_als(X, R, 25, 0.0, init=init, precision="fp32")
        assert abs(r.fit - d.fit) <= 1e-4, (X.shape, R, r.fit, d.fit)
    b.close()


def test_c4_instances_vs_fp64_oracle(orc):
    """The first 48 instances of the 512-instance workload itself (seed 0xC4:
    sizes U{16..96}, ranks U{4..16}, low-rank N(0,1) + 1% noise), batched in
    one run of 25 iterations, against the FP64 oracle's cp_als
    (cp/core.rs:59-182) from the same injected init.

    Some instances are still leaving an ALS swamp at iteration 25, where the
    trajectory itself is unstable: perturbing the init by 1e-7 relative (the
    scale of FP32 rounding) moves the FP64 oracle's own 25-iteration fit by up
    to ~3e-4. Each instance is therefore held to max(1e-4, 3x that measured
    sensitivity), and at least 90% of the instances to 1e-4 outright. Near
    convergence the reference's oscillation rule (a fit lower than the last,
    more than 5 times after iteration 10) can also fire one sweep apart on
    either side, so the stopping iteration must agree only when neither run
    stopped for oscillation."""
    inst = synth.batched_instances(512, 0xC4)[:48]
    tensors = [X.astype(np.float32) for X, _, _ in inst]
    ranks = [R for _, R, _ in inst]
    inits = [init for _, _, init in inst]
    b = tb.BatchedCpAls(tensors, ranks)
    res = b.cp_als(25, 0.0, init=inits)
    rng = np.random.default_rng(0xC4)
    within, worst = 0, 0.0
    for X, R, init, r in zip(tensors, ranks, inits, res):
        f64 = [f.astype(np.float64) for f in init]
        _, info = orc.cp_als(X.astype(np.float64), R, 25, 0.0, f64)
        pert = [f * (1 + 1e-7 * rng.standard_normal(f.shape)) for f in f64]
        _, info_p = orc.cp_als(X.astype(np.float64), R, 25, 0.0, pert)
        if "Oscillation" not in (r.convergence.reason, info["reason"]):
            assert r.iters == info["iters"] == 25, (X.shape, R, r.iters, info["iters"])
        err = abs(r.fit - info["fit"])
        tol = max(1e-4, 3.0 * abs(info_p["fit"] - info["fit"]))
        assert err <= tol, (X.shape, R, r.fit, info["fit"], tol)
        within += err <= 1e-4
        worst = max(worst, err)
    assert within >= 0.9 * len(inst), (within, len(inst))
    print(f"C4 instances: {within}/{len(inst)} within 1e-4 of the fp64 oracle, worst {worst:.2e}")
    b.close()
