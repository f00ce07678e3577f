"""The f64 instantiation (mttkrp<f64>, cp_als<f64>) against the oracle's
FP64 restatement (the C++ port of mttkrp.rs:74-146 and cp/core.rs:59-182
templated on double), and the reference's own MTTKRP golden vectors.

Tolerances: FP64 on both sides, different summation orders: MTTKRP within
1e-12 relative, CP-ALS fit history within 1e-9 from the same injected
factors with the same iterations and stop reason."""
import numpy as np
import pytest

import tenrso_b200 as tb
from tenrso_b200 import synth

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("shape,R", [((6, 5, 4), 3), ((64, 64, 64), 8), ((256, 256, 256), 64),
                                     ((20, 9, 8, 7), 5), ((30, 40), 6), ((3, 70, 33), 130)])
def test_mttkrp_f64_vs_oracle(orc, shape, R):
    rng = np.random.default_rng(R + len(shape))
    X = rng.standard_normal(shape)
    fs = [rng.standard_normal((n, R)) for n in shape]
    for mode in range(len(shape)):
        got = tb.mttkrp_f64(X, fs, mode)
        ref = orc.mttkrp(X, fs, mode)
        assert got.dtype == np.float64 and got.shape == (shape[mode], R)
        assert _rel(got, ref) <= 1e-12, (mode, _rel(got, ref))


def test_mttkrp_f64_golden(kats):
    for case in kats["mttkrp"]:
        X = np.array(case["tensor"], np.float64).reshape(case["shape"])
        fs = [np.array(f, np.float64) for f in case["factors"]]
        got = tb.mttkrp_f64(X, fs, case["mode"])
        assert np.allclose(got, np.array(case["expected"], np.float64), rtol=0, atol=1e-12)


def test_mttkrp_f64_errors():
    X = np.zeros((4, 5, 6))
    fs = [np.zeros((4, 2)), np.zeros((5, 2)), np.zeros((6, 2))]
    with pytest.raises(tb.TenrsoError, match="Mode 3 out of bounds for tensor with rank 3"):
        tb.mttkrp_f64(X, fs, 3)
    with pytest.raises(tb.TenrsoError, match="Factor matrix 1 has 3 columns, expected 2"):
        tb.mttkrp_f64(X, [fs[0], np.zeros((5, 3)), fs[2]], 0)


@pytest.mark.parametrize("shape,R,tol,iters", [((64, 64, 64), 8, 0.0, 10),
                                               ((256, 256, 256), 64, 0.0, 4),
                                               ((20, 16, 12, 9), 4, 1e-6, 40)])
def test_cp_als_f64_vs_oracle(orc, shape, R, tol, iters):
    X, _ = synth.dense_lowrank(shape, R, seed=0xF6, dist="uniform", noise=0.01,
                               dtype=np.float64)
    init = [synth.uniform(0xF6, 200 + m, (n, R)) for m, n in enumerate(shape)]
    res = tb.cp_als_f64(X, R, iters, tol, init=init)
    U, info = orc.cp_als(X, R, iters, tol, init)
    assert res.iters == info["iters"] and res.convergence.reason == info["reason"]
    assert np.abs(res.convergence.fit_history - info["fit_history"]).max() <= 1e-9
    for a, b in zip(res.factors, U):
        assert a.dtype == np.float64
        assert _rel(a, b) <= 1e-6


def test_cp_als_f64_seeded_random_init_and_validation(orc):
    shape = (12, 10, 8)
    X, _ = synth.dense_lowrank(shape, 3, seed=1, dist="normal", noise=0.01, dtype=np.float64)
    a = tb.cp_als_f64(X, 3, 5, 0.0, seed=9)
    init = [synth.uniform(9, 200 + m, (n, 3)) for m, n in enumerate(shape)]
    _, info = orc.cp_als(X, 3, 5, 0.0, init)
    assert np.abs(a.convergence.fit_history - info["fit_history"]).max() <= 1e-9
    with pytest.raises(tb.TenrsoError, match="Invalid rank: 0"):
        tb.cp_als_f64(X, 0, 5, 0.0)
    with pytest.raises(tb.TenrsoError, match="Invalid tolerance"):
        tb.cp_als_f64(X, 2, 5, 1.0)
