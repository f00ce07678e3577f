"""InitStrategy (crates/tenrso-decomp/src/cp/types.rs:39-59) through
initialize_factors (cp/helpers.rs:192-377): the device against the FP64
oracle restatement (oracle.initialize_factors, numpy's thin SVD with the same
column orientation) and cp_als from each strategy against the oracle's cp_als
from the oracle's factors.

Tolerances: Random and RandomNormal factors are the same seeded draws (fp32
rounding of the same doubles; RandomNormal within 1e-6 relative, the host
libm and numpy may differ in the last bit). SVD-based factors within 1e-5 of
the oracle's per column (relative to the column norm) on tensors whose
leading singular values are well separated: the device forms u_r as an
eigenvector of the FP64 Gram X_(n) X_(n)^T, whose accuracy goes with the
eigenvalue gaps."""
import numpy as np
import pytest

import tenrso_b200 as tb
from tenrso_b200 import synth

STRATS = ["random", "random_normal", "svd", "nnsvd", "leverage_score"]


def decaying(shape, R, seed):
    """sum_r 2^-r/2 a_r o b_r o c_r (N(0,1) factors) + 1e-3 relative noise:
    distinct leading singular values in every unfolding."""
    fs = [synth.normal(seed, 100 + m, (n, R)) for m, n in enumerate(shape)]
    fs[0] = fs[0] * (2.0 ** (-0.5 * np.arange(R)))[None, :]
    kr = fs[1]
    for f in fs[2:]:
        kr = (kr[:, None, :] * f[None, :, :]).reshape(-1, R)
    X = (fs[0] @ kr.T).reshape(shape)
    X += 1e-3 * np.linalg.norm(X) / np.sqrt(X.size) * synth.normal(seed, 9, shape)
    return X.astype(np.float32)


def test_oracle_strategy_properties(orc):
    X = decaying((12, 10, 8), 4, 3).astype(np.float64)
    Fs = orc.initialize_factors(X, 5, "svd", 7)
    for F, n in zip(Fs, X.shape):
        k = min(5, n, X.size // n)
        assert np.allclose(F[:, :k].T @ F[:, :k], np.eye(k), atol=1e-12)
        i = np.argmax(np.abs(F[:, :k]), axis=0)
        assert np.all(F[i, np.arange(k)] > 0)
    assert all(np.all(F >= 0) for F in orc.initialize_factors(X, 5, "nnsvd", 7))
    r = orc.initialize_factors(X, 3, "random", 11)
    assert np.array_equal(r[1], synth.uniform(11, 201, (10, 3)))
    g = orc.initialize_factors(X, 3, "random_normal", 11)
    assert np.array_equal(g[2], synth.normal(11, 402, (8, 3)))
    # more components than the unfolding's rank: N(0, 0.01) padding
    small = decaying((3, 4, 5), 2, 5).astype(np.float64)
    F0 = orc.initialize_factors(small, 4, "svd", 2)[0]
    assert np.allclose(F0[:, 3], synth.normal(2, 500, (3, 1))[:, 0] * 0.01)


@pytest.mark.gpu
@pytest.mark.parametrize("strategy", STRATS)
@pytest.mark.parametrize("shape,R", [((64, 64, 64), 8), ((30, 24, 20, 16), 6),
                                     ((3, 40, 5), 4), ((128, 96, 64), 10)])
def test_device_factors_vs_oracle(orc, strategy, shape, R):
    X = decaying(shape, R, 0xC1)
    got = tb.initialize_factors(X, R, strategy, seed=0xC1)
    ref = orc.initialize_factors(X.astype(np.float64), R, strategy, 0xC1)
    for m, (g, r) in enumerate(zip(got, ref)):
        assert g.shape == r.shape == (shape[m], R)
        if strategy == "random":
            assert np.array_equal(g, r.astype(np.float32))
            continue
        tol = 1e-6 if strategy == "random_normal" else 1e-5
        scale = np.maximum(np.linalg.norm(r, axis=0), 1e-30)
        err = np.abs(g - r).max(axis=0) / scale
        assert err.max() <= tol, (strategy, m, err)


@pytest.mark.gpu
@pytest.mark.parametrize("strategy", ["svd", "nnsvd", "leverage_score", "random_normal"])
def test_cp_als_from_strategy_vs_oracle(orc, strategy):
    shape, R = (64, 64, 64), 8
    X = decaying(shape, R, 0xC1)
    res = tb.cp_als(X, R, 10, 0.0, init=strategy, seed=0xC1)
    init = orc.initialize_factors(X.astype(np.float64), R, strategy, 0xC1)
    _, info = orc.cp_als(X.astype(np.float64), R, 10, 0.0, init)
    assert res.iters == info["iters"] == 10
    assert abs(res.fit - info["fit"]) <= 1e-4, (strategy, res.fit, info["fit"])
    acc = tb.cp_als_accelerated(X, R, 6, 1e-9, init=strategy, seed=0xC1)
    assert 0.0 <= acc.fit <= 1.0


@pytest.mark.gpu
def test_init_errors():
    X = decaying((8, 8, 8), 2, 1)
    with pytest.raises(tb.TenrsoError) as e:
        tb.initialize_factors(X, 0, "svd")
    assert e.value.status == 5
    with pytest.raises(ValueError):
        tb.initialize_factors(X, 2, "qr")
    with pytest.raises(tb.TenrsoError) as e:
        tb.initialize_factors(np.zeros((1100, 2, 2), np.float32), 2, "svd")
    assert e.value.status == 14
