"""cp_als_constrained (crates/tenrso-decomp/src/cp/core.rs:225-400): host-side
validation in tenrso's order and wording (CPU), and GPU runs against the FP64
restatement in the oracle (fit within 1e-4 after the same iterations from the
same injected factors)."""
import numpy as np
import pytest

import tenrso_b200 as tb
from tenrso_b200 import synth

CC = tb.CpConstraints
RT = tb.RegularizationType


def test_regularization_components_and_validation():
    assert CC.l2_regularized(0.3).effective_l2() == 0.3
    assert CC.l1_regularized(0.2).effective_l1() == 0.2
    en = CC.elastic_net(1.0, 0.25)
    assert (en.effective_l2(), en.effective_l1()) == (0.75, 0.25)
    assert CC.tikhonov(0.5, 0).effective_l2() == 0.5
    assert CC.tikhonov(0.5, 1).effective_l2() == 0.0
    assert CC(l2_reg=0.4).effective_l2() == 0.4  # legacy field when regularization is None
    assert CC(l2_reg=0.4, regularization=RT.l1(0.1)).effective_l2() == 0.0  # overridden
    for c, msg in ((CC.l2_regularized(-1.0), "L2 lambda must be >= 0, got -1"),
                   (CC.l1_regularized(-0.5), "L1 lambda must be >= 0, got -0.5"),
                   (CC.elastic_net(1.0, 1.5), "ElasticNet alpha must be in \\[0, 1\\], got 1.5"),
                   (CC.tikhonov(-2.0, 1), "Tikhonov lambda must be >= 0, got -2")):
        with pytest.raises(tb.TenrsoError, match="Invalid regularization parameter: " + msg) as e:
            tb.cp_als_constrained(np.ones((4, 4, 4)), 2, 1, 0.0, constraints=c)
        assert e.value.status == 19


@pytest.mark.parametrize("rank,tol,c,status,msg", [
    (0, 0.0, CC(), 5, "Invalid rank: 0"),
    (5, 0.0, CC(), 5, "Invalid rank: 5"),
    (2, 1.0, CC(), 6, "Invalid tolerance: 1"),
    (2, 0.0, CC(l2_reg=-0.5), 6, "Invalid tolerance: -0.5"),
])
def test_validation_order_without_device(rank, tol, c, status, msg):
    with pytest.raises(tb.TenrsoError, match=msg) as e:
        tb.cp_als_constrained(np.ones((4, 4, 4)), rank, 3, tol, constraints=c)
    assert e.value.status == status


def test_oracle_tikhonov_penalty_and_qr(orc):
    """apply_tikhonov_to_gram (helpers.rs:630-700) as matrices, and the
    orthonormalization's sign convention."""
    assert not orc.tikhonov_penalty(1, 1).any()
    D1 = np.diff(np.eye(4), axis=0)
    assert np.array_equal(orc.tikhonov_penalty(4, 1), D1.T @ D1)
    P = orc.tikhonov_penalty(6, 2)
    assert np.diag(P).tolist() == [1, 5, 6, 6, 5, 1]
    assert np.diag(P, 1).tolist() == [-2, -4, -4, -4, -2] and np.diag(P, 2).tolist() == [1] * 4
    assert np.array_equal(orc.tikhonov_penalty(2, 2), np.eye(2))
    F = np.random.default_rng(0).standard_normal((9, 3))
    Q = orc.orthonormalize(F)
    assert np.allclose(Q.T @ Q, np.eye(3)) and np.all(np.diag(Q.T @ F) > 0)


def test_oracle_without_constraints_is_cp_als(orc):
    X, _ = synth.dense_lowrank((20, 16, 12), 3, seed=5, dist="uniform", noise=0.01)
    init = [f.astype(np.float64) for f in synth.init_factors(X.shape, 3, 5)]
    U, info = orc.cp_als_constrained(X, 3, 10, 0.0, init)
    V, ref = orc.cp_als(X.astype(np.float64), 3, 10, 0.0, init)
    assert abs(info["fit"] - ref["fit"]) < 1e-12
    for a, b in zip(U, V):
        assert np.allclose(a, b, rtol=1e-9, atol=1e-12)


def _case(shape, rank, seed, dist):
    X, _ = synth.dense_lowrank(shape, rank, seed=seed, dist=dist, noise=0.01)
    return X, synth.init_factors(shape, rank, seed)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
@pytest.mark.parametrize("name,c,kw", [
    ("nonneg", CC.nonnegative_only(), dict(nonneg=True)),
    ("l2", CC.l2_regularized(0.5), dict(l2=0.5)),
    ("elastic", CC.elastic_net(0.02, 0.5), dict(l2=0.01, l1=0.01)),
    ("nonneg+l2", CC(nonnegative=True, l2_reg=0.25), dict(l2=0.25, nonneg=True)),
    ("orthogonal", CC.orthogonal_only(), dict(orthogonal=True)),
    ("orthogonal+l2", CC(orthogonal=True, l2_reg=0.1), dict(orthogonal=True, l2=0.1)),
    ("tikhonov1", CC.tikhonov(0.3, 1), dict(tikhonov=(0.3, 1))),
    ("tikhonov2", CC.tikhonov(0.05, 2), dict(tikhonov=(0.05, 2))),
])
def test_constrained_fit_vs_oracle(orc, precision, name, c, kw):
    X, init = _case((48, 40, 36), 6, 0xC2, "uniform")
    res = tb.cp_als_constrained(X, 6, 10, 0.0, init=init, constraints=c, precision=precision)
    U, info = orc.cp_als_constrained(X, 6, 10, 0.0, [f.astype(np.float64) for f in init], **kw)
    assert res.iters == info["iters"] == 10
    assert abs(res.fit - info["fit"]) <= 1e-4, (name, precision, res.fit, info["fit"])
    assert np.allclose(res.convergence.fit_history, info["fit_history"], atol=1e-4)
    for a, b in zip(res.factors, U):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 2e-3, name
    if kw.get("nonneg"):
        assert all((f >= 0).all() for f in res.factors)


@pytest.mark.gpu
@pytest.mark.parametrize("R,order", [(1, 1), (2, 2), (3, 2)])
def test_tikhonov_small_rank_rules(orc, R, order):
    """Order 1 adds nothing at rank 1; order 2 falls back to the ridge below
    rank 3 (helpers.rs:649, 695-699)."""
    X, init = _case((12, 10, 9), R, 11, "uniform")
    res = tb.cp_als_constrained(X, R, 6, 0.0, init=init, constraints=CC.tikhonov(0.2, order))
    _, info = orc.cp_als_constrained(X, R, 6, 0.0, [f.astype(np.float64) for f in init],
                                     tikhonov=(0.2, order))
    assert np.allclose(res.convergence.fit_history, info["fit_history"], atol=1e-4)


@pytest.mark.gpu
def test_orthogonal_factors_are_orthonormal():
    X, init = _case((30, 25, 20), 4, 13, "normal")
    res = tb.cp_als_constrained(X, 4, 5, 0.0, init=init, constraints=CC.orthogonal_only())
    for f in res.factors:
        assert np.allclose(f.T @ f, np.eye(4), atol=1e-5)


@pytest.mark.gpu
def test_no_constraints_equals_cp_als():
    """Same kernels and sweep graph; the Grams and the fit are FP64 atomic
    sums across CTAs, so two runs agree to FP64 rounding, not bit for bit."""
    X, init = _case((32, 24, 20), 4, 7, "normal")
    a = tb.cp_als(X, 4, 8, 0.0, init=init)
    b = tb.cp_als_constrained(X, 4, 8, 0.0, init=init, constraints=CC())
    assert a.iters == b.iters == 8
    assert abs(a.fit - b.fit) <= 1e-12
    for x, y in zip(a.factors, b.factors):
        assert np.allclose(x, y, rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_nonneg_input_check():
    X, init = _case((16, 12, 10), 3, 3, "uniform")
    Xn = X.copy()
    Xn[3, 4, 5] = -1e-3
    with pytest.raises(tb.TenrsoError, match="Non-negative constraint violated") as e:
        tb.cp_als_constrained(Xn, 3, 5, 0.0, init=init, constraints=CC.nonnegative_only())
    assert e.value.status == 18
    # with the check off the run projects as usual
    c = CC(nonnegative=True, validate_nonneg_input=False)
    res = tb.cp_als_constrained(Xn, 3, 5, 0.0, init=init, constraints=c)
    assert res.iters == 5 and all((f >= 0).all() for f in res.factors)
    # the plain path still runs after the rejected call
    assert tb.cp_als(X, 3, 5, 0.0, init=init).iters == 5


@pytest.mark.gpu
def test_constrained_dev_and_negative_init(orc):
    import torch
    X, init = _case((40, 30, 20), 5, 11, "uniform")
    init = [f - 0.3 for f in init]  # negative entries: projected before the first sweep
    flat = np.concatenate([f.ravel() for f in init]).astype(np.float32)
    dX = torch.from_numpy(X).cuda()
    di = torch.from_numpy(flat).cuda()
    do = torch.empty_like(di)
    fit, iters, _ = tb.cp_als_constrained_dev(dX.data_ptr(), X.shape, 5, 6, 0.0, di.data_ptr(),
                                              do.data_ptr(), constraints=CC.nonnegative_only())
    _, info = orc.cp_als_constrained(X, 5, 6, 0.0, [f.astype(np.float64) for f in init],
                                     nonneg=True)
    assert iters == 6 and abs(fit - info["fit"]) <= 1e-4
    assert (do.cpu().numpy() >= 0).all()


@pytest.mark.gpu
@pytest.mark.parametrize("rank,precision", [(40, "fp32"), (64, "bf16x3")])
def test_constrained_large_rank_vs_oracle(orc, rank, precision):
    """Ranks above 16 run the multi-block (RB = 3, 4) inverse and solve
    instances, whose diagonal blocks take the ridge."""
    X, init = _case((96, 80, 72), rank, 0xC2 + rank, "uniform")
    c = CC(nonnegative=True, l2_reg=0.5)
    res = tb.cp_als_constrained(X, rank, 6, 0.0, init=init, constraints=c, precision=precision)
    U, info = orc.cp_als_constrained(X, rank, 6, 0.0, [f.astype(np.float64) for f in init],
                                     l2=0.5, nonneg=True)
    assert res.iters == info["iters"] == 6
    assert abs(res.fit - info["fit"]) <= 1e-4, (rank, precision, res.fit, info["fit"])
    assert all((f >= 0).all() for f in res.factors)
    # factors of U(0,1) data at rank 40-64 are less well conditioned than
    # the fit; fp32 rounding in six sweeps moves them by up to about 1e-2
    for a, b in zip(res.factors, U):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 2e-2
