"""Dense MTTKRP / Khatri-Rao / CP-ALS on the GPU, through the C ABI, against
the oracle (FP64 restatement of tenrso's CPU code) on the same seeded inputs.

Tolerances (stated per test):
  FP32 MTTKRP          relative Frobenius error <= 1e-5 vs FP64 oracle
  BF16X3 MTTKRP        relative Frobenius error <= 1e-4 vs FP64 oracle
  CP-ALS fit           |fit - fit_oracle_fp64| <= 1e-4 after the same iterations
"""
import numpy as np
import pytest

import tenrso_b200 as tb
from tenrso_b200 import synth

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def rand_problem(shape, R, seed, dist="normal"):
    rng = np.random.default_rng(seed)
    if dist == "normal":
        X = rng.standard_normal(shape).astype(np.float32)
        fs = [rng.standard_normal((n, R)).astype(np.float32) for n in shape]
    else:
        X = rng.random(shape).astype(np.float32)
        fs = [rng.random((n, R)).astype(np.float32) for n in shape]
    return X, fs


def test_khatri_rao_golden(kats):
    for case in kats["khatri_rao"]:
        c = tb.khatri_rao(np.array(case["a"], np.float32), np.array(case["b"], np.float32))
        if "c" in case:
            assert np.array_equal(c, np.array(case["c"], np.float32)), case["src"]
        else:
            assert np.array_equal(c[:, 0], np.array(case["c_col0"], np.float32)), case["src"]


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_mttkrp_golden(kats, orc, precision):
    case = kats["mttkrp"][0]
    X = np.array(case["tensor"], np.float32).reshape(case["shape"])
    fs = [np.array(f, np.float32) for f in case["factors"]]
    out = tb.mttkrp(X, fs, case["mode"], precision=precision)
    # small integers and halves are exact in bf16: exact result on both paths
    assert np.array_equal(out, np.array(case["expected"], np.float32))
    for mode in range(3):
        ref = orc.mttkrp(X.astype(np.float64), [f.astype(np.float64) for f in fs], mode)
        assert np.array_equal(tb.mttkrp(X, fs, mode, precision=precision), ref.astype(np.float32))


SHAPES = [
    ((17, 33, 9), 5),
    ((64, 64, 64), 8),
    ((3, 5, 7, 11), 3),
    ((2, 3), 1),
    ((1, 40, 7), 1),
    ((129, 70, 31), 20),
    ((200, 16, 12), 64),
    ((33, 41, 18), 100),
    ((8, 9, 10, 3, 4), 6),
]


@pytest.mark.parametrize("shape,R", SHAPES)
@pytest.mark.parametrize("precision,tol", [("fp32", 1e-5), ("bf16x3", 1e-4)])
def test_mttkrp_parity(orc, shape, R, precision, tol):
    X, fs = rand_problem(shape, R, seed=hash((shape, R)) & 0xFFFF, dist="uniform")
    X64 = X.astype(np.float64)
    f64 = [f.astype(np.float64) for f in fs]
    for mode in range(len(shape)):
        out = tb.mttkrp(X, fs, mode, precision=precision)
        ref = orc.mttkrp(X64, f64, mode)
        e = rel_err(out, ref)
        assert e <= tol, (shape, R, mode, precision, e)


# Shapes whose fastest other mode is a multiple of 8 (at most 384 once padded
# to 64) take the tensor-core path that scales U_last per run of KR rows;
# these cover run lengths 8..384 (whole and zero-padded 64-wide k-blocks),
# ranks that are not multiples of 16, partial 128-row tiles, 4-way run weights
# and up to 16 runs per CTA.
RUN_SHAPES = [
    ((130, 5, 192), 40),
    ((70, 6, 4, 128), 17),
    ((40, 7, 384), 64),
    ((300, 64, 64), 16),
    ((128, 1024, 64), 8),
    ((33, 2, 3, 64), 1),
    ((70, 6, 48), 17),
    ((16, 12, 8, 48), 32),
    ((50, 9, 104), 20),
    ((24, 40, 8), 5),
]


@pytest.mark.parametrize("shape,R", RUN_SHAPES)
def test_mttkrp_run_scaled_path(orc, shape, R):
    X, fs = rand_problem(shape, R, seed=hash((shape, R)) & 0xFFFF, dist="normal")
    X64 = X.astype(np.float64)
    f64 = [f.astype(np.float64) for f in fs]
    for mode in range(len(shape)):
        out = tb.mttkrp(X, fs, mode, precision="bf16x3")
        ref = orc.mttkrp(X64, f64, mode)
        e = rel_err(out, ref)
        assert e <= 1e-4, (shape, R, mode, e)


# 3-way tensors whose last mode is a multiple of 8 (middle and last modes at
# most 384) take the single-layout tensor-core path: one bf16 hi/lo copy of X
# read by every mode (modes 0 and 1 K-major, mode 2 MN-major), the contracted
# factor as a prebuilt B image. These cover partial 128-row tiles in every
# mode (mode 2's rows are the last mode: 136 ends inside a second 64-wide
# box, 40 inside the first), contracted lengths that are not multiples of 64
# (zero-filled boxes), middle modes that are not multiples of 8, ranks 1-64
# (n_pad 32 and 64), single runs and the largest supported L.
SINGLE_LAYOUT_SHAPES = [
    ((37, 50, 72), 33),
    ((5, 300, 16), 64),
    ((129, 128, 136), 48),
    ((64, 384, 384), 64),
    ((20, 13, 40), 7),
    ((1, 1, 8), 1),
    ((300, 3, 24), 32),
    ((17, 260, 200), 31),
]


@pytest.mark.parametrize("shape,R", SINGLE_LAYOUT_SHAPES)
def test_mttkrp_single_layout_path(orc, shape, R):
    X, fs = rand_problem(shape, R, seed=hash((shape, R)) & 0xFFFF, dist="normal")
    X64 = X.astype(np.float64)
    f64 = [f.astype(np.float64) for f in fs]
    for mode in range(3):
        out = tb.mttkrp(X, fs, mode, precision="bf16x3")
        ref = orc.mttkrp(X64, f64, mode)
        e = rel_err(out, ref)
        assert e <= 1e-4, (shape, R, mode, e)


@pytest.mark.parametrize("precision,tol", [("fp32", 1e-5), ("bf16x3", 1e-4)])
def test_mttkrp_signed_data(orc, precision, tol):
    X, fs = rand_problem((48, 40, 36), 16, seed=3, dist="normal")
    for mode in range(3):
        out = tb.mttkrp(X, fs, mode, precision=precision)
        ref = orc.mttkrp(X.astype(np.float64), [f.astype(np.float64) for f in fs], mode)
        assert rel_err(out, ref) <= tol


def test_mttkrp_c2_size(orc):
    """256^3 rank 64 (the CP-ALS benchmark tensor) on every mode, both paths."""
    X, fs = synth.dense_lowrank((256, 256, 256), 64, seed=0xC2, dist="uniform", noise=0.005)
    init = synth.init_factors(X.shape, 64, 0xC2)
    X64 = X.astype(np.float64)
    f64 = [f.astype(np.float64) for f in init]
    for mode in range(3):
        ref = orc.mttkrp(X64, f64, mode)
        e32 = rel_err(tb.mttkrp(X, init, mode, precision="fp32"), ref)
        e16 = rel_err(tb.mttkrp(X, init, mode, precision="bf16x3"), ref)
        assert e32 <= 1e-5, (mode, e32)
        assert e16 <= 1e-4, (mode, e16)


def test_mttkrp_strided_view(orc):
    X, fs = rand_problem((20, 30, 40), 7, seed=5)
    Xt = np.transpose(X, (2, 0, 1))  # non-standard strides
    fst = [fs[2], fs[0], fs[1]]
    for mode in range(3):
        out = tb.mttkrp(Xt, fst, mode)
        ref = orc.mttkrp(np.ascontiguousarray(Xt).astype(np.float64),
                         [f.astype(np.float64) for f in fst], mode)
        assert rel_err(out, ref) <= 1e-5


def test_mttkrp_variants_and_all_modes(orc):
    X, fs = rand_problem((12, 14, 16), 4, seed=9)
    base = [tb.mttkrp(X, fs, m) for m in range(3)]
    allm = tb.mttkrp_all_modes(X, fs)
    for m in range(3):
        assert np.array_equal(allm[m], base[m])
        assert np.array_equal(tb.mttkrp_blocked(X, fs, m, 16), base[m])
        assert np.array_equal(tb.mttkrp_fused(X, fs, m), base[m])


def _c1():
    X, _ = synth.dense_lowrank((64, 64, 64), 8, seed=0xC1, dist="normal", noise=0.01)
    init = synth.init_factors(X.shape, 8, 0xC1)
    return X, init


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_cp_als_c1_fit_parity(orc, precision):
    X, init = _c1()
    ref64, info64 = orc.cp_als(X.astype(np.float64), 8, 10, 0.0,
                               [f.astype(np.float64) for f in init])
    res = tb.cp_als(X, 8, 10, 0.0, init=init, precision=precision)
    assert res.iters == 10 == info64["iters"]
    assert res.convergence.reason == "MaxIterations"
    assert abs(res.fit - info64["fit"]) <= 1e-4, (res.fit, info64["fit"])
    # mid-trajectory fits move fast (0.64 -> 0.92 in two sweeps), so a 1e-5
    # perturbation shifts them more than the converged end point
    assert np.max(np.abs(res.convergence.fit_history - info64["fit_history"])) <= 1e-3
    assert res.weights is None
    assert [f.shape for f in res.factors] == [(64, 8)] * 3


def test_cp_als_c1_vs_f32_reference(orc):
    """Against the restated f32 instantiation (the reference's own T=f32 path):
    its factors, with their fit evaluated in FP64, match ours within 1e-4.
    (Its self-reported f32 fit is not comparable: the sequential f32 sum of
    squares in compute_norm_squared, helpers.rs:498-510, and the cancellation in
    ||X||^2 + ||Xhat||^2 - 2<X,Xhat> (helpers.rs:524) move it by ~6e-3 here.)"""
    X, init = _c1()
    f32_factors, _ = orc.cp_als(X, 8, 10, 0.0, init, faithful=True)
    Xh = orc.cp_reconstruct(f32_factors)
    X64 = X.astype(np.float64)
    fit_ref = 1.0 - np.linalg.norm(X64 - Xh) / np.linalg.norm(X64)
    res = tb.cp_als(X, 8, 10, 0.0, init=init)
    assert abs(res.fit - fit_ref) <= 1e-4, (res.fit, fit_ref)


# 3-way shapes whose middle and last sizes are multiples of 8 build every
# unfolding (and ||X||^2) in one fused pass; these cover partial 32-wide j
# tiles, partial 64-wide k tiles and odd first modes.
@pytest.mark.parametrize("shape,R", [((37, 24, 40), 5), ((5, 8, 72), 3), ((70, 136, 16), 7)])
@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_cp_als_fused_unfold_shapes(orc, shape, R, precision):
    X, _ = synth.dense_lowrank(shape, R, seed=0xF0 + R, dist="normal", noise=0.01)
    init = synth.init_factors(shape, R, 0xF0 + R)
    _, info = orc.cp_als(X.astype(np.float64), R, 6, 0.0, [f.astype(np.float64) for f in init])
    res = tb.cp_als(X, R, 6, 0.0, init=init, precision=precision)
    assert res.iters == 6
    assert abs(res.fit - info["fit"]) <= 1e-4, (shape, precision, res.fit, info["fit"])


def test_cp_als_tolerance_stop(orc):
    X, init = _c1()
    _, info = orc.cp_als(X.astype(np.float64), 8, 50, 1e-3,
                         [f.astype(np.float64) for f in init])
    res = tb.cp_als(X, 8, 50, 1e-3, init=init)
    assert info["reason"] == "FitTolerance"
    assert res.convergence.reason == "FitTolerance"
    assert abs(res.iters - info["iters"]) <= 1
    assert res.convergence.final_fit_change < 1e-3


def test_cp_als_time_limit_zero():
    X, init = _c1()
    res = tb.cp_als(X, 8, 10, 0.0, init=init, time_limit=0.0)
    assert res.convergence.reason == "TimeLimit"
    assert res.iters == 0


def test_cp_als_seeded_random_init_matches_synth():
    X, init = _c1()
    a = tb.cp_als(X, 8, 3, 0.0, init="random", seed=0xC1)
    b = tb.cp_als(X, 8, 3, 0.0, init=init)
    # same initial factors; FP64 atomics in the Gram sums may reorder additions
    assert abs(a.fit - b.fit) <= 1e-12
    for fa, fb in zip(a.factors, b.factors):
        assert np.allclose(fa, fb, rtol=1e-5, atol=1e-6)


def test_cp_als_4way(orc):
    X, _ = synth.dense_lowrank((16, 12, 10, 8), 4, seed=0xC5, dist="normal", noise=0.01)
    init = synth.init_factors(X.shape, 4, 0xC5)
    _, info = orc.cp_als(X.astype(np.float64), 4, 8, 0.0, [f.astype(np.float64) for f in init])
    for precision in ("fp32", "bf16x3"):
        res = tb.cp_als(X, 4, 8, 0.0, init=init, precision=precision)
        assert abs(res.fit - info["fit"]) <= 1e-4


def test_cp_als_rank_deficient_ridge(orc):
    """A rank-1 tensor decomposed at rank 3 from duplicated initial columns:
    the Gram is singular and the ridge fallback (cp/helpers.rs:477-490) runs."""
    a = np.ones(4, dtype=np.float32)  # exact arithmetic: the pivot is exactly 0
    X = np.einsum("i,j,k->ijk", a, a, a).astype(np.float32)
    init = [np.tile(a[:, None], (1, 3)).astype(np.float32) for _ in range(3)]
    try:
        res = tb.cp_als(X, 3, 2, 0.0, init=init)
    except tb.TenrsoError as e:
        assert e.code == "TSR_E_NOT_SPD"
    else:
        assert res.ridge_used
