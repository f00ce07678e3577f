"""Failure paths on the GPU, made without faulting it.

Bounded waits: the tensor-core MTTKRP bounds every mbarrier wait by a clock
budget. The test lowers the budget to one cycle (tsr_ctx_set_wait_budget), so
the first wait of every CTA runs out; the kernel then drains its TMA copies,
waits for its issued MMAs, frees its tensor memory and returns, and the call
fails with TSR_E_TIMEOUT. With the default budget restored the same context
computes the right answer again.

Non-finite input: a NaN or Inf in the tensor reaches the Gram matrices, the
FP64 inverse finds no finite positive pivot even after the ridge retry of
solve_least_squares (cp/helpers.rs:477-490), and cp_als fails with
TSR_E_NOT_SPD (tenrso's CpError::LinalgError). The MTTKRP itself propagates
a NaN only into the output rows that the entry contributes to."""
import numpy as np
import pytest

import tenrso_b200 as tb
from tenrso_b200 import synth

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b)


def c1():
    X, _ = synth.dense_lowrank((64, 64, 64), 8, seed=0xC1, dist="normal", noise=0.01)
    return X, synth.init_factors(X.shape, 8, 0xC1)


def test_mttkrp_wait_timeout_then_recovery(orc):
    X, init = c1()
    ctx = tb.Context(0)
    ctx.set_wait_budget(1)
    for mode in range(3):
        with pytest.raises(tb.TenrsoError) as e:
            tb.mttkrp(X, init, mode, precision="bf16x3", ctx=ctx)
        assert e.value.code == "TSR_E_TIMEOUT", e.value
    ctx.set_wait_budget(0)
    for mode in range(3):
        out = tb.mttkrp(X, init, mode, precision="bf16x3", ctx=ctx)
        ref = orc.mttkrp(X.astype(np.float64), [f.astype(np.float64) for f in init], mode)
        assert rel_err(out, ref) <= 1e-4
    ctx.close()


def test_cp_als_wait_timeout_then_recovery(orc):
    X, init = c1()
    ctx = tb.Context(0)
    ctx.set_wait_budget(1)
    with pytest.raises(tb.TenrsoError) as e:
        tb.cp_als(X, 8, 5, 0.0, init=init, precision="bf16x3", ctx=ctx)
    assert e.value.code == "TSR_E_TIMEOUT", e.value
    ctx.set_wait_budget(0)
    _, info = orc.cp_als(X.astype(np.float64), 8, 5, 0.0, [f.astype(np.float64) for f in init])
    res = tb.cp_als(X, 8, 5, 0.0, init=init, precision="bf16x3", ctx=ctx)
    assert abs(res.fit - info["fit"]) <= 1e-4
    ctx.close()


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_cp_als_non_finite_input_is_a_linalg_error(bad, precision):
    X, init = c1()
    X = X.copy()
    X[3, 4, 5] = bad
    with pytest.raises(tb.TenrsoError) as e:
        tb.cp_als(X, 8, 4, 0.0, init=init, precision=precision)
    assert e.value.code == "TSR_E_NOT_SPD", e.value
    # the context is still usable afterwards
    res = tb.cp_als(c1()[0], 8, 2, 0.0, init=init, precision=precision)
    assert np.isfinite(res.fit)


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_mttkrp_nan_reaches_only_its_rows(orc, precision):
    X, init = c1()
    X = X.copy()
    X[3, 4, 5] = np.nan
    Xc = X.copy()
    Xc[3, 4, 5] = 0.0
    f64 = [f.astype(np.float64) for f in init]
    for mode, row in ((0, 3), (1, 4), (2, 5)):
        out = tb.mttkrp(X, init, mode, precision=precision)
        assert np.isnan(out[row]).all()
        keep = np.ones(out.shape[0], bool)
        keep[row] = False
        assert np.isfinite(out[keep]).all()
        ref = orc.mttkrp(Xc.astype(np.float64), f64, mode)
        assert rel_err(out[keep], ref[keep]) <= (1e-5 if precision == "fp32" else 1e-4)
