"""n-mode products and Tucker operators (crates/tenrso-kernels/src/nmode.rs)
on the device against the FP64 oracle restatement (oracle.nmode_product) and
the reference's own tests (nmode.rs:256-330, 620-770).

Tolerance: fp32 products with fp32 accumulation (the reference sums in T):
1e-5 relative (Frobenius) to the FP64 result; the reference's integer-valued
known answers exactly."""
import ctypes as C

import numpy as np
import pytest

import tenrso_b200 as tb
from tenrso_b200 import _lib


def arange(shape):
    return np.arange(int(np.prod(shape)), dtype=np.float64).reshape(shape)


def test_oracle_known_answers(orc):
    """nmode.rs:313-330: [[1,2,3],[4,5,6]] x_0 [[1,0],[0,1],[1,1]]."""
    X = np.array([[1.0, 2, 3], [4, 5, 6]])
    M = np.array([[1.0, 0], [0, 1], [1, 1]])
    assert orc.nmode_product(X, M, 0).tolist() == [[1, 2, 3], [4, 5, 6], [5, 7, 9]]
    T = arange((2, 3, 4))
    assert orc.nmode_product(T, np.eye(3), 1).tolist() == T.tolist()
    assert orc.nmode_product(T, np.ones((5, 3)), 1).shape == (2, 5, 4)


def test_validation_without_device():
    """nmode.rs:86-101 messages through the C ABI (checked before the
    context is touched)."""
    lib = _lib.load()
    X = np.zeros((2, 3, 4), np.float32)
    M = np.zeros((5, 3), np.float32)
    shape = np.array([2, 3, 4], np.int64)
    rc = lib.tsr_nmode_product_f32(None, X.ctypes.data, 3, shape.ctypes.data, M.ctypes.data,
                                   5, 3, 3, X.ctypes.data)
    assert rc == 1 and b"Mode 3 out of bounds for tensor with rank 3" in lib.tsr_last_error()
    rc = lib.tsr_nmode_product_f32(None, X.ctypes.data, 3, shape.ctypes.data, M.ctypes.data,
                                   5, 3, 0, X.ctypes.data)
    assert rc == 15
    assert b"Matrix columns (3) must match tensor mode-0 size (2)" in lib.tsr_last_error()
    rows = np.array([2, 2], np.int64)
    cols = np.array([2, 1], np.int64)
    ptrs = (C.c_void_p * 2)(M.ctypes.data, M.ctypes.data)
    out_shape = np.zeros(2, np.int64)
    core = np.array([2, 2], np.int64)
    rc = lib.tsr_tucker_reconstruct_f32(None, X.ctypes.data, 2, core.ctypes.data, 1, ptrs,
                                        rows.ctypes.data, cols.ctypes.data, None,
                                        out_shape.ctypes.data)
    assert rc == 2 and b"Number of factor matrices (1) must match core rank (2)" in \
        lib.tsr_last_error()
    rc = lib.tsr_tucker_reconstruct_f32(None, X.ctypes.data, 2, core.ctypes.data, 2, ptrs,
                                        rows.ctypes.data, cols.ctypes.data, None,
                                        out_shape.ctypes.data)
    assert rc == 3 and b"Factor matrix 1 has 1 columns, expected 2 (core mode-1 size)" in \
        lib.tsr_last_error()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.gpu
@pytest.mark.parametrize("shape,mode,J", [
    ((2, 3, 4), 1, 5), ((2, 3), 0, 3), ((7,), 0, 4), ((256, 256, 256), 0, 64),
    ((256, 256, 256), 1, 64), ((256, 256, 256), 2, 64), ((128, 96, 64, 48), 2, 32),
    ((33, 17, 9, 5, 3), 4, 7), ((33, 17, 9, 5, 3), 0, 70), ((1000, 70, 3), 2, 1),
])
def test_nmode_product_vs_fp64(orc, shape, mode, J):
    rng = np.random.default_rng(sum(shape) + mode)
    X = rng.standard_normal(shape).astype(np.float32)
    M = rng.standard_normal((J, shape[mode])).astype(np.float32)
    got = tb.nmode_product(X, M, mode)
    ref = orc.nmode_product(X, M, mode)
    assert got.shape == ref.shape
    assert _rel(got, ref) <= 1e-5, _rel(got, ref)


@pytest.mark.gpu
def test_reference_cases_on_device():
    T = arange((2, 3, 4)).astype(np.float32)
    X = np.array([[1.0, 2, 3], [4, 5, 6]], np.float32)
    assert tb.nmode_product(X, np.array([[1.0, 0], [0, 1], [1, 1]]), 0).tolist() == \
        [[1, 2, 3], [4, 5, 6], [5, 7, 9]]
    assert np.array_equal(tb.nmode_product(T, np.eye(3), 1), T)
    r = tb.nmode_products_seq(T, [(np.eye(2), 0), (np.eye(3)[:2], 1)])
    assert r.shape == (2, 2, 4)
    # tucker_operator (nmode.rs:623-660)
    assert tb.tucker_operator(X, {0: np.eye(2)}).shape == (2, 3)
    assert tb.tucker_operator(T, {0: np.eye(2), 2: np.eye(4)[:2]}).shape == (2, 3, 2)
    assert np.array_equal(tb.tucker_operator(np.ones((2, 3), np.float32), {}),
                          np.ones((2, 3), np.float32))
    assert tb.tucker_operator_ordered(T, [(0, np.eye(2)), (1, np.eye(3)[:2]),
                                          (2, np.eye(4)[:2])]).shape == (2, 2, 2)
    # tucker_reconstruct (nmode.rs:684-720)
    rec = tb.tucker_reconstruct(np.eye(2), [np.eye(2), np.eye(2)])
    assert rec.tolist() == [[1, 0], [0, 1]]
    core = np.zeros((2, 2, 2), np.float32)
    core[0, 0, 0] = core[1, 1, 1] = 1.0
    rec = tb.tucker_reconstruct(core, [np.array([[1.0, 0], [0, 1], [1, 1]]), np.eye(2),
                                       np.array([[1.0, 0], [0, 1], [0.5, 0.5]])])
    assert rec.shape == (3, 2, 3)
    with pytest.raises(tb.TenrsoError):
        tb.tucker_operator(np.ones((2, 3), np.float32), {5: np.ones((1, 1))})
    red = tb.tucker_operator(arange((4, 5, 6)).astype(np.float32),
                             {0: np.ones((2, 4)), 1: np.ones((3, 5)), 2: np.ones((4, 6))})
    assert red.shape == (2, 3, 4) and np.allclose(red, arange((4, 5, 6)).sum())


@pytest.mark.gpu
def test_tucker_chain_vs_fp64(orc):
    """HOOI-style chain on the 256^3 tensor: X x_1 U1^T x_2 U2^T (a 256 x 64 x 64
    projection) and the full reconstruction from a 64^3 core."""
    rng = np.random.default_rng(7)
    X = rng.standard_normal((256, 256, 256)).astype(np.float32)
    U = [np.linalg.qr(rng.standard_normal((256, 64)))[0].astype(np.float32) for _ in range(3)]
    got = tb.tucker_operator(X, {1: U[1].T, 2: U[2].T})
    ref = orc.nmode_product(orc.nmode_product(X, U[1].T, 1), U[2].T, 2)
    assert _rel(got, ref) <= 1e-5
    core = rng.standard_normal((64, 64, 64)).astype(np.float32)
    got = tb.tucker_reconstruct(core, U)
    ref = core.astype(np.float64)
    for m in range(3):
        ref = orc.nmode_product(ref, U[m], m)
    assert _rel(got, ref) <= 1e-5
