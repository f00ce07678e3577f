"""n-mode products (TTM) and the Tucker operators over the C ABI.

  nmode_product            crates/tenrso-kernels/src/nmode.rs:72-131
  nmode_products_seq       nmode.rs:241-254
  tucker_operator          nmode.rs:442-480 (ascending rows / mode size)
  tucker_operator_ordered  nmode.rs:517-531
  tucker_reconstruct       nmode.rs:576-611

Every product runs on the device (a strided batched fp32 GEMM, no unfolding
copy); errors come back as TenrsoError with the reference's messages.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import check
from .dense import _ctx_handle, _f32, _i64, _ptr


def nmode_product(tensor, matrix, mode: int, ctx=None) -> np.ndarray:
    """tensor x_mode matrix (matrix J x I_mode)."""
    t = _f32(tensor)
    m = _f32(matrix)
    if m.ndim != 2:
        raise ValueError("matrix must be 2-D")
    shape = list(t.shape)
    out_shape = list(shape)
    if 0 <= mode < t.ndim:
        out_shape[mode] = m.shape[0]
    out = np.zeros(int(np.prod(out_shape)) if out_shape else 1, np.float32)
    check(_lib.load().tsr_nmode_product_f32(_ctx_handle(ctx), _ptr(t), t.ndim, _ptr(_i64(shape)),
                                            _ptr(m), m.shape[0], m.shape[1], mode, _ptr(out)))
    return out.reshape(out_shape)


def _chain(fn, tensor, pairs: Sequence[Tuple[int, np.ndarray]], ctx):
    t = _f32(tensor)
    mats = [_f32(m) for _, m in pairs]
    modes = np.array([int(md) for md, _ in pairs] or [0], np.int32)
    ptrs = (C.c_void_p * max(len(pairs), 1))(*[m.ctypes.data for m in mats])
    rows = _i64([m.shape[0] for m in mats] or [0])
    cols = _i64([m.shape[1] for m in mats] or [0])
    oshape = np.zeros(max(t.ndim, 1), np.int64)
    check(fn(_ctx_handle(ctx), _ptr(t), t.ndim, _ptr(_i64(t.shape)), len(pairs), _ptr(modes),
             ptrs, _ptr(rows), _ptr(cols), None, _ptr(oshape)))
    out = np.zeros(max(int(np.prod(oshape[:t.ndim])), 1), np.float32)
    check(fn(_ctx_handle(ctx), _ptr(t), t.ndim, _ptr(_i64(t.shape)), len(pairs), _ptr(modes),
             ptrs, _ptr(rows), _ptr(cols), _ptr(out), _ptr(oshape)))
    return out[:int(np.prod(oshape[:t.ndim]))].reshape([int(v) for v in oshape[:t.ndim]])


def nmode_products_seq(tensor, matrices: Sequence[Tuple[np.ndarray, int]], ctx=None):
    """Products in the given order; matrices = [(matrix, mode), ...]."""
    return _chain(_lib.load().tsr_nmode_products_seq_f32, tensor,
                  [(md, m) for m, md in matrices], ctx)


def tucker_operator_ordered(tensor, mode_matrix_pairs: Sequence[Tuple[int, np.ndarray]],
                            ctx=None):
    """Products in the given order; pairs = [(mode, matrix), ...]."""
    return _chain(_lib.load().tsr_nmode_products_seq_f32, tensor, list(mode_matrix_pairs), ctx)


def tucker_operator(tensor, factor_matrices: Dict[int, np.ndarray], ctx=None):
    """A mode -> matrix map, applied in ascending order of rows / mode size."""
    return _chain(_lib.load().tsr_tucker_operator_f32, tensor,
                  sorted(factor_matrices.items()), ctx)


def tucker_reconstruct(core, factors: Sequence[np.ndarray], ctx=None):
    """core x_0 U_0 ... x_{N-1} U_{N-1}."""
    c = _f32(core)
    fs = [_f32(f) for f in factors]
    ptrs = (C.c_void_p * max(len(fs), 1))(*[f.ctypes.data for f in fs])
    rows = _i64([f.shape[0] for f in fs] or [0])
    cols = _i64([f.shape[1] for f in fs] or [0])
    oshape = np.zeros(max(c.ndim, 1), np.int64)
    fn = _lib.load().tsr_tucker_reconstruct_f32
    check(fn(_ctx_handle(ctx), _ptr(c), c.ndim, _ptr(_i64(c.shape)), len(fs), ptrs, _ptr(rows),
             _ptr(cols), None, _ptr(oshape)))
    out = np.zeros(max(int(np.prod(oshape[:c.ndim])), 1), np.float32)
    check(fn(_ctx_handle(ctx), _ptr(c), c.ndim, _ptr(_i64(c.shape)), len(fs), ptrs, _ptr(rows),
             _ptr(cols), _ptr(out), _ptr(oshape)))
    return out[:int(np.prod(oshape[:c.ndim]))].reshape([int(v) for v in oshape[:c.ndim]])
