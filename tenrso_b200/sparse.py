"""Python mirror of tenrso's sparse types on the CP-ALS path.

  CooTensor (new/sort/deduplicate/to_dense)   crates/tenrso-sparse/src/coo.rs:73-347
  CsfTensor.from_coo + accessors              crates/tenrso-sparse/src/csf.rs:137-331
  HiCooTensor.from_coo + accessors + MTTKRP    crates/tenrso-sparse/src/hicoo.rs:79-359
  SparseTensor: device-resident per-mode CSF for the sparse MTTKRP and sparse
  CP-ALS, which tenrso does not implement (csf.rs:42 only names MTTKRP).

The arrays CsfTensor exposes are those tenrso's from_coo builds, including its
nnz-offset fptr at every level (csf.rs:193-254).
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import CpInfo, TenrsoError, check
from .dense import REASONS, ConvergenceInfo, CpDecomp, _ctx_handle, _i64, _ptr


class CooError(ValueError):
    """coo.rs CooError: construction-time validation failures."""


class CooTensor:
    """Coordinate storage: indices (nnz x ndim), values (nnz), shape."""

    def __init__(self, indices, values, shape):
        shape = [int(s) for s in shape]
        idx = np.asarray(indices, dtype=np.int64)
        vals = np.asarray(values, dtype=np.float32)
        if idx.ndim == 1 and idx.size == 0:
            idx = idx.reshape(0, len(shape))
        # coo.rs:107-149, same order of checks and wording
        if idx.shape[0] != vals.shape[0]:
            raise CooError(f"Length mismatch: {idx.shape[0]} indices but {vals.shape[0]} values")
        if len(shape) == 0:
            raise CooError("Invalid shape: Shape cannot be empty")
        if 0 in shape:
            raise CooError("Invalid shape: Shape cannot contain zeros")
        if idx.shape[0] and idx.shape[1] != len(shape):
            raise CooError(f"Shape mismatch: indices have {idx.shape[1]} elements but shape has "
                           f"{len(shape)} dimensions")
        if idx.shape[0]:
            bad = np.any((idx < 0) | (idx >= np.asarray(shape)[None, :]), axis=1)
            if bad.any():
                k = int(np.argmax(bad))
                raise CooError(f"Index out of bounds: index {idx[k].tolist()} exceeds shape "
                               f"{shape}")
        self._idx = np.ascontiguousarray(idx.reshape(-1, len(shape)))
        self._vals = np.ascontiguousarray(vals)
        self._shape = shape

    @classmethod
    def zeros(cls, shape):
        return cls(np.zeros((0, len(shape)), np.int64), np.zeros(0, np.float32), shape)

    def push(self, index, value):
        """coo.rs:213-234 (bounds-checked append)."""
        index = [int(i) for i in index]
        if len(index) != len(self._shape):
            raise CooError(f"Shape mismatch: indices have {len(index)} elements but shape has "
                           f"{len(self._shape)} dimensions")
        if any(i < 0 or i >= s for i, s in zip(index, self._shape)):
            raise CooError(f"Index out of bounds: index {index} exceeds shape {self._shape}")
        self._idx = np.concatenate([self._idx, np.asarray([index], np.int64)])
        self._vals = np.concatenate([self._vals, np.asarray([value], np.float32)])

    def nnz(self) -> int:
        return int(self._idx.shape[0])

    def shape(self) -> List[int]:
        return list(self._shape)

    def rank(self) -> int:
        return len(self._shape)

    def indices(self) -> np.ndarray:
        return self._idx

    def values(self) -> np.ndarray:
        return self._vals

    def density(self) -> float:
        return self.nnz() / float(np.prod(self._shape))

    def sort(self, ctx=None):
        """Stable lexicographic sort on the device (coo.rs:239-257)."""
        idx = self._idx.copy()
        vals = self._vals.copy()
        check(_lib.load().tsr_coo_sort_f32(_ctx_handle(ctx) if self.nnz() > 1 else None,
                                           _ptr(idx), _ptr(vals), self.nnz(), self.rank(),
                                           _ptr(_i64(self._shape))))
        self._idx, self._vals = idx, vals

    def deduplicate(self, ctx=None):
        """Sort, then sum equal coordinates in fp32 left to right
        (coo.rs:320-347), on the device."""
        idx = self._idx.copy()
        vals = self._vals.copy()
        n = C.c_int64(0)
        check(_lib.load().tsr_coo_deduplicate_f32(
            _ctx_handle(ctx) if self.nnz() > 1 else None, _ptr(idx), _ptr(vals), self.nnz(),
            self.rank(), _ptr(_i64(self._shape)), C.byref(n)))
        self._idx, self._vals = idx[:n.value].copy(), vals[:n.value].copy()

    def to_dense(self) -> np.ndarray:
        out = np.zeros(self._shape, np.float32)
        if self.nnz():
            out[tuple(self._idx.T)] = self._vals  # last write wins, as coo.rs:282-294
        return out


class CsfError(ValueError):
    """csf.rs CsfError."""


class CsfTensor:
    """The reference CSF arrays, built on the device by from_coo."""

    def __init__(self, shape, mode_order, nnz, fptr, fids, vals):
        self._shape = list(shape)
        self._mode_order = list(mode_order)
        self._nnz = nnz
        self._fptr = fptr
        self._fids = fids
        self._vals = vals

    @classmethod
    def from_coo(cls, coo: CooTensor, mode_order: Sequence[int], ctx=None) -> "CsfTensor":
        ndim = coo.rank()
        nnz = coo.nnz()
        mo = _i64(list(mode_order) if len(mode_order) else [0])
        fptr = np.zeros((ndim, nnz + 1), np.int64)
        fids = np.zeros((ndim, max(nnz, 1)), np.int64)
        vals = np.zeros(max(nnz, 1), np.float32)
        lens = np.zeros(2 * ndim, np.int64)
        h = _ctx_handle(ctx) if nnz > 0 else None
        rc = _lib.load().tsr_csf_from_coo_f32(h, _ptr(coo.indices()), _ptr(coo.values()), nnz,
                                              ndim, _ptr(_i64(coo.shape())), _ptr(mo),
                                              len(mode_order), _ptr(fptr), _ptr(fids),
                                              _ptr(vals), _ptr(lens))
        if rc == 13:
            raise CsfError(_lib.load().tsr_last_error().decode())
        check(rc)
        fp = [fptr[l, :lens[2 * l]].copy() for l in range(ndim)]
        fi = [fids[l, :lens[2 * l + 1]].copy() for l in range(ndim)]
        nv = nnz if ndim > 1 else 0
        return cls(coo.shape(), mode_order, nnz, fp, fi, vals[:nv].copy())

    def shape(self):
        return list(self._shape)

    def ndim(self):
        return len(self._shape)

    def nnz(self):
        return self._nnz

    def mode_order(self):
        return list(self._mode_order)

    def density(self):
        total = float(np.prod(self._shape))
        return self._nnz / total if total else 0.0

    def fptr(self, level: int) -> np.ndarray:
        return self._fptr[level]

    def fids(self, level: int) -> np.ndarray:
        return self._fids[level]

    def vals(self) -> np.ndarray:
        return self._vals

    def to_coo(self) -> CooTensor:
        """A correct inverse of the layout (every fptr level holds nnz
        offsets). tenrso's own CsfIterator (csf.rs:423-495) reconstructs wrong
        indices for fibers of more than one entry, so this is not a port of it."""
        nd = self.ndim()
        n = len(self._fids[-1]) if nd > 1 else 0
        idx = np.zeros((n, nd), np.int64)
        pos = np.arange(n)
        for level in range(nd - 1):
            f = np.searchsorted(self._fptr[level], pos, side="right") - 1
            idx[:, self._mode_order[level]] = self._fids[level][f]
        if nd > 1:
            idx[:, self._mode_order[-1]] = self._fids[-1]
        return CooTensor(idx, self._vals, self._shape)


class HiCooTensor:
    """HiCooTensor (hicoo.rs:79-359): block coordinates, cumulative block
    pointers, within-block local coordinates and values, built on the device
    by from_coo. The device copy stays attached for the HiCOO MTTKRP."""

    def __init__(self, handle, ctx, shape, block_shape, block_coords, block_ptrs, local_coords,
                 values):
        self._h = handle
        self._ctx = ctx
        self._shape = list(shape)
        self._block_shape = list(block_shape)
        self._block_coords = block_coords
        self._block_ptrs = block_ptrs
        self._local = local_coords
        self._values = values

    @classmethod
    def from_coo(cls, coo: CooTensor, block_shape: Sequence[int], ctx=None) -> "HiCooTensor":
        """hicoo.rs:118-203. Raises TenrsoError (TSR_E_BLOCK_SHAPE) with
        hicoo.rs's messages for a block_shape of the wrong length or with a
        zero."""
        ndim, nnz = coo.rank(), coo.nnz()
        bs = list(block_shape)
        if len(bs) != ndim:
            raise TenrsoError(20, f"Invalid block shape: block_shape length {len(bs)} != "
                                  f"ndim {ndim}")
        if 0 in bs:
            raise TenrsoError(20, "Invalid block shape: block_shape cannot contain zeros")
        lib = _lib.load()
        h = C.c_void_p()
        check(lib.tsr_hicoo_create_f32(_ctx_handle(ctx), _ptr(coo.indices()), _ptr(coo.values()),
                                       nnz, ndim, _ptr(_i64(coo.shape())),
                                       _ptr(_i64(bs or [0])), len(bs), C.byref(h)))
        n, nb = C.c_int64(0), C.c_int64(0)
        check(lib.tsr_hicoo_info(h, C.byref(n), C.byref(nb)))
        bc = np.zeros((max(nb.value, 1), ndim), np.int64)
        bp = np.zeros(nb.value + 1, np.int64)
        lc = np.zeros((max(n.value, 1), ndim), np.int64)
        vals = np.zeros(max(n.value, 1), np.float32)
        check(lib.tsr_hicoo_export(_ctx_handle(ctx), h, _ptr(bc), _ptr(bp), _ptr(lc), _ptr(vals)))
        return cls(h, ctx, coo.shape(), bs, bc[:nb.value], bp, lc[:n.value], vals[:n.value])

    def shape(self):
        return list(self._shape)

    def block_shape(self):
        return list(self._block_shape)

    def ndim(self):
        return len(self._shape)

    def nnz(self):
        return len(self._values)

    def num_blocks(self):
        return len(self._block_coords)

    def density(self):
        """hicoo.rs:240-247."""
        total = float(np.prod(self._shape))
        return self.nnz() / total if total else 0.0

    def block_coords(self) -> np.ndarray:
        return self._block_coords

    def block_ptrs(self) -> np.ndarray:
        return self._block_ptrs

    def local_coords(self) -> np.ndarray:
        return self._local

    def values(self) -> np.ndarray:
        return self._values

    def _global_indices(self) -> np.ndarray:
        counts = np.diff(self._block_ptrs)
        blocks = np.repeat(np.arange(self.num_blocks()), counts)
        bs = np.asarray(self._block_shape, np.int64)
        return self._block_coords[blocks] * bs + self._local

    def iter(self):
        """(indices, value) in block-major order (hicoo.rs:298-359)."""
        for idx, v in zip(self._global_indices(), self._values):
            yield [int(i) for i in idx], float(v)

    def to_coo(self) -> CooTensor:
        """hicoo.rs:285-293: the entries in block-major order."""
        return CooTensor(self._global_indices(), self._values.copy(), self._shape)

    def to_dense(self) -> np.ndarray:
        """hicoo.rs:311-321: each entry assigned in block-major order (a later
        duplicate overwrites an earlier one)."""
        out = np.zeros(self._shape, np.float32)
        idx = self._global_indices()
        if len(idx):
            lin = np.ravel_multi_index(tuple(idx.T), self._shape)
            # last occurrence of each position wins
            rev = lin[::-1]
            _, first = np.unique(rev, return_index=True)
            keep = len(lin) - 1 - first
            out.ravel()[lin[keep]] = self._values[keep]
        return out

    def mttkrp(self, factors, mode: int) -> np.ndarray:
        """Sparse MTTKRP on the device's HiCOO layout (fp32 out, FP64 sums)."""
        fs = [np.ascontiguousarray(f, dtype=np.float32) for f in factors]
        if not 0 <= mode < self.ndim():
            raise TenrsoError(1, f"Mode {mode} out of bounds for tensor with rank {self.ndim()}")
        if len(fs) != self.ndim():
            raise ValueError("one factor matrix per mode is required")
        R = fs[0].shape[1]
        ptrs = (C.c_void_p * len(fs))(*[f.ctypes.data for f in fs])
        out = np.zeros((self._shape[mode], R), np.float32)
        check(_lib.load().tsr_mttkrp_hicoo_f32(_ctx_handle(self._ctx), self._h, ptrs, R, mode,
                                               _ptr(out)))
        return out

    def mttkrp_dev(self, d_factors, rank: int, mode: int, d_out: int):
        ptrs = (C.c_void_p * len(d_factors))(*d_factors)
        check(_lib.load().tsr_mttkrp_hicoo_dev_f32(_ctx_handle(self._ctx), self._h, ptrs, rank,
                                                   mode, C.c_void_p(d_out)))

    def close(self):
        if self._h:
            _lib.load().tsr_hicoo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def synth_zipf_coo_dev(shape, nnz: int, seed: int, d_indices: int, d_values: int,
                       capacity: int, s: float = 1.2, ctx=None) -> int:
    """Device version of synth.zipf_coo: writes the raw COO (duplicates
    included) to device buffers and returns its entry count."""
    n = C.c_int64(0)
    check(_lib.load().tsr_synth_zipf_coo_dev(_ctx_handle(ctx), len(shape), _ptr(_i64(shape)),
                                             nnz, seed, float(s), capacity,
                                             C.c_void_p(d_indices), C.c_void_p(d_values),
                                             C.byref(n)))
    return n.value


def coo_deduplicate_dev(d_indices: int, d_values: int, nnz: int, shape, ctx=None) -> int:
    """CooTensor::deduplicate on device arrays; returns the merged count."""
    n = C.c_int64(0)
    check(_lib.load().tsr_coo_deduplicate_dev_f32(_ctx_handle(ctx), C.c_void_p(d_indices),
                                                  C.c_void_p(d_values), nnz, len(shape),
                                                  _ptr(_i64(shape)), C.byref(n)))
    return n.value


class SparseTensor:
    """Device-resident sparse tensor for MTTKRP / CP-ALS (one CSF per mode)."""

    def __init__(self, coo: Optional[CooTensor] = None, ctx=None, *, d_indices: int = 0,
                 d_values: int = 0, nnz: int = 0, shape=None):
        from .dense import default_context
        self._ctx = ctx or default_context()
        self._lib = _lib.load()
        h = C.c_void_p()
        if coo is not None:
            check(self._lib.tsr_sparse_create_f32(self._ctx.handle, _ptr(coo.indices()),
                                                  _ptr(coo.values()), coo.nnz(), coo.rank(),
                                                  _ptr(_i64(coo.shape())), C.byref(h)))
            self.shape = coo.shape()
            self.nnz = coo.nnz()
        else:
            check(self._lib.tsr_sparse_create_dev_f32(self._ctx.handle, C.c_void_p(d_indices),
                                                      C.c_void_p(d_values), nnz, len(shape),
                                                      _ptr(_i64(shape)), C.byref(h)))
            self.shape = list(shape)
            self.nnz = nnz
        self.handle = h

    def info(self, mode: int):
        nnz, roots, fibers = C.c_int64(), C.c_int64(), C.c_int64()
        check(self._lib.tsr_sparse_info(self.handle, mode, C.byref(nnz), C.byref(roots),
                                        C.byref(fibers)))
        return {"nnz": nnz.value, "roots": roots.value, "fibers": fibers.value}

    def mttkrp(self, factors, mode: int) -> np.ndarray:
        fs = [np.ascontiguousarray(np.asarray(f, np.float32)) for f in factors]
        R = fs[0].shape[1]
        out = np.zeros((self.shape[mode], R), np.float32)
        ptrs = (C.c_void_p * len(fs))(*[f.ctypes.data for f in fs])
        check(self._lib.tsr_mttkrp_csf_f32(self._ctx.handle, self.handle, ptrs, R, mode,
                                           _ptr(out)))
        return out

    def mttkrp_dev(self, d_factors, rank: int, mode: int, d_out: int):
        ptrs = (C.c_void_p * len(d_factors))(*d_factors)
        check(self._lib.tsr_mttkrp_csf_dev_f32(self._ctx.handle, self.handle, ptrs, rank, mode,
                                               C.c_void_p(d_out)))

    def profile_mttkrp_dev(self, d_factors, rank: int, mode: int, iters=10, flush_l2=True):
        ptrs = (C.c_void_p * len(d_factors))(*d_factors)
        ms = C.c_double(0)
        check(self._lib.tsr_profile_mttkrp_csf_dev_f32(self._ctx.handle, self.handle, ptrs, rank,
                                                       mode, iters, int(flush_l2),
                                                       C.byref(ms)))
        return ms.value

    def cp_als(self, rank: int, max_iters: int, tol: float, init="random",
               time_limit: Optional[float] = None, seed: int = 0) -> CpDecomp:
        total = int(sum(n * rank for n in self.shape))
        out = np.zeros(max(total, 1), np.float32)
        if isinstance(init, str):
            init_ptr = None
        else:
            flat = np.concatenate([np.asarray(f, np.float32).ravel() for f in init])
            init_ptr = _ptr(flat)
        hist = np.zeros(max(max_iters, 1), np.float64)
        info = CpInfo()
        info.fit_history = hist.ctypes.data_as(C.POINTER(C.c_double))
        check(self._lib.tsr_cp_als_sparse_f32(self._ctx.handle, self.handle, rank, max_iters,
                                              float(tol), init_ptr, seed,
                                              -1.0 if time_limit is None else float(time_limit),
                                              _ptr(out), C.byref(info)))
        factors, off = [], 0
        for n in self.shape:
            factors.append(out[off:off + n * rank].reshape(n, rank).copy())
            off += n * rank
        conv = ConvergenceInfo(fit_history=hist[:info.iters].copy(), reason=REASONS[info.reason],
                               oscillated=bool(info.oscillated),
                               oscillation_count=int(info.oscillation_count),
                               final_fit_change=float(info.final_fit_change))
        return CpDecomp(factors=factors, weights=None, fit=float(info.fit), iters=int(info.iters),
                        convergence=conv, ridge_used=bool(info.ridge_used))

    def cp_als_dev(self, rank, max_iters, tol, d_init: int, d_out: int, time_limit=None):
        hist = np.zeros(max(max_iters, 1), np.float64)
        info = CpInfo()
        info.fit_history = hist.ctypes.data_as(C.POINTER(C.c_double))
        check(self._lib.tsr_cp_als_sparse_dev_f32(
            self._ctx.handle, self.handle, rank, max_iters, float(tol), C.c_void_p(d_init),
            -1.0 if time_limit is None else float(time_limit), C.c_void_p(d_out),
            C.byref(info)))
        return float(info.fit), int(info.iters), hist[:info.iters].copy()

    def close(self):
        if getattr(self, "handle", None):
            self._lib.tsr_sparse_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
