"""Batched CP-ALS over the C ABI: many independent 3-way instances of uneven
shape and rank in one persistent launch. Each instance follows tenrso's
cp_als (crates/tenrso-decomp/src/cp/core.rs:59-182) from its own initial
factors; tenrso itself has no batched entry point (it would loop cp_als).

Factors of the whole batch live in one packed float32 array: instance b at
offset ``offsets[b]`` holds A (I0 x R) | B (I1 x R) | C (I2 x R), row-major.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import CpInfo, check
from .dense import REASONS, Context, ConvergenceInfo, CpDecomp, _ctx_handle, _f32, _i64, _ptr


class BatchedCpAls:
    """A device-resident batch of dense 3-way tensors with their ranks."""

    def __init__(self, tensors: Sequence, ranks: Sequence[int], ctx: Optional[Context] = None):
        ts = [_f32(t) for t in tensors]
        for t in ts:
            if t.ndim != 3:
                raise ValueError("batched CP-ALS takes 3-way tensors")
        self.shapes = [tuple(int(x) for x in t.shape) for t in ts]
        self.ranks = [int(r) for r in ranks]
        if len(self.ranks) != len(ts):
            raise ValueError("one rank per tensor")
        self.ctx = ctx
        self._lib = _lib.load()
        shp = _i64([s for sh in self.shapes for s in sh]) if ts else _i64([0])
        rk = _i64(self.ranks) if ts else _i64([0])
        ptrs = (C.c_void_p * max(len(ts), 1))(*[t.ctypes.data for t in ts])
        h = C.c_void_p()
        check(self._lib.tsr_batch_create_f32(_ctx_handle(ctx), len(ts), _ptr(shp), _ptr(rk),
                                             ptrs, C.byref(h)))
        self.handle = h
        total = C.c_int64(0)
        offs = np.zeros(len(ts), dtype=np.int64)
        check(self._lib.tsr_batch_factor_layout(self.handle, C.byref(total), _ptr(offs)))
        self.total = int(total.value)
        self.offsets = offs

    def __len__(self):
        return len(self.shapes)

    # -- packing -------------------------------------------------------------
    def pack(self, factors_per_instance) -> np.ndarray:
        """[[A, B, C], ...] -> the packed float32 array."""
        out = np.zeros(self.total, dtype=np.float32)
        for b, fs in enumerate(factors_per_instance):
            flat = np.concatenate([_f32(f).ravel() for f in fs])
            out[self.offsets[b]:self.offsets[b] + flat.size] = flat
        return out

    def unpack(self, packed) -> List[List[np.ndarray]]:
        res = []
        for b, (sh, R) in enumerate(zip(self.shapes, self.ranks)):
            off, fs = int(self.offsets[b]), []
            for n in sh:
                fs.append(np.asarray(packed[off:off + n * R]).reshape(n, R).copy())
                off += n * R
            res.append(fs)
        return res

    # -- configuration -------------------------------------------------------
    @property
    def config(self):
        t, s, c = C.c_int(), C.c_int(), C.c_int()
        check(self._lib.tsr_batch_get_config(self.handle, C.byref(t), C.byref(s), C.byref(c)))
        return {"threads": t.value, "sweeps_per_launch": s.value, "ctas_per_sm": c.value}

    def set_config(self, threads=256, sweeps_per_launch=0, ctas_per_sm=2):
        check(self._lib.tsr_batch_set_config(self.handle, threads, sweeps_per_launch,
                                             ctas_per_sm))

    def autotune(self, max_iters: int, d_init: int, cache_path: Optional[str] = None):
        """Time the launch configurations on this batch; returns (config,
        from_cache)."""
        fc = C.c_int(0)
        check(self._lib.tsr_batch_autotune(
            _ctx_handle(self.ctx), self.handle, max_iters, C.c_void_p(d_init),
            None if cache_path is None else str(cache_path).encode(), C.byref(fc)))
        return self.config, bool(fc.value)

    # -- runs ------------------------------------------------------------------
    def _infos(self, max_iters):
        infos = (CpInfo * len(self))()
        hists = [np.zeros(max(max_iters, 1), dtype=np.float64) for _ in range(len(self))]
        for i, h in enumerate(hists):
            infos[i].fit_history = h.ctypes.data_as(C.POINTER(C.c_double))
        return infos, hists

    def cp_als(self, max_iters: int, tol: float, init="random", seed: int = 0) -> List[CpDecomp]:
        """cp_als on every instance; init = "random" or [[A, B, C], ...]."""
        init_ptr, keep = None, None
        if not isinstance(init, str):
            keep = self.pack(init)
            init_ptr = _ptr(keep)
        elif init.lower() != "random":
            raise ValueError("only InitStrategy::Random or injected factors are supported")
        out = np.zeros(max(self.total, 1), dtype=np.float32)
        infos, hists = self._infos(max_iters)
        check(self._lib.tsr_cp_als_batched_f32(_ctx_handle(self.ctx), self.handle, max_iters,
                                               float(tol), init_ptr, seed, _ptr(out), infos))
        res = []
        for b, fs in enumerate(self.unpack(out)):
            I = infos[b]
            conv = ConvergenceInfo(fit_history=hists[b][:I.iters].copy(),
                                   reason=REASONS[I.reason], oscillated=bool(I.oscillated),
                                   oscillation_count=int(I.oscillation_count),
                                   final_fit_change=float(I.final_fit_change))
            res.append(CpDecomp(factors=fs, weights=None, fit=float(I.fit), iters=int(I.iters),
                                convergence=conv, ridge_used=bool(I.ridge_used)))
        return res

    def cp_als_dev(self, max_iters: int, tol: float, d_init: int, d_out: int,
                   want_info: bool = False):
        """Device-resident run; returns [(fit, iters, reason)] when want_info
        (that synchronizes), else None."""
        infos = (CpInfo * len(self))() if want_info else None
        check(self._lib.tsr_cp_als_batched_dev_f32(_ctx_handle(self.ctx), self.handle,
                                                   max_iters, float(tol), C.c_void_p(d_init),
                                                   C.c_void_p(d_out), infos))
        if not want_info:
            return None
        return [(float(I.fit), int(I.iters), REASONS[I.reason]) for I in infos]

    def close(self):
        if getattr(self, "handle", None):
            self._lib.tsr_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
