"""The C-ABI boundary without a GPU: the library loads, exports every symbol
include/tenrso_b200.h declares, and reproduces tenrso's argument validation
(messages from mttkrp.rs / khatri_rao.rs / cp/core.rs) before any device
work. No call here reaches a kernel."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import tenrso_b200 as tb
from tenrso_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "tenrso_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tsr_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"


def test_version_and_status_strings():
    lib = _lib.load()
    assert b"sm_100a" in lib.tsr_version()
    assert lib.tsr_status_string(0) == b"ok"


@pytest.mark.parametrize("case", range(3))
def test_mttkrp_error_messages(kats, case):
    k = kats["mttkrp_errors"][case]
    X = np.ones(k["shape"], dtype=np.float32)
    fs = [np.array(f, dtype=np.float32) for f in k["factors"]]
    with pytest.raises(tb.TenrsoError, match=k["expect"]):
        tb.mttkrp(X, fs, k["mode"])


def test_mttkrp_exact_wording():
    X = np.ones((2, 3), dtype=np.float32)
    with pytest.raises(tb.TenrsoError) as e:
        tb.mttkrp(X, [np.ones((2, 1)), np.ones((3, 1))], 5)
    assert str(e.value) == "Mode 5 out of bounds for tensor with rank 2"
    with pytest.raises(tb.TenrsoError) as e:
        tb.mttkrp(X, [np.ones((2, 1)), np.ones((4, 1))], 0)
    assert str(e.value) == "Factor matrix 1 has 4 rows, expected 3 (tensor mode-1 size)"
    with pytest.raises(tb.TenrsoError) as e:
        tb.mttkrp(np.ones(4, np.float32), [np.ones((4, 1))], 0)
    assert str(e.value) == "Need at least 2 factor matrices for MTTKRP"


def test_blocked_tile_size_zero():
    X = np.ones((2, 3, 4), dtype=np.float32)
    fs = [np.ones((n, 2), np.float32) for n in X.shape]
    with pytest.raises(tb.TenrsoError, match="Tile size must be greater than 0"):
        tb.mttkrp_blocked(X, fs, 0, 0)


def test_khatri_rao_column_mismatch(kats):
    k = kats["khatri_rao_errors"][0]
    with pytest.raises(tb.TenrsoError, match=k["expect"]):
        tb.khatri_rao(np.array(k["a"], np.float32), np.array(k["b"], np.float32))


def test_cp_als_validation():
    X = np.ones((3, 4, 5), dtype=np.float32)
    with pytest.raises(tb.TenrsoError, match="Invalid rank: 0"):
        tb.cp_als(X, 0, 5, 0.0)
    with pytest.raises(tb.TenrsoError, match="Invalid rank: 4"):
        tb.cp_als(X, 4, 5, 0.0)
    with pytest.raises(tb.TenrsoError, match="Invalid tolerance"):
        tb.cp_als(X, 2, 5, 1.0)
    with pytest.raises(tb.TenrsoError, match="Invalid tolerance"):
        tb.cp_als(X, 2, 5, -0.1)


def test_no_cpu_fallback_without_device():
    """Valid arguments need a device: without one the call fails loudly."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = C.c_void_p()
    rc = lib.tsr_ctx_create(0, None, C.byref(h))
    assert rc == 9  # TSR_E_CUDA
    assert lib.tsr_last_error()


def test_cp_reconstruct_errors(kats):
    k = kats["cp_reconstruct_errors"][0]
    with pytest.raises(tb.TenrsoError, match=k["expect"]):
        tb.cp_reconstruct([np.array(f, np.float32) for f in k["factors"]])
    with pytest.raises(tb.TenrsoError, match="Factor 1 has 1 columns, expected 2"):
        tb.cp_reconstruct([np.array(f, np.float32) for f in k["factors"]])
    with pytest.raises(tb.TenrsoError,
                       match="Need at least one factor matrix for CP reconstruction"):
        tb.cp_reconstruct([])
    with pytest.raises(tb.TenrsoError, match="Weights length 3 must match rank 2"):
        tb.cp_reconstruct([np.ones((2, 2), np.float32)] * 2, weights=[1, 2, 3])


def test_cp_reconstruction_grad_errors():
    fs = [np.ones((n, 2), np.float32) for n in (3, 4, 5)]
    g = tb.CpReconstructionGrad(fs)
    with pytest.raises(tb.TenrsoError, match="Gradient rank 2 doesn't match number of factors 3"):
        g.compute_factor_gradients(np.ones((3, 4), np.float32))
    one = tb.CpReconstructionGrad([np.ones((3, 2), np.float32)])
    with pytest.raises(tb.TenrsoError, match="Need at least one factor for Khatri-Rao product"):
        one.compute_factor_gradients(np.ones((3,), np.float32))


def test_batched_validation():
    X = np.ones((4, 5, 6), np.float32)
    with pytest.raises(tb.TenrsoError, match="instance 1: Invalid rank: 5"):
        tb.BatchedCpAls([X, X], [2, 5])
    with pytest.raises(tb.TenrsoError, match="instance 0: Invalid rank: 0"):
        tb.BatchedCpAls([X], [0])
    Y = np.ones((20, 20, 20), np.float32)
    with pytest.raises(tb.TenrsoError, match="rank <= 16"):
        tb.BatchedCpAls([Y], [17])
    with pytest.raises(ValueError, match="3-way"):
        tb.BatchedCpAls([np.ones((3, 3), np.float32)], [1])


def test_cp_als_accelerated_validation():
    """advanced.rs:71-77 in the Python mirror and in the C ABI itself (the C
    checks run before the context is touched, so a NULL context is fine)."""
    X = np.ones((3, 4, 5), dtype=np.float32)
    with pytest.raises(tb.TenrsoError, match="Invalid rank: 0"):
        tb.cp_als_accelerated(X, 0, 5, 1e-4)
    for tol in (0.0, 1.0, -0.1):
        with pytest.raises(tb.TenrsoError, match="Invalid tolerance"):
            tb.cp_als_accelerated(X, 2, 5, tol)
    lib = _lib.load()
    shape = np.array(X.shape, dtype=np.int64)
    out = np.zeros(12 * 4, dtype=np.float32)
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = lib.tsr_cp_als_accelerated_f32(None, ptr(X), 3, ptr(shape), 0, 5, 1e-4, None, 0, 0, -1.0,
                                        ptr(out), None)
    assert rc == 5 and b"Invalid rank: 0" in lib.tsr_last_error()
    for tol in (0.0, 1.0):
        rc = lib.tsr_cp_als_accelerated_f32(None, ptr(X), 3, ptr(shape), 2, 5, tol, None, 0, 0,
                                            -1.0, ptr(out), None)
        assert rc == 6 and b"Invalid tolerance" in lib.tsr_last_error()
