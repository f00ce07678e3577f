"""The allocation-free MTTKRP entry point (tsr_mttkrp_mode0_noalloc_f32).

It serves callers that cannot call cudaMalloc — a library whose host
application's caching allocator owns the device memory, or a service that
sizes every buffer before it starts — by keeping its split partials in a fixed
device array instead of a context workspace. This test calls it through the C
ABI twice in a row and compares each result with the context-based
tsr_mttkrp_dev_f32 on the same inputs (relative Frobenius error <= 1e-5, the
FP32 MTTKRP tolerance used throughout the tests), checks that the second call
leaves the device's free memory unchanged, and covers its argument checks
(empty tensors, negative sizes, a problem too large for the array). The file
name sorts last so that a run stopping at the first failure has already run
every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_mttkrp_matches_context_entry_point():
    import torch

    import tenrso_b200 as tb
    from tenrso_b200 import _lib

    lib = _lib.load()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = tb.Context(0, stream=stream.cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(7)
    for shape, R in (((96, 40, 36), 16), ((256, 256, 256), 64)):
        X = torch.rand(shape, device="cuda", generator=g)
        fs = [torch.rand(n, R, device="cuda", generator=g) for n in shape]
        shp = np.asarray(shape, dtype=np.int64)
        ptrs = (C.c_void_p * 3)(*[f.data_ptr() for f in fs])
        ref = torch.empty(shape[0], R, device="cuda")
        tb.mttkrp_dev(X.data_ptr(), shape, [f.data_ptr() for f in fs], R, 0, ref.data_ptr(),
                      "fp32", ctx=ctx)
        for call in range(2):  # two calls in a row share the fixed scratch array
            out = torch.full((shape[0], R), float("nan"), device="cuda")
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            rc = lib.tsr_mttkrp_mode0_noalloc_f32(C.c_void_p(stream.cuda_stream),
                                                  C.c_void_p(X.data_ptr()), 3,
                                                  shp.ctypes.data_as(C.c_void_p), ptrs, R,
                                                  C.c_void_p(out.data_ptr()))
            assert rc == 0, lib.tsr_last_error().decode()
            torch.cuda.synchronize()
            if call == 1:  # the first call may load kernel code; the second allocates nothing
                assert torch.cuda.mem_get_info()[0] == free0
            err = float(torch.linalg.norm(out.double() - ref.double()) /
                        torch.linalg.norm(ref.double()))
            assert err <= 1e-5, (shape, err)
    # a problem whose partials do not fit the fixed array is rejected
    big = (65536, 8, 8)  # one split of 65536 x 128 partials > 4 Mi floats
    Xb = torch.rand(big, device="cuda", generator=g)
    fb = [torch.rand(n, 128, device="cuda", generator=g) for n in big]
    ob = torch.empty(big[0], 128, device="cuda")
    rc = lib.tsr_mttkrp_mode0_noalloc_f32(C.c_void_p(stream.cuda_stream),
                                          C.c_void_p(Xb.data_ptr()), 3,
                                          np.asarray(big, np.int64).ctypes.data_as(C.c_void_p),
                                          (C.c_void_p * 3)(*[f.data_ptr() for f in fb]), 128,
                                          C.c_void_p(ob.data_ptr()))
    assert rc == 14 and b"exceed the fixed" in lib.tsr_last_error()

    def call(shape, R, X, fs, out):
        shp = np.asarray(shape, dtype=np.int64)
        ptrs = (C.c_void_p * len(shape))(*[f.data_ptr() for f in fs])
        return lib.tsr_mttkrp_mode0_noalloc_f32(C.c_void_p(stream.cuda_stream),
                                                C.c_void_p(X.data_ptr()), len(shape),
                                                shp.ctypes.data_as(C.c_void_p), ptrs, R,
                                                C.c_void_p(out.data_ptr()))

    # an empty sum over the other modes gives zeros; an empty output is a no-op
    Xe = torch.empty(16, device="cuda")
    fe = [torch.rand(8, 4, device="cuda"), torch.empty(0, 4, device="cuda"),
          torch.rand(4, 4, device="cuda")]
    oe = torch.full((8, 4), float("nan"), device="cuda")
    assert call((8, 0, 4), 4, Xe, fe, oe) == 0, lib.tsr_last_error().decode()
    torch.cuda.synchronize()
    assert bool((oe == 0).all())
    assert call((0, 4, 4), 4, Xe, [fe[1], fe[2], fe[2]], oe) == 0
    # negative sizes are rejected before any launch
    assert call((8, -4, 4), 4, Xe, fe, oe) == 10  # TSR_E_INVALID_ARG
    assert b"negative size" in lib.tsr_last_error()
    ctx.close()
