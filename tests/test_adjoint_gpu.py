"""CP reconstruction and its adjoint on the GPU against the oracle:
cp_reconstruct within 1e-6 relative Frobenius of the FP64 definition (exact on
tenrso's integer known-answer vectors), CpReconstructionGrad within 1e-5 of
the FP64 restatement, and the loss/gradient of ||X - [[A,B,C,D]]||^2 +
1e-3 sum ||U||^2 at 128x96x64x48, R=32 checked against the CPU VJP and against
FP64 central differences (h=1e-6) on 64 seeded entries per factor."""
import numpy as np
import pytest

import tenrso_b200 as tb

pytestmark = pytest.mark.gpu

C5_SHAPE = (128, 96, 64, 48)
C5_RANK = 32
C5_REG = 1e-3


def rel_err(a, b):
    b = np.asarray(b, np.float64)
    return np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300)


def c5_inputs(seed=0xC5):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal(C5_SHAPE).astype(np.float32)
    fs = [rng.standard_normal((n, C5_RANK)).astype(np.float32) for n in C5_SHAPE]
    return X, fs


def test_reconstruct_golden(kats):
    for case in kats["cp_reconstruct"]:
        fs = [np.array(f, np.float32) for f in case["factors"]]
        Xh = tb.cp_reconstruct(fs, case["weights"])
        assert list(Xh.shape) == case["shape"], case["src"]
        assert np.array_equal(Xh, np.array(case["expected"], np.float32)), case["src"]


@pytest.mark.parametrize("shape,R", [((7,), 3), ((5, 9), 4), ((33, 17, 5), 7), ((6, 5, 4, 3), 40),
                                     ((70, 3, 2), 16), ((2, 3, 2, 3, 2, 3), 5), ((130, 200), 1)])
@pytest.mark.parametrize("weighted", [False, True])
def test_reconstruct_parity(orc, shape, R, weighted):
    rng = np.random.default_rng(len(shape) * 100 + R)
    fs = [rng.standard_normal((n, R)).astype(np.float32) for n in shape]
    w = rng.random(R).astype(np.float32) if weighted else None
    Xh = tb.cp_reconstruct(fs, w)
    ref = orc.cp_reconstruct([f.astype(np.float64) for f in fs],
                             None if w is None else w.astype(np.float64))
    assert Xh.shape == tuple(shape)
    assert rel_err(Xh, ref) <= 1e-6


def test_reconstruction_grad_golden(kats):
    for case in kats["cp_grad"]:
        fs = [np.array(f, np.float32) for f in case["factors"]]
        g = tb.CpReconstructionGrad(fs, case["weights"])
        outs = g.compute_factor_gradients(np.ones(case["shape"], np.float32))
        assert len(outs) == len(fs)
        for o, f, e in zip(outs, fs, case["expected"]):
            assert o.shape == f.shape
            assert rel_err(o, e) <= 1e-6, case["src"]


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
@pytest.mark.parametrize("shape,R", [((20, 30, 10), 8), ((9, 8, 7, 6), 32), ((40, 64), 5)])
def test_reconstruction_grad_parity(orc, shape, R, precision):
    rng = np.random.default_rng(R)
    fs = [rng.standard_normal((n, R)).astype(np.float32) for n in shape]
    w = rng.random(R).astype(np.float32)
    G = rng.standard_normal(shape).astype(np.float32)
    op = tb.CpReconstructionOp(fs, w, precision)
    outs = op.backward([G])
    ref = orc.cp_reconstruction_grad([f.astype(np.float64) for f in fs], G.astype(np.float64),
                                     w.astype(np.float64))
    for n in range(len(shape)):
        assert rel_err(outs[n], ref[n]) <= 1e-5, (n, rel_err(outs[n], ref[n]))
    (Xh,) = op.forward()
    assert rel_err(Xh, orc.cp_reconstruct([f.astype(np.float64) for f in fs],
                                          w.astype(np.float64))) <= 1e-6
    assert op.name() == "cp_reconstruct" and op.num_inputs() == len(shape)
    assert op.num_outputs() == 1


@pytest.fixture(scope="module")
def c5_reference(orc):
    X, fs = c5_inputs()
    loss, grads = orc.cp_loss_grad_vjp(X, fs, C5_REG)
    return X, fs, loss, grads


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_loss_grad_vs_cpu_vjp(c5_reference, precision):
    X, fs, loss_ref, grads_ref = c5_reference
    loss, grads = tb.cp_loss_grad(X, fs, C5_REG, precision)
    assert abs(loss - loss_ref) <= 1e-6 * abs(loss_ref), (loss, loss_ref)
    for n in range(4):
        assert rel_err(grads[n], grads_ref[n]) <= 1e-5, (n, rel_err(grads[n], grads_ref[n]))


# Routes of the loss/gradient on 3+ mode tensors (trailing-two-modes view
# A x J x K, C = J K). BF16x3: the two-sided contraction (R <= 32, C % 8 == 0)
# with ragged A and C blocks (128), R % 4 != 0, three and five modes and K % 8
# != 0; the three-pass single-layout view (32 < R <= 64); the per-mode path.
# FP32: the 2-way view's two MTTKRPs (R <= 32), else one MTTKRP per mode.
@pytest.mark.parametrize("shape,R", [((10, 9, 8, 16), 7), ((5, 6, 24, 40), 12),
                                     ((3, 4, 5, 6, 16), 8), ((7, 6, 10, 12), 5),
                                     ((6, 5, 8, 16), 40), ((9, 7, 5, 3), 6),
                                     ((200, 24, 56), 16), ((33, 17, 8), 5),
                                     ((40, 24, 56), 48)])
@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_loss_grad_routes(orc, shape, R, precision):
    rng = np.random.default_rng(sum(shape) + R)
    X = rng.standard_normal(shape).astype(np.float32)
    fs = [rng.standard_normal((n, R)).astype(np.float32) for n in shape]
    loss_ref, grads_ref = orc.cp_loss_grad_vjp(X, fs, C5_REG)
    loss, grads = tb.cp_loss_grad(X, fs, C5_REG, precision)
    assert abs(loss - loss_ref) <= 1e-6 * abs(loss_ref), (loss, loss_ref)
    for n in range(len(shape)):
        assert rel_err(grads[n], grads_ref[n]) <= 1e-5, (n, rel_err(grads[n], grads_ref[n]))


def test_vjp_path_matches_gram_form(c5_reference):
    """Residual G = 2(Xhat - X) on the GPU, then the reconstruction adjoint
    (tenrso-ad's rule) on G, plus 2 reg U: the recompute form of the same
    gradient."""
    import torch
    X, fs, loss_ref, grads_ref = c5_reference
    dX = torch.from_numpy(X).cuda()
    dF = [torch.from_numpy(f).cuda() for f in fs]
    dG = torch.empty_like(dX)
    outs = [torch.empty_like(f) for f in dF]
    ptrs = [f.data_ptr() for f in dF]
    torch.cuda.synchronize()  # the library's default context runs on its own stream
    sq = tb.cp_residual_dev(dX.data_ptr(), C5_SHAPE, ptrs, C5_RANK, dG.data_ptr(), alpha=2.0)
    tb.reconstruction_grad_dev(dG.data_ptr(), C5_SHAPE, ptrs, C5_RANK,
                               [o.data_ptr() for o in outs])
    torch.cuda.synchronize()
    loss = sq + C5_REG * sum(float((f.double() ** 2).sum()) for f in dF)
    assert abs(loss - loss_ref) <= 1e-6 * abs(loss_ref)
    for n in range(4):
        g = outs[n].cpu().numpy().astype(np.float64) + 2 * C5_REG * fs[n].astype(np.float64)
        assert rel_err(g, grads_ref[n]) <= 1e-5, n


def test_loss_grad_vs_central_differences(orc, c5_reference):
    """FP64 central differences (h=1e-6) of the loss on 64 seeded entries per
    factor, each from the loss restricted to the slice the entry changes."""
    X, fs, _, _ = c5_reference
    _, grads = tb.cp_loss_grad(X, fs, C5_REG, "fp32")
    rng = np.random.default_rng(0xFD)
    for n in range(4):
        ent = [(int(rng.integers(C5_SHAPE[n])), int(rng.integers(C5_RANK))) for _ in range(64)]
        fd = orc.fd_grad_entries(X, fs, C5_REG, n, ent, h=1e-6)
        an = np.array([grads[n][i, r] for i, r in ent], np.float64)
        assert rel_err(an, fd) <= 1e-5, (n, rel_err(an, fd))


def test_dense_tensor_reuse_and_errors():
    import torch
    X, fs = c5_inputs(7)
    dX = torch.from_numpy(X).cuda()
    dF = [torch.from_numpy(f).cuda() for f in fs]
    gs = [torch.empty_like(f) for f in dF]
    torch.cuda.synchronize()
    d = tb.DenseTensor(dX.data_ptr(), C5_SHAPE, "fp32")
    l1 = d.loss_grad_dev([f.data_ptr() for f in dF], C5_RANK, C5_REG, [g.data_ptr() for g in gs])
    g1 = [g.clone() for g in gs]
    l2 = d.loss_grad_dev([f.data_ptr() for f in dF], C5_RANK, C5_REG, [g.data_ptr() for g in gs])
    # FP64 atomics in the Gram kernel may reorder the last bits between calls
    assert abs(l1 - l2) <= 1e-12 * abs(l1)
    for a, b in zip(g1, gs):
        assert torch.allclose(a, b, rtol=1e-6, atol=0)
    with pytest.raises(tb.TenrsoError, match="Invalid rank"):
        d.loss_grad_dev([f.data_ptr() for f in dF], 0, C5_REG, [g.data_ptr() for g in gs])
    d.close()
