"""The FP64 inverse that the CP-ALS solve applies (tsr_gram_inverse_f64, the
2 x 2-block Gauss-Jordan kernel standing in for solve_least_squares' lstsq,
cp/helpers.rs:455-495) against numpy's FP64 inverse.

Tolerance: relative Frobenius error of G^-1 at most 1e-12 * cond(G) (FP64
elimination on the unit-diagonal scaled matrix); the ridge retry and the
not-SPD report follow helpers.rs:477-490."""
import numpy as np
import pytest

import tenrso_b200 as tb

pytestmark = pytest.mark.gpu


def spd(R, rows, seed, corr=0.0):
    rng = np.random.default_rng(seed)
    F = rng.random((rows, R))
    if corr:
        F[:, 1:] = (1 - corr) * F[:, 1:] + corr * F[:, :1]
    return F.T @ F


@pytest.mark.parametrize("R", [1, 2, 3, 5, 16, 17, 31, 32, 33, 48, 63, 64, 65, 100, 112])
def test_gram_inverse_matches_numpy(R):
    for seed, corr in ((R, 0.0), (R + 1000, 0.9)):
        G = spd(R, 3 * R + 7, seed, corr)
        inv, ridge, _ = tb.gram_inverse(G)
        ref = np.linalg.inv(G)
        cond = np.linalg.cond(G)
        err = np.linalg.norm(inv - ref) / np.linalg.norm(ref)
        assert ridge == 0
        assert err <= 1e-12 * max(cond, 1.0), (R, corr, err, cond)


def test_gram_inverse_hadamard_of_factor_grams():
    """The matrices CP-ALS inverts: Hadamards of factor Grams (256 x 64 U(0,1))."""
    rng = np.random.default_rng(7)
    A, B = rng.random((256, 64)), rng.random((256, 64))
    G = (A.T @ A) * (B.T @ B)
    inv, ridge, ms = tb.gram_inverse(G, iters=20)
    ref = np.linalg.inv(G)
    assert ridge == 0
    assert np.linalg.norm(inv - ref) / np.linalg.norm(ref) <= 1e-12 * np.linalg.cond(G)
    print(f"inverse R=64: {ms * 1e3:.2f} us per launch")


def test_gram_inverse_singular_takes_the_ridge():
    """Rank-deficient G (duplicated columns): not SPD as given, so the
    eps*rank*10 ridge is added as in solve_least_squares; the result inverts
    G + ridge*I."""
    a = np.ones((6, 1))
    F = np.hstack([a, a, np.arange(6.0)[:, None]])
    G = F.T @ F
    inv, ridge, _ = tb.gram_inverse(G)
    assert ridge in (1, 2)
    eps = np.finfo(np.float32).eps * 3 * 10
    scale = 1.0 if ridge == 1 else np.mean(np.abs(np.diag(G)))
    ref = np.linalg.inv(G + eps * max(scale, 1.0) * np.eye(3))
    assert np.linalg.norm(inv - ref) / np.linalg.norm(ref) <= 1e-6


def test_gram_inverse_not_spd_reports():
    G = -np.eye(4)
    with pytest.raises(tb.TenrsoError) as e:
        tb.gram_inverse(G)
    assert e.value.code == "TSR_E_NOT_SPD"
