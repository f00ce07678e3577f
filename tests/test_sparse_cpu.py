"""Sparse host-side logic without a GPU: CooTensor construction checks in
tenrso's wording (coo.rs:101-149), CsfTensor mode-order validation through the
C ABI (csf.rs:141-156), and the seeded Zipf COO generator's dedup count."""
import numpy as np
import pytest

import tenrso_b200 as tb
from tenrso_b200 import synth


def test_coo_construction_errors():
    with pytest.raises(tb.CooError, match="Length mismatch: 2 indices but 1 values"):
        tb.CooTensor([[0, 0], [1, 1]], [1.0], [2, 2])
    with pytest.raises(tb.CooError, match="Shape cannot contain zeros"):
        tb.CooTensor([[0, 0]], [1.0], [2, 0])
    with pytest.raises(tb.CooError, match="Shape cannot be empty"):
        tb.CooTensor(np.zeros((0, 0)), [], [])
    with pytest.raises(tb.CooError, match=r"Index out of bounds: index \[0, 5\] exceeds shape"):
        tb.CooTensor([[0, 5]], [1.0], [2, 2])
    coo = tb.CooTensor.zeros([3, 4])
    coo.push([1, 2], 2.0)
    assert coo.nnz() == 1 and coo.density() == pytest.approx(1 / 12)
    with pytest.raises(tb.CooError, match="Index out of bounds"):
        coo.push([3, 0], 1.0)


def test_csf_mode_order_errors_without_device():
    coo = tb.CooTensor.zeros([3, 3, 3])
    with pytest.raises(tb.CsfError, match=r"mode_order length 2 != ndim 3"):
        tb.CsfTensor.from_coo(coo, [0, 1])
    with pytest.raises(tb.CsfError, match=r"mode_order \[0, 0, 1\] is not a permutation of 0..3"):
        tb.CsfTensor.from_coo(coo, [0, 0, 1])
    csf = tb.CsfTensor.from_coo(coo, [2, 0, 1])  # empty: no device work
    assert csf.nnz() == 0 and csf.mode_order() == [2, 0, 1]


def test_zipf_coo_dedups_to_exact_nnz(orc):
    shape = (1000, 800, 100)
    idx, vals, dups = synth.zipf_coo(shape, 20000, seed=0xC3)
    oi, ov = orc.coo_deduplicate(idx, vals)
    assert oi.shape[0] == 20000
    assert idx.shape[0] == 20000 + dups
    # Zipf(1.2): the most frequent root index holds a large share
    counts = np.bincount(idx[:, 0], minlength=shape[0])
    assert counts.max() > 0.05 * idx.shape[0]
