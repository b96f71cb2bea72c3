"""The PCA's tensor-core products (S D through the blocked layout: column masks, values
as fp16 hi/lo pairs of the scaled value, kind::f16 MMAs with A in tensor memory and f64
flushes), one at a time through kg_diag_spmm, against a plain f64 product.

Bar: |device - f64| <= 2^-15 sum |s| |d| per entry (both operands to about 2^-22 in their
fp16 parts; f32 sums of at most 512 products between f64 flushes), and counts (the ones
mode) exact. A layout or indexing fault shows as an O(1) error. Shapes cover ragged tiles
(rows not a multiple of 128, columns not a multiple of 32), empty rows and blocks, fully
dense rows, values over six decades, and K split over several 16,384-wide segments."""

import numpy as np
import pytest

import kyto_b200 as K
from kyto_b200 import synthetic

pytestmark = pytest.mark.gpu


def _dense(indptr, indices, values, n_cols):
    n = len(indptr) - 1
    m = np.zeros((n, n_cols))
    rows = np.repeat(np.arange(n), np.diff(indptr).astype(np.int64))
    m[rows, indices.astype(np.int64)] = values.astype(np.float64)
    return m


def _check(got, s, d):
    ref = s @ d
    bound = (np.abs(s) @ np.abs(d)) * 2.0**-15 + 1e-300
    err = np.abs(got - ref)
    assert np.all(err <= bound), float(np.max(err / bound))


@pytest.fixture(scope="module")
def log1p_cells():
    return synthetic.log1p_csr(20_000, 700, 120, 5, 50, seed=11, device="cpu")


@pytest.mark.parametrize("transposed", [False, True])
def test_product_matches_f64(log1p_cells, transposed):
    x = log1p_cells
    s = _dense(x.indptr, x.indices, x.values, x.n_genes)
    s = s.T if transposed else s
    rng = np.random.default_rng(3 + transposed)
    d = rng.uniform(-1.0, 1.0, (s.shape[1], 60))
    got = K.product(x.indptr, x.indices, x.values, x.n_genes, d, transposed)
    assert got.shape == (s.shape[0], 60)
    _check(got, s, d)


def _ragged():
    """300 x 77: empty rows, a fully dense row, an empty column block, wide values."""
    rng = np.random.default_rng(5)
    n, g = 300, 77
    dense = (rng.random((n, g)) < 0.3) * np.exp(rng.uniform(np.log(1e-3), np.log(1e3), (n, g)))
    dense[10] = 0.0                      # empty rows
    dense[200:210] = 0.0
    dense[42] = rng.uniform(0.5, 2.0, g)  # a fully dense row
    dense[128:256, 32:64] = 0.0          # an empty block (tile 1, chunk 1)
    dense[:, 70] = rng.uniform(1.0, 2.0, n)  # a full column in the last, ragged chunk
    indptr = np.zeros(n + 1, dtype=np.uint64)
    idx, val = [], []
    for r in range(n):
        nz = np.flatnonzero(dense[r])
        idx.append(nz.astype(np.uint32))
        val.append(dense[r, nz].astype(np.float32))
        indptr[r + 1] = indptr[r] + len(nz)
    vals = np.concatenate(val)
    return indptr, np.concatenate(idx), vals, g, _dense(indptr, np.concatenate(idx), vals, g)


@pytest.mark.parametrize("transposed", [False, True])
def test_ragged_edges_and_value_modes(transposed):
    indptr, idx, vals, g, s = _ragged()
    s = s.T if transposed else s
    rows, k = s.shape
    rng = np.random.default_rng(9)
    d = rng.uniform(-3.0, 3.0, (k, 64))
    _check(K.product(indptr, idx, vals, g, d, transposed), s, d)
    # Ones: each row's stored values counted, exactly.
    ones = K.product(indptr, idx, vals, g, None, transposed, value_mode=2)
    assert np.array_equal(ones[:, 0], (s != 0).sum(axis=1).astype(np.float64))
    # Centred squares over the stored values: sum of (v - mean_row)^2 where v is stored.
    means = rng.uniform(0.0, 5.0, rows)
    sq = K.product(indptr, idx, vals, g, None, transposed, value_mode=1, row_means=means)
    stored = s != 0
    want = np.where(stored, (s - means[:, None]) ** 2, 0.0).sum(axis=1)
    scale = np.where(stored, (np.abs(s) + means[:, None]) ** 2, 0.0).sum(axis=1)
    assert np.all(np.abs(sq[:, 0] - want) <= scale * 2.0**-14 + 1e-300)


def test_a_single_row_and_column():
    indptr = np.array([0, 1], dtype=np.uint64)
    idx = np.array([0], dtype=np.uint32)
    vals = np.array([2.5], dtype=np.float32)
    d = np.array([[0.75, -1.0]])
    got = K.product(indptr, idx, vals, 1, d, False)
    assert np.array_equal(got, np.array([[1.875, -2.5]]))
