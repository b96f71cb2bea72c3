"""The pipeline at two of the benchmark's configurations, end to end through the C ABI,
against the oracle:

- C1: 2,700 cells x 32,738 genes of u32 counts (negative binomial, log-normal gene means
  mu 0.5, sigma 1.5, dispersion 0.2, about 2.5% dense), normalize_total(1e4) -> log1p ->
  seurat HVG top 2,000 -> PCA 50 (seed 0) -> exact kNN (n_neighbors 15);
- C2: 100,000 cells x 20,000 genes (about 2,000 stored counts a cell, gene means mu 0,
  sigma 1.5, dispersion 0.3, 20 planted cell types each shifting 200 genes), the same
  pipeline with the PCA's input pushed in blocks of 8,192 cells.

Bars: HVG flags equal to the oracle's (the device moments carry the oracle's bits);
singular values within 1e-4 relative of the f64 oracle PCA; the kNN of the oracle's
embedding (kyto's parity rule: the same embedding input) equal to the oracle's exact
search bit for bit, indices and f32 distances. Seeded synthetic counts stand in for the
benchmark's data (its shapes and distributions)."""

import numpy as np
import pytest

import kyto_b200 as K
from kyto_b200 import synthetic
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return K.Context(0)


def _pipeline(ctx, x, n_top, block_cells=None):
    n_genes = x.n_genes
    hv = K.highly_variable_genes(x.indptr, x.indices, x.values, n_genes, n_top, ctx=ctx)
    logx = O.normalize_log1p(O.Csr(x.indptr, x.indices, x.values, n_genes))
    s, q, p = O.hvg_moments(logx)
    flags = O.hvg_seurat(s, q, p, x.n_cells, n_top)[3]
    assert np.array_equal(hv.highly_variable, flags)
    assert flags.sum() >= n_top
    res = K.pca(x.indptr, x.indices, x.values, n_genes, 50, seed=0, gene_set=flags,
                target_sum=1e4, log1p=True, block_cells=block_cells, ctx=ctx)
    ref = O.pca(logx, 50, 0, gene_set=flags)
    sv = np.abs(np.sqrt(res.variance) - np.sqrt(ref.variance)) / np.sqrt(ref.variance)
    assert sv.max() <= 1e-4, sv.max()
    assert res.passes_run == ref.passes_run
    return res, ref


def _knn_bits(ctx, emb):
    g = K.neighbors(emb, 15, ctx=ctx)
    keys, rows, _ = O.knn_ranked(emb, 15, "exact")
    o = O.ranked_to_graph(keys, rows)
    assert np.array_equal(g.indptr, o.indptr)
    assert np.array_equal(g.indices, o.indices)
    assert np.array_equal(g.distances.view(np.uint32), o.distances.view(np.uint32))


def test_c1_counts_hvg_pca_knn(ctx):
    x = synthetic.counts_csr(2700, 32738, 0.025 * 32738, 1, 0, mu=0.5, sigma=1.5,
                             dispersion=0.2, seed=0)
    density = x.nnz / (2700 * 32738)
    assert 0.015 <= density <= 0.035, density
    res, ref = _pipeline(ctx, x, 2000)
    _knn_bits(ctx, ref.embedding)


def test_c2_streamed_in_blocks(ctx):
    x = synthetic.counts_csr(100_000, 20_000, 2000.0, 20, 200, mu=0.0, sigma=1.5,
                             dispersion=0.3, seed=2)
    assert 1500 <= x.nnz / x.n_cells <= 2500
    res, ref = _pipeline(ctx, x, 2000, block_cells=8192)
    # One push or 13 blocks of 8,192 cells: the same bits (the held input is one matrix).
    flags = np.zeros(x.n_genes, dtype=bool)
    flags[np.flatnonzero(np.any(res.loadings != 0, axis=1))] = True
    one = K.pca(x.indptr, x.indices, x.values, x.n_genes, 50, seed=0, gene_set=flags,
                target_sum=1e4, log1p=True, ctx=ctx)
    assert np.array_equal(one.embedding.view(np.uint32), res.embedding.view(np.uint32))
    _knn_bits(ctx, ref.embedding)
