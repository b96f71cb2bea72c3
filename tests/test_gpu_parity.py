"""Parity of the CUDA path (through the C ABI) with the oracle and kyto's goldens.

Bars: normalize/log1p, HVG moments and flags, and every kNN row (indices and f32
distances) bit for bit; PCA within kyto's own GPU-vs-CPU agreement bar, tightened:
singular values (variances) 1e-6 relative to the FP64 oracle (the product path
accumulates in f64), loadings/embedding columns 1e-5 of their largest value.
"""

import json

import numpy as np
import pytest

import kyto_b200 as K
from kyto_b200 import synthetic
from oracle import oracle as O
from tests.conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return K.Context(0)


@pytest.fixture(scope="module")
def counts():
    g = load_golden("synthetic_counts")
    return O.Csr(g["indptr"], g["indices"], g["counts"], int(g["n_genes"][0]))


def test_normalize_log1p_bits(ctx, counts):
    gold = load_golden("synthetic_normalize_log1p")
    norm = K.normalize_log1p(counts.indptr, counts.values, 1e4, False, ctx=ctx)
    assert np.array_equal(norm.view(np.uint32), gold["normalized"].view(np.uint32))
    gpu = K.normalize_log1p(counts.indptr, counts.values, 1e4, True, ctx=ctx)
    cpu = O.normalize_log1p(counts, 1e4, True).values
    assert np.array_equal(gpu.view(np.uint32), cpu.view(np.uint32))


def test_normalize_f32_values_and_empty_rows(ctx):
    rng = np.random.default_rng(3)
    x = synthetic.counts_csr(300, 500, 40, 3, 20, seed=3, device="cpu")
    vals = (x.values.astype(np.float32) * rng.uniform(0.1, 3.0, x.nnz).astype(np.float32))
    # Empty rows (no counts) keep divisor 1.
    indptr = x.indptr.copy()
    gpu = K.normalize_log1p(indptr, vals, 1e4, True, ctx=ctx)
    cpu = O.normalize_log1p(O.Csr(indptr, x.indices, vals, x.n_genes), 1e4, True).values
    assert np.array_equal(gpu.view(np.uint32), cpu.view(np.uint32))


def test_hvg_moments_and_flags(ctx, counts):
    gold = load_golden("synthetic_hvg")
    res = K.highly_variable_genes(counts.indptr, counts.indices, counts.values, counts.n_genes,
                                  n_top_genes=100, ctx=ctx)
    assert np.array_equal(res.highly_variable, gold["highly_variable"])
    log1p = O.normalize_log1p(counts)
    s, q, p = O.hvg_moments(log1p)
    # The moments carry the oracle's bits (each gene's cells summed in cell order).
    n = counts.n_genes
    gs, gq, gp = np.empty(n), np.empty(n), np.empty(n, dtype=np.uint64)
    K._check(K.library().kg_hvg_moments(
        ctx.handle, K._ptr(counts.indptr), K._ptr(counts.indices), K._ptr(counts.values),
        K.KG_U32, counts.n_rows, n, 1e4, 1, K._ptr(gs), K._ptr(gq), K._ptr(gp)))
    assert np.array_equal(gs.view(np.uint64), s.view(np.uint64))
    assert np.array_equal(gq.view(np.uint64), q.view(np.uint64))
    assert np.array_equal(gp, p)
    # The derived statistics go through the host's libm (log, log1p): to its ulps.
    om, od, on, of = O.hvg_seurat(s, q, p, counts.n_rows, 100)
    np.testing.assert_allclose(res.means, om, rtol=1e-15, atol=0)
    fin = np.isfinite(on)
    np.testing.assert_allclose(res.dispersions_norm[fin], on[fin], rtol=1e-12, atol=1e-15)


def _col_diff(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


# The two product engines: tensor cores (fp16 hi/lo parts, f32 sums of at most 512 terms
# flushed into f64) and the SIMT pipes (f64 throughout). Bars against the FP64 oracle:
# variances (singular values squared) and loadings/embedding columns.
PRODUCTS = {"tc": (2e-5, 2e-4), "simt": (1e-6, 1e-5)}


@pytest.fixture(params=sorted(PRODUCTS))
def products(request, monkeypatch):
    monkeypatch.setenv("KYTO_GPU_PCA_PRODUCTS", request.param)
    return PRODUCTS[request.param]


def _angle(a, b):
    qa, _ = np.linalg.qr(a.astype(np.float64))
    qb, _ = np.linalg.qr(b.astype(np.float64))
    s = np.linalg.svd(qa.T @ qb, compute_uv=False)
    return float(np.arccos(np.clip(s.min(), -1.0, 1.0)))


def test_pca_synthetic_golden(ctx, counts, products):
    var_tol, col_tol = products
    hv = load_golden("synthetic_hvg")["highly_variable"]
    gold = load_golden("synthetic_pca")
    res = K.pca(counts.indptr, counts.indices, counts.values, counts.n_genes, 20, seed=0,
                gene_set=hv, target_sum=1e4, log1p=True, ctx=ctx)
    assert np.max(np.abs(res.variance - gold["variance"]) / gold["variance"]) <= 1e-3
    ref = O.pca(O.normalize_log1p(counts), 20, 0, gene_set=hv)
    assert np.max(np.abs(res.variance - ref.variance) / ref.variance) <= var_tol
    for c in range(20):
        assert _col_diff(res.loadings[:, c], ref.loadings[:, c]) <= col_tol
        assert _col_diff(res.embedding[:, c], ref.embedding[:, c]) <= col_tol
    assert res.passes_run == ref.passes_run


@pytest.fixture(scope="module")
def planted():
    x = synthetic.counts_csr(6000, 3000, 300, 12, 100, seed=1, dispersion=0.3)
    return x


def test_pca_planted_with_hvg_matches_oracle(ctx, planted, products):
    var_tol, col_tol = products
    x = planted
    hv = K.highly_variable_genes(x.indptr, x.indices, x.values, x.n_genes, 1000, ctx=ctx)
    logx = O.normalize_log1p(O.Csr(x.indptr, x.indices, x.values, x.n_genes))
    s, q, p = O.hvg_moments(logx)
    assert np.array_equal(hv.highly_variable, O.hvg_seurat(s, q, p, x.n_cells, 1000)[3])
    res = K.pca(x.indptr, x.indices, x.values, x.n_genes, 50, seed=0,
                gene_set=hv.highly_variable, target_sum=1e4, log1p=True, ctx=ctx)
    ref = O.pca(logx, 50, 0, gene_set=hv.highly_variable)
    rel = np.abs(res.variance - ref.variance) / ref.variance
    assert rel.max() <= var_tol, rel.max()
    assert np.allclose(res.variance_ratio, ref.variance_ratio, rtol=var_tol)
    for c in range(10):
        assert _col_diff(res.embedding[:, c], ref.embedding[:, c]) <= col_tol
    assert _angle(res.loadings[hv.highly_variable][:, :10],
                  ref.loadings[hv.highly_variable][:, :10]) <= 1e-3


def test_pca_blocks_give_the_same_bits(ctx, planted):
    x = planted
    one = K.pca(x.indptr, x.indices, x.values, x.n_genes, 20, target_sum=1e4, log1p=True, ctx=ctx)
    blocks = K.pca(x.indptr, x.indices, x.values, x.n_genes, 20, target_sum=1e4, log1p=True,
                   block_cells=37, ctx=ctx)
    again = K.pca(x.indptr, x.indices, x.values, x.n_genes, 20, target_sum=1e4, log1p=True, ctx=ctx)
    assert np.array_equal(one.embedding, blocks.embedding)
    assert np.array_equal(one.embedding, again.embedding)
    assert np.array_equal(one.variance, again.variance)


def test_pca_refusals(ctx):
    indptr = np.array([0, 1], dtype=np.uint64)
    with pytest.raises(K.KytoError) as e:
        K.pca(indptr, np.array([0], np.uint32), np.array([1.0], np.float32), 3, 1, ctx=ctx)
    assert e.value.code == "KY-E215"
    indptr = np.array([0, 1, 2], dtype=np.uint64)
    with pytest.raises(K.KytoError):
        K.pca(indptr, np.array([0, 1], np.uint32), np.array([1.0, 2.0], np.float32), 3, 3, ctx=ctx)
    with pytest.raises(K.KytoError):
        K.pca(indptr, np.array([0, 1], np.uint32), np.array([1.0, np.nan], np.float32), 3, 1,
              ctx=ctx)


@pytest.mark.parametrize("offset", [1e6, 1e7])
def test_pca_large_means_are_centred_row_by_row(ctx, offset):
    # kyto's tests/it/pca.rs:486-506: values * 8 + offset, a rank-3 spread. The
    # tensor-core products cannot resolve the spread under such means, so the session
    # takes the f64 products; the result must still match the f64 oracle.
    rng = np.random.default_rng(int(offset) % 97)
    basis = rng.normal(size=(3, 12))
    dense = (rng.normal(size=(200, 3)) @ basis + 0.01 * rng.normal(size=(200, 12))) * 8 + offset
    dense = dense.astype(np.float32)
    indptr = np.arange(0, 201 * 12, 12, dtype=np.uint64)
    idx = np.tile(np.arange(12, dtype=np.uint32), 200)
    vals = dense.reshape(-1)
    res = K.pca(indptr, idx, vals, 12, 3, ctx=ctx)
    ref = O.pca(O.Csr(indptr, idx, vals, 12), 3)
    assert np.max(np.abs(res.variance - ref.variance) / ref.variance) <= 1e-6
    for c in range(3):
        assert _col_diff(res.embedding[:, c], ref.embedding[:, c]) <= 1e-5


def test_pca_rank_deficient_completes_loadings(ctx, products):
    # Two distinct cells: one direction of variance; kyto completes the loadings with
    # orthonormal zero-variance directions (pca_dense.rs complement).
    var_tol, _ = products
    indptr = np.array([0, 2, 4, 6], dtype=np.uint64)
    idx = np.array([0, 1, 0, 1, 0, 1], dtype=np.uint32)
    val = np.array([1, 2, 1, 2, 3, 1], dtype=np.float32)
    res = K.pca(indptr, idx, val, 4, 3, ctx=ctx)
    ref = O.pca(O.Csr(indptr, idx, val, 4), 3)
    np.testing.assert_allclose(res.variance, ref.variance, rtol=var_tol,
                               atol=1e-12 * ref.variance[0])
    l = res.loadings.astype(np.float64)
    np.testing.assert_allclose(l.T @ l, np.eye(3), atol=1e-6)


def _graph_equal(gpu: K.Graph, cpu: O.Graph):
    assert np.array_equal(gpu.indptr, cpu.indptr)
    assert np.array_equal(gpu.indices, cpu.indices)
    assert np.array_equal(gpu.distances.view(np.uint32), cpu.distances.view(np.uint32))


def test_knn_pbmc3k_bits_and_scanpy(ctx):
    g = load_golden("pbmc3k_neighbors")
    gpu = K.neighbors(g["embedding"], 15, ctx=ctx)
    _graph_equal(gpu, O.neighbors(g["embedding"], 15))
    assert np.array_equal(gpu.indices.astype(np.int64), g["indices"])


def test_knn_synthetic_duplicates(ctx):
    emb = load_golden("synthetic_pca")["embedding"]
    _graph_equal(K.neighbors(emb, 15, ctx=ctx), O.neighbors(emb, 15))


def test_knn_clusters_ties_and_duplicates(ctx):
    pts, _ = synthetic.gaussian_mixture(6000, 50, 40, seed=5, device="cpu")
    pts[100:140] = pts[7]  # a block of exact duplicates (ties past the candidates)
    pts[200:230] = np.round(pts[200:230])
    _graph_equal(K.neighbors(pts, 31, ctx=ctx), O.neighbors(pts, 31))


@pytest.mark.parametrize("candidate_filter", ["fp16", "split", "bf16", "simt"])
def test_knn_every_filter_gives_the_exact_graph(ctx, monkeypatch, candidate_filter):
    # The tensor-core filter in fp16, split fp16 (hi and lo parts, a tighter slack) or
    # bf16 (wider slack, more candidates) and the SIMT f32 filter all end in the same
    # exact ranking.
    monkeypatch.setenv("KYTO_GPU_KNN_FILTER", candidate_filter)
    pts, _ = synthetic.gaussian_mixture(5000, 50, 30, seed=11, device="cpu")
    pts[40:60] = pts[3]
    gpu = K.neighbors(pts, 16, ctx=ctx)
    _graph_equal(gpu, O.neighbors(pts, 16))
    assert gpu.stats.candidates >= 5000 * 15


@pytest.mark.parametrize("candidate_filter", ["fp16", "split"])
def test_knn_tensor_core_tiles_past_the_end(ctx, monkeypatch, candidate_filter):
    # n not a multiple of the 128-point tile or the query block; one CTA per SM walks
    # several query blocks (more blocks than SMs).
    monkeypatch.setenv("KYTO_GPU_KNN_FILTER", candidate_filter)
    pts, _ = synthetic.gaussian_mixture(148 * 256 + 77, 12, 25, seed=12, device="cpu")
    _graph_equal(K.neighbors(pts, 10, ctx=ctx), O.neighbors(pts, 10))


def test_knn_split_filter_keeps_tight_clusters_off_the_full_search(ctx, monkeypatch):
    # Components with sigma 0.2 hold hundreds of points inside fp16's slack (2^-9 of
    # |q| R), so their queries overflow the 512 candidate slots and go through the
    # overflow retry (every tile, the tiles split into ranges between copies of the
    # overflowed queries and the copies' candidates merged); the split operands' slack (about 2^-14 of
    # |q| R) keeps them near k. Same graph either way, and no row searched in full.
    pts, _ = synthetic.gaussian_mixture(20_000, 50, 40, seed=13, device="cpu")
    ref = O.neighbors(pts, 15)
    stats = {}
    for f in ("fp16", "split"):
        monkeypatch.setenv("KYTO_GPU_KNN_FILTER", f)
        g = K.neighbors(pts, 15, ctx=ctx)
        _graph_equal(g, ref)
        stats[f] = g.stats
    assert stats["split"].candidates * 2 < stats["fp16"].candidates, (
        stats["split"].candidates, stats["fp16"].candidates)
    assert stats["split"].rows_full == 0 and stats["fp16"].rows_full == 0
    # Without a choice the filter kind is tuned on the data (a pilot of both kinds).
    monkeypatch.delenv("KYTO_GPU_KNN_FILTER")
    g = K.neighbors(pts, 15, ctx=ctx)
    _graph_equal(g, ref)
    assert g.stats.rows_full == 0


@pytest.mark.parametrize("candidate_filter", ["fp16", "split"])
def test_knn_bounds_skip_far_tiles_and_keep_the_graph(ctx, monkeypatch, candidate_filter):
    # Well-separated clusters: the bounded scan (rows by k-means part, each query block's
    # tiles nearest first) proves most tiles hold no neighbour of the block and skips
    # them; the same order without bounds, and the Morton order, scan every tile. All
    # three give the oracle's graph.
    monkeypatch.setenv("KYTO_GPU_KNN_FILTER", candidate_filter)
    pts, _ = synthetic.gaussian_mixture(30_000, 50, 24, spread=6.0, seed=21, device="cpu")
    ref = O.neighbors(pts, 15)
    got = {}
    for order in ("bounded", "cluster", "morton"):
        monkeypatch.setenv("KYTO_GPU_KNN_ORDER", order)
        g = K.neighbors(pts, 15, ctx=ctx)
        _graph_equal(g, ref)
        got[order] = g.stats
    total = got["bounded"].tiles_total
    assert total == ((30_000 + 255) // 256) * ((30_000 + 127) // 128)
    assert got["cluster"].tiles_scanned == total and got["morton"].tiles_scanned == total
    assert 0 < got["bounded"].tiles_scanned < total // 2, (got["bounded"].tiles_scanned, total)


@pytest.mark.parametrize("n_neighbors,n_components", [(2, None), (16, 7), (64, 1)])
def test_knn_edges(ctx, n_neighbors, n_components):
    pts, _ = synthetic.gaussian_mixture(1500, 50, 10, seed=9, device="cpu")
    ref_pts = pts if n_components is None else pts[:, :n_components]
    gpu = K.neighbors(pts, n_neighbors, n_components, ctx=ctx)
    _graph_equal(gpu, O.neighbors(ref_pts, n_neighbors))


def test_knn_every_row_a_neighbour(ctx):
    pts, _ = synthetic.gaussian_mixture(97, 20, 3, seed=2, device="cpu")
    _graph_equal(K.neighbors(pts, 97, ctx=ctx), O.neighbors(pts, 97))


def test_knn_line_known_answer(ctx):
    g = K.neighbors(np.array([[0.0], [1.0], [3.0], [7.0]], np.float32), 3, ctx=ctx)
    assert g.indices.tolist() == [1, 2, 0, 2, 0, 1, 1, 2]
    assert g.distances.tolist() == [1.0, 3.0, 1.0, 2.0, 3.0, 2.0, 6.0, 4.0]


def test_knn_refusals(ctx):
    pts = np.zeros((5, 3), np.float32)
    for bad in (1, 6):
        with pytest.raises(K.KytoError) as e:
            K.neighbors(pts, bad, ctx=ctx)
        assert e.value.code == "KY-E215"
    pts[2, 1] = np.nan
    with pytest.raises(K.KytoError) as e:
        K.neighbors(pts, 2, ctx=ctx)
    assert "row 2, component 1" in str(e.value)


def test_knn_huge_norms_search_every_row(ctx):
    pts, _ = synthetic.gaussian_mixture(300, 8, 3, seed=4, device="cpu")
    pts[5] = 1e18
    gpu = K.neighbors(pts, 5, ctx=ctx)
    _graph_equal(gpu, O.neighbors(pts, 5))


@pytest.mark.parametrize("candidate_filter", ["fp16", "split"])
def test_knn_batch_equals_each_sample_alone(ctx, monkeypatch, candidate_filter):
    # Samples of uneven sizes (not multiples of the 128-row tile or the 256-row query
    # block, one as small as n_neighbors) searched in one launch: every sample's graph
    # equals the exact search of that sample alone, with columns numbered from its own
    # first row.
    monkeypatch.setenv("KYTO_GPU_KNN_FILTER", candidate_filter)
    rng = np.random.default_rng(21)
    sizes = [16, 300, 1000, 2049, 77, 5000, 130]
    samples = []
    for i, m in enumerate(sizes):
        pts, _ = synthetic.gaussian_mixture(m, 30, 5, seed=30 + i, device="cpu")
        samples.append(pts + rng.normal(0, 5, 30).astype(np.float32))  # each its own offset
    samples[2][10:20] = samples[2][3]  # duplicates inside one sample
    graphs = K.neighbors_batch(samples, 16, ctx=ctx)
    assert len(graphs) == len(samples)
    for pts, g in zip(samples, graphs):
        _graph_equal(g, O.neighbors(pts, 16))


def test_knn_batch_refusals(ctx):
    small = np.zeros((4, 3), np.float32)
    with pytest.raises(K.KytoError) as e:
        K.neighbors_batch([np.ones((40, 3), np.float32), small], 5, ctx=ctx)
    assert e.value.code == "KY-E215" and "sample 1" in str(e.value)


def test_pca_neighbors_batch_equals_each_sample_alone(ctx):
    # The batching form: samples of uneven sizes, PCA 30 + kNN 15 each, sessions run side
    # by side and one batched search; each sample's embedding, variances and graph equal
    # the single-sample calls' bit for bit.
    sizes = [500, 3100, 257, 1200, 9000, 640]
    samples = []
    for i, m in enumerate(sizes):
        x = synthetic.counts_csr(m, 400, 40, 4, 30, seed=50 + i, device="cpu")
        samples.append((x.indptr, x.indices, x.values))
    out, stats = K.pca_neighbors_batch(samples, 400, 30, 15, seed=0, target_sum=1e4, log1p=True,
                                       ctx=ctx)
    assert stats.workers == len(sizes)
    for (indptr, idx, vals), (res, g) in zip(samples, out):
        one = K.pca(indptr, idx, vals, 400, 30, seed=0, target_sum=1e4, log1p=True, ctx=ctx)
        assert np.array_equal(res.embedding.view(np.uint32), one.embedding.view(np.uint32))
        assert np.array_equal(res.variance.view(np.uint64), one.variance.view(np.uint64))
        _graph_equal(g, K.neighbors(one.embedding, 15, ctx=ctx))


def test_pca_neighbors_batch_stages_large_host_blocks(ctx):
    # Samples whose index and value arrays pass 4 MB are copied by the batching workers
    # through page-locked staging buffers (16 MB halves, the second sample spanning
    # several); the results equal the single-sample calls' (the driver's own copies)
    # bit for bit.
    samples = []
    for i, (m, per_cell) in enumerate([(20_000, 60), (70_000, 80), (700, 40)]):
        x = synthetic.counts_csr(m, 400, per_cell, 4, 30, seed=80 + i, device="cpu")
        samples.append((x.indptr, x.indices, x.values))
    assert samples[1][2].nbytes > (16 << 20)
    out, _ = K.pca_neighbors_batch(samples, 400, 20, 10, seed=0, target_sum=1e4, log1p=True,
                                   ctx=ctx)
    for (indptr, idx, vals), (res, g) in zip(samples, out):
        one = K.pca(indptr, idx, vals, 400, 20, seed=0, target_sum=1e4, log1p=True, ctx=ctx)
        assert np.array_equal(res.embedding.view(np.uint32), one.embedding.view(np.uint32))
        assert np.array_equal(res.variance.view(np.uint64), one.variance.view(np.uint64))
        _graph_equal(g, K.neighbors(one.embedding, 10, ctx=ctx))


# ------------------------------------------------------------ connectivities ----------

from oracle import connectivities as OC  # noqa: E402


def _conn_equal_edges(gpu, ref):
    assert np.array_equal(gpu.indptr, np.asarray(ref[0], dtype=np.uint64))
    assert np.array_equal(gpu.indices, np.asarray(ref[1], dtype=np.uint32))


@pytest.mark.parametrize("name", ["synthetic", "pbmc3k"])
def test_connectivities_match_scanpy_and_the_oracle(ctx, name):
    # Scanpy's own distance graph in (kyto's connectivities_parity.rs): the same edges as
    # scanpy's connectivities, weights within 1e-5, and the oracle's weights.
    g = load_golden(f"{name}_connectivities")
    ip = g["dist_indptr"].astype(np.uint64)
    k = int(ip[1] - ip[0])
    graph = K.Graph(ip, g["dist_indices"].astype(np.uint32), g["dist_data"].astype(np.float32))
    gpu = K.connectivities(graph, ctx=ctx)
    _conn_equal_edges(gpu, (g["indptr"], g["indices"]))
    assert np.abs(gpu.weights.astype(np.float64) - g["weights"]).max() <= 1e-5
    ref = OC.connectivities(ip, graph.indices, graph.distances, k + 1)
    _conn_equal_edges(gpu, ref)
    assert np.abs(gpu.weights.astype(np.float64) - ref[2]).max() <= 1e-6
    assert (gpu.weights.view(np.uint32) == ref[2].view(np.uint32)).mean() > 0.999


def test_connectivities_known_answers_on_the_device(ctx):
    # kyto's connectivities.rs in-file cases (:279-397) through the C ABI.
    def graph(rows):
        k = len(rows[0])
        return K.Graph(np.arange(len(rows) + 1, dtype=np.uint64) * k,
                       np.array([c for row in rows for c, _ in row], dtype=np.uint32),
                       np.array([d for row in rows for _, d in row], dtype=np.float32))

    line = K.connectivities(graph([[(1, 1.0), (2, 3.0)], [(0, 1.0), (2, 2.0)],
                                   [(0, 3.0), (1, 2.0)]]), ctx=ctx)
    assert line.indptr.tolist() == [0, 2, 4, 6] and line.indices.tolist() == [1, 2, 0, 2, 0, 1]
    assert line.weights[0] == 1.0 and 0.0 < line.weights[1] < 1.0
    same = K.connectivities(graph([[(1, 0.0), (2, 0.0)], [(0, 0.0), (2, 0.0)],
                                   [(0, 0.0), (1, 0.0)]]), ctx=ctx)
    assert same.weights.tolist() == [1.0] * 6
    far = K.connectivities(graph([[(1, 1.0), (2, 1.0), (3, 1e6)], [(0, 1.0), (2, 1.0), (3, 1.0)],
                                  [(0, 1.0), (1, 1.0), (3, 1.0)],
                                  [(0, 1e6), (1, 1.0), (2, 1.0)]]), ctx=ctx)
    assert far.indptr.tolist() == [0, 2, 5, 8, 10]
    assert far.indices.tolist() == [1, 2, 0, 2, 3, 0, 1, 3, 1, 2]


def test_connectivities_of_the_device_graph_with_duplicate_groups(ctx):
    # A 20,000-row graph from the device search, with a group of 30 identical rows (their
    # distances all 0: rho 0, the global floor) and rows listing ties: the oracle's edges
    # and weights.
    pts, _ = synthetic.gaussian_mixture(20_000, 30, 25, seed=17, device="cpu")
    pts[500:530] = pts[499]
    graph = K.neighbors(pts, 15, ctx=ctx)
    gpu = K.connectivities(graph, ctx=ctx)
    ref = OC.connectivities(graph.indptr, graph.indices, graph.distances, 15)
    _conn_equal_edges(gpu, ref)
    assert np.abs(gpu.weights.astype(np.float64) - ref[2]).max() <= 1e-6
    assert (gpu.weights.view(np.uint32) == ref[2].view(np.uint32)).mean() > 0.999
    rows = np.repeat(np.arange(20_000), np.diff(gpu.indptr.astype(np.int64)))
    dense_pairs = set(zip(rows.tolist(), gpu.indices.tolist()))
    assert all((c, r) in dense_pairs for r, c in list(dense_pairs)[:5000])  # symmetric


def test_connectivities_refusals(ctx):
    g = K.Graph(np.array([0, 2, 3], dtype=np.uint64), np.array([1, 0, 0], dtype=np.uint32),
                np.ones(3, dtype=np.float32))
    with pytest.raises(K.KytoError):
        K.connectivities(g, ctx=ctx)  # uneven rows
    g = K.Graph(np.array([0, 2, 4], dtype=np.uint64), np.array([1, 0, 1, 0], dtype=np.uint32),
                np.ones(4, dtype=np.float32))
    with pytest.raises(K.KytoError):
        K.connectivities(g, ctx=ctx)  # columns not increasing in row 1


@pytest.mark.parametrize("candidate_filter", ["fp16", "split", "bf16"])
def test_filter_query_operand_in_tmem_or_smem_gives_the_same_keys(ctx, monkeypatch,
                                                                  candidate_filter):
    # The filter's MMAs read the query tiles from tensor memory (copied once per block) or
    # from shared memory, into two whole or three or four half accumulator slots: the same
    # products, so the same approximate keys, candidates, full-row searches and graph
    # bits; and on ordinary data no row needs a full search with fp16 or split operands
    # (bf16's 8-bit significands leave slacks wide enough that some rows keep too many
    # candidates and are searched in full, the same rows every way).
    monkeypatch.setenv("KYTO_GPU_KNN_FILTER", candidate_filter)
    x, _ = synthetic.gaussian_mixture(60_000, dim=50, n_components=40, seed=21, device="cpu")
    monkeypatch.setenv("KYTO_GPU_FILTER_A", "smem")
    a = K.neighbors(x, 15, ctx=ctx)
    for mode in ("tmem", "half"):  # A in tensor memory; A in shared memory, half slots
        monkeypatch.setenv("KYTO_GPU_FILTER_A", mode)
        b = K.neighbors(x, 15, ctx=ctx)
        assert np.array_equal(a.indices, b.indices), mode
        assert np.array_equal(a.distances.view(np.uint32), b.distances.view(np.uint32)), mode
        assert a.stats.candidates == b.stats.candidates, mode
        assert a.stats.rows_full == b.stats.rows_full, mode
    if candidate_filter != "bf16":
        assert a.stats.rows_full == 0
    o = O.neighbors(x[:5000], 15, method="exact")
    c = K.neighbors(x[:5000], 15, ctx=ctx)
    assert np.array_equal(c.indices, o.indices)
    assert np.array_equal(c.distances.view(np.uint32), o.distances.view(np.uint32))


def test_filter_choice_is_tuned_once_and_kept_in_the_cache_file(ctx, monkeypatch, tmp_path):
    # An unusual shape class (no earlier test tuned it in this process): the first search
    # pilots both operand kinds in every query-operand mode, keeps the cheapest in the
    # cache file under (GPU, class), and the graph is the oracle's whichever it picked.
    path = tmp_path / "tune.json"
    monkeypatch.setenv("KYTO_GPU_TUNE_CACHE", str(path))
    monkeypatch.delenv("KYTO_GPU_KNN_FILTER", raising=False)
    monkeypatch.delenv("KYTO_GPU_FILTER_A", raising=False)
    pts, _ = synthetic.gaussian_mixture(3000, 7, 12, seed=31, device="cpu")
    g = K.neighbors(pts, 9, ctx=ctx)
    _graph_equal(g, O.neighbors(pts, 9))
    doc = json.loads(path.read_text())
    (entry,) = [e for e in doc["entries"] if e["class"] == "knn_filter/n2^12/d7/k8"]
    assert entry["choice"]["kind"] in ("fp16", "split")
    assert entry["choice"]["a_mode"] in ("smem", "tmem", "half")
    assert "SMs" in entry["gpu"] and entry["ms"] > 0
