"""The oracle pinned against kyto's checked-in golden vectors (scanpy references).

Tolerances are kyto's own (tests/parity/tolerances.toml in kyto): normalize_total bit
for bit, log1p 1e-6 relative, HVG statistics 1e-6 and flags exact, PCA variance 1e-3
relative / leading angle 1e-3 rad / all angle 1e-2 rad / loadings and embedding 1e-3,
neighbour rows equal (all of pbmc3k; synthetic's 10 documented duplicate/tie rows
excepted) with distances within 2e-7 relative.
"""

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import load_golden


@pytest.fixture(scope="module")
def counts():
    g = load_golden("synthetic_counts")
    return O.Csr(g["indptr"], g["indices"], g["counts"], int(g["n_genes"][0]))


@pytest.fixture(scope="module")
def log1p(counts):
    return O.normalize_log1p(counts, 1e4, True)


def test_normalize_total_is_bit_exact(counts):
    g = load_golden("synthetic_normalize_log1p")
    assert np.array_equal(g["indptr"], counts.indptr.astype(np.int64))
    norm = O.normalize_log1p(counts, 1e4, False)
    assert np.array_equal(norm.values.view(np.uint32), g["normalized"].view(np.uint32))


def test_log1p_within_one_ulp(log1p):
    g = load_golden("synthetic_normalize_log1p")
    ref = g["log1p"]
    ulps = np.abs(log1p.values.view(np.int32).astype(np.int64) - ref.view(np.int32))
    assert ulps.max() <= 1
    assert np.max(np.abs(log1p.values - ref) / np.abs(ref)) <= 1e-6


def test_log1p_is_the_rounded_f64_value(log1p):
    g = load_golden("synthetic_normalize_log1p")
    expect = np.log1p(g["normalized"].astype(np.float64)).astype(np.float32)
    assert np.array_equal(log1p.values, expect)


def test_hvg_seurat_matches_scanpy(log1p):
    g = load_golden("synthetic_hvg")
    sums, squares, positives = O.hvg_moments(log1p)
    means, disp, norm, flags = O.hvg_seurat(sums, squares, positives, log1p.n_rows, 100)
    assert np.array_equal(flags, g["highly_variable"])
    assert flags.sum() == 100
    assert np.allclose(means, g["means"], rtol=1e-6, atol=0)
    fin = np.isfinite(g["dispersions"])
    assert np.array_equal(fin, np.isfinite(disp))
    assert np.allclose(disp[fin], g["dispersions"][fin], rtol=1e-6, atol=0)
    fin = np.isfinite(g["dispersions_norm"])
    assert np.allclose(norm[fin], g["dispersions_norm"][fin], rtol=0, atol=1e-6)


def _angle(a: np.ndarray, b: np.ndarray) -> float:
    qa, _ = np.linalg.qr(a)
    qb, _ = np.linalg.qr(b)
    s = np.linalg.svd(qa.T @ qb, compute_uv=False)
    return float(np.arccos(np.clip(s.min(), -1, 1)))


def test_pca_matches_scanpy(log1p):
    hv = load_golden("synthetic_hvg")["highly_variable"]
    g = load_golden("synthetic_pca")
    res = O.pca(log1p, 20, seed=0, gene_set=hv)
    k = 20
    assert res.embedding.shape == (500, k)
    assert np.max(np.abs(res.variance - g["variance"]) / g["variance"]) <= 1e-3
    assert np.max(np.abs(res.variance_ratio - g["variance_ratio"]) / g["variance_ratio"]) <= 1e-3
    load = res.loadings[hv].astype(np.float64)
    comp = g["components"].astype(np.float64)
    assert _angle(load[:, :3], comp[:, :3]) <= 1e-3
    assert _angle(load, comp) <= 1e-2
    for c in range(3):
        assert np.max(np.abs(load[:, c] - comp[:, c])) / np.max(np.abs(comp[:, c])) <= 1e-3
        e, r = res.embedding[:, c].astype(np.float64), g["embedding"][:, c].astype(np.float64)
        assert np.max(np.abs(e - r)) / np.max(np.abs(r)) <= 1e-3
    # 100 genes, width 30: the basis spans every gene, so kyto's PCA is exact there and
    # the seed changes nothing (pca_parity.rs in kyto).
    other = O.pca(log1p, 20, seed=1, gene_set=hv)
    assert np.max(np.abs(other.variance - res.variance) / res.variance) <= 1e-9


def _rows_equal(graph, g):
    n = len(g["indptr"]) - 1
    k = int(g["indptr"][1] - g["indptr"][0])
    mine = graph.indices.reshape(n, k).astype(np.int64)
    ref = g["indices"].reshape(n, k)
    equal = np.all(np.sort(mine, axis=1) == np.sort(ref, axis=1), axis=1)
    return mine, ref, equal


def test_knn_matches_scanpy_pbmc3k_every_row():
    g = load_golden("pbmc3k_neighbors")
    graph = O.neighbors(g["embedding"], 15, method="brute")
    mine, ref, equal = _rows_equal(graph, g)
    assert equal.all()
    # scanpy's rows are sorted by column too.
    assert np.array_equal(mine, ref)
    d = graph.distances.astype(np.float64)
    assert np.max(np.abs(d - g["distances"]) / g["distances"]) <= 2e-7


def test_knn_matches_scanpy_synthetic_but_documented_rows():
    g = load_golden("synthetic_neighbors")
    emb = load_golden("synthetic_pca")["embedding"]
    graph = O.neighbors(emb, 15, method="brute")
    _, _, equal = _rows_equal(graph, g)
    # kyto's deviations.md: 490 of 500 rows equal, the other 10 at duplicate cells.
    assert equal.sum() == 490


def test_filtered_exact_equals_brute_force():
    g = load_golden("pbmc3k_neighbors")
    emb = g["embedding"]
    kb, rb, _ = O.knn_ranked(emb, 15, "brute")
    ke, re_, fallbacks = O.knn_ranked(emb, 15, "exact")
    assert np.array_equal(rb, re_)
    assert np.array_equal(kb.view(np.uint64), ke.view(np.uint64))
    assert fallbacks < 50


def test_line_of_points_known_answer():
    # neighbors.rs:563-576 in kyto: rows at 0, 1, 3, 7 on a line, n_neighbors 3.
    pts = np.array([[0.0], [1.0], [3.0], [7.0]], dtype=np.float32)
    graph = O.neighbors(pts, 3)
    assert graph.indptr.tolist() == [0, 2, 4, 6, 8]
    assert graph.indices.tolist() == [1, 2, 0, 2, 0, 1, 1, 2]
    assert graph.distances.tolist() == [1.0, 3.0, 1.0, 2.0, 3.0, 2.0, 6.0, 4.0]


def test_ties_go_to_the_lower_row():
    # neighbors.rs:555-561 in kyto: equal keys rank by row.
    pts = np.array([[0.0], [1.0], [-1.0], [1.0]], dtype=np.float32)
    keys, rows, _ = O.knn_ranked(pts, 3)
    assert rows[0].tolist() == [1, 2]
    assert rows[1].tolist() == [3, 0]


# ------------------------------------------------------------ connectivities ----------

from oracle import connectivities as OC  # noqa: E402


def _golden_connectivities(name):
    g = load_golden(f"{name}_connectivities")
    ip = g["dist_indptr"]
    k = int(ip[1] - ip[0])
    return g, k


@pytest.mark.parametrize("name", ["synthetic", "pbmc3k"])
def test_connectivities_match_scanpy(name):
    # kyto's connectivities_parity.rs: scanpy's own distances in, the same edges out and
    # every weight within connectivities.weights (1e-5 absolute).
    g, k = _golden_connectivities(name)
    indptr, indices, weights = OC.connectivities(g["dist_indptr"], g["dist_indices"],
                                                 g["dist_data"].astype(np.float32), k + 1)
    assert np.array_equal(indptr, g["indptr"].astype(np.uint64))
    assert np.array_equal(indices, g["indices"].astype(np.uint32))
    diff = np.abs(weights.astype(np.float64) - g["weights"].astype(np.float64))
    assert diff.max() <= 1e-5, diff.max()
    # The f32 exponential rounded once from f64 against numba's expf: a few last bits.
    assert (weights.view(np.uint32) == g["weights"].view(np.uint32)).mean() > 0.99


def _graph(rows):
    k = len(rows[0])
    indptr = np.arange(len(rows) + 1, dtype=np.uint64) * k
    indices = np.array([c for row in rows for c, _ in row], dtype=np.uint32)
    dist = np.array([d for row in rows for _, d in row], dtype=np.float32)
    return indptr, indices, dist, k + 1


def test_connectivities_known_answers():
    # The in-file cases of kyto's connectivities.rs tests (:279-397).
    line = _graph([[(1, 1.0), (2, 3.0)], [(0, 1.0), (2, 2.0)], [(0, 3.0), (1, 2.0)]])
    ip, ix, w = OC.connectivities(*line)
    assert ip.tolist() == [0, 2, 4, 6] and ix.tolist() == [1, 2, 0, 2, 0, 1]
    dense = np.zeros((3, 3), dtype=np.float32)
    for r in range(3):
        dense[r, ix[ip[r]:ip[r + 1]]] = w[ip[r]:ip[r + 1]]
    assert np.array_equal(dense, dense.T)
    assert dense[0, 1] == 1.0 and dense[1, 2] >= 1.0 - np.finfo(np.float32).eps
    assert 0.0 < dense[0, 2] < 1.0
    # sigma's floor rounds once, as umap: bits 983688805.
    ranked = np.array([[0, 0, 0, 0, 2.4006681, 2.417103, 2.4605973, 2.4799116, 2.5937085]],
                      dtype=np.float32)
    sigma, rho = OC.smooth_knn(ranked, 10)
    assert rho[0] == np.float32(2.4006681) and int(sigma.view(np.uint32)[0]) == 983688805
    # Duplicates weigh one, the row itself zero (dropped by the union).
    dup = _graph([[(1, 0.0), (2, 1.0)], [(0, 0.0), (2, 1.0)], [(1, 1.0), (2, 0.0)]])
    ip, ix, w = OC.connectivities(*dup)
    assert ip.tolist() == [0, 2, 4, 6] and ix.tolist() == [1, 2, 0, 2, 0, 1]
    assert w[0] == 1.0 and np.all((w > 0) & (w <= 1))
    # Rows of zero distances take the global floor: every membership 1.
    same = _graph([[(1, 0.0), (2, 0.0)], [(0, 0.0), (2, 0.0)], [(0, 0.0), (1, 0.0)]])
    assert OC.connectivities(*same)[2].tolist() == [1.0] * 6
    # Underflowing weights are dropped unless the other side holds them.
    far = _graph([[(1, 1.0), (2, 1.0), (3, 1e6)], [(0, 1.0), (2, 1.0), (3, 1.0)],
                  [(0, 1.0), (1, 1.0), (3, 1.0)], [(0, 1e6), (1, 1.0), (2, 1.0)]])
    ip, ix, _ = OC.connectivities(*far)
    assert ip.tolist() == [0, 2, 5, 8, 10] and ix.tolist() == [1, 2, 0, 2, 3, 0, 1, 3, 1, 2]
