"""The learned-partition kNN: the network's device gradients against the CPU oracle's
(bf16 operands emulated, f64 sums), and the search's recall against the exact graph,
with and without training (what the trained network gains)."""

import numpy as np
import pytest

import kyto_b200 as K
from kyto_b200 import synthetic
from oracle import partitioner as O

pytestmark = pytest.mark.gpu


def _pack(params: O.Params, offsets, total):
    flat = np.zeros(total, dtype=np.float32)
    for l in range(3):
        w, b = params.w[l], params.b[l]
        flat[offsets[2 * l]:offsets[2 * l] + w.size] = w.ravel()
        flat[offsets[2 * l + 1]:offsets[2 * l + 1] + b.size] = b
    return flat


def _unpack(flat, params: O.Params, offsets):
    ws, bs = [], []
    for l in range(3):
        w, b = params.w[l], params.b[l]
        ws.append(flat[offsets[2 * l]:offsets[2 * l] + w.size].reshape(w.shape))
        bs.append(flat[offsets[2 * l + 1]:offsets[2 * l + 1] + b.size])
    return ws, bs


@pytest.mark.parametrize("rows,din,hidden,parts,L", [(96, 50, 64, 128, 5), (257, 50, 256, 1024, 15)])
def test_gradients_match_the_oracle(rows, din, hidden, parts, L):
    rng = np.random.default_rng(rows)
    params = O.init_params([din, hidden, hidden, parts], seed=rows)
    for b in params.b:  # non-zero biases, so every term is exercised
        b[:] = rng.normal(0, 0.1, b.shape).astype(np.float32)
    x = rng.normal(0, 1.0, (rows, din)).astype(np.float32)
    labels = rng.integers(0, parts, (rows, L)).astype(np.uint32)
    offsets, total = K.learned_layout(din, hidden, parts)
    flat = _pack(params, offsets, total)
    grads, loss, logits = K.learned_gradients(flat, x, labels, hidden, parts)
    targets = np.zeros((rows, parts))
    for j in range(L):
        np.add.at(targets, (np.arange(rows), labels[:, j]), 1.0 / L)
    o_loss, o_gw, o_gb = O.loss_and_grads(params, x, targets)
    o_logits, _ = O.forward(params, x)
    # f32 sums against f64: an activation may land on the other side of a bf16 rounding
    # (2^-8 relative), so the logits agree to 1e-3 of their norm overall and 1e-2 of
    # their scale everywhere; the loss to 1e-4; each gradient block to 2e-3 of its norm.
    scale = np.abs(o_logits).max()
    assert np.linalg.norm(logits - o_logits) <= 1e-3 * np.linalg.norm(o_logits)
    np.testing.assert_allclose(logits, o_logits, rtol=0, atol=1e-2 * scale)
    assert abs(float(loss.mean()) - o_loss) <= 1e-4 * max(1.0, abs(o_loss))
    gw, gb = _unpack(grads, params, offsets)
    for l in range(3):
        for got, want in ((gw[l], o_gw[l]), (gb[l], o_gb[l])):
            err = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30)
            assert err < 2e-3, (l, err)


def _recall(graph: K.Graph, exact: K.Graph) -> float:
    n = len(exact.indptr) - 1
    k = len(exact.indices) // n
    a = graph.indices.reshape(n, k).astype(np.int64)
    b = exact.indices.reshape(n, k).astype(np.int64)
    hits = sum(len(np.intersect1d(a[i], b[i], assume_unique=True)) for i in range(n))
    return hits / b.size


@pytest.mark.parametrize("candidate_filter", ["fp16", "split"])
def test_learned_search_recall_and_what_training_gains(monkeypatch, candidate_filter):
    monkeypatch.setenv("KYTO_GPU_KNN_FILTER", candidate_filter)
    x, _ = synthetic.gaussian_mixture(60_000, dim=50, n_components=60, seed=3, device="cpu")
    x = np.ascontiguousarray(x, dtype=np.float32)
    ctx = K.Context(0)
    exact = K.neighbors(x, 15, ctx=ctx)
    common = dict(n_parts=512, hidden=128, n_probe=8, confidence=0.0, train_cells=30_000,
                  batch=2048, learning_rate=2e-3, seed=1)
    g1, s1 = K.neighbors_learned(x, 15, params=K.LearnedParams(epochs=8, **common), ctx=ctx)
    # Without training: the network as initialised, the k-means parts' nearest-centre
    # classifier (k-means centroid probing), and random weights.
    gk, sk = K.neighbors_learned(x, 15, params=K.LearnedParams(epochs=0, **common), ctx=ctx)
    g0, s0 = K.neighbors_learned(x, 15, params=K.LearnedParams(epochs=0, random_init=True,
                                                               **common), ctx=ctx)
    r1, rk, r0 = _recall(g1, exact), _recall(gk, exact), _recall(g0, exact)
    # Every distance returned is the true distance of its pair (the exact re-rank).
    n = x.shape[0]
    rows = np.repeat(np.arange(n), 14)
    d_true = np.sqrt(((x[rows].astype(np.float64) - x[g1.indices.astype(np.int64)]) ** 2).sum(1))
    np.testing.assert_allclose(g1.distances, d_true, rtol=1e-5, atol=1e-5)
    assert s1.fallback_rows == 0 and np.isfinite(s1.final_loss)
    # What training gains: the trained network's proposals find more of the neighbours
    # than k-means centroid probing while its query blocks scan fewer tiles, and a
    # fraction of the tiles an untrained random network makes them scan (random parts
    # spread over nearly every tile).
    assert r1 > 0.95, r1
    assert r1 >= rk and s1.scanned_tiles < sk.scanned_tiles, (r1, rk, s1.scanned_tiles,
                                                              sk.scanned_tiles)
    assert s1.scanned_tiles < 0.5 * s0.scanned_tiles, (s1.scanned_tiles, s0.scanned_tiles, r1, r0)
    n_tiles = (n + 127) // 128
    n_blocks = (n + 255) // 256
    assert s1.scanned_tiles < 0.5 * n_tiles * n_blocks
    # The distance bounds skip listed tiles that cannot hold a neighbour of the block.
    assert 0 < s1.tiles_computed <= s1.scanned_tiles, (s1.tiles_computed, s1.scanned_tiles)


@pytest.mark.parametrize("candidate_filter", ["fp16", "split"])
def test_confidence_above_one_falls_back_to_the_exact_graph(monkeypatch, candidate_filter):
    monkeypatch.setenv("KYTO_GPU_KNN_FILTER", candidate_filter)
    x, _ = synthetic.gaussian_mixture(5_000, dim=20, n_components=10, seed=4, device="cpu")
    x = np.ascontiguousarray(x, dtype=np.float32)
    ctx = K.Context(0)
    exact = K.neighbors(x, 10, ctx=ctx)
    p = K.LearnedParams(n_parts=16, hidden=32, n_probe=2, confidence=1.01, train_cells=2_000,
                        epochs=1, batch=512, seed=2)
    g, s = K.neighbors_learned(x, 10, params=p, ctx=ctx)
    assert s.fallback_rows == x.shape[0]
    assert np.array_equal(g.indices, exact.indices)
    assert np.array_equal(g.distances.view(np.uint32), exact.distances.view(np.uint32))
