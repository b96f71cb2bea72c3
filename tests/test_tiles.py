"""Tiled store layers joined into CSR rows on the device (kg_tiles_to_csr,
kg_pca_push_tiles) against the oracle's restatement of kyto-store's tile_decode.rs.

CPU: the oracle is pinned to kyto's own in-file cases (tile_encode.rs:87-109,
tile_decode.rs:238-338): the 3 x 5 matrix in 2 x 2 tiles, each corrupt tile's wording,
and the vectorised encoder against the loop restatement.
GPU: the device join equals the oracle's bit for bit (host and device inputs, ragged last
cell and gene blocks, empty tiles and rows, u32 and f32 values), reports the oracle's
first problem in kyto's wording (KY-E107) for every corruption of a valid layer, and a
PCA pushed as tiles equals the PCA of the same rows pushed as CSR, bit for bit.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import tiles as T

# kyto's test matrix (tile_encode.rs:87-109): rows [1 0 2 0 3], [0 0 0 0 0],
# [0 4 0 -0.0 5], stored zeros included (the writer drops them).
M_INDPTR = np.array([0, 4, 4, 8], dtype=np.uint64)
M_INDICES = np.array([0, 1, 2, 4, 1, 2, 3, 4], dtype=np.uint32)
M_DATA = np.array([1.0, 0.0, 2.0, 3.0, 4.0, 0.0, -0.0, 5.0], dtype=np.float32)
GRID = T.TileGrid(3, 5, 2, 2)
OFFSETS = np.array([0, 1, 2, 3, 4, 4, 5], dtype=np.uint64)
INDICES = np.array([0, 0, 0, 1, 0], dtype=np.uint32)
DATA = np.array([1.0, 2.0, 3.0, 4.0, 5.0], dtype=np.float32)
GOOD0 = [0, 1, 1, 0, 1, 1, 0, 1, 1]
GOOD1 = [0, 1, 1, 0, 0, 0, 0, 1, 1]

# (block, shard, indices, the problem kyto reports): tile_decode.rs:270-320.
CORRUPT = [
    (0, [1, 1, 1, 0, 1, 1, 0, 1, 1], INDICES, "tile (0, 0): indptr does not start at 0"),
    (0, [0, 1, 2, 0, 1, 1, 0, 1, 1], INDICES, "tile_offsets gives 1"),
    (0, [0, 1, 1, 0, 1, 1, 0, 2, 1], INDICES, "tile (0, 2): indptr decreases"),
    (0, GOOD0, np.array([2, 0, 0, 1, 0], np.uint32),
     "local gene index 2 is not below the block width 2"),
    (0, GOOD0, np.array([0, 0, 1, 1, 0], np.uint32),
     "tile (0, 2): row 0: local gene index 1 is not below the block width 1"),
    (1, [0, 1, 1, 0, 0, 0, 0, 0, 1], INDICES,
     "tile (1, 2): indptr is not flat after the last row 1"),
]


def _oracle_problem(grid, block, shard, offsets, indices, data):
    try:
        T.decode_cell_block(grid, block, shard, offsets, indices, data)
    except T.CorruptLayer as e:
        return str(e)
    return None


def test_oracle_encodes_kytos_test_matrix():
    shards, offsets, idx, vals = T.encode(M_INDPTR, M_INDICES, M_DATA, GRID)
    assert shards[0].ravel().tolist() == GOOD0
    assert shards[1].ravel().tolist() == GOOD1
    assert offsets.tolist() == OFFSETS.tolist()
    assert idx.tolist() == INDICES.tolist() and vals.tolist() == DATA.tolist()
    fast = T.encode_fast(M_INDPTR, M_INDICES, M_DATA, GRID)
    assert all(np.array_equal(a, b) for a, b in zip(fast[0], shards))
    assert np.array_equal(fast[1], offsets) and np.array_equal(fast[2], idx)


def test_oracle_decodes_kytos_rows():
    p0, i0, d0 = T.decode_cell_block(GRID, 0, GOOD0, OFFSETS, INDICES, DATA)
    p1, i1, d1 = T.decode_cell_block(GRID, 1, GOOD1, OFFSETS, INDICES, DATA)
    # kyto's joined layer: indptr [0, 3, 3, 5], indices [0, 2, 4, 1, 4].
    assert p0.tolist() == [0, 3, 3] and p1.tolist() == [0, 2]
    assert np.concatenate([i0, i1]).tolist() == [0, 2, 4, 1, 4]
    assert np.concatenate([d0, d1]).tolist() == [1.0, 2.0, 3.0, 4.0, 5.0]


@pytest.mark.parametrize("block,shard,indices,problem", CORRUPT)
def test_oracle_reports_kytos_corrupt_tiles(block, shard, indices, problem):
    assert problem in _oracle_problem(GRID, block, shard, OFFSETS, indices, DATA)


def test_oracle_reports_kytos_tile_offsets_and_unsorted_rows():
    with pytest.raises(T.CorruptLayer, match="n_tiles \\+ 1 is 7"):
        T.check_tile_offsets(GRID, OFFSETS[:6], 5)
    with pytest.raises(T.CorruptLayer, match="\\[0\\] is not 0"):
        T.check_tile_offsets(GRID, [1, 1, 2, 3, 4, 4, 5], 5)
    with pytest.raises(T.CorruptLayer, match="decreases after tile 1"):
        T.check_tile_offsets(GRID, [0, 2, 1, 3, 4, 4, 5], 5)
    with pytest.raises(T.CorruptLayer, match="hold 6 entries"):
        T.check_tile_offsets(GRID, OFFSETS, 6)
    one = T.TileGrid(1, 4, 1, 4)
    assert "row 0: gene indices are not strictly increasing" in _oracle_problem(
        one, 0, [0, 2], [0, 2], np.array([3, 1], np.uint32), np.array([1.0, 2.0], np.float32))


def _layer(n_cells, n_genes, per_cell, seed, dtype=np.float32, empty_rows=0.05):
    """A sorted random CSR with some empty rows and a few stored zeros."""
    rng = np.random.default_rng(seed)
    counts = rng.poisson(per_cell, n_cells).clip(0, n_genes)
    counts[rng.random(n_cells) < empty_rows] = 0
    indptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    indices = np.concatenate([np.sort(rng.choice(n_genes, c, replace=False)) for c in counts]
                             ).astype(np.uint32) if counts.sum() else np.zeros(0, np.uint32)
    if dtype == np.float32:
        data = rng.lognormal(0, 1, len(indices)).astype(np.float32)
    else:
        data = rng.integers(1, 50, len(indices)).astype(np.uint32)
    data[rng.random(len(data)) < 0.01] = 0
    return indptr, indices, data


def test_oracle_fast_encoder_equals_the_loop():
    for n_cells, n_genes, c, g in [(37, 23, 8, 5), (64, 40, 16, 64), (10, 9, 3, 1)]:
        grid = T.TileGrid(n_cells, n_genes, c, g)
        layer = _layer(n_cells, n_genes, 6, seed=n_cells)
        slow, fast = T.encode(*layer, grid), T.encode_fast(*layer, grid)
        assert all(np.array_equal(a, b) for a, b in zip(slow[0], fast[0]))
        for a, b in zip(slow[1:], fast[1:]):
            assert np.array_equal(a, b)


def test_entries_shorter_than_tile_offsets_are_refused_on_the_host():
    """The binding refuses a block whose tile_offsets run past the entries it was given
    (kyto's check_tile_offsets wording, KY-E107) before any device work."""
    import kyto_b200 as K

    with pytest.raises(K.KytoError) as e:
        K.tiles_to_csr(0, 2, 2, 3, 5, np.array(GOOD0, np.uint32), OFFSETS, INDICES[:2],
                       DATA[:2])
    assert e.value.code == "KY-E107" and "hold 2 and 2 entries" in str(e.value)


# ---------------------------------------------------------------- device ----------------

@pytest.fixture(scope="module")
def ctx():
    import kyto_b200 as K

    return K.Context(0)


def _device_join(grid, block, shard, offsets, indices, data, ctx, on_device=False):
    import kyto_b200 as K

    if on_device:
        import torch

        shard = torch.from_numpy(np.ascontiguousarray(shard).view(np.int32)).cuda()
        offsets = torch.from_numpy(offsets.view(np.int64)).cuda()
        indices = torch.from_numpy(indices.view(np.int32)).cuda()
        data = torch.from_numpy(data).cuda() if data.dtype == np.float32 else \
            torch.from_numpy(data.view(np.int32)).cuda()
    return K.tiles_to_csr(block, grid.cell_block_size, grid.gene_block_size, grid.n_cells,
                          grid.n_genes, shard, offsets, indices, data, ctx=ctx)


def _same(a, b):
    return all(np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))
               for x, y in zip(a, b))


@pytest.mark.gpu
def test_device_join_of_kytos_test_matrix(ctx):
    for block, shard in ((0, GOOD0), (1, GOOD1)):
        shard = np.array(shard, np.uint32)
        ref = T.decode_cell_block(GRID, block, shard, OFFSETS, INDICES, DATA)
        for on_device in (False, True):
            got = _device_join(GRID, block, shard, OFFSETS, INDICES, DATA, ctx, on_device)
            assert _same(got, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("n_cells,n_genes,c,g,dtype", [
    (5000, 3000, 1024, 512, np.float32),   # ragged last cell and gene blocks
    (4096, 2000, 4096, 1024, np.uint32),   # kyto's default tiling, one cell block
    (777, 64, 100, 7, np.float32),         # many narrow gene blocks, empty tiles
    (300, 50, 64, 64, np.uint32),          # one gene block wider than the genes
    (129, 33, 1, 4, np.float32),           # one-row cell blocks
])
def test_device_join_equals_the_oracle(ctx, n_cells, n_genes, c, g, dtype):
    grid = T.TileGrid(n_cells, n_genes, c, g)
    layer = _layer(n_cells, n_genes, min(40, n_genes // 2), seed=n_cells + c, dtype=dtype)
    shards, offsets, idx, vals = T.encode_fast(*layer, grid)
    blocks = list(range(grid.n_cell_blocks))
    if len(blocks) > 8:
        blocks = blocks[:4] + blocks[-4:]
    for b in blocks:
        ref = T.decode_cell_block(grid, b, shards[b], offsets, idx, vals)
        assert _same(_device_join(grid, b, shards[b], offsets, idx, vals, ctx), ref)
        assert _same(_device_join(grid, b, shards[b], offsets, idx, vals, ctx, True), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("block,shard,indices,problem", CORRUPT)
def test_device_reports_kytos_corrupt_tiles(ctx, block, shard, indices, problem):
    import kyto_b200 as K

    with pytest.raises(K.KytoError) as e:
        _device_join(GRID, block, np.array(shard, np.uint32), OFFSETS, indices, DATA, ctx)
    assert e.value.code == "KY-E107"
    assert problem in str(e.value)
    assert _oracle_problem(GRID, block, shard, OFFSETS, indices, DATA) in str(e.value)


@pytest.mark.gpu
def test_device_reports_the_oracles_first_problem_for_every_corruption(ctx):
    """Valid layers with one or two values changed (an indptr value raised or lowered, a
    local index moved past the width or before its neighbour): the device reports the
    oracle's first problem word for word, or passes exactly when the oracle does (and
    then gives its rows)."""
    import kyto_b200 as K

    rng = np.random.default_rng(7)
    grid = T.TileGrid(300, 70, 64, 16)
    layer = _layer(300, 70, 12, seed=3)
    shards, offsets, idx, vals = T.encode_fast(*layer, grid)
    n_gb = grid.n_gene_blocks
    for trial in range(120):
        b = int(rng.integers(grid.n_cell_blocks))
        shard = shards[b].copy()
        local = idx.copy()
        for _ in range(1 + trial % 2):
            if rng.random() < 0.5:
                g, r = int(rng.integers(n_gb)), int(rng.integers(grid.indptr_len))
                shard[g, r] = max(0, int(shard[g, r]) + int(rng.choice([-3, -1, 1, 2, 40])))
            else:
                lo = int(offsets[b * n_gb])
                hi = int(offsets[(b + 1) * n_gb])
                if hi > lo:
                    e = int(rng.integers(lo, hi))
                    local[e] = int(rng.choice([0, 1, 15, 16, 99]))
        expected = _oracle_problem(grid, b, shard, offsets, local, vals)
        if expected is None:
            ref = T.decode_cell_block(grid, b, shard, offsets, local, vals)
            assert _same(_device_join(grid, b, shard, offsets, local, vals, ctx), ref)
        else:
            with pytest.raises(K.KytoError) as e:
                _device_join(grid, b, shard, offsets, local, vals, ctx)
            assert e.value.code == "KY-E107" and expected in str(e.value), (expected, str(e.value))


@pytest.mark.gpu
def test_pca_pushed_as_tiles_equals_the_csr_push(ctx):
    """kg_pca_push_tiles (cells b C + r) and kg_pca_push_block of the oracle's joined rows
    (cells numbered on) give the same PCA, bit for bit, with normalize/log1p and a gene
    map applied by the session."""
    import kyto_b200 as K
    from kyto_b200 import synthetic

    x = synthetic.counts_csr(6000, 1500, 120, 6, 60, seed=4, device="cpu")
    grid = T.TileGrid(6000, 1500, 1024, 512)
    shards, offsets, idx, vals = T.encode_fast(x.indptr, x.indices, x.values, grid)
    gene_set = np.zeros(1500, dtype=bool)
    gene_set[::3] = True
    results = []
    for as_tiles in (False, True):
        sess = K.PcaSession(20, 1500, seed=0, gene_set=gene_set, target_sum=1e4, log1p=True,
                            ctx=ctx)
        for b in range(grid.n_cell_blocks):
            if as_tiles:
                sess.push_tiles(b, grid.cell_block_size, grid.gene_block_size, grid.n_cells,
                                shards[b], offsets, idx, vals)
            else:
                sess.push(*T.decode_cell_block(grid, b, shards[b], offsets, idx, vals))
        sess.run()
        results.append(sess.results())
        sess.close()
    a, b = results
    assert np.array_equal(a.embedding.view(np.uint32), b.embedding.view(np.uint32))
    assert np.array_equal(a.variance.view(np.uint64), b.variance.view(np.uint64))
