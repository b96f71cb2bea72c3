"""The shards of kyto's tiled layers decoded on the host (kg_shard_read, kg_chunk_read),
against the oracle's restatement of the layout (oracle/shards.py: Zarr v3
sharding_indexed with zstd inner chunks, CRC-32C index; docs/format.md §4.4).

Host code only: these tests need no GPU. A whole tiled layer (oracle/tiles.py's encoder,
kyto's default-like tiling) is written as shards, read back through the library and
joined by the oracle into the original rows; every unreadable shard returns KY-E110."""

from __future__ import annotations

import numpy as np
import pytest

import kyto_b200 as K
from oracle import shards as S
from oracle import tiles as T


def test_oracle_crc32c_known_answers():
    # The Castagnoli CRC's published check value, and the empty input.
    assert S.crc32c(b"123456789") == 0xE3069283
    assert S.crc32c(b"") == 0


@pytest.mark.parametrize("dtype", [np.uint32, np.float32, np.uint64])
def test_ranges_of_shards_read_back(dtype):
    rng = np.random.default_rng(1)
    n, k, s = 10_000, 256, 2048
    v = (rng.integers(1, 1 << 30, n) if dtype != np.float32 else rng.random(n)).astype(dtype)
    v[1000:3000] = 0  # whole chunks of the fill value are not stored
    shards = S.write_shards(v, k, s)
    assert len(shards) == 5
    for first, count in [(0, n), (0, 1), (255, 2), (1000, 2000), (2047, 3), (9999, 1),
                         (513, 7000), (4096, 2048)]:
        got = K.read_sharded(shards, k, s, dtype, first, count)
        assert np.array_equal(got.view(np.uint8), v[first:first + count].view(np.uint8))
        ref = S.read_range(shards, k, s, first, count, dtype)
        assert np.array_equal(got.view(np.uint8), ref.view(np.uint8))
    # Past the array's end, inside the last shard: the fill value.
    assert not K.read_sharded(shards, k, s, dtype, n, 240).any()


def test_tile_offsets_chunk_reads_back():
    offsets = np.cumsum(np.random.default_rng(2).integers(0, 900, 65_536)).astype(np.uint64)
    got = K.chunk_read(S.write_chunk(offsets), len(offsets), np.uint64)
    assert np.array_equal(got, offsets)
    with pytest.raises(K.KytoError) as e:
        K.chunk_read(S.write_chunk(offsets[:-1]), len(offsets), np.uint64)
    assert e.value.code == "KY-E110" and "decodes to" in str(e.value)


def test_a_tiled_layer_read_from_its_shards_gives_its_rows():
    """Every cell block: its indptr shard (one inner chunk a tile) and its entries (the
    range tile_offsets gives, across the indices and data shards) decoded by the library,
    then joined by the oracle: the layer's rows, zeros dropped as kyto's writer drops
    them."""
    rng = np.random.default_rng(3)
    n_cells, n_genes, c, g = 3000, 1500, 512, 256
    counts = rng.poisson(40, n_cells).clip(0, n_genes)
    indptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    indices = np.concatenate([np.sort(rng.choice(n_genes, x, replace=False)) for x in counts]
                             ).astype(np.uint32)
    values = rng.integers(1, 30, len(indices)).astype(np.uint32)
    grid = T.TileGrid(n_cells, n_genes, c, g)
    shards, offsets, local, vals = T.encode_fast(indptr, indices, values, grid)
    kc, sc = 1024, 8192  # inner chunk and shard of the entry arrays
    idx_shards = S.write_shards(local, kc, sc)
    val_shards = S.write_shards(vals, kc, sc)
    ptr_shards = [S.write_shards(sh.ravel(), c + 1, grid.n_gene_blocks * (c + 1))[0]
                  for sh in shards]
    offsets_back = K.chunk_read(S.write_chunk(offsets), len(offsets), np.uint64)
    assert np.array_equal(offsets_back, offsets)
    n_gb = grid.n_gene_blocks
    rows = []
    for b in range(grid.n_cell_blocks):
        shard = K.shard_read(ptr_shards[b], n_gb, c + 1, np.uint32, 0, n_gb * (c + 1))
        assert np.array_equal(shard, shards[b].ravel())
        lo, hi = int(offsets_back[b * n_gb]), int(offsets_back[(b + 1) * n_gb])
        got_idx = np.zeros(len(local), np.uint32)
        got_val = np.zeros(len(vals), np.uint32)
        got_idx[lo:hi] = K.read_sharded(idx_shards, kc, sc, np.uint32, lo, hi - lo)
        got_val[lo:hi] = K.read_sharded(val_shards, kc, sc, np.uint32, lo, hi - lo)
        rows.append(T.decode_cell_block(grid, b, shard, offsets_back, got_idx, got_val))
    out_ptr = np.concatenate([[0], np.concatenate(
        [p[1:] + sum(len(r[1]) for r in rows[:i]) for i, (p, _, _) in enumerate(rows)])])
    assert np.array_equal(out_ptr.astype(np.uint64), indptr)
    assert np.array_equal(np.concatenate([r[1] for r in rows]), indices)
    assert np.array_equal(np.concatenate([r[2] for r in rows]), values)


def _shard():
    v = np.arange(1, 4097, dtype=np.uint32)
    return S.write_shards(v, 512, 4096)[0], v


def test_unreadable_shards_return_kytos_store_error():
    shard, v = _shard()
    assert np.array_equal(K.shard_read(shard, 8, 512, np.uint32, 0, 4096), v)
    cases = {
        "short": shard[:100],
        "checksum": shard[:-5] + bytes([shard[-5] ^ 1]) + shard[-4:],
        "index past": None,
        "bad frame": None,
    }
    # An index entry pointing past the chunks (with a checksum that matches it).
    body_len = len(shard) - (16 * 8 + 4)
    index = bytearray(shard[body_len:-4])
    index[0:8] = (body_len + 10).to_bytes(8, "little")
    cases["index past"] = shard[:body_len] + bytes(index) + S.crc32c(bytes(index)).to_bytes(
        4, "little")
    # A frame whose bytes are damaged (same index).
    broken = bytearray(shard)
    broken[5:9] = b"\x00\x00\x00\x00"
    cases["bad frame"] = bytes(broken)
    words = {"short": "fewer than its index", "checksum": "CRC-32C",
             "index past": "lies outside", "bad frame": "inner chunk 0"}
    for name, data in cases.items():
        with pytest.raises(K.KytoError) as e:
            K.shard_read(data, 8, 512, np.uint32, 0, 4096)
        assert e.value.code == "KY-E110", name
        assert words[name] in str(e.value), (name, str(e.value))


def test_shard_read_refuses_ranges_past_the_shard():
    shard, _ = _shard()
    with pytest.raises(K.KytoError) as e:
        K.shard_read(shard, 8, 512, np.uint32, 4000, 100)
    assert e.value.code == "KY-E215"


def test_threaded_decode_reports_the_lowest_damaged_chunk():
    """A read of 8 MB decodes on several threads; with chunks 20 and 5 damaged the error
    names chunk 5 on every run (the hand-out goes in chunk order and every chunk handed
    out before a failure finishes)."""
    v = np.arange(1, 2 * 1024 * 1024 + 1, dtype=np.uint32)
    k = 65536
    shard = bytearray(S.write_shards(v, k, len(v))[0])
    n_chunks = len(v) // k
    index = np.frombuffer(bytes(shard[len(shard) - 16 * n_chunks - 4:-4]), dtype="<u8")
    for c in (20, 5):
        off = int(index[2 * c])
        shard[off + 5:off + 9] = b"\x00\x00\x00\x00"
    for _ in range(5):
        with pytest.raises(K.KytoError) as e:
            K.shard_read(bytes(shard), n_chunks, k, np.uint32, 0, len(v))
        assert e.value.code == "KY-E110" and "inner chunk 5" in str(e.value), str(e.value)
    good = S.write_shards(v, k, len(v))[0]
    assert np.array_equal(K.shard_read(good, n_chunks, k, np.uint32, 0, len(v)), v)


def test_bench_store_writer_and_block_reader_give_the_rows():
    """bench.py's store leg on the host: its tiled-layer writer (the store's layout) and
    its block reader (kg_shard_read into the buffers the join reads) give, through the
    oracle's join, the rows of the CSR it wrote."""
    import bench

    rng = np.random.default_rng(5)
    n_cells, n_genes = 9000, 2000
    counts = rng.poisson(60, n_cells).clip(0, n_genes)
    indptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    indices = np.concatenate([np.sort(rng.choice(n_genes, x, replace=False)) for x in counts]
                             ).astype(np.uint32)
    values = rng.integers(1, 50, len(indices)).astype(np.uint32)
    store = bench.tiled_store(indptr, indices, values, n_genes, inner=4096, per_shard=8)
    grid = T.TileGrid(n_cells, n_genes, 4096, 1024)
    n_gb, c = store["n_gb"], 4096
    shard = np.zeros(n_gb * (c + 1), np.uint32)
    idx = np.zeros(len(indices), np.uint32)
    val = np.zeros(len(indices), np.uint32)
    joined = []
    for b in range(store["n_cb"]):
        lo, m = bench.read_cell_block(store, b, shard, idx, val)
        # read_cell_block wrote the entries at the front of the buffers; the oracle's
        # join wants them at the layer's offsets.
        layer_idx = np.zeros(len(indices), np.uint32)
        layer_val = np.zeros(len(indices), np.uint32)
        layer_idx[lo:lo + m], layer_val[lo:lo + m] = idx[:m], val[:m]
        joined.append(T.decode_cell_block(grid, b, shard, store["offsets"], layer_idx,
                                          layer_val))
    assert np.array_equal(np.concatenate([j[1] for j in joined]), indices)
    assert np.array_equal(np.concatenate([j[2] for j in joined]), values)
    ends = np.cumsum([len(j[1]) for j in joined])
    starts = np.concatenate([[0], ends[:-1]])
    ptr = np.concatenate([[0]] + [j[0][1:] + s for j, s in zip(joined, starts)])
    assert np.array_equal(ptr.astype(np.uint64), indptr)


def test_bench_shard_writer_writes_the_oracles_bytes():
    """bench.py keeps its own copy of the shard writer (its device legs use no oracle);
    it writes the same bytes as the oracle's restatement of the layout."""
    import bench

    rng = np.random.default_rng(9)
    v = rng.integers(0, 5, 70_000).astype(np.uint32)
    v[10_000:30_000] = 0
    assert bench.write_shards(v, 4096, 4) == S.write_shards(v, 4096, 4 * 4096)
    assert bench._crc32c(b"123456789") == 0xE3069283
