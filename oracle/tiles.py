"""Oracle (test infrastructure only): kyto's tiled sparse layers, restated in numpy.

The checker for the device tile join (``kg_tiles_to_csr`` / ``kg_pca_push_tiles``);
nothing on the product path imports this file.

- ``encode_cell_block`` follows crates/kyto-store/src/tile_encode.rs:38-81: cell block
  ``b``'s indptr shard (every gene block, padding rows repeating the tile's nnz) and its
  tiles' entries, gene blocks in increasing order, local gene indices, zeros dropped.
- ``decode_cell_block`` follows crates/kyto-store/src/tile_decode.rs:74-127 with its
  checks (``check_tile_indptr`` :129-164, ``check_tile_rows`` :166-196): every tile of
  the block is checked in gene-block order, the first problem raised as ``CorruptLayer``
  with kyto's wording (KY-E107), then the rows are joined with global gene indices.
- ``check_tile_offsets`` follows tile_decode.rs:29-66.
- ``TileGrid`` follows crates/kyto-store/src/tiling.rs:43-149 (rows, widths, indptr
  length; the limits of format.md §4.5 are the writer's and are not restated).

The layout itself is docs/format.md §4.1-4.3: tile (b, g) holds cells [bC, bC + rows(b))
and genes [gG, gG + width(g)); its entries sit at tile_offsets[t] + indptr[b, g, r] ..
tile_offsets[t] + indptr[b, g, r + 1], t = b n_gene_blocks + g.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


class CorruptLayer(ValueError):
    """kyto's KytoError::CorruptLayer (KY-E107): the message names the tile and the
    invariant that fails."""


@dataclass(frozen=True)
class TileGrid:
    n_cells: int
    n_genes: int
    cell_block_size: int
    gene_block_size: int

    @property
    def n_cell_blocks(self) -> int:
        return -(-self.n_cells // self.cell_block_size)

    @property
    def n_gene_blocks(self) -> int:
        return -(-self.n_genes // self.gene_block_size)

    @property
    def n_tiles(self) -> int:
        return self.n_cell_blocks * self.n_gene_blocks

    def rows(self, block: int) -> int:
        return min(self.cell_block_size, self.n_cells - block * self.cell_block_size)

    def width(self, gene_block: int) -> int:
        return min(self.gene_block_size, self.n_genes - gene_block * self.gene_block_size)

    @property
    def indptr_len(self) -> int:
        return self.cell_block_size + 1


def encode_cell_block(indptr, indices, data, grid: TileGrid, block: int,
                      tile_offsets: list, out_indices: list, out_data: list) -> np.ndarray:
    """Cell block ``block`` of a sorted CSR (u64 indptr, u32 global indices): appends its
    tiles' entries to ``out_indices`` / ``out_data`` and their ends to ``tile_offsets``
    (which starts as [0]); returns its indptr shard (n_gene_blocks x (C + 1), u32)."""
    c = grid.cell_block_size
    first = block * c
    rows = grid.rows(block)
    shard = np.zeros((grid.n_gene_blocks, c + 1), dtype=np.uint32)
    cursor = [int(indptr[first + r]) for r in range(rows)]
    for g in range(grid.n_gene_blocks):
        g0 = g * grid.gene_block_size
        g1 = g0 + grid.width(g)
        nnz = 0
        for r in range(rows):
            end = int(indptr[first + r + 1])
            while cursor[r] < end and int(indices[cursor[r]]) < g1:
                v = data[cursor[r]]
                if v != 0:
                    out_indices.append(int(indices[cursor[r]]) - g0)
                    out_data.append(v)
                    nnz += 1
                cursor[r] += 1
            shard[g, r + 1] = nnz
        shard[g, rows + 1:] = nnz
        tile_offsets.append(tile_offsets[-1] + nnz)
    return shard


def encode(indptr, indices, data, grid: TileGrid):
    """Every cell block of a CSR: (list of indptr shards, tile_offsets u64, local indices
    u32, values in the data's dtype)."""
    offsets, idx, vals = [0], [], []
    shards = [encode_cell_block(indptr, indices, data, grid, b, offsets, idx, vals)
              for b in range(grid.n_cell_blocks)]
    dtype = np.asarray(data).dtype
    return (shards, np.asarray(offsets, dtype=np.uint64), np.asarray(idx, dtype=np.uint32),
            np.asarray(vals, dtype=dtype))


def check_tile_offsets(grid: TileGrid, tile_offsets, nnz: int) -> None:
    """tile_decode.rs:29-66."""
    to = [int(v) for v in tile_offsets]
    if len(to) != grid.n_tiles + 1:
        raise CorruptLayer(f"tile_offsets has {len(to)} values but n_tiles + 1 is "
                           f"{grid.n_tiles + 1}")
    if to[0] != 0:
        raise CorruptLayer("tile_offsets[0] is not 0")
    for t in range(len(to) - 1):
        if to[t + 1] < to[t]:
            raise CorruptLayer(f"tile_offsets decreases after tile {t}")
    if to[-1] != nnz:
        raise CorruptLayer(f"tile_offsets ends at Some({to[-1]}) but indices and data hold "
                           f"{nnz} entries")


def _check_tile_indptr(b, g, tp, rows, tile_nnz):
    """tile_decode.rs:129-164."""
    where = f"tile ({b}, {g}): "
    if int(tp[0]) != 0:
        raise CorruptLayer(where + "indptr does not start at 0")
    if int(tp[-1]) != tile_nnz:
        raise CorruptLayer(where + f"indptr ends at Some({int(tp[-1])}) but tile_offsets gives "
                           f"{tile_nnz} entries")
    for r in range(len(tp) - 1):
        if int(tp[r + 1]) < int(tp[r]):
            raise CorruptLayer(where + f"indptr decreases after row {r}")
    if any(int(v) != int(tp[rows]) for v in tp[rows + 1:]):
        raise CorruptLayer(where + f"indptr is not flat after the last row {rows}")


def _check_tile_rows(b, g, tp, rows, width, tile_indices):
    """tile_decode.rs:166-196 (the rows of one tile whose indptr passed)."""
    where = f"tile ({b}, {g}): "
    for r in range(rows):
        row = [int(v) for v in tile_indices[int(tp[r]):int(tp[r + 1])]]
        wide = [v for v in row if v >= width]
        if wide:
            raise CorruptLayer(where + f"row {r}: local gene index {wide[0]} is not below the "
                               f"block width {width}")
        if any(row[i + 1] <= row[i] for i in range(len(row) - 1)):
            raise CorruptLayer(where + f"row {r}: gene indices are not strictly increasing")


def decode_cell_block(grid: TileGrid, block: int, shard, tile_offsets, indices, data):
    """Cell block ``block`` joined into CSR rows (u64 indptr from 0, u32 global gene
    indices, values), after kyto's checks of every tile. ``tile_offsets``, ``indices``
    and ``data`` are the whole layer's (tile_offsets checked by the caller)."""
    shard = np.asarray(shard, dtype=np.uint32).reshape(grid.n_gene_blocks, grid.indptr_len)
    rows = grid.rows(block)
    first_tile = block * grid.n_gene_blocks
    for g in range(grid.n_gene_blocks):
        start = int(tile_offsets[first_tile + g])
        tile_nnz = int(tile_offsets[first_tile + g + 1]) - start
        _check_tile_indptr(block, g, shard[g], rows, tile_nnz)
        _check_tile_rows(block, g, shard[g], rows, grid.width(g),
                         indices[start:start + tile_nnz])
    out_ptr = [0]
    out_idx, out_val = [], []
    for r in range(rows):
        for g in range(grid.n_gene_blocks):
            start = int(tile_offsets[first_tile + g])
            a, e = start + int(shard[g, r]), start + int(shard[g, r + 1])
            out_idx.append(indices[a:e].astype(np.uint64) + g * grid.gene_block_size)
            out_val.append(data[a:e])
        out_ptr.append(out_ptr[-1] + sum(len(x) for x in out_idx[-grid.n_gene_blocks:]))
    idx = (np.concatenate(out_idx).astype(np.uint32) if out_idx
           else np.zeros(0, dtype=np.uint32))
    val = np.concatenate(out_val) if out_val else np.zeros(0, dtype=np.asarray(data).dtype)
    return np.asarray(out_ptr, dtype=np.uint64), idx, val


def encode_fast(indptr, indices, data, grid: TileGrid):
    """``encode`` vectorised for larger layers (the same arrays: entries ordered by cell
    block, gene block, row, then gene; zeros dropped; padding rows flat)."""
    indptr = np.asarray(indptr, dtype=np.uint64)
    indices = np.asarray(indices, dtype=np.uint64)
    data = np.asarray(data)
    c, gs, n_gb = grid.cell_block_size, grid.gene_block_size, grid.n_gene_blocks
    rows = np.repeat(np.arange(grid.n_cells, dtype=np.uint64), np.diff(indptr).astype(np.int64))
    keep = data != 0
    rows, idx, vals = rows[keep], indices[keep], data[keep]
    b, r, g = rows // c, rows % c, idx // gs
    order = np.lexsort((r, g, b))  # stable: each row's genes stay increasing
    local = (idx - g * gs).astype(np.uint32)[order]
    tiles = (b * n_gb + g).astype(np.int64)
    counts = np.bincount(tiles, minlength=grid.n_tiles)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    per_row = np.bincount((tiles * c + r.astype(np.int64)), minlength=grid.n_tiles * c)
    per_row = per_row.reshape(grid.n_cell_blocks, n_gb, c)
    shards = []
    for blk in range(grid.n_cell_blocks):
        sh = np.zeros((n_gb, c + 1), dtype=np.uint32)
        sh[:, 1:] = np.cumsum(per_row[blk], axis=1)
        shards.append(sh)
    return shards, offsets, local, vals[order]
