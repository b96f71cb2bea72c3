// The device join of a tiled layer's cell block into CSR rows (kg_tiles.cu).
#pragma once

#include "kg_internal.cuh"

namespace kg {

// The joined block's shape, read on the host from the block's tile_offsets (after the
// argument checks and the check that they never decrease).
struct TileShape {
  uint32_t n_gene_blocks = 0;
  uint64_t first = 0;            // tile_offsets of the block's first tile
  uint64_t nnz = 0;              // the block's entries
  std::vector<uint64_t> start;   // each tile's first entry, from the block's first
};

// Checks the block's arguments (KG_ERR_INVALID) and that its tile_offsets never
// decrease (KG_ERR_CORRUPT), reading them (host or device memory) on `s`.
TileShape tile_shape(const kg_tile_block* tb, cudaStream_t s);

// Joins the block's tiles (kyto's checks first; KG_ERR_CORRUPT on the first problem)
// into device outputs on `s`: indptr rows + 1 values, indices and values shape.nnz
// entries (values as their 4-byte words). Waits for the checks' verdict on the host.
void join_tiles(kg_ctx* ctx, cudaStream_t s, const kg_tile_block* tb, const TileShape& shape,
                uint64_t* d_indptr, uint32_t* d_indices, uint32_t* d_values);

}  // namespace kg
