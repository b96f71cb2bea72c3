/*
 * kyto_gpu.h - the C ABI of libkyto_gpu.so, a B200 (sm_100a) backend for kyto's
 * PCA -> exact-kNN hot path.
 *
 * It replaces, for this path, the Rust type `kyto_gpu::DeviceKernels` of datavil/kyto
 * (crates/kyto-gpu/src/launch.rs:42-93, launch_matrix.rs:183-287) with coarser,
 * device-resident calls: a whole PCA (all 11 Krylov passes, the input held in HBM) or a
 * whole exact-kNN search per call instead of one host round trip per fold.
 *
 * Conventions (all entry points):
 *  - Plain pointers and sizes only. Array arguments may be host or device (CUDA)
 *    pointers unless a comment says otherwise; host arrays are only read or written
 *    during the call.
 *  - Every call returns a kg_status; no C++ exception crosses the ABI. After an error
 *    kg_last_error() gives the message (kyto's KytoError text goes there).
 *  - Status -> kyto error code: KG_ERR_INVALID -> KY-E215, KG_ERR_DEVICE / KG_ERR_OOM /
 *    KG_ERR_TIMEOUT / KG_ERR_STATE -> KY-E505, KG_CANCELLED -> KY-E503
 *    (kyto errors.toml:635,790,826,839).
 *  - A kg_ctx may be used from several threads for distinct sessions (each session
 *    has its own CUDA stream); one session is used from one thread at a time.
 *  - Results are the same bits run to run (no floating-point atomics on any path).
 */
#ifndef KYTO_GPU_H
#define KYTO_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define KG_API __attribute__((visibility("default")))
#else
#define KG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum kg_status {
  KG_OK = 0,
  KG_ERR_INVALID = 1,   /* input outside the contract (kyto: KY-E215) */
  KG_ERR_DEVICE = 2,    /* a CUDA call failed (kyto: KY-E505) */
  KG_ERR_OOM = 3,       /* device memory exhausted (KY-E505, "lower memory_limit") */
  KG_CANCELLED = 4,     /* the cancel flag was set (kyto: KY-E503) */
  KG_ERR_TIMEOUT = 5,   /* a bounded wait on the device ran out (KY-E505) */
  KG_ERR_STATE = 6,     /* calls out of order, e.g. results before run (KY-E505) */
  KG_ERR_CORRUPT = 7,   /* a tiled layer breaks the store format (kyto: KY-E107) */
  KG_ERR_STORE = 8      /* a stored shard or chunk cannot be read (kyto: KY-E110) */
} kg_status;

/* Value type of a CSR block: kyto's CellValues::{U32, F32}
 * (crates/kyto-store/src/cell_block.rs). */
typedef enum kg_dtype { KG_U32 = 0, KG_F32 = 1 } kg_dtype;

typedef struct kg_ctx kg_ctx;
typedef struct kg_pca kg_pca;

/* ---------------------------------------------------------------- context --------- */

/* Open device `device` (a CUDA ordinal). Replaces DeviceKernels::open
 * (crates/kyto-gpu/src/launch.rs:81-93). */
KG_API kg_status kg_open(int device, kg_ctx** out);
/* Close a context; every PCA session begun on it must be freed first (a freed session
 * returns its stream and solver handles to the context for the next session). */
KG_API void kg_close(kg_ctx* ctx);

/* The last error's message, NUL-terminated into buf (truncated to len); returns the
 * message length. Thread-local per context. */
KG_API size_t kg_last_error(const kg_ctx* ctx, char* buf, size_t len);

/* A flag polled between passes and query tiles; nonzero cancels the running call
 * with KG_CANCELLED. Replaces RunControl::check (crates/kyto-exec/src/run_control.rs,
 * called at neighbors_gpu.rs:95). NULL clears it. */
KG_API kg_status kg_set_cancel_flag(kg_ctx* ctx, const volatile int32_t* flag);

/* How long a call waits for its device work before it returns KG_ERR_TIMEOUT (default
 * 900 s). The host stops waiting; the work already queued on the device still runs to its
 * end, and may still write the call's outputs: synchronize the device (or close the
 * context) before reusing or freeing them. No kyto counterpart (kyto's GPU calls block
 * without a limit); a deadline for serving processes. */
KG_API kg_status kg_set_wait_limit(kg_ctx* ctx, double seconds);

/* Reserve `bytes` of device memory for the library's allocations up front. Every device
 * buffer of this library comes from its own stream-ordered pool on the device (created at
 * the first kg_open there, never the device's default pool), which keeps what it frees
 * until the process ends: later calls carve their buffers out of the reserve instead of
 * growing the pool, whose driver calls can block the host for tens to hundreds of
 * milliseconds mid-call. Other allocators in the process (a PyTorch caching allocator, a
 * CuPy pool) cannot use memory this pool holds. No kyto counterpart (a deployment knob of
 * this library); 0 does nothing. */
KG_API kg_status kg_reserve(kg_ctx* ctx, uint64_t bytes);

/* Work done / total of the running or last call, in cells (all passes counted), as
 * RunControl::progress. */
KG_API kg_status kg_progress(const kg_ctx* ctx, uint64_t* done, uint64_t* total);

/* ---------------------------------------------------------------- maps ------------ */

/* normalize_total(target_sum) then log1p of one CSR block, into out (nnz f32):
 * total = the row's values summed in f64 (8 lanes, kyto's fixed tree), divisor =
 * f32(total) / f32(target_sum) (0 -> 1), value = f32(v) / divisor (IEEE f32
 * division), log1p = f32(log1p(f64(v))). target_sum NaN skips normalize_total;
 * log1p 0 skips log1p. Replaces DeviceKernels::{row_sums, divide_rows, log1p}
 * (crates/kyto-gpu/src/launch.rs:106-173) as kyto-exec/src/elementwise.rs:205-235
 * calls them. */
KG_API kg_status kg_normalize_log1p(kg_ctx* ctx, const uint64_t* indptr, const void* values,
                             kg_dtype dtype, uint64_t n_rows, double target_sum,
                             int32_t log1p, float* out);

/* The seurat statistics pass of highly_variable_genes over one CSR block, with
 * normalize_total/log1p (as kg_normalize_log1p) fused in: per gene sum of
 * t = f32(expm1(f64(x))), sum of f32(t*t) (both f64) and the cells with x > 0.
 * Replaces HvgAccumulator::fold_rows (crates/kyto-exec/src/hvg_pass.rs:157-219).
 * Each gene's sums add its cells in cell order (the bits of one kyto leaf). */
KG_API kg_status kg_hvg_moments(kg_ctx* ctx, const uint64_t* indptr, const uint32_t* indices,
                         const void* values, kg_dtype dtype, uint64_t n_rows,
                         uint32_t n_genes, double target_sum, int32_t log1p,
                         double* sums, double* sums_of_squares, uint64_t* positives);

/* kg_hvg_moments without any allocation. No counterpart in the reference: kyto's
 * fold_rows allocates freely; this variant is for callers that cannot, such as a
 * process whose device memory is already held by another allocator's pool (a PyTorch
 * caching allocator, a fixed arena), where a fresh cudaMallocAsync can fail with
 * out-of-memory while the pool still has room, or a per-block fold deep in a long
 * streaming pass that must not fail late for lack of memory.
 * Same arguments and results as kg_hvg_moments, with these limits:
 * - indptr, indices and values must be device memory (staging host inputs would
 *   allocate); the outputs may be host or device memory;
 * - at most 1,048,576 stored values per block and 65,536 genes; larger inputs return
 *   KG_ERR_INVALID before any launch.
 * Its scratch is one fixed 22.1 MB array of static device memory per device. The first
 * call on a device sets it up (cudaGetSymbolAddress, which loads the code module there
 * and with it the array): that first call takes the 22.1 MB from the device and can
 * itself fail with KG_ERR_OOM on a full device, so make it early (at start-up, before
 * the device fills and before any stream capture); later calls take no memory. Every
 * call on a device shares the
 * array: calls that overlap in time (two contexts on one device from two threads, or a
 * call made while the kernels of a call that returned KG_CANCELLED or KG_ERR_TIMEOUT
 * still run) race on it and give wrong results. */
KG_API kg_status kg_hvg_moments_noalloc(kg_ctx* ctx, const uint64_t* indptr,
                                        const uint32_t* indices, const void* values,
                                        kg_dtype dtype, uint64_t n_rows, uint32_t n_genes,
                                        double target_sum, int32_t log1p, double* sums,
                                        double* sums_of_squares, uint64_t* positives);

/* seurat flags from the moments (host arithmetic on n_genes values, as kyto runs it on
 * the host): crates/kyto-exec/src/hvg.rs:284-361,393-437,501-580. n_top_genes < 0
 * uses scanpy's mean/dispersion cutoffs. Outputs are host arrays of n_genes. */
KG_API kg_status kg_hvg_seurat(const double* sums, const double* sums_of_squares,
                        const uint64_t* positives, uint64_t n_cells, uint32_t n_genes,
                        int64_t n_top_genes, double* means, double* dispersions,
                        double* dispersions_norm, uint8_t* highly_variable);

/* ---------------------------------------------------------------- PCA ------------- */

typedef struct kg_pca_params {
  uint32_t n_components;     /* k (kyto: pca(n_components=...)) */
  uint32_t n_genes;          /* genes of the pushed blocks (the stream's genes) */
  uint64_t seed;             /* kyto: pca(seed=...), drives Omega (pca.rs:936-950) */
  const uint32_t* gene_map;  /* NULL: every gene; else n_genes entries, the gene's
                                position among the PCA's genes or 0xFFFFFFFF to skip
                                it (pca.rs:352-372: pca(genes=...) / HVG selection) */
  double target_sum;         /* normalize_total before the PCA; NaN: none */
  int32_t log1p;             /* nonzero: log1p after normalize_total */
  uint32_t reserved;
} kg_pca_params;

/* Start a PCA session (kyto's PcaAccumulator::new, pca.rs:343-403). */
KG_API kg_status kg_pca_begin(kg_ctx* ctx, const kg_pca_params* params, kg_pca** out);

/* Push the next block of cells in stream order (kyto's store cell blocks). The block
 * is copied to the device, normalized/log1p'd/gene-selected there in one kernel and
 * held in HBM for every pass (kyto's held input, held_input.rs). cells: each row's
 * table position (Omega's seed input); NULL numbers the rows on from the last
 * block. */
KG_API kg_status kg_pca_push_block(kg_pca* pca, const uint64_t* indptr, const uint32_t* indices,
                            const void* values, kg_dtype dtype, uint64_t n_rows,
                            const uint64_t* cells);

/* kg_pca_push_block without waiting: the block's host->device copies and pack kernels
 * are queued on the session's own stream and the call returns at once, so the copies
 * (cudaMemcpyAsync, truly asynchronous from pinned host memory) run beside other work on
 * the device, such as another session's passes or a kNN search (kyto's streaming of
 * store blocks through pinned buffers, kyto-exec/src/block_stream.rs:65-303). The host
 * arrays stay in use until kg_pca_run returns: the caller keeps them alive and
 * unchanged until then. Gene indices are checked when the run starts (KG_ERR_INVALID
 * there); without a gene map and with a host indptr the call does not wait on the
 * device at all. */
KG_API kg_status kg_pca_push_block_async(kg_pca* pca, const uint64_t* indptr,
                                         const uint32_t* indices, const void* values,
                                         kg_dtype dtype, uint64_t n_rows, const uint64_t* cells);

/* One cell block of a tiled sparse layer as kyto's store holds it (docs/format.md
 * 4.1-4.3): tile (b, g) covers cells [b C, b C + rows) and genes [g G, g G + width(g)),
 * width(g) = min(G, n_genes - g G); its entries are a CSR of local gene indices. The
 * arrays are those kyto-store's reader decodes from the layer's shards (zstd inner
 * chunks), host (page-locked or not) or device memory. */
typedef struct kg_tile_block {
  uint64_t block;               /* cell block number b */
  uint32_t rows;                /* rows(b): C, or fewer in the last cell block */
  uint32_t cell_block_size;     /* C */
  uint64_t gene_block_size;     /* G */
  uint64_t n_genes;             /* the layer's genes; n_gene_blocks = ceil(n_genes / G) */
  const uint32_t* indptr;       /* the block's indptr shard, n_gene_blocks x (C + 1) */
  const uint64_t* tile_offsets; /* the layer's tile_offsets[b n_gene_blocks ..
                                   (b + 1) n_gene_blocks], n_gene_blocks + 1 values */
  const uint32_t* indices;      /* the block's entries: the layer's indices from
                                   tile_offsets[b n_gene_blocks] on (local gene indices) */
  const void* data;             /* the same entries' values */
  kg_dtype dtype;
  uint32_t reserved;
} kg_tile_block;

/* Join one cell block's tiles into CSR rows with global gene indices, on the device,
 * after kyto's checks of every tile (indptr starts at 0, ends at the tile's nnz, never
 * decreases and is flat over padding rows; each row's local indices strictly increase
 * below the block width). Replaces decode_cell_block and its checks
 * (crates/kyto-store/src/tile_decode.rs:74-196); the first problem, in kyto's order (tile,
 * then check, then row), returns KG_ERR_CORRUPT with kyto's wording, and no entry is
 * read through an indptr that failed its check. Outputs (host or device): indptr
 * rows + 1 values from 0; indices and values tile_offsets[last] - tile_offsets[0]
 * entries, each row's genes in increasing order. */
KG_API kg_status kg_tiles_to_csr(kg_ctx* ctx, const kg_tile_block* block, uint64_t* indptr,
                                 uint32_t* indices, void* values);

/* Elements [first, first + count) of one shard of a sharded array of kyto's tiled
 * layers (indptr, indices or data: Zarr v3 sharding_indexed, inner chunks
 * [bytes(little), zstd], index [bytes(little), crc32c] at the shard's end; docs/format.md
 * 4.4), decoded on the host into `out` (elem_bytes 4 or 8; a page-locked buffer lets the
 * tile join's copies run at the link's rate). shard: the shard file's bytes;
 * chunks_per_shard and chunk_elems: the array's shard and inner chunk shapes (an indptr
 * shard: n_gene_blocks chunks of C + 1; indices and data: S / K chunks of K); first: from
 * the shard's first element. A chunk the range covers whole decodes straight into `out`;
 * a chunk that is not stored reads as zeros. A short shard, an index whose CRC-32C does
 * not match, a chunk outside the shard or one that does not decode to its full shape
 * returns KG_ERR_STORE (KY-E110). Replaces the read of a tile's arrays through kyto's
 * Zarr crate (crates/kyto-store/src/tile_reader.rs:304-383, read_subset :444-452).
 * Host code: needs no device. */
KG_API kg_status kg_shard_read(const uint8_t* shard, uint64_t shard_bytes,
                               uint64_t chunks_per_shard, uint64_t chunk_elems,
                               uint32_t elem_bytes, uint64_t first, uint64_t count, void* out);

/* One unsharded chunk ([bytes(little), zstd]: tile_offsets' chunks, docs/format.md 4.4)
 * decoded into `out` (elems elements of elem_bytes 4 or 8). KG_ERR_STORE if it does not
 * decode to exactly that. Host code: needs no device. */
KG_API kg_status kg_chunk_read(const uint8_t* chunk, uint64_t chunk_bytes, uint64_t elems,
                               uint32_t elem_bytes, void* out);

/* kg_pca_push_block of one tiled cell block: the tiles are joined on the device
 * (kg_tiles_to_csr, into the session's scratch) and pushed as they are, each row's
 * table position b C + r as its cell (Omega's seed input). Replaces the host row
 * rebuild of crates/kyto-exec/src/pca/gpu.rs:73-115 for a tiled store: no CSR is built
 * on the host. Returns once the block is held on the device. */
KG_API kg_status kg_pca_push_tiles(kg_pca* pca, const kg_tile_block* block);

/* Run all passes on the device (pass 0 sketch, 9 Krylov products, the embedding pass)
 * with the FP64 orthonormalisation and Rayleigh-Ritz steps between them. Replaces
 * the folds of pca/gpu.rs:149-219 and PcaAccumulator::end_pass (pca.rs:699-801). */
KG_API kg_status kg_pca_run(kg_pca* pca);

/* Results (kyto's PcaStatistics, pca.rs:804-845): embedding n_cells x k f32 (row-major,
 * cell order), loadings n_genes x k f32 (zeros outside the gene set), variance and
 * variance_ratio k f64, means (one per PCA gene) f64. Any pointer may be NULL. */
KG_API kg_status kg_pca_results(kg_pca* pca, float* embedding, float* loadings, double* variance,
                         double* variance_ratio, double* means);

/* Sizes after run: cells pushed, PCA genes, passes run (fewer than 11 when the basis
 * spans the data early). */
KG_API kg_status kg_pca_info(const kg_pca* pca, uint64_t* n_cells, uint32_t* n_pca_genes,
                      uint32_t* passes_run);

/* The device address of the f32 embedding (n_cells x k) after run, valid until
 * kg_pca_free: lets kg_knn_exact search it without a host round trip. */
KG_API kg_status kg_pca_embedding_device(const kg_pca* pca, const float** out);

/* Device time of the last run's sparse x dense products (the PCA's HBM-bound hot loop:
 * the sketch X^T Omega, each pass's X Q and X^T W, the embedding pass X V, and the gene
 * statistics), from CUDA events around each launch on the session's stream, with their
 * algorithmic bytes (8 nnz + 4 (n + 1) + 4 g l + 4 n l each, l the product's width): the
 * figures a roofline of the products is computed from. No kyto counterpart (kyto's
 * GPU path times nothing); zero launches when the products ran on the SIMT path. */
typedef struct kg_pca_stats {
  uint32_t product_launches;
  uint32_t passes_run;
  double product_ms;
  double product_bytes;
  double run_ms;           /* kg_pca_run's host wall time */
} kg_pca_stats;

KG_API kg_status kg_pca_run_stats(const kg_pca* pca, kg_pca_stats* out);

/* A PCA result kept on the device and handed over as a DLPack tensor (DLPack's C ABI,
 * kDLCUDA on the session's device, kDLFloat 32, row-major, no strides): which =
 * KG_RESULT_EMBEDDING (n_cells x k) or KG_RESULT_LOADINGS (n_genes x k). The tensor owns
 * a device copy (cudaMalloc) that outlives the session; its deleter frees it (cudaFree,
 * which waits for queued work, so a consumer may drop it from any thread at any time).
 * Hand it to a consumer (torch.from_dlpack, CuPy, JAX) or give it back with
 * kg_dlpack_free. Replaces the host copy of kyto's embedding for a device consumer
 * (Implementation Plan.md:144, kDLCUDA export). */
#define KG_RESULT_EMBEDDING 0
#define KG_RESULT_LOADINGS 1
struct DLManagedTensor;
KG_API kg_status kg_pca_result_dlpack(kg_pca* pca, int32_t which, struct DLManagedTensor** out);

/* Calls a DLPack tensor's deleter (for a tensor no consumer took). */
KG_API void kg_dlpack_free(struct DLManagedTensor* tensor);

/* DLPack tensors this library handed out and whose deleter has not run yet. */
KG_API kg_status kg_diag_dlpack_live(int64_t* count);

KG_API void kg_pca_free(kg_pca* pca);

/* ---------------------------------------------------------------- exact kNN ------- */

typedef struct kg_knn_stats {
  uint64_t candidates;     /* approximate candidates ranked by their exact keys */
  uint64_t rows_full;      /* rows searched against every row (filter could not prove
                              its candidates complete) */
  double filter_ms;        /* device time of the candidate filter */
  double rank_ms;          /* device time of the exact re-rank (and full rows) */
  uint64_t tiles_scanned;  /* (query block, point tile) products the filter computed */
  uint64_t tiles_total;    /* of the query blocks x point tiles a full scan computes (the
                              rest skipped on proven distance bounds or not listed) */
} kg_knn_stats;

/* Each row's n_neighbors - 1 nearest other rows of `embedding` (n_rows x width f32,
 * row-major; the first n_components used, 0 = all) by kyto's exact key (the f64 sum of
 * squared f64 differences in kyto's 8-lane order), ties to the lower row, the row
 * itself excluded by position. Output: kyto's NeighborGraph CSR (neighbors.rs:412-435):
 * indptr n_rows+1 (u64), indices and distances n_rows*(n_neighbors-1), each row's
 * columns increasing, distance f32(sqrt(key)). The same graph as kyto's CPU exact
 * search (neighbors_exact.rs:50-356) bit for bit. Replaces neighbors_gpu::exact +
 * DeviceKernels::nearest_keys (neighbors_gpu.rs:70-127, launch_matrix.rs:253-287). */
KG_API kg_status kg_knn_exact(kg_ctx* ctx, const float* embedding, uint64_t n_rows,
                       uint32_t width, uint32_t n_components, uint32_t n_neighbors,
                       uint64_t* indptr, uint32_t* indices, float* distances,
                       kg_knn_stats* stats);

/* Exact kNN of a batch of samples in one search (the batching form): sample
 * s is rows [sample_rows[s], sample_rows[s + 1]) of `embedding` (sample_rows: host array
 * of n_samples + 1 offsets from 0 to n_rows); each row gets the n_neighbors - 1 nearest
 * rows of its own sample, exactly as kg_knn_exact on that sample alone. One filter launch
 * covers every sample (each block of query rows scans only its samples' point tiles).
 * Outputs: the samples' CSR graphs one after another: sample s's indptr (its rows + 1
 * entries, from 0) at indptr + sample_rows[s] + s (n_rows + n_samples entries in all),
 * its columns (numbered from its own first row) and distances at
 * sample_rows[s] * (n_neighbors - 1). */
KG_API kg_status kg_knn_batch(kg_ctx* ctx, const float* embedding, uint64_t n_rows,
                              uint32_t width, uint32_t n_components, uint32_t n_neighbors,
                              const uint64_t* sample_rows, uint32_t n_samples,
                              uint64_t* indptr, uint32_t* indices, float* distances,
                              kg_knn_stats* stats);

/* One sample of a batch: a CSR block (as kg_pca_push_block takes it). */
typedef struct kg_batch_sample {
  const uint64_t* indptr;
  const uint32_t* indices;
  const void* values;
  kg_dtype dtype;
  uint32_t reserved;
  uint64_t n_rows;
} kg_batch_sample;

typedef struct kg_batch_stats {
  double pca_ms;           /* all samples' PCA (host wall time) */
  double knn_ms;           /* the batched search and its graphs */
  uint32_t workers;        /* PCA sessions run at once */
  uint32_t reserved;
  kg_knn_stats knn;        /* the batched search's counters */
} kg_batch_stats;

/* The batching form end to end: kyto's pca(n_components, seed) and neighbors(n_neighbors)
 * on each of n_samples samples of uneven sizes (each as kg_pca_begin/push/run and
 * kg_knn_exact on that sample alone would give it). The samples' PCA sessions run
 * concurrently, each on its own stream with its own solver handles, so the GPU
 * interleaves the small samples' kernels; the embeddings are then searched in one
 * batched kNN launch (kg_knn_batch). Outputs: embedding (all samples' rows one after
 * another, n_components each, f32), variance (n_samples x n_components), and the
 * graphs laid out as kg_knn_batch's. */
KG_API kg_status kg_pca_knn_batch(kg_ctx* ctx, const kg_pca_params* params, uint32_t n_samples,
                                  const kg_batch_sample* samples, uint32_t n_neighbors,
                                  float* embedding, double* variance, uint64_t* indptr,
                                  uint32_t* indices, float* distances, kg_batch_stats* stats);

/* ---------------------------------------------------------------- connectivities -- */

/* scanpy's UMAP connectivities of a kNN graph (pp.neighbors(method="umap"): umap-learn's
 * fuzzy_simplicial_set with set_op_mix_ratio 1, local_connectivity 1), as kyto computes
 * them: per row rho (its smallest distance above 0) and sigma (a 64-step f64 bisection to
 * log2(n_neighbors) within 1e-5, floored at 1e-3 of the row's mean distance, of every
 * distance for rows whose distances are all 0), memberships exp(-max(0, d - rho) / sigma)
 * in f32 (0 for an entry naming its own row), and the fuzzy union w + w^T - w o w^T in f32
 * with zeros dropped. Input: a graph as kg_knn_exact writes it (indptr n_rows + 1 = r *
 * (n_neighbors - 1); each row's columns strictly increasing; f32 distances), host or
 * device pointers. Output: the symmetric CSR (out_indptr n_rows + 1, columns increasing in
 * each row) with *out_nnz entries; out_indices / out_weights must hold
 * 2 * n_rows * (n_neighbors - 1) entries. Replaces kyto's
 * connectivities::connectivities (crates/kyto-exec/src/connectivities.rs:84-131), called
 * at pipeline.rs:638 and umap.rs:607. */
KG_API kg_status kg_connectivities(kg_ctx* ctx, const uint64_t* indptr, const uint32_t* indices,
                                   const float* distances, uint64_t n_rows,
                                   uint32_t n_neighbors, uint64_t* out_indptr,
                                   uint32_t* out_indices, float* out_weights,
                                   uint64_t* out_nnz);

/* ------------------------------------------------------- learned-partition kNN ---- */

/* No counterpart in kyto: the learned-partition form of the search. A BF16 MLP (n_components ->
 * hidden -> hidden -> n_parts, ReLU) is trained on the device on the exact kNN graph of
 * train_cells evenly strided rows (it starts as the k-means parts' nearest-centre
 * classifier; targets: the parts of a row and of its n_neighbors - 1 neighbours;
 * soft-target cross-entropy, Adam, `epochs` seeded shuffles of `batch` rows). Every row
 * then gets its n_probe most probable parts and lives in the most probable one; rows in
 * that order form blocks of 256 query rows, and a row is searched exactly (kg_knn_exact's
 * filter and re-rank) among the rows of the parts its block probes (the union of the
 * block's rows' n_probe parts), or against every row when its probability in those
 * parts is below `confidence`. The probability is the softmax at a temperature
 * calibrated on the sample: the one whose top-n_probe mass best predicts, by
 * cross-entropy, the share of a sample row's exact neighbours living in those parts. */
typedef struct kg_learned_params {
  uint32_t n_parts;        /* partitions (>= 2) */
  uint32_t hidden;         /* hidden width */
  uint32_t n_probe;        /* parts searched per row (1..64) */
  float confidence;        /* below: the row is searched against every row */
  uint64_t train_cells;    /* sampled rows whose exact graph trains the network (0: all) */
  uint32_t epochs;         /* passes over the sample */
  uint32_t batch;          /* rows per training step */
  float learning_rate;     /* Adam's */
  uint32_t flags;          /* KG_LEARNED_RANDOM_INIT: start from random weights instead of
                              the sample's nearest-part classifier */
  uint64_t seed;
} kg_learned_params;

#define KG_LEARNED_RANDOM_INIT 1u

typedef struct kg_learned_stats {
  uint64_t fallback_rows;  /* rows searched against every row (low confidence) */
  uint64_t scanned_tiles;  /* point tiles (128 rows) in the query blocks' probe lists, in
                              all: what the network proposes */
  uint64_t candidates;     /* approximate candidates ranked by their exact keys */
  uint64_t rows_full;      /* rows searched in full by the exact re-rank's own checks */
  double train_ms;         /* sample graph, parts and training (host wall time) */
  double index_ms;         /* every row's parts */
  double search_ms;        /* the restricted exact search and the graph */
  float final_loss;        /* mean cross-entropy of the last training batch */
  float temperature;       /* the confidence's calibrated temperature (logits scale) */
  uint64_t tiles_computed; /* of those, the (block, tile) products the filter computed (the
                              rest skipped on proven distance bounds) */
} kg_learned_stats;

/* The graph (as kg_knn_exact's: CSR, rows sorted by column, f32 distances) of each
 * row's n_neighbors - 1 nearest rows among those the learned partitions propose. */
KG_API kg_status kg_knn_learned(kg_ctx* ctx, const float* embedding, uint64_t n_rows,
                                uint32_t width, uint32_t n_components, uint32_t n_neighbors,
                                const kg_learned_params* params, uint64_t* indptr,
                                uint32_t* indices, float* distances, kg_learned_stats* stats);

/* Offsets (floats) of W1, b1, W2, b2, W3, b3 in the network's packed f32 parameters
 * (W row-major out x in) and their total. */
KG_API kg_status kg_learned_layout(uint32_t din, uint32_t hidden, uint32_t parts,
                                   uint64_t* offsets /* 6 */, uint64_t* total);

/* One forward and backward pass of the network on `rows` rows of x (rows x din f32):
 * the gradients of the mean soft-target cross-entropy (targets: each row's n_labels
 * part labels, equally weighted) with respect to the packed parameters, each row's loss
 * and (if not NULL) the logits (rows x parts). For checking the device kernels. */
KG_API kg_status kg_learned_gradients(kg_ctx* ctx, uint32_t din, uint32_t hidden,
                                      uint32_t parts, const float* params, const float* x,
                                      uint32_t rows, const uint32_t* labels,
                                      uint32_t n_labels, float* grads, float* row_loss,
                                      float* logits);

/* ---------------------------------------------------------------- diagnostics ----- */

/* Kernels of this library launched since it was loaded (library calls such as cuBLAS
 * not counted): lets a benchmark state how many of its own kernels a timed region ran.
 * No counterpart in kyto (diagnostics only). */
KG_API kg_status kg_diag_kernel_launches(uint64_t* count);

/* The library's device pool on `device`: bytes reserved from the driver, bytes in use by
 * live buffers, and the high-water mark of bytes in use (reset to the current use when
 * reset_high is nonzero). Any pointer may be NULL. No kyto counterpart (diagnostics). */
KG_API kg_status kg_diag_pool_usage(int device, uint64_t* reserved, uint64_t* used,
                                    uint64_t* used_high, int32_t reset_high);

/* Test hook: after `after` more device allocations by this library, every allocation fails
 * as out of memory (the call returns KG_ERR_OOM and frees what it allocated); UINT64_MAX
 * turns the injection off. No kyto counterpart (tests the KG_ERR_OOM path without
 * exhausting a GPU). */
KG_API kg_status kg_diag_fail_allocations(uint64_t after);

/* One of the PCA's tensor-core products on a caller's CSR matrix (n_rows x n_cols, f32
 * values, columns strictly increasing in each row; host or device arrays), through the
 * same blocked layout and kernel the PCA uses: out (rows x width, column-major f64) =
 * S D, with S the matrix (transposed = 0: rows = n_rows, K = n_cols) or its transpose
 * (transposed = 1: rows = n_cols, K = n_rows), each stored value first mapped by
 * value_mode (0: as is; 1: (v - row_means[row])^2; 2: 1), and D the K x width
 * column-major f64 `dense` (value modes 1 and 2: D is a column of ones and `dense` is
 * ignored). width 1..64, n_cols <= 65,535. No kyto counterpart (diagnostics: lets a test
 * check the layout and the product against a plain f64 product). */
KG_API kg_status kg_diag_spmm(kg_ctx* ctx, const uint64_t* indptr, const uint32_t* indices,
                              const float* values, uint64_t n_rows, uint32_t n_cols,
                              int32_t transposed, int32_t value_mode, const double* row_means,
                              const double* dense, uint32_t width, double* out);

/* Omega's rows as the device PCA draws them (pca.rs:936-950, omega_row: SplitMix64
 * seeded from (seed, cells[r]), values (x >> 11) 2^-52 - 1), n x width f64 row-major;
 * cells host or device, out host or device, width 1..64. The device kernels of the PCA
 * take Omega from the same generator; this export lets a test pin its bits against
 * kyto's. No kyto counterpart (diagnostics only). */
KG_API kg_status kg_diag_omega(kg_ctx* ctx, uint64_t seed, const uint64_t* cells, uint64_t n,
                               uint32_t width, double* out);

/* The tuner's cache (no kyto counterpart; kyto's Config/flags layer chooses execution
 * knobs, this caches the device choices that cannot change a result). The library tunes
 * the kNN filter's operand kind and query-operand mode once per (GPU, shape class) and
 * keeps the choice in a versioned JSON file: KYTO_GPU_TUNE_CACHE (a path, or "off"),
 * else $XDG_CACHE_HOME/kyto_b200/tune.json, else $HOME/.cache/kyto_b200/tune.json;
 * KYTO_GPU_TUNE=retune tunes again and replaces the entry. These two entry points read
 * and write such a file directly (no GPU needed).
 *
 * kg_tune_lookup: the value of `field` in the choice stored for (gpu, cls) in the file
 * at `path`, NUL-terminated into out (out_len bytes). Returns 1 when found, 0 when
 * there is no such entry (or the file is missing, unreadable, malformed or of another
 * version), -1 for a NULL argument or a value longer than out_len - 1. */
KG_API int kg_tune_lookup(const char* path, const char* gpu, const char* cls,
                          const char* field, char* out, size_t out_len);

/* kg_tune_store: records the choice (keys and values: ';'-separated lists of the same
 * length) and its measured cost (ms) for (gpu, cls) in the file at `path`, replacing an
 * earlier entry for the same key and dropping entries of another version; the file is
 * written to a temporary and renamed over. Returns 1 on success, 0 if the file could not
 * be written, -1 for a NULL argument or lists of different lengths. */
KG_API int kg_tune_store(const char* path, const char* gpu, const char* cls, const char* keys,
                         const char* values, double ms);

#ifdef __cplusplus
}
#endif

#endif /* KYTO_GPU_H */
