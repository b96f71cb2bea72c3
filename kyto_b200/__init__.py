"""kyto_b200: kyto's PCA -> exact-kNN hot path on a B200, behind a C ABI.

The compute lives in ``libkyto_gpu.so`` (CUDA for sm_100a, C ABI in
``include/kyto_gpu.h``). This module is the host-side mirror of kyto's operator
interface for the path (kyto's ``Atlas.pca`` / ``Atlas.neighbors``, crates/kyto-py/src/
atlas.rs:823-966, over ``kyto_gpu::DeviceKernels``): the same argument names and
meanings, errors raised with kyto's codes. There is no CPU fallback: without the built
library or a CUDA device every call raises.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libkyto_gpu.so"

(KG_OK, KG_ERR_INVALID, KG_ERR_DEVICE, KG_ERR_OOM, KG_CANCELLED, KG_ERR_TIMEOUT, KG_ERR_STATE,
 KG_ERR_CORRUPT, KG_ERR_STORE) = range(9)
KG_U32, KG_F32 = 0, 1
KG_LEARNED_RANDOM_INIT = 1
NO_GENE = 0xFFFFFFFF

# kyto's error registry (errors.toml): the status a call returns -> kyto's code.
KYTO_CODE = {
    KG_ERR_INVALID: "KY-E215",
    KG_ERR_DEVICE: "KY-E505",
    KG_ERR_OOM: "KY-E505",
    KG_CANCELLED: "KY-E503",
    KG_ERR_TIMEOUT: "KY-E505",
    KG_ERR_STATE: "KY-E505",
    KG_ERR_CORRUPT: "KY-E107",
    KG_ERR_STORE: "KY-E110",
}

# Every entry point of include/kyto_gpu.h.
EXPORTS = (
    "kg_open", "kg_close", "kg_last_error", "kg_set_cancel_flag", "kg_reserve", "kg_progress",
    "kg_normalize_log1p", "kg_hvg_moments", "kg_hvg_moments_noalloc", "kg_hvg_seurat",
    "kg_pca_begin", "kg_pca_push_block", "kg_pca_run", "kg_pca_results", "kg_pca_info",
    "kg_pca_embedding_device", "kg_pca_free", "kg_pca_knn_batch", "kg_knn_exact",
    "kg_knn_batch", "kg_knn_learned",
    "kg_learned_layout", "kg_learned_gradients", "kg_diag_kernel_launches", "kg_connectivities",
    "kg_pca_run_stats", "kg_diag_omega", "kg_diag_pool_usage", "kg_diag_fail_allocations",
    "kg_tune_lookup", "kg_tune_store",
    "kg_set_wait_limit", "kg_diag_spmm", "kg_pca_push_block_async",
    "kg_tiles_to_csr", "kg_pca_push_tiles", "kg_pca_result_dlpack", "kg_dlpack_free",
    "kg_diag_dlpack_live", "kg_shard_read", "kg_chunk_read",
)


class KytoError(RuntimeError):
    """A failed call: ``code`` is kyto's error code, ``status`` the C ABI's."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.code = KYTO_CODE.get(status, "KY-E505")
        super().__init__(f"{self.code}: {message}")


class TileBlock(ctypes.Structure):
    """kg_tile_block: one cell block of a tiled sparse layer (kyto's store format)."""

    _fields_ = [
        ("block", ctypes.c_uint64),
        ("rows", ctypes.c_uint32),
        ("cell_block_size", ctypes.c_uint32),
        ("gene_block_size", ctypes.c_uint64),
        ("n_genes", ctypes.c_uint64),
        ("indptr", ctypes.c_void_p),
        ("tile_offsets", ctypes.c_void_p),
        ("indices", ctypes.c_void_p),
        ("data", ctypes.c_void_p),
        ("dtype", ctypes.c_int),
        ("reserved", ctypes.c_uint32),
    ]


class _PcaParams(ctypes.Structure):
    _fields_ = [
        ("n_components", ctypes.c_uint32),
        ("n_genes", ctypes.c_uint32),
        ("seed", ctypes.c_uint64),
        ("gene_map", ctypes.c_void_p),
        ("target_sum", ctypes.c_double),
        ("log1p", ctypes.c_int32),
        ("reserved", ctypes.c_uint32),
    ]


class KnnStats(ctypes.Structure):
    _fields_ = [
        ("candidates", ctypes.c_uint64),
        ("rows_full", ctypes.c_uint64),
        ("filter_ms", ctypes.c_double),
        ("rank_ms", ctypes.c_double),
        ("tiles_scanned", ctypes.c_uint64),
        ("tiles_total", ctypes.c_uint64),
    ]


class PcaStats(ctypes.Structure):
    """kg_pca_stats: the last run's sparse x dense products (device ms from CUDA events
    around each launch, algorithmic bytes) and the run's host wall time."""

    _fields_ = [
        ("product_launches", ctypes.c_uint32),
        ("passes_run", ctypes.c_uint32),
        ("product_ms", ctypes.c_double),
        ("product_bytes", ctypes.c_double),
        ("run_ms", ctypes.c_double),
    ]


class _BatchSample(ctypes.Structure):
    _fields_ = [
        ("indptr", ctypes.c_void_p),
        ("indices", ctypes.c_void_p),
        ("values", ctypes.c_void_p),
        ("dtype", ctypes.c_int32),
        ("reserved", ctypes.c_uint32),
        ("n_rows", ctypes.c_uint64),
    ]


class BatchStats(ctypes.Structure):
    _fields_ = [
        ("pca_ms", ctypes.c_double),
        ("knn_ms", ctypes.c_double),
        ("workers", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("knn", KnnStats),
    ]


class LearnedParams(ctypes.Structure):
    """kg_learned_params: the learned-partition kNN's settings (defaults: 1,024 parts,
    256 hidden, top-4 probes, fallback below confidence 0.3, 100,000 training rows, 4
    epochs of 8,192-row batches: the fastest setting of a sweep on a 4M-row,
    200-component Gaussian mixture at recall@15 >= 0.999)."""

    _fields_ = [
        ("n_parts", ctypes.c_uint32),
        ("hidden", ctypes.c_uint32),
        ("n_probe", ctypes.c_uint32),
        ("confidence", ctypes.c_float),
        ("train_cells", ctypes.c_uint64),
        ("epochs", ctypes.c_uint32),
        ("batch", ctypes.c_uint32),
        ("learning_rate", ctypes.c_float),
        ("flags", ctypes.c_uint32),
        ("seed", ctypes.c_uint64),
    ]

    def __init__(self, n_parts=1024, hidden=256, n_probe=4, confidence=0.3,
                 train_cells=100_000, epochs=4, batch=8192, learning_rate=1e-3, seed=0,
                 random_init=False):
        super().__init__(n_parts, hidden, n_probe, confidence, train_cells, epochs, batch,
                         learning_rate, KG_LEARNED_RANDOM_INIT if random_init else 0, seed)


class LearnedStats(ctypes.Structure):
    _fields_ = [
        ("fallback_rows", ctypes.c_uint64),
        ("scanned_tiles", ctypes.c_uint64),
        ("candidates", ctypes.c_uint64),
        ("rows_full", ctypes.c_uint64),
        ("train_ms", ctypes.c_double),
        ("index_ms", ctypes.c_double),
        ("search_ms", ctypes.c_double),
        ("final_loss", ctypes.c_float),
        ("temperature", ctypes.c_float),
        ("tiles_computed", ctypes.c_uint64),
    ]


_lib = None


def library() -> ctypes.CDLL:
    """The loaded ``libkyto_gpu.so``; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise KytoError(KG_ERR_DEVICE, f"{LIB_PATH} is missing: run `python -m kyto_b200.build`")
        lib = ctypes.CDLL(str(LIB_PATH))
        P, U64, U32, I32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int32
        sig = {
            "kg_open": [ctypes.c_int, ctypes.POINTER(P)],
            "kg_last_error": [P, ctypes.c_char_p, ctypes.c_size_t],
            "kg_set_cancel_flag": [P, P],
            "kg_reserve": [P, U64],
            "kg_set_wait_limit": [P, ctypes.c_double],
            "kg_progress": [P, P, P],
            "kg_normalize_log1p": [P, P, P, ctypes.c_int, U64, ctypes.c_double, I32, P],
            "kg_hvg_moments": [P, P, P, P, ctypes.c_int, U64, U32, ctypes.c_double, I32, P, P, P],
            "kg_hvg_moments_noalloc": [P, P, P, P, ctypes.c_int, U64, U32, ctypes.c_double, I32,
                                       P, P, P],
            "kg_hvg_seurat": [P, P, P, U64, U32, ctypes.c_int64, P, P, P, P],
            "kg_pca_begin": [P, ctypes.POINTER(_PcaParams), ctypes.POINTER(P)],
            "kg_pca_push_block": [P, P, P, P, ctypes.c_int, U64, P],
            "kg_pca_push_block_async": [P, P, P, P, ctypes.c_int, U64, P],
            "kg_tiles_to_csr": [P, ctypes.POINTER(TileBlock), P, P, P],
            "kg_pca_push_tiles": [P, ctypes.POINTER(TileBlock)],
            "kg_pca_result_dlpack": [P, I32, ctypes.POINTER(P)],
            "kg_diag_dlpack_live": [ctypes.POINTER(ctypes.c_int64)],
            "kg_shard_read": [P, U64, U64, U64, U32, U64, U64, P],
            "kg_chunk_read": [P, U64, U64, U32, P],
            "kg_pca_run": [P],
            "kg_pca_results": [P, P, P, P, P, P],
            "kg_pca_info": [P, P, P, P],
            "kg_pca_embedding_device": [P, ctypes.POINTER(P)],
            "kg_knn_exact": [P, P, U64, U32, U32, U32, P, P, P, ctypes.POINTER(KnnStats)],
            "kg_connectivities": [P, P, P, P, U64, U32, P, P, P, ctypes.POINTER(U64)],
            "kg_knn_batch": [P, P, U64, U32, U32, U32, P, U32, P, P, P,
                             ctypes.POINTER(KnnStats)],
            "kg_pca_knn_batch": [P, ctypes.POINTER(_PcaParams), U32, ctypes.POINTER(_BatchSample),
                                 U32, P, P, P, P, P, ctypes.POINTER(BatchStats)],
            "kg_knn_learned": [P, P, U64, U32, U32, U32, ctypes.POINTER(LearnedParams), P, P, P,
                               ctypes.POINTER(LearnedStats)],
            "kg_learned_layout": [U32, U32, U32, P, P],
            "kg_learned_gradients": [P, U32, U32, U32, P, P, U32, P, U32, P, P, P],
            "kg_diag_kernel_launches": [P],
            "kg_pca_run_stats": [P, ctypes.POINTER(PcaStats)],
            "kg_diag_omega": [P, U64, P, U64, U32, P],
            "kg_diag_pool_usage": [ctypes.c_int, P, P, P, I32],
            "kg_diag_fail_allocations": [U64],
            "kg_tune_lookup": [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                               ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t],
            "kg_tune_store": [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                              ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double],
            "kg_diag_spmm": [P, P, P, P, U64, U32, I32, I32, P, P, U32, P],
        }
        for name, args in sig.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        lib.kg_close.argtypes = [P]
        lib.kg_close.restype = None
        lib.kg_pca_free.argtypes = [P]
        lib.kg_pca_free.restype = None
        lib.kg_dlpack_free.argtypes = [P]
        lib.kg_dlpack_free.restype = None
        lib.kg_last_error.restype = ctypes.c_size_t
        _lib = lib
    return _lib


def _check(status: int) -> None:
    if status != KG_OK:
        buf = ctypes.create_string_buffer(4096)
        library().kg_last_error(None, buf, len(buf))
        raise KytoError(status, buf.value.decode(errors="replace"))


def _ptr(a):
    """A numpy array's data pointer, a torch tensor's (host or CUDA), or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(ctypes.c_void_p)
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    raise TypeError(f"not an array: {type(a)}")


class Context:
    """An open device (kg_open); closes itself when collected or on ``close()``."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        _check(library().kg_open(int(device), ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().kg_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_cancel_flag(self, flag: np.ndarray | None) -> None:
        _check(library().kg_set_cancel_flag(self._h, _ptr(flag)))

    def reserve(self, nbytes: int) -> None:
        """Reserve ``nbytes`` of device memory for this library's buffers up front
        (kg_reserve): later calls do not grow the device pool mid-call."""
        _check(library().kg_reserve(self._h, int(nbytes)))

    def set_wait_limit(self, seconds: float) -> None:
        """Seconds a call waits for its device work before KG_ERR_TIMEOUT."""
        _check(library().kg_set_wait_limit(self._h, float(seconds)))

    def progress(self) -> tuple[int, int]:
        done, total = ctypes.c_uint64(), ctypes.c_uint64()
        _check(library().kg_progress(self._h, ctypes.byref(done), ctypes.byref(total)))
        return done.value, total.value


_default: Context | None = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context(0)
    return _default


def _dtype_code(values) -> int:
    dt = values.dtype if isinstance(values, np.ndarray) else values.dtype
    name = str(dt)
    if name in ("uint32", "torch.uint32", "torch.int32", "int32"):
        return KG_U32
    if name in ("float32", "torch.float32"):
        return KG_F32
    raise TypeError(f"values must be uint32 counts or float32 values, not {name}")


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64) if isinstance(a, np.ndarray) else a


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32) if isinstance(a, np.ndarray) else a


def product(indptr, indices, values, n_cols: int, dense=None, transposed: bool = False,
            value_mode: int = 0, row_means=None, width: int | None = None,
            ctx: Context | None = None) -> np.ndarray:
    """One of the PCA's tensor-core products (kg_diag_spmm): S D as f64, rows x width."""
    ctx = ctx or default_context()
    indptr = _u64(indptr)
    n_rows = len(indptr) - 1
    rows = n_cols if transposed else n_rows
    K = n_rows if transposed else n_cols
    if dense is not None:
        dense = np.asfortranarray(dense, dtype=np.float64)
        assert dense.shape[0] == K
        width = dense.shape[1]
    width = int(width or 1)
    out = np.empty((width, rows))  # column-major rows x width
    means = None if row_means is None else np.ascontiguousarray(row_means, dtype=np.float64)
    _check(library().kg_diag_spmm(
        ctx.handle, _ptr(indptr), _ptr(_u32(indices)),
        _ptr(np.ascontiguousarray(values, dtype=np.float32)), n_rows, int(n_cols),
        int(bool(transposed)), int(value_mode), _ptr(means),
        None if dense is None else dense.ctypes.data_as(ctypes.c_void_p), width, _ptr(out)))
    return out.T


def omega(seed: int, cells, width: int, ctx: Context | None = None) -> np.ndarray:
    """Omega's rows as the device PCA draws them (kg_diag_omega): len(cells) x width f64."""
    ctx = ctx or default_context()
    cells = np.ascontiguousarray(cells, dtype=np.uint64)
    out = np.empty((len(cells), int(width)))
    _check(library().kg_diag_omega(ctx.handle, int(seed), _ptr(cells), len(cells), int(width),
                                   _ptr(out)))
    return out


def pool_usage(device: int = 0, reset_high: bool = False) -> dict:
    """The library's device pool: reserved, used and high-water bytes (kg_diag_pool_usage)."""
    r, u, h = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    _check(library().kg_diag_pool_usage(int(device), ctypes.byref(r), ctypes.byref(u),
                                        ctypes.byref(h), int(bool(reset_high))))
    return {"reserved": r.value, "used": u.value, "used_high": h.value}


def fail_allocations(after: int | None) -> None:
    """Test hook: fail every allocation after ``after`` more (None: stop failing)."""
    _check(library().kg_diag_fail_allocations(0xFFFFFFFFFFFFFFFF if after is None else int(after)))


def tune_lookup(path, gpu: str, cls: str, field: str) -> str | None:
    """The value of ``field`` in the tuner cache entry for (gpu, cls) in the file at
    ``path`` (kg_tune_lookup), or None."""
    buf = ctypes.create_string_buffer(256)
    r = library().kg_tune_lookup(str(path).encode(), gpu.encode(), cls.encode(), field.encode(),
                                 buf, len(buf))
    if r < 0:
        raise KytoError(KG_ERR_INVALID, "kg_tune_lookup: bad argument")
    return buf.value.decode() if r == 1 else None


def tune_store(path, gpu: str, cls: str, choice: dict, ms: float) -> bool:
    """Record ``choice`` (str -> str) for (gpu, cls) in the tuner cache file at ``path``
    (kg_tune_store); False if the file could not be written."""
    keys = ";".join(choice)
    values = ";".join(str(choice[k]) for k in choice)
    r = library().kg_tune_store(str(path).encode(), gpu.encode(), cls.encode(), keys.encode(),
                                values.encode(), float(ms))
    if r < 0:
        raise KytoError(KG_ERR_INVALID, "kg_tune_store: bad argument")
    return r == 1


def kernel_launches() -> int:
    """Kernels this library has launched since it was loaded."""
    c = ctypes.c_uint64()
    _check(library().kg_diag_kernel_launches(ctypes.byref(c)))
    return c.value


# ------------------------------------------------------------------ maps -------------
def normalize_log1p(indptr, values, target_sum: float | None = 1e4, log1p: bool = True,
                    ctx: Context | None = None) -> np.ndarray:
    """normalize_total(target_sum) then log1p of a CSR block's values (f32, one per
    stored value). ``target_sum=None`` skips normalize_total."""
    ctx = ctx or default_context()
    indptr = _u64(indptr)
    n_rows = len(indptr) - 1
    out = np.empty(int(indptr[-1]), dtype=np.float32)
    _check(library().kg_normalize_log1p(
        ctx.handle, _ptr(indptr), _ptr(values), _dtype_code(values), n_rows,
        math.nan if target_sum is None else float(target_sum), int(bool(log1p)), _ptr(out)))
    return out


@dataclass
class HvgResult:
    means: np.ndarray
    dispersions: np.ndarray
    dispersions_norm: np.ndarray
    highly_variable: np.ndarray


def highly_variable_genes(indptr, indices, values, n_genes: int, n_top_genes: int | None = 2000,
                          target_sum: float | None = 1e4, log1p: bool = True,
                          ctx: Context | None = None) -> HvgResult:
    """kyto's ``highly_variable_genes(flavor="seurat")`` on the log1p of normalized
    counts: the statistics pass on the device, the flags on the host."""
    ctx = ctx or default_context()
    indptr, indices = _u64(indptr), _u32(indices)
    n_rows = len(indptr) - 1
    sums = np.empty(n_genes)
    squares = np.empty(n_genes)
    positives = np.empty(n_genes, dtype=np.uint64)
    L = library()
    _check(L.kg_hvg_moments(
        ctx.handle, _ptr(indptr), _ptr(indices), _ptr(values), _dtype_code(values), n_rows,
        int(n_genes), math.nan if target_sum is None else float(target_sum), int(bool(log1p)),
        _ptr(sums), _ptr(squares), _ptr(positives)))
    means, disp, norm = np.empty(n_genes), np.empty(n_genes), np.empty(n_genes)
    flags = np.empty(n_genes, dtype=np.uint8)
    _check(L.kg_hvg_seurat(
        _ptr(sums), _ptr(squares), _ptr(positives), n_rows, int(n_genes),
        -1 if n_top_genes is None else int(n_top_genes), _ptr(means), _ptr(disp), _ptr(norm),
        _ptr(flags)))
    return HvgResult(means, disp, norm, flags.astype(bool))


# ------------------------------------------------------------------ PCA --------------
@dataclass
class PcaResult:
    """kyto's PcaStatistics (crates/kyto-exec/src/pca.rs:51-120)."""

    embedding: np.ndarray
    loadings: np.ndarray
    variance: np.ndarray
    variance_ratio: np.ndarray
    means: np.ndarray
    passes_run: int


class PcaSession:
    """One ``pca`` node: push the blocks in stream order, run, read the results."""

    def __init__(self, n_components: int, n_genes: int, seed: int = 0,
                 gene_set: np.ndarray | None = None, target_sum: float | None = None,
                 log1p: bool = False, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self._map = None
        if gene_set is not None:
            flags = np.asarray(gene_set, dtype=bool)
            if flags.shape != (n_genes,):
                raise KytoError(KG_ERR_INVALID, "gene_set must flag every gene")
            self._map = np.full(n_genes, NO_GENE, dtype=np.uint32)
            self._map[flags] = np.arange(int(flags.sum()), dtype=np.uint32)
        p = _PcaParams(int(n_components), int(n_genes), int(seed),
                       None if self._map is None else self._map.ctypes.data,
                       math.nan if target_sum is None else float(target_sum),
                       int(bool(log1p)), 0)
        h = ctypes.c_void_p()
        _check(library().kg_pca_begin(self.ctx.handle, ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.n_components = int(n_components)
        self.n_genes = int(n_genes)

    def push(self, indptr, indices, values, cells=None, wait: bool = True) -> None:
        """Push the next block. ``wait=False`` queues its copies and returns at once
        (kg_pca_push_block_async): the arrays must stay alive and unchanged until
        ``run()`` returns (the session keeps references to them until then)."""
        indptr, indices = _u64(indptr), _u32(indices)
        n_rows = (len(indptr) if isinstance(indptr, np.ndarray) else indptr.shape[0]) - 1
        fn = library().kg_pca_push_block if wait else library().kg_pca_push_block_async
        cells = _u64(cells) if cells is not None else None
        _check(fn(self._h, _ptr(indptr), _ptr(indices), _ptr(values), _dtype_code(values),
                  n_rows, _ptr(cells)))
        if not wait:
            self._held = getattr(self, "_held", []) + [indptr, indices, values, cells]

    def push_tiles(self, block: int, cell_block_size: int, gene_block_size: int, n_cells: int,
                   shard, tile_offsets, indices, data) -> None:
        """Push cell block ``block`` of a tiled layer (kg_pca_push_tiles): the tiles are
        joined into rows on the device after kyto's checks; arguments as
        ``tiles_to_csr``. Returns once the block is held on the device."""
        tb, keep = _tile_block(block, cell_block_size, gene_block_size, n_cells, self.n_genes,
                               shard, tile_offsets, indices, data)
        _check(library().kg_pca_push_tiles(self._h, ctypes.byref(tb)))
        del keep

    def result_dlpack(self, which: str = "embedding") -> "DeviceResult":
        """A PCA result kept on the device (kg_pca_result_dlpack) for a DLPack consumer:
        ``torch.from_dlpack(result)`` (or CuPy / JAX) takes it without a host copy. The
        result owns a device copy that outlives the session; one consumer may take it,
        else ``close()`` (or collection) gives it back."""
        code = {"embedding": 0, "loadings": 1}[which]
        out = ctypes.c_void_p()
        _check(library().kg_pca_result_dlpack(self._h, code, ctypes.byref(out)))
        return DeviceResult(out.value)

    def run(self) -> None:
        try:
            _check(library().kg_pca_run(self._h))
        finally:
            self._held = []

    def info(self) -> tuple[int, int, int]:
        n, g, p = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(library().kg_pca_info(self._h, ctypes.byref(n), ctypes.byref(g), ctypes.byref(p)))
        return n.value, g.value, p.value

    def stats(self) -> PcaStats:
        st = PcaStats()
        _check(library().kg_pca_run_stats(self._h, ctypes.byref(st)))
        return st

    def embedding_device_ptr(self) -> int:
        out = ctypes.c_void_p()
        _check(library().kg_pca_embedding_device(self._h, ctypes.byref(out)))
        return out.value

    def results(self) -> PcaResult:
        n, g, passes = self.info()
        k = self.n_components
        emb = np.empty((n, k), dtype=np.float32)
        load = np.empty((self.n_genes, k), dtype=np.float32)
        var, ratio, means = np.empty(k), np.empty(k), np.empty(g)
        _check(library().kg_pca_results(self._h, _ptr(emb), _ptr(load), _ptr(var),
                                        _ptr(ratio), _ptr(means)))
        return PcaResult(emb, load, var, ratio, means, passes)

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().kg_pca_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pca(indptr, indices, values, n_genes: int, n_components: int = 50, seed: int = 0,
        gene_set: np.ndarray | None = None, target_sum: float | None = None,
        log1p: bool = False, block_cells: int | None = None,
        ctx: Context | None = None) -> PcaResult:
    """kyto's ``pca(n_components, seed, genes=...)`` on a CSR matrix (optionally after
    normalize_total/log1p), pushed in blocks of ``block_cells`` cells."""
    sess = PcaSession(n_components, n_genes, seed, gene_set, target_sum, log1p, ctx)
    indptr = np.ascontiguousarray(indptr, dtype=np.uint64)
    n = len(indptr) - 1
    step = n if not block_cells else int(block_cells)
    for a in range(0, n, max(step, 1)):
        b = min(n, a + step)
        s, e = int(indptr[a]), int(indptr[b])
        sess.push(indptr[a:b + 1] - np.uint64(s), indices[s:e], values[s:e],
                  np.arange(a, b, dtype=np.uint64))
    sess.run()
    res = sess.results()
    sess.close()
    return res


# ------------------------------------------------------------------ neighbors --------
@dataclass
class Graph:
    """kyto's NeighborGraph: k = n_neighbors - 1 entries a row, columns increasing
    within a row, f32 distances."""

    indptr: np.ndarray
    indices: np.ndarray
    distances: np.ndarray
    stats: KnnStats | None = None


def neighbors(embedding, n_neighbors: int = 15, n_components: int | None = None,
              ctx: Context | None = None) -> Graph:
    """kyto's exact ``neighbors(n_neighbors, n_components, metric="euclidean")``."""
    ctx = ctx or default_context()
    if isinstance(embedding, np.ndarray):
        embedding = np.ascontiguousarray(embedding, dtype=np.float32)
    n, width = embedding.shape
    k = int(n_neighbors) - 1
    indptr = np.empty(n + 1, dtype=np.uint64)
    indices = np.empty(max(n * k, 0), dtype=np.uint32)
    dist = np.empty(max(n * k, 0), dtype=np.float32)
    stats = KnnStats()
    _check(library().kg_knn_exact(ctx.handle, _ptr(embedding), n, width,
                                  0 if n_components is None else int(n_components),
                                  int(n_neighbors), _ptr(indptr), _ptr(indices), _ptr(dist),
                                  ctypes.byref(stats)))
    return Graph(indptr, indices, dist, stats)


@dataclass
class Connectivities:
    """kyto's ConnectivityGraph: symmetric CSR, columns increasing in each row, f32
    weights in (0, 1]."""

    indptr: np.ndarray
    indices: np.ndarray
    weights: np.ndarray


def connectivities(graph: Graph, ctx: Context | None = None) -> Connectivities:
    """kyto's ``connectivities`` of a neighbour graph (scanpy's UMAP weights): the graph as
    ``neighbors`` returns it, n_neighbors - 1 entries a row."""
    ctx = ctx or default_context()
    indptr = np.ascontiguousarray(graph.indptr, dtype=np.uint64)
    indices = np.ascontiguousarray(graph.indices, dtype=np.uint32)
    dist = np.ascontiguousarray(graph.distances, dtype=np.float32)
    n = len(indptr) - 1
    k = len(indices) // n if n else 0
    out_indptr = np.empty(n + 1, dtype=np.uint64)
    out_indices = np.empty(max(2 * n * k, 1), dtype=np.uint32)
    out_weights = np.empty(max(2 * n * k, 1), dtype=np.float32)
    nnz = ctypes.c_uint64()
    _check(library().kg_connectivities(ctx.handle, _ptr(indptr), _ptr(indices), _ptr(dist), n,
                                       k + 1, _ptr(out_indptr), _ptr(out_indices),
                                       _ptr(out_weights), ctypes.byref(nnz)))
    m = nnz.value
    return Connectivities(out_indptr, out_indices[:m].copy(), out_weights[:m].copy())


def neighbors_batch(embeddings, n_neighbors: int = 15, n_components: int | None = None,
                    ctx: Context | None = None) -> list[Graph]:
    """Exact ``neighbors`` of every sample of a batch in one search (kg_knn_batch): one
    graph per sample, each equal to ``neighbors`` of that sample alone."""
    ctx = ctx or default_context()
    mats = [np.ascontiguousarray(e, dtype=np.float32) for e in embeddings]
    if not mats:
        raise ValueError("neighbors_batch: no samples")
    width = mats[0].shape[1]
    sizes = np.array([m.shape[0] for m in mats], dtype=np.uint64)
    first = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    x = np.ascontiguousarray(np.concatenate(mats, axis=0))
    n, S = int(first[-1]), len(mats)
    k = int(n_neighbors) - 1
    indptr = np.empty(n + S, dtype=np.uint64)
    indices = np.empty(max(n * k, 0), dtype=np.uint32)
    dist = np.empty(max(n * k, 0), dtype=np.float32)
    stats = KnnStats()
    _check(library().kg_knn_batch(ctx.handle, _ptr(x), n, width,
                                  0 if n_components is None else int(n_components),
                                  int(n_neighbors), _ptr(first), S, _ptr(indptr),
                                  _ptr(indices), _ptr(dist), ctypes.byref(stats)))
    out = []
    for s in range(S):
        a, b = int(first[s]), int(first[s + 1])
        out.append(Graph(indptr[a + s:b + s + 1].copy(), indices[a * k:b * k].copy(),
                         dist[a * k:b * k].copy(), stats))
    return out


def pca_neighbors_batch(samples, n_genes: int, n_components: int = 30, n_neighbors: int = 15,
                        seed: int = 0, target_sum: float | None = None, log1p: bool = False,
                        ctx: Context | None = None):
    """The batching form (kg_pca_knn_batch): ``pca`` then exact ``neighbors`` on each
    sample, every sample a CSR block ``(indptr, indices, values)``. Returns one
    ``(PcaResult, Graph)`` per sample (loadings and means not returned: None) and the
    batch's counters."""
    ctx = ctx or default_context()
    keep = []
    arr = (_BatchSample * len(samples))()
    for i, (indptr, indices, values) in enumerate(samples):
        indptr, indices = _u64(indptr), _u32(indices)
        keep += [indptr, indices, values]
        n_rows = (len(indptr) if isinstance(indptr, np.ndarray) else indptr.shape[0]) - 1
        arr[i] = _BatchSample(_ptr(indptr), _ptr(indices), _ptr(values), _dtype_code(values), 0,
                              n_rows)
    sizes = [int(arr[i].n_rows) for i in range(len(samples))]
    n, S, kc, k = sum(sizes), len(samples), int(n_components), int(n_neighbors) - 1
    p = _PcaParams(kc, int(n_genes), int(seed), None,
                   math.nan if target_sum is None else float(target_sum), int(bool(log1p)), 0)
    emb = np.empty((n, kc), dtype=np.float32)
    var = np.empty((S, kc), dtype=np.float64)
    indptr = np.empty(n + S, dtype=np.uint64)
    indices = np.empty(max(n * k, 0), dtype=np.uint32)
    dist = np.empty(max(n * k, 0), dtype=np.float32)
    stats = BatchStats()
    _check(library().kg_pca_knn_batch(ctx.handle, ctypes.byref(p), S, arr, int(n_neighbors),
                                      _ptr(emb), _ptr(var), _ptr(indptr), _ptr(indices),
                                      _ptr(dist), ctypes.byref(stats)))
    out, a = [], 0
    for s, m in enumerate(sizes):
        b = a + m
        res = PcaResult(embedding=emb[a:b].copy(), loadings=None, variance=var[s].copy(),
                        variance_ratio=None, means=None, passes_run=0)
        g = Graph(indptr[a + s:b + s + 1].copy(), indices[a * k:b * k].copy(),
                  dist[a * k:b * k].copy(), stats.knn)
        out.append((res, g))
        a = b
    return out, stats


def neighbors_learned(embedding, n_neighbors: int = 15, n_components: int | None = None,
                      params: LearnedParams | None = None,
                      ctx: Context | None = None) -> tuple[Graph, LearnedStats]:
    """The learned-partition kNN (kg_knn_learned): the graph of each row's n_neighbors - 1
    nearest rows among those its learned partitions propose, and the run's counters."""
    ctx = ctx or default_context()
    if isinstance(embedding, np.ndarray):
        embedding = np.ascontiguousarray(embedding, dtype=np.float32)
    n, width = embedding.shape
    k = int(n_neighbors) - 1
    indptr = np.empty(n + 1, dtype=np.uint64)
    indices = np.empty(max(n * k, 0), dtype=np.uint32)
    dist = np.empty(max(n * k, 0), dtype=np.float32)
    stats = LearnedStats()
    params = params or LearnedParams()
    _check(library().kg_knn_learned(ctx.handle, _ptr(embedding), n, width,
                                    0 if n_components is None else int(n_components),
                                    int(n_neighbors), ctypes.byref(params), _ptr(indptr),
                                    _ptr(indices), _ptr(dist), ctypes.byref(stats)))
    return Graph(indptr, indices, dist), stats


def learned_layout(din: int, hidden: int, parts: int) -> tuple[list[int], int]:
    """Offsets of W1, b1, W2, b2, W3, b3 in the network's packed parameters, and the total."""
    off = np.zeros(6, dtype=np.uint64)
    total = ctypes.c_uint64()
    _check(library().kg_learned_layout(din, hidden, parts, _ptr(off), ctypes.byref(total)))
    return [int(v) for v in off], total.value


def learned_gradients(params: np.ndarray, x: np.ndarray, labels: np.ndarray, hidden: int,
                      parts: int, ctx: Context | None = None):
    """One forward/backward pass of the partitioner network on the device: (gradients of
    the packed parameters, per-row losses, logits)."""
    ctx = ctx or default_context()
    x = np.ascontiguousarray(x, dtype=np.float32)
    labels = np.ascontiguousarray(labels, dtype=np.uint32)
    rows, din = x.shape
    grads = np.empty(params.shape, dtype=np.float32)
    loss = np.empty(rows, dtype=np.float32)
    logits = np.empty((rows, parts), dtype=np.float32)
    _check(library().kg_learned_gradients(
        ctx.handle, din, hidden, parts, _ptr(np.ascontiguousarray(params, dtype=np.float32)),
        _ptr(x), rows, _ptr(labels), labels.shape[1], _ptr(grads), _ptr(loss), _ptr(logits)))
    return grads, loss, logits


def _tile_block(block, cell_block_size, gene_block_size, n_cells, n_genes, shard, tile_offsets,
                indices, data):
    """A TileBlock for cell block ``block`` from the layer's arrays (the block's slices are
    taken here), and the arrays it points into (kept alive by the caller)."""
    c, g = int(cell_block_size), int(gene_block_size)
    n_gb = -(-int(n_genes) // g)
    rows = min(c, int(n_cells) - int(block) * c)
    to = tile_offsets[int(block) * n_gb:(int(block) + 1) * n_gb + 1]
    if isinstance(to, np.ndarray):
        to = np.ascontiguousarray(to, dtype=np.uint64)
    lo, hi = int(to[0]), int(to[-1])
    if hi < lo or hi > len(indices) or len(data) != len(indices):
        raise KytoError(KG_ERR_CORRUPT, f"the layer is corrupt: tile_offsets of cell block "
                                        f"{int(block)} end at {hi} but indices and data hold "
                                        f"{len(indices)} and {len(data)} entries")
    idx = indices[lo:hi] if hi > lo else indices
    val = data[lo:hi] if hi > lo else data
    if isinstance(shard, np.ndarray):
        shard = np.ascontiguousarray(shard, dtype=np.uint32)
    if isinstance(idx, np.ndarray):
        idx = np.ascontiguousarray(idx, dtype=np.uint32)
    tb = TileBlock(int(block), rows, c, g, int(n_genes), _ptr(shard).value if _ptr(shard) else None,
                   _ptr(to).value, _ptr(idx).value if len(idx) else None,
                   _ptr(val).value if len(val) else None, _dtype_code(data), 0)
    return tb, (shard, to, idx, val)


def _bytes_ptr(b):
    """A bytes-like object's data pointer (bytes, bytearray, numpy u8) and the object to
    keep alive while it is used."""
    a = np.frombuffer(b, dtype=np.uint8) if isinstance(b, (bytes, bytearray, memoryview)) else b
    return _ptr(a), a


def shard_read(shard, chunks_per_shard: int, chunk_elems: int, dtype, first: int, count: int,
               out=None) -> np.ndarray:
    """Elements [first, first + count) of one shard of a tiled layer's sharded array
    (kg_shard_read), decoded on the host into ``out`` (a new array if None; a page-locked
    torch tensor works too). A shard that cannot be read raises KytoError KY-E110."""
    dtype = np.dtype(dtype)
    if out is None:
        out = np.empty(int(count), dtype=dtype)
    p, keep = _bytes_ptr(shard)
    _check(library().kg_shard_read(p, len(keep), int(chunks_per_shard), int(chunk_elems),
                                   dtype.itemsize, int(first), int(count), _ptr(out)))
    return out


def read_sharded(shards, chunk_elems: int, shard_elems: int, dtype, first: int, count: int,
                 out=None) -> np.ndarray:
    """Elements [first, first + count) of a sharded array given as its shards' bytes in
    order (each read with ``shard_read`` into its part of ``out``)."""
    dtype = np.dtype(dtype)
    if out is None:
        out = np.empty(int(count), dtype=dtype)
    e, end = int(first), int(first) + int(count)
    while e < end:
        s = e // shard_elems
        stop = min(end, (s + 1) * shard_elems)
        shard_read(shards[s], shard_elems // chunk_elems, chunk_elems, dtype, e - s * shard_elems,
                   stop - e, out[e - first:stop - first])
        e = stop
    return out


def chunk_read(chunk, elems: int, dtype) -> np.ndarray:
    """One unsharded chunk (tile_offsets') decoded on the host (kg_chunk_read)."""
    dtype = np.dtype(dtype)
    out = np.empty(int(elems), dtype=dtype)
    p, keep = _bytes_ptr(chunk)
    _check(library().kg_chunk_read(p, len(keep), int(elems), dtype.itemsize, _ptr(out)))
    return out


def tiles_to_csr(block: int, cell_block_size: int, gene_block_size: int, n_cells: int,
                 n_genes: int, shard, tile_offsets, indices, data, ctx: Context | None = None):
    """Cell block ``block`` of a tiled layer joined into CSR rows on the device
    (kg_tiles_to_csr; kyto-store's decode_cell_block with its checks). ``shard``: the
    block's indptr shard (n_gene_blocks x (C + 1)); ``tile_offsets``, ``indices`` and
    ``data``: the whole layer's arrays (numpy, or torch tensors on the device). Returns
    (indptr u64 from 0, global gene indices u32, values) as numpy arrays; a corrupt tile
    raises KytoError with kyto's code KY-E107."""
    tb, keep = _tile_block(block, cell_block_size, gene_block_size, n_cells, n_genes, shard,
                           tile_offsets, indices, data)
    ctx = ctx or default_context()
    nnz = int(keep[1][-1]) - int(keep[1][0])
    out_ptr = np.empty(tb.rows + 1, dtype=np.uint64)
    out_idx = np.empty(nnz, dtype=np.uint32)
    vdt = np.float32 if tb.dtype == KG_F32 else np.uint32
    out_val = np.empty(nnz, dtype=vdt)
    _check(library().kg_tiles_to_csr(ctx.handle, ctypes.byref(tb), _ptr(out_ptr), _ptr(out_idx),
                                     _ptr(out_val)))
    return out_ptr, out_idx, out_val


_capsule_new = ctypes.pythonapi.PyCapsule_New
_capsule_new.restype = ctypes.py_object
_capsule_new.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]


class DeviceResult:
    """A DLPack tensor the library handed out (a DLManagedTensor owning a device copy),
    exported once through the DLPack protocol (``__dlpack__``: a "dltensor" capsule the
    consumer takes over, its deleter run when the consumer drops the tensor). Until
    then ``close()`` (or collection) runs the deleter here."""

    def __init__(self, managed: int):
        self._m = managed
        # DLTensor.device.device_id: after the data pointer and the device type.
        self._device = ctypes.c_int32.from_address(managed + 12).value

    def __dlpack_device__(self):
        return (2, self._device)  # kDLCUDA

    def __dlpack__(self, stream=None, max_version=None, dl_device=None, copy=None):
        # The copy is complete when the library returns it, so any consumer stream may
        # read it at once; the legacy capsule is what this producer offers.
        if self._m is None:
            raise BufferError("this result was already exported or closed")
        m, self._m = self._m, None
        return _capsule_new(m, b"dltensor", None)

    def close(self) -> None:
        m, self._m = self._m, None
        if m:
            library().kg_dlpack_free(m)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dlpack_live() -> int:
    """DLPack tensors handed out by the library whose deleter has not run yet."""
    n = ctypes.c_int64()
    _check(library().kg_diag_dlpack_live(ctypes.byref(n)))
    return int(n.value)
