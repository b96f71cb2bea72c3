"""Test infrastructure, not product code: the CPU oracle for kyto's PCA -> exact-kNN path.

Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import
this module, and only as the checker. It restates kyto's CPU algorithms (datavil/kyto,
paths within that project): the per-row and per-gene folds run in ``kyto_oracle.cpp``
(C++, OpenMP, no FMA contraction); the small dense FP64 steps (kyto's faer calls) run on
numpy's LAPACK here, so parity at that boundary holds to rounding, not to bits.

Pinned against kyto's checked-in golden vectors by ``tests/test_oracle_golden.py``.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libkyto_oracle.so"

PCA_POWER_ITERATIONS = 9  # crates/kyto-plan/src/physical_plan.rs:73
PCA_OVERSAMPLES = 10  # crates/kyto-plan/src/estimate.rs:153
PCA_PASSES = 2 + PCA_POWER_ITERATIONS  # crates/kyto-exec/src/pca.rs:123
DROP_TOLERANCE = 1e-10  # crates/kyto-exec/src/pca_dense.rs:30
N_BINS = 20  # crates/kyto-exec/src/hvg.rs:34
NO_GENE = 0xFFFFFFFF

_P = ctypes.c_void_p
_U64 = ctypes.c_uint64
_U32 = ctypes.c_uint32


def build(force: bool = False) -> Path:
    """Compile ``kyto_oracle.cpp`` into ``libkyto_oracle.so`` (beside it)."""
    src = HERE / "kyto_oracle.cpp"
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(
            ["make", "-C", str(HERE), "-s", "libkyto_oracle.so"], check=True
        )
    return LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        _lib.ko_knn_exact.restype = ctypes.c_uint64
        _lib.ko_knn_exact_range.restype = ctypes.c_uint64
        _lib.ko_knn_prepare.restype = ctypes.c_void_p
        _lib.ko_knn_prepare.argtypes = [_P, _U64, _U32]
        _lib.ko_knn_search.restype = ctypes.c_uint64
        _lib.ko_knn_search.argtypes = [ctypes.c_void_p, _U32, _U64, _U64, _P, _P]
        _lib.ko_knn_free.argtypes = [ctypes.c_void_p]
        _lib.ko_knn_search_rows.restype = ctypes.c_uint64
        _lib.ko_knn_search_rows.argtypes = [ctypes.c_void_p, _U32, _P, _U64, _P, _P]
        _lib.ko_key.restype = ctypes.c_double
        _lib.ko_key.argtypes = [_P, _U32, _U64, _U64]
        _lib.ko_max_threads.restype = ctypes.c_int
    return _lib


def set_threads(n: int) -> None:
    lib().ko_set_threads(ctypes.c_int(int(n)))


def max_threads() -> int:
    return int(lib().ko_max_threads())


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_P)


@dataclass
class Csr:
    """One block of cells x genes: u64 indptr, u32 gene indices, u32 counts or f32 values."""

    indptr: np.ndarray
    indices: np.ndarray
    values: np.ndarray
    n_genes: int

    @property
    def n_rows(self) -> int:
        return len(self.indptr) - 1

    def checked(self) -> "Csr":
        return Csr(
            np.ascontiguousarray(self.indptr, dtype=np.uint64),
            np.ascontiguousarray(self.indices, dtype=np.uint32),
            np.ascontiguousarray(self.values),
            int(self.n_genes),
        )


# ----------------------------------------------------------------------------------
# normalize_total + log1p (crates/kyto-exec/src/elementwise.rs:149-269)
# ----------------------------------------------------------------------------------
def normalize_log1p(x: Csr, target_sum: float | None = 1e4, log1p: bool = True) -> Csr:
    x = x.checked()
    dtype = 0 if x.values.dtype == np.uint32 else 1
    values = x.values if dtype == 0 else np.ascontiguousarray(x.values, dtype=np.float32)
    out = np.empty(len(values), dtype=np.float32)
    lib().ko_normalize_log1p(
        _ptr(x.indptr), _ptr(values), ctypes.c_int(dtype), _U64(x.n_rows),
        ctypes.c_double(math.nan if target_sum is None else float(target_sum)),
        ctypes.c_int(1 if log1p else 0), _ptr(out),
    )
    return Csr(x.indptr, x.indices, out, x.n_genes)


# ----------------------------------------------------------------------------------
# highly_variable_genes(flavor="seurat") (hvg_pass.rs:157-219, statistics.rs:153-168,
# hvg.rs:284-361,393-437,501-580)
# ----------------------------------------------------------------------------------
def hvg_moments(x: Csr) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    x = x.checked()
    values = np.ascontiguousarray(x.values, dtype=np.float32)
    sums = np.empty(x.n_genes)
    squares = np.empty(x.n_genes)
    positives = np.empty(x.n_genes, dtype=np.uint64)
    lib().ko_hvg_moments(
        _ptr(x.indptr), _ptr(x.indices), _ptr(values), _U64(x.n_rows), _U32(x.n_genes),
        _ptr(sums), _ptr(squares), _ptr(positives),
    )
    return sums, squares, positives


def _kahan_mean(values: np.ndarray) -> float:
    total, compensation, count = 0.0, 0.0, 0
    for value in values:
        if math.isnan(value):
            continue
        count += 1
        y = value - compensation
        t = total + y
        compensation = t - total - y
        if math.isnan(compensation):
            compensation = 0.0
        total = t
    return math.nan if count == 0 else total / count


def _welford_std(values: np.ndarray) -> float:
    count, mean, squared = 0, 0.0, 0.0
    for value in values:
        if math.isnan(value):
            continue
        count += 1
        previous = mean
        mean += (value - previous) / count
        squared += (value - mean) * (value - previous)
    return math.nan if count <= 1 else math.sqrt(squared / (count - 1))


def _equal_width_bins(values: np.ndarray) -> np.ndarray:
    finite = values[~np.isnan(values)]
    bins = np.full(len(values), -1, dtype=np.int64)
    if len(finite) == 0:
        return bins
    low, high = float(finite.min()), float(finite.max())
    if low == high:
        lo = low - (0.001 if low == 0.0 else 0.001 * abs(low))
        hi = high + (0.001 if high == 0.0 else 0.001 * abs(high))
        edges = _linspace(lo, hi, N_BINS + 1)
    else:
        edges = _linspace(low, high, N_BINS + 1)
        edges[0] -= (high - low) * 0.001
    for i, value in enumerate(values):
        if math.isnan(value):
            continue
        index = max(int(np.searchsorted(edges, value, side="left")), 1)
        if index < len(edges):
            bins[i] = index - 1
    return bins


def _linspace(start: float, stop: float, num: int) -> np.ndarray:
    step = (stop - start) / (num - 1)
    values = np.array([i * step + start for i in range(num)])
    values[num - 1] = stop
    return values


def hvg_seurat(sums, squares, positives, n_cells: int, n_top_genes: int | None):
    """scanpy's seurat flavor on one group's moments: (means, dispersions,
    dispersions_norm, highly_variable). hvg.rs:284-361."""
    n = float(n_cells)
    mean = sums / n
    variance = squares / n - mean * mean
    if n_cells != 1:
        variance = variance * (n / (n - 1.0))
    mean = np.where(mean == 0.0, 1e-12, mean)
    with np.errstate(divide="ignore", invalid="ignore"):
        dispersion = variance / mean
        dispersion = np.where(dispersion == 0.0, np.nan, dispersion)
        dispersion = np.log(dispersion)
    mean = np.log1p(mean)
    bins = _equal_width_bins(mean)
    stats = []
    for b in range(N_BINS):
        members = dispersion[bins == b]
        average = _kahan_mean(members)
        deviation = _welford_std(members)
        stats.append((0.0, average) if math.isnan(deviation) else (average, deviation))
    normalized = np.full(len(mean), np.nan)
    for i in range(len(mean)):
        if bins[i] >= 0:
            average, deviation = stats[bins[i]]
            with np.errstate(divide="ignore", invalid="ignore"):
                normalized[i] = (dispersion[i] - average) / deviation
    if n_top_genes is not None:
        finite = np.sort(normalized[~np.isnan(normalized)])[::-1]
        count = min(int(n_top_genes), len(mean), len(finite))
        if count == 0:
            flags = np.zeros(len(mean), dtype=bool)
        else:
            cutoff = finite[count - 1]
            big = np.finfo(np.float64).max
            as_num = np.where(normalized == np.inf, big, normalized)
            as_num = np.where(as_num == -np.inf, -big, as_num)
            as_num = np.where(np.isnan(as_num), -np.inf, as_num)
            flags = as_num >= cutoff
    else:
        nz = np.where(np.isnan(normalized), 0.0, normalized)
        flags = (mean > 0.0125) & (mean < 3.0) & (nz > 0.5) & (nz < np.inf)
    return mean, dispersion, normalized, flags


# ----------------------------------------------------------------------------------
# PCA (crates/kyto-exec/src/pca.rs, pca_dense.rs)
# ----------------------------------------------------------------------------------
def omega_rows(seed: int, cells: np.ndarray, width: int) -> np.ndarray:
    """Omega's rows for the cells at these table positions (pca.rs:936-950, omega_row):
    len(cells) x width f64."""
    cells = np.ascontiguousarray(cells, dtype=np.uint64)
    out = np.empty((len(cells), int(width)))
    lib().ko_omega_rows(_U64(seed), _ptr(cells), _U64(len(cells)), _U32(width), _ptr(out))
    return out


def _splitmix_mix(v: int) -> int:
    m = (1 << 64) - 1
    v = ((v ^ (v >> 30)) * 0xBF58476D1CE4E5B9) & m
    v = ((v ^ (v >> 27)) * 0x94D049BB133111EB) & m
    return v ^ (v >> 31)


def omega_row_reference(seed: int, cell: int, width: int) -> list[float]:
    """pca.rs:936-950 in pure Python integers (checks the C restatement's bits)."""
    m = (1 << 64) - 1
    golden = 0x9E3779B97F4A7C15
    state = _splitmix_mix((seed ^ _splitmix_mix((cell + golden) & m)) & m)
    out = []
    for _ in range(width):
        state = (state + golden) & m
        out.append(float(_splitmix_mix(state) >> 11) * 2.0**-52 - 1.0)
    return out
def extend_basis(basis: np.ndarray, block: np.ndarray) -> np.ndarray:
    """pca_dense.rs:105-129: CGS twice, thin SVD, keep sigma > 1e-10 |block|_F."""
    scale = float(np.linalg.norm(block))
    if scale == 0.0 or block.shape[1] == 0:
        return np.zeros((block.shape[0], 0))
    rest = block.copy()
    if basis.shape[1] > 0:
        for _ in range(2):
            rest = rest - basis @ (basis.T @ rest)
    u, s, _ = np.linalg.svd(rest, full_matrices=False)
    keep = 0
    while keep < len(s) and s[keep] > DROP_TOLERANCE * scale:
        keep += 1
    return u[:, :keep].copy()


def _complement(columns: np.ndarray, count: int) -> np.ndarray:
    """pca_dense.rs:225-253."""
    allc = columns.copy()
    added = np.zeros((columns.shape[0], 0))
    for _ in range(count):
        covered = (allc * allc).sum(axis=1)
        gene = int(np.argmin(covered)) if len(covered) else 0
        vector = np.zeros(allc.shape[0])
        vector[gene] = 1.0
        for _ in range(2):
            vector = vector - allc @ (allc.T @ vector)
        vector = vector / np.linalg.norm(vector)
        allc = np.hstack([allc, vector[:, None]])
        added = np.hstack([added, vector[:, None]])
    return added


def flip_signs(loadings: np.ndarray) -> np.ndarray:
    """pca_dense.rs:257-275: each column's largest |value| (first on ties) positive."""
    out = loadings.copy()
    for c in range(out.shape[1]):
        col = out[:, c]
        largest, sign = 0.0, 1.0
        for v in col:
            if abs(v) > largest:
                largest, sign = abs(v), math.copysign(1.0, v)
        if sign < 0:
            out[:, c] = -col
    return out


def rayleigh_ritz(basis: np.ndarray, products: np.ndarray, k: int):
    """pca_dense.rs:141-174."""
    loadings = np.zeros((basis.shape[0], 0))
    eigenvalues: list[float] = []
    if basis.shape[1] > 0:
        projected = basis.T @ products
        symmetric = 0.5 * (projected + projected.T)
        values, vectors = np.linalg.eigh(symmetric)
        n = len(values)
        taken = min(k, n)
        order = [n - 1 - i for i in range(taken)]
        eigenvalues = [max(float(values[i]), 0.0) for i in order]
        loadings = basis @ vectors[:, order]
    missing = k - len(eigenvalues)
    if missing > 0:
        loadings = np.hstack([loadings, _complement(loadings, missing)])
        eigenvalues += [0.0] * missing
    return np.array(eigenvalues), flip_signs(loadings)


@dataclass
class PcaResult:
    embedding: np.ndarray  # n x k f32
    loadings: np.ndarray  # genes x k f32 (zeros outside the gene set)
    variance: np.ndarray
    variance_ratio: np.ndarray
    means: np.ndarray
    eigenvalues: np.ndarray
    passes_run: int


def pca(x: Csr, n_components: int, seed: int = 0, gene_set: np.ndarray | None = None,
        cells: np.ndarray | None = None) -> PcaResult:
    """kyto's streamed Krylov PCA over one leaf holding every cell (pca.rs:343-862).

    ``x`` holds the values the node sees (f32: normalize/log1p already applied);
    ``gene_set`` flags the stream's genes the components use (None: all)."""
    x = x.checked()
    values = np.ascontiguousarray(x.values, dtype=np.float32)
    n_rows, stream_genes = x.n_rows, x.n_genes
    if gene_set is None:
        gene_map = None
        n_genes = stream_genes
    else:
        flags = np.asarray(gene_set, dtype=bool)
        gene_map = np.full(stream_genes, NO_GENE, dtype=np.uint32)
        gene_map[flags] = np.arange(flags.sum(), dtype=np.uint32)
        n_genes = int(flags.sum())
    cells = (np.arange(n_rows, dtype=np.uint64) if cells is None
             else np.ascontiguousarray(cells, dtype=np.uint64))
    k = int(n_components)
    if n_rows < 2 or k > min(n_rows, n_genes):
        raise ValueError("pca needs at least 2 cells and n_components <= min(cells, genes)")
    width = min(k + PCA_OVERSAMPLES, n_genes)
    L = lib()
    common = (_ptr(x.indptr), _ptr(x.indices), _ptr(values), _U64(n_rows),
              _ptr(gene_map), _U32(stream_genes), _U32(n_genes))

    # Pass 0: sketch.
    sums = np.empty(n_genes)
    omega_sums = np.empty(width)
    sketch = np.empty((n_genes, width))
    L.ko_pca_sketch(*common, _ptr(cells), _U64(seed), _U32(width), _ptr(sums),
                    _ptr(omega_sums), _ptr(sketch))
    means = sums / float(n_rows)
    if not np.all(np.isfinite(means)):
        raise ValueError("a gene holds a value that is not finite")
    sketch -= means[:, None] * omega_sums[None, :]
    basis = np.zeros((n_genes, 0))
    products = np.zeros((n_genes, 0))
    state = {"loadings": None}

    def block_means_of(block):
        out = np.zeros(block.shape[1])
        for g in range(n_genes):  # gene order, as set_block
            out += means[g] * block[g]
        return out

    def finish(basis, products):
        eig, loadings = rayleigh_ritz(basis, products, k)
        mean_projection = np.zeros(k)
        for g in range(n_genes):
            mean_projection += means[g] * loadings[g]
        state["loadings"] = loadings
        state["eig"] = eig
        state["mean_projection"] = mean_projection

    block = extend_basis(basis, sketch)
    if block.shape[1] == 0:
        finish(basis, products)
    passes_run = 1
    for p in range(1, PCA_PASSES - 1):
        if state["loadings"] is not None:
            break
        w = block.shape[1]
        bm = block_means_of(block)
        product = np.empty((n_genes, w))
        wsums = np.empty(w)
        L.ko_pca_product(*common, _ptr(np.ascontiguousarray(block)), _ptr(bm), _U32(w),
                         _ptr(product), _ptr(wsums))
        passes_run += 1
        product -= means[:, None] * wsums[None, :]
        basis = np.hstack([basis, block])
        products = np.hstack([products, product])
        if p == PCA_PASSES - 2:
            finish(basis, products)
        else:
            block = extend_basis(basis, product)
            if block.shape[1] == 0:
                finish(basis, products)
    loadings = np.ascontiguousarray(state["loadings"])
    rows = np.empty((n_rows, k))
    squares = np.empty(n_genes)
    stored = np.empty(n_genes, dtype=np.uint64)
    L.ko_pca_rows(*common, _ptr(loadings), _ptr(state["mean_projection"]), _U32(k),
                  _ptr(means), _ptr(rows), _ptr(squares), _ptr(stored))
    passes_run += 1
    n = float(n_rows)
    total = 0.0
    for g in range(n_genes):
        total += squares[g] + float(n_rows - int(stored[g])) * means[g] * means[g]
    total_variance = total / (n - 1.0)
    eig = state["eig"]
    variance = np.zeros(k) if total_variance == 0.0 else eig / (n - 1.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = variance / total_variance
    full_loadings = np.zeros((stream_genes, k), dtype=np.float32)
    if gene_map is None:
        full_loadings[:] = loadings.astype(np.float32)
    else:
        full_loadings[np.asarray(gene_set, dtype=bool)] = loadings.astype(np.float32)
    return PcaResult(rows.astype(np.float32), full_loadings, variance, ratio, means, eig,
                     passes_run)


# ----------------------------------------------------------------------------------
# Exact kNN (crates/kyto-exec/src/neighbors.rs, neighbors_exact.rs)
# ----------------------------------------------------------------------------------
@dataclass
class Graph:
    """kyto's NeighborGraph (neighbors.rs:412-435): k = n_neighbors - 1 entries a row,
    columns increasing within a row, f32 distances sqrt(f64 key)."""

    indptr: np.ndarray
    indices: np.ndarray
    distances: np.ndarray


def ranked_to_graph(keys: np.ndarray, rows: np.ndarray) -> Graph:
    n, k = rows.shape
    order = np.argsort(rows, axis=1, kind="stable")
    idx = np.take_along_axis(rows, order, axis=1)
    dist = np.sqrt(np.take_along_axis(keys, order, axis=1)).astype(np.float32)
    indptr = np.arange(n + 1, dtype=np.uint64) * np.uint64(k)
    return Graph(indptr, idx.reshape(-1).astype(np.uint32), dist.reshape(-1))


def knn_ranked(points: np.ndarray, n_neighbors: int, method: str = "brute"):
    """Each row's k = n_neighbors - 1 nearest other rows by (f64 key, row), ranked."""
    points = np.ascontiguousarray(points, dtype=np.float32)
    n, width = points.shape
    k = int(n_neighbors) - 1
    if not (2 <= n_neighbors <= n):
        raise ValueError("n_neighbors must be in [2, n]")
    keys = np.empty((n, k))
    rows = np.empty((n, k), dtype=np.uint32)
    if method == "brute":
        lib().ko_knn_brute(_ptr(points), _U64(n), _U32(width), _U32(k), _ptr(keys), _ptr(rows))
        fallbacks = n
    else:
        fallbacks = lib().ko_knn_exact(_ptr(points), _U64(n), _U32(width), _U32(k),
                                       _ptr(keys), _ptr(rows))
    return keys, rows, int(fallbacks)


def knn_exact_sample(points: np.ndarray, n_neighbors: int, q_begin: int, q_end: int):
    """kyto's CPU exact search (the filtered path) for queries [q_begin, q_end) against
    every row: the CPU baseline's timed sample."""
    points = np.ascontiguousarray(points, dtype=np.float32)
    n, width = points.shape
    k = int(n_neighbors) - 1
    keys = np.empty((q_end - q_begin, k))
    rows = np.empty((q_end - q_begin, k), dtype=np.uint32)
    fb = lib().ko_knn_exact_range(_ptr(points), _U64(n), _U32(width), _U32(k), _U64(q_begin),
                                  _U64(q_end), _ptr(keys), _ptr(rows))
    return keys, rows, int(fb)


class KnnIndex:
    """kyto's CPU exact search split as kyto splits it (neighbors_exact.rs:98-160
    ``Prepared::new``, then ``search_block`` per 128 queries): ``prepare`` centres the
    rows, computes the offsets and slacks and lays out the point tiles once; ``search``
    ranks any range of query rows against every row. The timed CPU baseline pays the
    setup once and samples the per-query cost on enough queries to keep every host
    thread busy."""

    def __init__(self, points: np.ndarray):
        self.points = np.ascontiguousarray(points, dtype=np.float32)
        n, width = self.points.shape
        self.n, self.width = n, width
        self._h = lib().ko_knn_prepare(_ptr(self.points), n, width)

    def search(self, n_neighbors: int, q_begin: int, q_end: int):
        """(keys, rows, fallbacks) of queries [q_begin, q_end), ranked by (key, row)."""
        k = int(n_neighbors) - 1
        keys = np.empty((q_end - q_begin, k))
        rows = np.empty((q_end - q_begin, k), dtype=np.uint32)
        fb = lib().ko_knn_search(self._h, k, q_begin, q_end, _ptr(keys), _ptr(rows))
        return keys, rows, int(fb)

    def search_rows(self, n_neighbors: int, rows: np.ndarray):
        """(keys, rows, fallbacks) of the given query rows, in their order."""
        rows = np.ascontiguousarray(rows, dtype=np.uint64)
        k = int(n_neighbors) - 1
        keys = np.empty((len(rows), k))
        out = np.empty((len(rows), k), dtype=np.uint32)
        fb = lib().ko_knn_search_rows(self._h, k, _ptr(rows), len(rows), _ptr(keys), _ptr(out))
        return keys, out, int(fb)

    def close(self) -> None:
        if self._h:
            lib().ko_knn_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def neighbors(points: np.ndarray, n_neighbors: int = 15, method: str = "brute") -> Graph:
    keys, rows, _ = knn_ranked(points, n_neighbors, method)
    return ranked_to_graph(keys, rows)


def exact_key(points: np.ndarray, q: int, p: int) -> float:
    points = np.ascontiguousarray(points, dtype=np.float32)
    return float(lib().ko_key(_ptr(points), _U32(points.shape[1]), _U64(q), _U64(p)))


if __name__ == "__main__":
    build(force=True)
    print(LIB_PATH, max_threads(), os.cpu_count())
