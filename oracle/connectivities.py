"""CPU restatement of kyto's UMAP connectivities — test infrastructure only (the checker the
parity tests compare the device path with), never called by the library.

kyto's ``connectivities`` (crates/kyto-exec/src/connectivities.rs:84-131) reproduces
scanpy's ``pp.neighbors(method="umap")`` weights (umap-learn's ``fuzzy_simplicial_set``
with ``set_op_mix_ratio=1``, ``local_connectivity=1``) on a kNN graph with n_neighbors - 1
stored neighbours per row:

1. each row's distances ranked by (distance in f32 total order, column) (:90-104);
2. per row ``rho`` = the first ranked distance above 0 and ``sigma`` by a 64-step f64
   bisection on sum_j exp(-max(0, d_j - rho) / sigma) = log2(n_neighbors) within 1e-5,
   floored at 1e-3 of the row's mean distance when rho > 0 (:133-176); rows with
   rho == 0 floored at 1e-3 of the mean of every distance (:108-116);
3. each entry's membership in f32: 0 for the row itself, 1 when d - rho <= 0 or sigma is
   0, else exp(-((d - rho) / sigma)) (:189-198);
4. the fuzzy union (w + w^T) - w o w^T in f32, zeros dropped (:200-258).

Means are f32 sums in sequence divided in f64 (:178-184). The f32 exponential of step 3
is evaluated here in f64 and rounded once to f32 (kyto calls the platform's expf); the
goldens of kyto's own parity test (scanpy's weights) pin that within its 1e-5 bar.
"""

from __future__ import annotations

import numpy as np

SMOOTH_K_ITERATIONS = 64      # connectivities.rs:26
SMOOTH_K_TOLERANCE = 1e-5     # connectivities.rs:28
MIN_K_DIST_SCALE = 1e-3       # connectivities.rs:30


def _total_order(d: np.ndarray) -> np.ndarray:
    """f32 values as int32 keys in IEEE total order (Rust's f32::total_cmp)."""
    bits = np.ascontiguousarray(d, dtype=np.float32).view(np.int32)
    return bits ^ ((bits >> 31) & np.int32(0x7FFFFFFF))


def ranked_rows(distances: np.ndarray, indices: np.ndarray, k: int) -> np.ndarray:
    """Each row's k distances by (distance, column) (connectivities.rs:90-104)."""
    d = np.asarray(distances, dtype=np.float32).reshape(-1, k)
    c = np.asarray(indices, dtype=np.int64).reshape(-1, k)
    order = np.lexsort((c, _total_order(d)), axis=-1)
    return np.take_along_axis(d, order, axis=1)


def _f32_sequential_sum(values: np.ndarray) -> np.float32:
    """A float32 fold in order (cumsum accumulates one value at a time)."""
    if values.size == 0:
        return np.float32(0.0)
    return np.cumsum(values.ravel(), dtype=np.float32)[-1]


def smooth_knn(ranked: np.ndarray, n_neighbors: int) -> tuple[np.ndarray, np.ndarray]:
    """(sigma, rho) per row (connectivities.rs:133-176), the row floor applied."""
    n, k = ranked.shape
    target = np.log2(float(n_neighbors))
    pos = ranked > 0
    first = np.argmax(pos, axis=1)
    rho = np.where(pos.any(axis=1), ranked[np.arange(n), first], np.float32(0.0)).astype(np.float32)
    # Two float32 values: a float32 difference, then widened.
    diff = (ranked - rho[:, None]).astype(np.float32).astype(np.float64)
    ceiling = float(np.finfo(np.float32).max)
    lo = np.zeros(n)
    hi = np.full(n, ceiling)
    mid = np.ones(n)
    active = np.ones(n, dtype=bool)
    for _ in range(SMOOTH_K_ITERATIONS):
        total = np.zeros(n)
        for j in range(k):  # the row's terms in order
            dj = diff[:, j]
            with np.errstate(over="ignore", under="ignore"):
                term = np.where(dj > 0, np.exp(-(dj / mid)), 1.0)
            total = total + term
        done = np.abs(total - target) < SMOOTH_K_TOLERANCE
        active &= ~done
        if not active.any():
            break
        up = active & (total > target)
        down = active & ~(total > target)
        hi = np.where(up, mid, hi)
        mid_up = (lo + hi) / 2.0
        lo = np.where(down, mid, lo)
        mid_down = np.where(hi >= ceiling, mid * 2.0, (lo + hi) / 2.0)
        mid = np.where(up, mid_up, np.where(down, mid_down, mid))
    sigma = mid.astype(np.float32)
    for r in np.nonzero(rho > 0)[0]:
        floor = MIN_K_DIST_SCALE * (float(_f32_sequential_sum(ranked[r])) / n_neighbors)
        if float(sigma[r]) < floor:
            sigma[r] = np.float32(floor)
    return sigma, rho


def memberships(distances: np.ndarray, indices: np.ndarray, k: int, sigma: np.ndarray,
                rho: np.ndarray) -> np.ndarray:
    """Each entry's f32 membership, entries in the graph's order (connectivities.rs:189-198)."""
    d = np.asarray(distances, dtype=np.float32).reshape(-1, k)
    c = np.asarray(indices, dtype=np.int64).reshape(-1, k)
    n = d.shape[0]
    t = (d - rho[:, None]).astype(np.float32)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore", under="ignore"):
        u = (t / sigma[:, None]).astype(np.float32)
        e = np.exp(-u.astype(np.float64)).astype(np.float32)
    w = np.where((t <= 0) | (sigma[:, None] == 0), np.float32(1.0), e).astype(np.float32)
    w[c == np.arange(n)[:, None]] = np.float32(0.0)
    return w.ravel()


def fuzzy_union(n: int, k: int, indices: np.ndarray, w: np.ndarray):
    """(w + w^T) - w o w^T in f32, zeros dropped, columns increasing (connectivities.rs:200-258)."""
    rows = np.repeat(np.arange(n, dtype=np.int64), k)
    cols = np.asarray(indices, dtype=np.int64)
    fkey = rows * n + cols
    tkey = cols * n + rows
    keys = np.union1d(fkey, tkey)
    wf = np.zeros(keys.size, dtype=np.float32)
    wt = np.zeros(keys.size, dtype=np.float32)
    wf[np.searchsorted(keys, fkey)] = w
    wt[np.searchsorted(keys, tkey)] = w
    weight = ((wf + wt).astype(np.float32) - (wf * wt).astype(np.float32)).astype(np.float32)
    keep = weight != 0
    keys, weight = keys[keep], weight[keep]
    out_rows = keys // n
    indptr = np.zeros(n + 1, dtype=np.uint64)
    np.add.at(indptr, out_rows + 1, 1)
    return np.cumsum(indptr).astype(np.uint64), (keys % n).astype(np.uint32), weight


def connectivities(indptr: np.ndarray, indices: np.ndarray, distances: np.ndarray,
                   n_neighbors: int):
    """kyto's connectivities of a kNN graph (n_neighbors - 1 entries a row, columns
    increasing): (indptr u64, indices u32, weights f32)."""
    n = len(indptr) - 1
    k = n_neighbors - 1
    ranked = ranked_rows(distances, indices, k)
    sigma, rho = smooth_knn(ranked, n_neighbors)
    if (rho == 0).any():
        floor = MIN_K_DIST_SCALE * (float(_f32_sequential_sum(ranked)) / (n * n_neighbors))
        low = (rho == 0) & (sigma.astype(np.float64) < floor)
        sigma[low] = np.float32(floor)
    w = memberships(distances, indices, k, sigma, rho)
    return fuzzy_union(n, k, indices, w)
