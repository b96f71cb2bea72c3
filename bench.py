"""Benchmark: cells/s of PCA50 + exact kNN15 at 1M cells on one B200.

Workload (``config.workload``): 1,000,000 cells x 2,000 genes, f32 log1p CSR with about
600 stored values per cell (negative-binomial counts, log-normal gene means, 50 planted
cell types, normalize_total(1e4) + log1p), seeded synthetic data of the benchmark's
shape; then kyto's PCA (50 components, seed 0, 11 passes) and exact Euclidean kNN
(n_neighbors 15 = 14 stored neighbours per cell, kyto's semantics).

One step = the whole path over the whole dataset: push the CSR to the PCA session
(held in HBM), run all passes, search the embedding's exact neighbours.
- ``value``: inputs already resident in HBM when the timed region starts (device CSR).
- ``e2e``: the same through the public API from pinned host CSR, host->device copy of
  the input and device->host copy of the graph inside every step; each step's input is
  pushed asynchronously before the previous step's search, so its copies overlap it.
Inputs (4.8 GB) are larger than L2 (126 MB), so no flush is needed between steps.

On one GPU the line also carries the metric's second half and the batching form:
- ``learned_vs_exact``: the learned-partition kNN against the exact search on 4M x 50
  Gaussian-mixture points (speed-up and recall@15 judged by the exact graph);
- ``batching``: 64 samples of uneven sizes (PCA 30 + kNN 15 each) through the batching
  form against one sample at a time;
- ``connectivities`` (the timed step's graph) and ``hvg_moments`` (the seurat moments
  pass over the benchmark's raw counts): the path's neighbouring rows, timed alone;
- ``tile_join``: the benchmark's raw counts cut into the store's default tiles and every
  cell block joined back into CSR rows on the device (kyto's tile checks included),
  checked bit for bit against the counts;
- ``store_path``: 200,000 of those cells as a tiled layer's zstd shards, every cell block
  decoded on the host into page-locked buffers and joined on the device, checked against
  the counts;
- ``parity.precision_form``: the precision form's search (n_neighbors 30, bf16
  distances, exact re-rank) on the timed 1M embedding, 4,096 rows checked against the
  oracle.

``--impl reference``: kyto's CPU algorithms (the C++ restatement in oracle/, all host
threads) timed on a bounded sample of the same workload: the PCA over a subset of the
cells (all 11 passes) and the exact search of a subset of query cells against every
cell; cells/s = 1 / (PCA seconds per cell + kNN seconds per query cell).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "cells/s PCA50+kNN15 at 1M cells"
WORKLOAD = "1M cells x 2,000 genes f32 log1p CSR (~600 nnz/cell, 50 planted types) -> PCA 50 (11 passes, seed 0) -> exact kNN n_neighbors 15"


def parse() -> argparse.Namespace:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # Eight timed steps: the end-to-end leg's one unhidden copy (the first step's input,
    # which has no step before it to run beside) then costs an eighth of a copy a step.
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=1_000_000)
    ap.add_argument("--genes", type=int, default=2000)
    ap.add_argument("--nnz", type=float, default=600.0)
    ap.add_argument("--types", type=int, default=50)
    ap.add_argument("--components", type=int, default=50)
    ap.add_argument("--neighbors", type=int, default=15)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-pca-cells", type=int, default=50_000,
                    help="reference arm: cells of each step's PCA sample")
    ap.add_argument("--cpu-knn-queries", type=int, default=16_384,
                    help="query rows of the CPU kNN sample (and of the 1M parity check)")
    ap.add_argument("--learned-cells", type=int, default=4_000_000,
                    help="C5 learned-vs-exact comparison rows (0: skip)")
    ap.add_argument("--batch-samples", type=int, default=64,
                    help="C4 batching-form samples (0: skip)")
    ap.add_argument("--hvg", type=int, default=1,
                    help="time the HVG moments pass over the benchmark's counts (0: skip)")
    ap.add_argument("--reserve-gb", type=int, default=40,
                    help="device memory reserved for the library's pool at open (kg_reserve)")
    return ap.parse_args()


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"],
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
            "source": "fallback"}


def filter_traffic(n: int, d: int) -> dict:
    """The filter's DRAM traffic per launch is not measured on the benchmark's launch: ncu
    captures beyond the launch list are kept to 400K rows or fewer, and the filter's DRAM
    bytes do not scale with its work from there (the operand kind the tuner picks and the
    L2 reuse both change with n). The 400K launch's bytes are in profiles/."""
    return {"value": None,
            "source": ("not captured at this size (captures are kept to 400K rows; "
                       "profiles/knn_filter_400k.md holds that launch's DRAM bytes)")}


class Clocks:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"kyto_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_data(args, rank: int):
    """The workload's CSR on the host (numpy) and the device (torch)."""
    import torch

    import kyto_b200 as K
    from kyto_b200 import synthetic

    x = synthetic.counts_csr(args.cells, args.genes, args.nnz, args.types, 200, mu=0.0,
                             sigma=1.5, dispersion=0.3, seed=rank, device="cuda")
    ctx = K.default_context()
    dev_indptr = torch.from_numpy(x.indptr.view(np.int64)).cuda()
    dev_idx = torch.from_numpy(x.indices.view(np.int32)).cuda()
    dev_counts = torch.from_numpy(x.values.view(np.int32)).cuda()
    dev_vals = torch.empty(x.nnz, dtype=torch.float32, device="cuda")
    # normalize_total(1e4) + log1p with the library's own map kernel (data preparation).
    K._check(K.library().kg_normalize_log1p(
        ctx.handle, K._ptr(dev_indptr), K._ptr(dev_counts), K.KG_U32, x.n_cells, 1e4, 1,
        K._ptr(dev_vals)))
    del dev_counts
    vals = dev_vals.cpu().numpy()
    torch.cuda.synchronize()
    return x, vals, dev_indptr, dev_idx, dev_vals


def run_step(args, ctx, indptr, idx, vals, out, host: bool):
    """One step through the public API: PCA session + exact kNN."""
    import kyto_b200 as K

    sess = K.PcaSession(args.components, args.genes, seed=0, ctx=ctx)
    sess.push(indptr, idx, vals)
    sess.run()
    n = args.cells
    emb_ptr = sess.embedding_device_ptr()
    stats = K.KnnStats()
    L = K.library()
    K._check(L.kg_knn_exact(ctx.handle, emb_ptr, n, args.components, 0, args.neighbors,
                            K._ptr(out[0]), K._ptr(out[1]), K._ptr(out[2]),
                            K.ctypes.byref(stats)))
    pstats = sess.stats()
    sess.close()
    return stats, pstats


def e2e_steps(args, ctx, indptr, idx, vals, out, steps: int) -> None:
    """``steps`` steps through the public API from pinned host memory, as a streaming
    caller runs them: each step's CSR goes to the device by an asynchronous push
    (kg_pca_push_block_async: its copies and packing kernels on the session's own
    stream), queued before the previous step's PCA so that they run beside that step's
    PCA and search; each step's graph comes back to host memory inside kg_knn_exact.
    Every step copies its own input and output."""
    import kyto_b200 as K

    def new_session():
        sess = K.PcaSession(args.components, args.genes, seed=0, ctx=ctx)
        sess.push(indptr, idx, vals, wait=False)
        return sess

    L = K.library()
    nxt = new_session()
    for i in range(steps):
        sess = nxt
        if i + 1 < steps:
            nxt = new_session()
        sess.run()
        K._check(L.kg_knn_exact(ctx.handle, sess.embedding_device_ptr(), args.cells,
                                args.components, 0, args.neighbors, K._ptr(out[0]),
                                K._ptr(out[1]), K._ptr(out[2]), None))
        sess.close()


def hvg_timing(args, ctx, x, d_indptr, d_idx) -> dict:
    """The seurat HVG moments pass over the benchmark's raw counts (kg_hvg_moments:
    normalize + log1p, expm1, a stable sort by gene, kyto's per-gene f64 folds), device
    arrays in and out, CUDA-event timed (median of 3 after one warm-up)."""
    import torch

    import kyto_b200 as K

    counts = torch.from_numpy(x.values.view(np.int32)).cuda()
    g = args.genes
    sums = torch.empty(g, dtype=torch.float64, device="cuda")
    sq = torch.empty(g, dtype=torch.float64, device="cuda")
    pos = torch.empty(g, dtype=torch.int64, device="cuda")
    times = []
    for i in range(4):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        K._check(K.library().kg_hvg_moments(ctx.handle, K._ptr(d_indptr), K._ptr(d_idx),
                                            K._ptr(counts), K.KG_U32, args.cells, g, 1e4, 1,
                                            K._ptr(sums), K._ptr(sq), K._ptr(pos)))
        b.record()
        torch.cuda.synchronize()
        if i:
            times.append(a.elapsed_time(b))
    del counts
    return {"workload": f"{args.cells:,} cells x {g:,} genes raw counts ({x.nnz:,} stored)",
            "ms": float(np.median(times))}


def tiles_timing(args, ctx, x, d_indptr, d_idx, cell_block=4096, gene_block=1024) -> dict:
    """The store's tile join (kg_tiles_to_csr) over the benchmark's raw counts as kyto's
    writer tiles them by default (4,096 cells x 1,024 genes a tile): every cell block
    joined back into CSR rows on the device (kyto's checks included), device arrays in
    and out, CUDA-event timed over all blocks after one warm-up pass. The joined rows
    must equal the counts' CSR bit for bit (join(tile(X)) = X: the counts hold no stored
    zeros). The tiles are cut on the device with torch (a sort of the entries by tile and
    row), as the store's writer lays them out (docs/format.md 4.3)."""
    import torch

    import kyto_b200 as K

    n, genes, c, gs = args.cells, args.genes, cell_block, gene_block
    n_gb, n_cb = -(-genes // gs), -(-n // c)
    indptr = d_indptr.to(torch.int64)
    counts = torch.from_numpy(x.values.view(np.int32)).cuda()
    idx = d_idx.to(torch.int64)
    rows = torch.repeat_interleave(torch.arange(n, device="cuda"), indptr[1:] - indptr[:-1])
    gb = idx // gs
    key = ((rows // c) * n_gb + gb) * c + rows % c
    del rows
    key, order = torch.sort(key, stable=True)
    t_idx = (idx[order] - gb[order] * gs).to(torch.int32)
    t_val = counts[order]
    del order, gb, idx
    per_row = torch.bincount(key, minlength=n_cb * n_gb * c).view(n_cb, n_gb, c)
    del key
    shards = torch.zeros(n_cb, n_gb, c + 1, dtype=torch.int32, device="cuda")
    shards[:, :, 1:] = torch.cumsum(per_row, dim=2).to(torch.int32)
    offsets = torch.zeros(n_cb * n_gb + 1, dtype=torch.int64, device="cuda")
    offsets[1:] = torch.cumsum(per_row.sum(dim=2).flatten(), 0)
    del per_row
    nnz = int(offsets[-1])
    out_ptr = torch.empty(n_cb * (c + 1), dtype=torch.int64, device="cuda")
    out_idx = torch.empty(nnz, dtype=torch.int32, device="cuda")
    out_val = torch.empty(nnz, dtype=torch.int32, device="cuda")
    # tile_offsets from host memory, as kyto's reader holds them (it checks the whole
    # array when it opens the layer); the shards and entries on the device.
    h_offsets = offsets.cpu().numpy().view(np.uint64)
    blocks = []
    for b in range(n_cb):
        lo = int(h_offsets[b * n_gb])
        to = h_offsets.ctypes.data + 8 * b * n_gb
        tb = K.TileBlock(b, min(c, n - b * c), c, gs, genes, shards[b].data_ptr(), to,
                         t_idx.data_ptr() + 4 * lo, t_val.data_ptr() + 4 * lo, K.KG_U32, 0)
        blocks.append((tb, out_ptr.data_ptr() + 8 * b * (c + 1), out_idx.data_ptr() + 4 * lo,
                       out_val.data_ptr() + 4 * lo))

    def join_all():
        for tb, p, i, v in blocks:
            K._check(K.library().kg_tiles_to_csr(ctx.handle, K.ctypes.byref(tb), p, i, v))

    join_all()
    torch.cuda.synchronize()
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    join_all()
    e.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(e)
    same_entries = bool(torch.equal(out_idx, d_idx.view(torch.int32)) and
                        torch.equal(out_val, counts))
    same_rows = True
    for b in range(n_cb):
        r = min(c, n - b * c)
        want = indptr[b * c:b * c + r + 1] - indptr[b * c]
        same_rows &= bool(torch.equal(out_ptr[b * (c + 1):b * (c + 1) + r + 1], want))
    shard_bytes = 4 * n_gb * (c + 1) * n_cb
    moved = 8 * nnz + 8 * nnz + 8 * (n + n_cb) + shard_bytes
    del t_idx, t_val, out_idx, out_val, shards, counts
    torch.cuda.empty_cache()
    return {"workload": (f"{n:,} cells x {genes:,} genes raw counts ({nnz:,} stored) in "
                         f"{c:,} x {gs:,} tiles: {n_cb} cell blocks of {n_gb} gene blocks"),
            "ms": ms, "ms_per_block": ms / n_cb,
            "gb_per_s": moved / (ms / 1e3) / 1e9,
            "algorithmic": ("8 nnz in + 8 nnz out + 8 (rows + 1) + the indptr shards per pass; "
                            "one host wait a block for the checks' verdict (tile_offsets "
                            "from host memory)"),
            "rows_equal": same_rows, "entries_equal": same_entries}


def _crc32c(data: bytes) -> int:
    """CRC-32C (Castagnoli, reflected 0x82F63B78): the shard index's checksum."""
    c = 0xFFFFFFFF
    for byte in data:
        c ^= byte
        for _ in range(8):
            c = (c >> 1) ^ 0x82F63B78 if c & 1 else c >> 1
    return c ^ 0xFFFFFFFF


def write_shards(values: np.ndarray, inner: int, per_shard: int) -> list[bytes]:
    """A 1-D array as the store writes a sharded array (docs/format.md 4.4): shards of
    ``per_shard`` inner chunks of ``inner`` elements, each chunk one zstd frame (none for
    a chunk of zeros), then the index of (offset, nbytes) little-endian u64 pairs and its
    CRC-32C. The bench's synthetic store input."""
    import pyarrow as pa

    values = np.ascontiguousarray(values)
    shards = []
    step = inner * per_shard
    for s0 in range(0, max(len(values), 1), step):
        body, index = [], []
        at = 0
        for c in range(per_shard):
            chunk = np.zeros(inner, dtype=values.dtype)
            part = values[s0 + c * inner:s0 + (c + 1) * inner]
            chunk[:len(part)] = part
            if not chunk.any():
                index.append((2**64 - 1, 2**64 - 1))
                continue
            frame = pa.compress(chunk.tobytes(), codec="zstd", asbytes=True)
            index.append((at, len(frame)))
            body.append(frame)
            at += len(frame)
        ib = np.array(index, dtype="<u8").tobytes()
        shards.append(b"".join(body) + ib + _crc32c(ib).to_bytes(4, "little"))
    return shards


def tiled_store(indptr, indices, values, n_genes: int, cell_block=4096, gene_block=1024,
                inner=65536, per_shard=64) -> dict:
    """A CSR (sorted rows) as a tiled layer's shards (docs/format.md 4.1-4.4): an indptr
    shard per cell block (one inner chunk a tile), the entries' local gene indices and
    values in sharded arrays, tile_offsets on the host (as a reader holds them)."""
    indptr = np.asarray(indptr, dtype=np.int64)
    n = len(indptr) - 1
    c, gs = cell_block, gene_block
    n_gb, n_cb = -(-n_genes // gs), -(-n // c)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(indptr))
    gb = np.asarray(indices, dtype=np.int64) // gs
    tile = (rows // c) * n_gb + gb
    # A stable sort by tile keeps rows, then genes, in order (16-bit keys sort by radix).
    key = tile.astype(np.int16) if n_cb * n_gb < (1 << 15) else tile
    order = np.argsort(key, kind="stable")
    del key
    local = (np.asarray(indices, dtype=np.int64) - gb * gs).astype(np.uint32)[order]
    vals = np.asarray(values)[order]
    per_row = np.bincount(tile * c + rows % c, minlength=n_cb * n_gb * c).reshape(n_cb, n_gb, c)
    offsets = np.zeros(n_cb * n_gb + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(per_row.sum(axis=2).ravel())
    ptr_shards = []
    for b in range(n_cb):
        sh = np.zeros((n_gb, c + 1), dtype=np.uint32)
        sh[:, 1:] = np.cumsum(per_row[b], axis=1)
        ptr_shards.append(write_shards(sh.ravel(), c + 1, n_gb)[0])
    return {"n_cells": n, "n_genes": n_genes, "cell_block": c, "gene_block": gs,
            "n_gb": n_gb, "n_cb": n_cb, "inner": inner, "per_shard": per_shard,
            "offsets": offsets, "indptr_shards": ptr_shards,
            "indices_shards": write_shards(local, inner, per_shard),
            "values_shards": write_shards(vals, inner, per_shard)}


def read_cell_block(store: dict, b: int, shard_out, idx_out, val_out) -> tuple[int, int]:
    """Cell block ``b`` decoded on the host into the given (page-locked) buffers, as a
    block stream reads it: its indptr shard whole, its entries' range across the entry
    shards (kg_shard_read). Returns the range (first entry, entries)."""
    import kyto_b200 as K

    n_gb, c = store["n_gb"], store["cell_block"]
    K.shard_read(store["indptr_shards"][b], n_gb, c + 1, np.uint32, 0, n_gb * (c + 1),
                 shard_out[:n_gb * (c + 1)])
    lo, hi = int(store["offsets"][b * n_gb]), int(store["offsets"][(b + 1) * n_gb])
    step = store["inner"] * store["per_shard"]
    K.read_sharded(store["indices_shards"], store["inner"], step, np.uint32, lo, hi - lo,
                   idx_out[:hi - lo])
    K.read_sharded(store["values_shards"], store["inner"], step, np.uint32, lo, hi - lo,
                   val_out[:hi - lo])
    return lo, hi - lo


def store_path_timing(args, ctx, x, d_indptr, d_idx, cells=200_000) -> dict:
    """kyto's store path, from the shards' bytes to the rows on the device: the first
    ``cells`` cells of the benchmark's raw counts as a tiled layer's shards (the store's
    default 4,096 x 1,024 tiles, 64K-element zstd inner chunks), then every cell block
    decoded on the host into page-locked buffers (kg_shard_read, all host threads) and
    joined on the device with kyto's checks (kg_tiles_to_csr). Host wall clock over all
    blocks after one warm-up pass; the joined rows must equal the counts' CSR."""
    import torch

    import kyto_b200 as K

    n = min(cells, args.cells)
    nnz = int(x.indptr[n])
    store = tiled_store(x.indptr[:n + 1], x.indices[:nnz], x.values[:nnz], args.genes)
    n_gb, c = store["n_gb"], store["cell_block"]
    most = int(max(store["offsets"][(b + 1) * n_gb] - store["offsets"][b * n_gb]
                   for b in range(store["n_cb"])))
    pin = lambda m: torch.empty(max(m, 1), dtype=torch.int32).pin_memory()  # noqa: E731
    h_shard, h_idx, h_val = pin(n_gb * (c + 1)), pin(most), pin(most)
    s_np, i_np, v_np = (t.numpy().view(np.uint32) for t in (h_shard, h_idx, h_val))
    out_ptr = torch.empty(store["n_cb"] * (c + 1), dtype=torch.int64, device="cuda")
    out_idx = torch.empty(nnz, dtype=torch.int32, device="cuda")
    out_val = torch.empty(nnz, dtype=torch.int32, device="cuda")
    offsets = store["offsets"]

    def one_pass() -> tuple[float, float]:
        decode = join = 0.0
        for b in range(store["n_cb"]):
            t0 = time.perf_counter()
            lo, m = read_cell_block(store, b, s_np, i_np, v_np)
            t1 = time.perf_counter()
            tb = K.TileBlock(b, min(c, n - b * c), c, store["gene_block"], args.genes,
                             h_shard.data_ptr(), offsets.ctypes.data + 8 * b * n_gb,
                             h_idx.data_ptr(), h_val.data_ptr(), K.KG_U32, 0)
            K._check(K.library().kg_tiles_to_csr(
                ctx.handle, K.ctypes.byref(tb), out_ptr.data_ptr() + 8 * b * (c + 1),
                out_idx.data_ptr() + 4 * lo, out_val.data_ptr() + 4 * lo))
            decode += t1 - t0
            join += time.perf_counter() - t1
        return decode, join

    one_pass()
    t0 = time.perf_counter()
    decode, join = one_pass()
    wall = time.perf_counter() - t0
    counts = torch.from_numpy(x.values[:nnz].view(np.int32)).cuda()
    same = bool(torch.equal(out_idx, d_idx[:nnz].view(torch.int32)) and torch.equal(out_val, counts))
    indptr = d_indptr[:n + 1].to(torch.int64)
    for b in range(store["n_cb"]):
        r = min(c, n - b * c)
        same &= bool(torch.equal(out_ptr[b * (c + 1):b * (c + 1) + r + 1],
                                 indptr[b * c:b * c + r + 1] - indptr[b * c]))
    stored = sum(len(s) for k in ("indptr_shards", "indices_shards", "values_shards")
                 for s in store[k])
    return {"workload": (f"{n:,} cells x {args.genes:,} genes raw counts ({nnz:,} stored) as "
                         f"a tiled layer's shards ({stored / 1e6:.0f} MB of zstd frames): "
                         f"{store['n_cb']} cell blocks of 4,096 x 1,024 tiles"),
            "ms": 1e3 * wall, "decode_ms": 1e3 * decode, "join_ms": 1e3 * join,
            "cells_per_s": n / wall, "decoded_gb_per_s": 8 * nnz / decode / 1e9,
            "host_threads": os.cpu_count(), "rows_equal_csr": same}


def connectivities_timing(args, ctx, graph) -> dict:
    """The step after the search (the next row of the path): UMAP connectivities of the
    timed step's 1M-row graph, device arrays in and out, CUDA-event timed (median of 3
    after one warm-up)."""
    import torch

    import kyto_b200 as K

    n, k = args.cells, args.neighbors - 1
    out = (torch.empty(n + 1, dtype=torch.int64, device="cuda"),
           torch.empty(2 * n * k, dtype=torch.int32, device="cuda"),
           torch.empty(2 * n * k, dtype=torch.float32, device="cuda"))
    nnz = K.ctypes.c_uint64()
    times = []
    for i in range(4):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        K._check(K.library().kg_connectivities(ctx.handle, K._ptr(graph[0]), K._ptr(graph[1]),
                                               K._ptr(graph[2]), n, args.neighbors,
                                               K._ptr(out[0]), K._ptr(out[1]), K._ptr(out[2]),
                                               K.ctypes.byref(nnz)))
        b.record()
        torch.cuda.synchronize()
        if i:
            times.append(a.elapsed_time(b))
    return {"workload": f"{n:,} rows x {k} neighbours (the timed step's graph)",
            "ms": statistics.median(times), "nnz": int(nnz.value)}


def precision_search(ctx, emb_ptr: int, n: int, d: int, n_neighbors: int = 30) -> dict:
    """The precision form's search on the timed PCA's device embedding: n_neighbors 30 with
    the bf16 tensor-core distances (f32 accumulation) picking the candidates, then their
    exact re-rank (kyto's f64 keys of every candidate inside the filter's proven slack,
    which holds at least the 4k candidates the form asks for). One untimed call, then
    one timed by host wall clock around a device synchronisation."""
    import torch

    import kyto_b200 as K

    k = n_neighbors - 1
    out = (torch.empty(n + 1, dtype=torch.int64, device="cuda"),
           torch.empty(n * k, dtype=torch.int32, device="cuda"),
           torch.empty(n * k, dtype=torch.float32, device="cuda"))
    st = K.KnnStats()
    os.environ["KYTO_GPU_KNN_FILTER"] = "bf16"
    try:
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            K._check(K.library().kg_knn_exact(
                ctx.handle, emb_ptr, n, d, 0, n_neighbors, K._ptr(out[0]), K._ptr(out[1]),
                K._ptr(out[2]), K.ctypes.byref(st)))
            torch.cuda.synchronize()
            ms = 1e3 * (time.perf_counter() - t0)
    finally:
        del os.environ["KYTO_GPU_KNN_FILTER"]
    return {"workload": f"{n:,} x {d} timed PCA embedding, n_neighbors {n_neighbors}",
            "filter": "bf16 operands, f32 accumulation; exact f64 re-rank", "ms": ms,
            "filter_ms": st.filter_ms, "rank_ms": st.rank_ms,
            "candidates_per_row": st.candidates / n, "rows_searched_in_full": st.rows_full,
            "n_neighbors": n_neighbors, "graph": tuple(t.cpu().numpy() for t in out)}


def spread_rows(n: int, q: int) -> np.ndarray:
    """q distinct rows spread evenly over [0, n) (every part of the search's scan order
    holds some of them)."""
    q = min(q, n)
    return np.unique(np.linspace(0, n - 1, q).round().astype(np.uint64))


def cpu_baseline_and_parity(args, x, vals, res, graph, precision=None) -> tuple[dict, dict]:
    """kyto's CPU path (the oracle's C++ restatement, all host threads) on the bench's
    workload, and the device results checked against it.

    - PCA: the oracle's whole PCA of the same 1M cells (all 11 passes), timed; its singular
      values and loadings check the device PCA (``res``) of the timed configuration.
    - kNN: kyto's exact search prepared once over the device embedding (timed), then the
      queries of ``spread_rows`` (timed); the 1M search is estimated as setup + per-query
      time x n. The same queries' rows of the device graph (``graph``, searched on the same
      embedding, as kyto's parity rule takes it) must equal the oracle's bit for bit.
    - ``precision``: the precision form's search (``precision_search``); 4,096 spread rows
      of its graph are checked against the oracle's search at its n_neighbors."""
    from oracle import oracle as O

    n, d, k = args.cells, args.components, args.neighbors - 1
    threads = O.max_threads()
    full = O.Csr(x.indptr, x.indices, vals, args.genes)
    t0 = time.perf_counter()
    ref = O.pca(full, d, 0)
    t_pca = time.perf_counter() - t0
    # Singular values sigma_i = sqrt(variance_i (n - 1)); the subspaces' largest angle.
    sv_err = float(np.max(np.abs(np.sqrt(res.variance) - np.sqrt(ref.variance))
                          / np.sqrt(ref.variance)))
    qa, _ = np.linalg.qr(res.loadings.astype(np.float64))
    qb, _ = np.linalg.qr(ref.loadings.astype(np.float64))
    cosines = np.linalg.svd(qa.T @ qb, compute_uv=False)
    angle = float(np.arccos(np.clip(cosines.min(), -1.0, 1.0)))
    del ref, full

    t0 = time.perf_counter()
    index = O.KnnIndex(res.embedding)
    t_prep = time.perf_counter() - t0
    rows = spread_rows(n, args.cpu_knn_queries)
    q = len(rows)
    t0 = time.perf_counter()
    keys, ranked, fallbacks = index.search_rows(args.neighbors, rows)
    t_q = time.perf_counter() - t0

    def rows_equal(keys, ranked, graph, sel):
        kk = ranked.shape[1]
        order = np.argsort(ranked, axis=1, kind="stable")
        o_idx = np.take_along_axis(ranked, order, axis=1)
        o_dist = np.sqrt(np.take_along_axis(keys, order, axis=1)).astype(np.float32)
        g_idx = graph[1].reshape(n, kk)[sel.astype(np.int64)]
        g_dist = graph[2].reshape(n, kk)[sel.astype(np.int64)]
        return (int(np.all(g_idx == o_idx, axis=1).sum()),
                int(np.all(g_dist.view(np.uint32) == o_dist.view(np.uint32), axis=1).sum()))

    idx_rows, dist_rows = rows_equal(keys, ranked, graph, rows)
    wide = None
    if precision is not None:
        # The precision form's wider search, judged the same way on its own rows.
        sel = spread_rows(n, 4096)
        wkeys, wranked, wfb = index.search_rows(precision["n_neighbors"], sel)
        wi, wd = rows_equal(wkeys, wranked, precision["graph"], sel)
        wide = {k2: v for k2, v in precision.items() if k2 != "graph"}
        wide.update({"query_rows": len(sel), "rows_indices_equal": wi,
                     "rows_distances_bit_equal": wd, "oracle_full_row_searches": wfb})
    index.close()
    t_knn = t_prep + t_q / q * n
    cpu = {
        "value": n / (t_pca + t_knn), "unit": "cells/s", "cores": threads, "kind": "port",
        "sample": (f"kyto's CPU path restated in C++ ({threads} threads): the whole PCA of the "
                   f"{n:,} cells, 11 passes, timed ({t_pca:.1f} s); the exact kNN prepared "
                   f"once over the {n:,}-row embedding ({t_prep:.2f} s) and {q:,} query rows "
                   f"spread over it searched against all rows ({t_q:.2f} s), the full search "
                   f"estimated as setup + {n:,} x per-query ({t_knn:.1f} s); "
                   f"cells/s = {n:,} / (PCA s + kNN s)"),
        "pca_s": t_pca, "knn_setup_s": t_prep, "knn_s_per_query": t_q / q,
        "knn_s_estimated": t_knn,
        "reference_published": ("kyto's own 1M numbers on an Apple M4 (10 threads): PCA "
                                "12.76 s, exact kNN 84.4 s (performance.md:935,1146)"),
    }
    parity = {
        "pca": {"cells": n, "singular_value_max_rel_err": sv_err,
                "largest_principal_angle_rad": angle, "bar": "singular values <= 1e-4",
                "against": "f64 oracle PCA (kyto's CPU PCA restated) of the same cells"},
        "knn": {"query_rows": q, "rows_indices_equal": idx_rows,
                "rows_distances_bit_equal": dist_rows, "oracle_full_row_searches": fallbacks,
                "against": ("kyto's exact search (oracle) on the device PCA's embedding, "
                            "the rows of the device graph of that embedding")},
    }
    if wide is not None:
        parity["precision_form"] = wide
    return cpu, parity


def learned_vs_exact(n: int, ctx) -> dict:
    """C5: n x 50 f32 points from a 200-component Gaussian mixture (weights Dirichlet(1),
    isotropic sigma log-uniform [0.2, 2]); the learned-partition kNN (1,024 parts, BF16
    MLP 50-256-256-1024 trained on the device on the exact graph of a 100,000-row sample,
    top-4 probes, fallback below 0.3 confidence) against the exact search, recall@15
    judged by the exact graph. Times: host wall clock around each call, inputs on the
    device, after one untimed call of each (the filter kind tuning is cached)."""
    import torch

    import kyto_b200 as K
    from kyto_b200 import synthetic

    x, _ = synthetic.gaussian_mixture(n, dim=50, n_components=200, spread=3.0, seed=5,
                                      device="cuda")
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()
    k = 14
    params = K.LearnedParams(n_parts=1024, hidden=256, n_probe=4, confidence=0.3,
                             train_cells=100_000, epochs=4, batch=8192, seed=0)

    def graph(fn):
        out = (torch.empty(n + 1, dtype=torch.int64, device="cuda"),
               torch.empty(n * k, dtype=torch.int32, device="cuda"),
               torch.empty(n * k, dtype=torch.float32, device="cuda"))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = fn(out)
        torch.cuda.synchronize()
        return out, st, time.perf_counter() - t0

    def exact(out):
        st = K.KnnStats()
        K._check(K.library().kg_knn_exact(ctx.handle, K._ptr(xd), n, 50, 0, 15, K._ptr(out[0]),
                                          K._ptr(out[1]), K._ptr(out[2]), K.ctypes.byref(st)))
        return st

    def learned(out):
        st = K.LearnedStats()
        K._check(K.library().kg_knn_learned(ctx.handle, K._ptr(xd), n, 50, 0, 15,
                                            K.ctypes.byref(params), K._ptr(out[0]),
                                            K._ptr(out[1]), K._ptr(out[2]),
                                            K.ctypes.byref(st)))
        return st

    graph(exact)
    ex, ex_st, t_ex = graph(exact)
    # The same exact search scanning every tile of every query block (the rows in Morton
    # order, no lists, no bounds): the brute-force work kyto's exact search does.
    os.environ["KYTO_GPU_KNN_ORDER"] = "morton"
    try:
        _, fs_st, t_fs = graph(exact)
    finally:
        del os.environ["KYTO_GPU_KNN_ORDER"]
    graph(learned)
    le, le_st, t_le = graph(learned)
    a = le[1].view(n, k).long()
    b = ex[1].view(n, k).long()
    hits = 0
    for i in range(0, n, 250_000):
        hits += int((a[i:i + 250_000, :, None] == b[i:i + 250_000, None, :]).any(2).sum())
    return {
        "workload": (f"{n:,} x 50 f32 Gaussian mixture (200 components, Dirichlet(1) weights, "
                     "sigma log-uniform [0.2, 2]), k = 15 (14 stored)"),
        "exact_ms": t_ex * 1e3, "learned_ms": t_le * 1e3, "speedup": t_ex / t_le,
        "recall_at_15": hits / (n * k),
        "exact_full_scan_ms": t_fs * 1e3, "speedup_vs_full_scan": t_fs / t_le,
        "learned": {"train_ms": le_st.train_ms, "index_ms": le_st.index_ms,
                    "search_ms": le_st.search_ms, "fallback_rows": le_st.fallback_rows,
                    "scanned_tiles": le_st.scanned_tiles,
                    "tiles_computed": le_st.tiles_computed, "temperature": le_st.temperature,
                    "final_loss": le_st.final_loss},
        "exact": {"filter_ms": ex_st.filter_ms, "rank_ms": ex_st.rank_ms,
                  "rows_searched_in_full": ex_st.rows_full,
                  "tiles_scanned": ex_st.tiles_scanned, "tiles_total": ex_st.tiles_total},
        "exact_full_scan": {"filter_ms": fs_st.filter_ms, "rank_ms": fs_st.rank_ms,
                            "tiles_scanned": fs_st.tiles_scanned},
    }


def batching(n_samples: int, ctx) -> dict:
    """C4: n_samples samples x 2,000 genes, cells log-uniform [500, 80,000] (seed 1),
    ~600 stored values per cell; PCA 30 + kNN 15 each through the batching form
    (kg_pca_knn_batch), against the same calls one sample at a time."""
    import kyto_b200 as K
    from kyto_b200 import synthetic

    rng = np.random.default_rng(1)
    sizes = np.exp(rng.uniform(np.log(500), np.log(80_000), n_samples)).astype(int)
    samples = []
    for i, m in enumerate(sizes):
        c = synthetic.counts_csr(int(m), 2000, 600.0, 20, 100, seed=100 + i, device="cuda")
        samples.append((c.indptr, c.indices, c.values))
    kw = dict(target_sum=1e4, log1p=True, ctx=ctx)
    # Warm-up: the whole batch once, so every worker's pooled session resources exist.
    K.pca_neighbors_batch(samples, 2000, 30, 15, **kw)
    t0 = time.perf_counter()
    out, st = K.pca_neighbors_batch(samples, 2000, 30, 15, **kw)
    t_batch = time.perf_counter() - t0
    t0 = time.perf_counter()
    for ip, ix, v in samples:
        r = K.pca(ip, ix, v, 2000, 30, seed=0, **kw)
        K.neighbors(r.embedding, 15, ctx=ctx)
    t_one = time.perf_counter() - t0
    cells = int(sizes.sum())
    return {
        "workload": (f"{n_samples} samples x 2,000 genes, {cells:,} cells (log-uniform "
                     "500-80,000 a sample), PCA 30 + exact kNN 15 each, host CSR in"),
        "batch_ms": t_batch * 1e3, "cells_per_s": cells / t_batch,
        "one_at_a_time_ms": t_one * 1e3, "speedup": t_one / t_batch,
        "pca_ms": st.pca_ms, "knn_ms": st.knn_ms, "workers": st.workers,
    }


def replica_barrier(dist, cuda: bool) -> None:
    """Every rank's queued device work done (cuda), then every rank at the same point."""
    if cuda:
        import torch

        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()


def replica_max(dist, v: float, device: str) -> float:
    """The largest of the ranks' values (the timing rule: a step takes as long as its
    slowest rank); ``v`` itself with one rank."""
    if dist is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job(world: int, cells: int, ms: float) -> float:
    """cells/s of the whole job: every rank searched its own ``cells`` (weak scaling)."""
    return world * cells / (ms / 1e3)


def main() -> int:
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import kyto_b200 as K

    ctx = K.Context(local)
    K._default = ctx
    # A serving process reserves the pool once at open; no step then grows it mid-call.
    ctx.reserve(args.reserve_gb << 30)
    x, vals, d_indptr, d_idx, d_vals = make_data(args, rank)
    n, k = args.cells, args.neighbors - 1
    out_dev = (torch.empty(n + 1, dtype=torch.int64, device="cuda"),
               torch.empty(n * k, dtype=torch.int32, device="cuda"),
               torch.empty(n * k, dtype=torch.float32, device="cuda"))

    def barrier():
        replica_barrier(dist, cuda=True)

    def max_over_ranks(v: float) -> float:
        return replica_max(dist, v, device="cuda")

    for _ in range(args.warmup):
        run_step(args, ctx, d_indptr, d_idx, d_vals, out_dev, host=False)
    clocks = Clocks(local)
    launches0 = K.kernel_launches()
    barrier()
    clocks.start()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    filter_ms = []
    product = {"launches": 0, "ms": 0.0, "bytes": 0.0}
    for _ in range(args.steps):
        # The range names the timed steps for a profiler's launch list (ncu --nvtx).
        torch.cuda.nvtx.range_push("kyto_step")
        st, pst = run_step(args, ctx, d_indptr, d_idx, d_vals, out_dev, host=False)
        torch.cuda.nvtx.range_pop()
        filter_ms.append(st.filter_ms)
        product["launches"] += pst.product_launches
        product["ms"] += pst.product_ms
        product["bytes"] += pst.product_bytes
        knn_stats = {"candidates_per_row": st.candidates / args.cells,
                     "rows_searched_in_full": st.rows_full,
                     "filter_ms": st.filter_ms, "rank_ms": st.rank_ms,
                     "tiles_scanned": st.tiles_scanned, "tiles_total": st.tiles_total}
    stop.record()
    barrier()
    clk = clocks.stop()
    launches = K.kernel_launches() - launches0
    ms = max_over_ranks(start.elapsed_time(stop) / args.steps)
    value = whole_job(world, n, ms)

    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(a).pin_memory()  # noqa: E731
        h_indptr = pin(x.indptr.view(np.int64))
        h_idx = pin(x.indices.view(np.int32))
        h_vals = pin(vals)
        out_host = (torch.empty(n + 1, dtype=torch.int64).pin_memory(),
                    torch.empty(n * k, dtype=torch.int32).pin_memory(),
                    torch.empty(n * k, dtype=torch.float32).pin_memory())
        e2e_steps(args, ctx, h_indptr, h_idx, h_vals, out_host, 1)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        e2e_steps(args, ctx, h_indptr, h_idx, h_vals, out_host, args.steps)
        e1.record()
        barrier()
        ems = max_over_ranks(e0.elapsed_time(e1) / args.steps)
        h2d = x.indptr.nbytes + x.indices.nbytes + vals.nbytes
        d2h = sum(t.numel() * t.element_size() for t in out_host)
        e2e = {"value": whole_job(world, n, ems), "unit": "cells/s", "ms_per_step": ems,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}

    pk = peaks()
    d = args.components
    fl = 2.0 * n * n * d
    f_ms = statistics.median(filter_ms)
    achieved = fl / (f_ms / 1e3) / 1e12
    traffic = filter_traffic(n, d)
    roofline = {
        "kernel": "kNN candidate filter (distance GEMM + selection)",
        "bound": "tensor", "achieved": achieved, "peak": pk["bf16_tflops"], "unit": "TFLOP/s",
        "frac": achieved / pk["bf16_tflops"], "traffic": traffic["value"],
        "traffic_source": traffic["source"],
        "peak_source": f"{pk['source']} (bf16 burst)", "launch_ms": f_ms,
        "algorithmic": f"2*n^2*d = {fl:.3e} flop per launch (n={n}, d={d})",
    }
    roofline_spmm = None
    if product["launches"]:
        gbs = product["bytes"] / (product["ms"] / 1e3) / 1e9
        roofline_spmm = {
            "kernel": "PCA sparse x dense products (X Q, X^T W, sketch, embedding, gene stats)",
            "bound": "hbm", "achieved": gbs, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": gbs / pk["hbm_gbs"], "traffic": None,
            "launches_per_step": product["launches"] / args.steps,
            "launch_ms": product["ms"] / product["launches"],
            "peak_source": f"{pk['source']} (HBM copy)",
            "algorithmic": ("8 nnz + 4 (n+1) + 4 g l + 4 n l bytes per launch (l its width), "
                            "CUDA events around each launch on the session stream"),
        }
    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sess = K.PcaSession(args.components, args.genes, seed=0, ctx=ctx)
        sess.push(d_indptr, d_idx, d_vals)
        sess.run()
        res = sess.results()
        K._check(K.library().kg_knn_exact(
            ctx.handle, sess.embedding_device_ptr(), n, d, 0, args.neighbors,
            K._ptr(out_dev[0]), K._ptr(out_dev[1]), K._ptr(out_dev[2]), None))
        graph = tuple(t.cpu().numpy() for t in out_dev)
        try:
            precision = precision_search(ctx, sess.embedding_device_ptr(), n, d)
        except Exception as e:  # a side measurement never costs the main line
            precision, precision_error = None, f"{type(e).__name__}: {e}"
        sess.close()
        cpu, parity = cpu_baseline_and_parity(args, x, vals, res, graph, precision)
        if precision is None:
            parity["precision_form"] = {"error": precision_error}
    extra = {}
    if rank == 0 and world == 1:
        try:
            extra["connectivities"] = connectivities_timing(args, ctx, out_dev)
        except Exception as e:  # a side measurement never costs the main line
            extra["connectivities"] = {"error": f"{type(e).__name__}: {e}"}
        if args.hvg:
            try:
                extra["hvg_moments"] = hvg_timing(args, ctx, x, d_indptr, d_idx)
            except Exception as e:  # a side measurement never costs the main line
                extra["hvg_moments"] = {"error": f"{type(e).__name__}: {e}"}
            try:
                extra["tile_join"] = tiles_timing(args, ctx, x, d_indptr, d_idx)
            except Exception as e:  # a side measurement never costs the main line
                extra["tile_join"] = {"error": f"{type(e).__name__}: {e}"}
            try:
                extra["store_path"] = store_path_timing(args, ctx, x, d_indptr, d_idx)
            except Exception as e:  # a side measurement never costs the main line
                extra["store_path"] = {"error": f"{type(e).__name__}: {e}"}
        for name, fn, on in (("learned_vs_exact", learned_vs_exact, args.learned_cells),
                             ("batching", batching, args.batch_samples)):
            if not on:
                continue
            try:
                extra[name] = fn(on, ctx)
            except Exception as e:  # a side measurement never costs the main line
                extra[name] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 values; f64 dense steps and exact keys", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells": n, "genes": args.genes,
                       "nnz": x.nnz, "n_components": d, "n_neighbors": args.neighbors,
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs (>4 GB) larger than L2; no flush",
                       "pool_reserve_gb": args.reserve_gb},
            "e2e": e2e, "roofline": roofline, "roofline_spmm": roofline_spmm,
            "cpu_baseline": cpu, "parity": parity,
            "clocks": clk, "gpu_launches": launches, "knn": knn_stats,
            **extra,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def reference_arm(args, rank: int, world: int) -> int:
    """kyto's CPU path (the oracle's C++ restatement) on the box's host cores; rank 0 only.

    Each step times a bounded sample of the workload and estimates the whole 1M step from
    it: the PCA of the sample's cells (all 11 passes), scaled past its fixed part (the
    dense steps, measured once before the steps from two sample sizes), and the exact kNN
    of a fixed set of query rows spread over 1M points, prepared once (setup timed once)."""
    if rank != 0:
        return 0
    from kyto_b200 import synthetic
    from oracle import oracle as O

    threads = O.max_threads()
    n, s = args.cells, min(args.cpu_pca_cells, args.cells)
    x = synthetic.counts_csr(s, args.genes, args.nnz, args.types, 200, seed=0, device="cpu")
    sub = O.normalize_log1p(O.Csr(x.indptr, x.indices, x.values, args.genes))
    quarter = max(2, s // 4)
    e = int(sub.indptr[quarter])
    small = O.Csr(sub.indptr[: quarter + 1], sub.indices[:e], sub.values[:e], args.genes)

    def timed(fn):
        t0 = time.perf_counter()
        fn()
        return time.perf_counter() - t0

    # The PCA's fixed part: t(s) = fixed + s x per-cell, from the quarter and the whole.
    timed(lambda: O.pca(small, args.components, 0))
    t_small = timed(lambda: O.pca(small, args.components, 0))
    t_whole = timed(lambda: O.pca(sub, args.components, 0))
    per_cell = max(0.0, (t_whole - t_small) / (s - quarter))
    fixed = max(0.0, t_small - per_cell * quarter)
    # kNN: points from a Gaussian mixture of 50 types in 50 dimensions stand in for the
    # 1M-cell PCA embedding, which needs the full PCA to exist.
    pts, _ = synthetic.gaussian_mixture(n, args.components, args.types, seed=0, device="cpu")
    t0 = time.perf_counter()
    index = O.KnnIndex(pts)
    t_prep = time.perf_counter() - t0
    rows = spread_rows(n, args.cpu_knn_queries // 2)
    q = len(rows)

    def step():
        t_pca = timed(lambda: O.pca(sub, args.components, 0))
        t_knn = timed(lambda: index.search_rows(args.neighbors, rows))
        return t_pca, t_knn

    for _ in range(args.warmup):
        step()
    times = [step() for _ in range(args.steps)]
    t_pca = statistics.median(t[0] for t in times)
    t_knn = statistics.median(t[1] for t in times)
    est_pca = fixed + (t_pca - fixed) * n / s
    est_knn = t_prep + t_knn * n / q
    value = n / (est_pca + est_knn)
    cpu = {"value": value, "unit": "cells/s", "cores": threads, "kind": "port",
           "sample": (f"per step: PCA of {s:,} cells, 11 passes ({t_pca:.2f} s; fixed part "
                      f"{fixed:.2f} s from {quarter:,} and {s:,} cells) and the exact kNN of "
                      f"{q:,} query rows against {n:,} points ({t_knn:.2f} s; setup once "
                      f"{t_prep:.2f} s); {n:,}-cell estimate PCA {est_pca:.1f} s + kNN "
                      f"{est_knn:.1f} s"),
           "pca_s_estimated": est_pca, "knn_s_estimated": est_knn}
    line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * (t_pca + t_knn), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32 (CPU)",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "cells": args.cells, "genes": args.genes,
                       "n_components": args.components, "n_neighbors": args.neighbors},
            "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    index.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
