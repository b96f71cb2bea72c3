"""kg_hvg_moments_noalloc (the HVG moments pass in fixed static scratch) against
kg_hvg_moments, through the C ABI. Collected last, so it runs both after the other
GPU tests and alone (``pytest tests/test_zz_no_alloc.py -m gpu``).

Both passes sort the stored values by gene (stably) and add each gene's values in cell
order, so they agree bit for bit. After the first call (which loads the scratch array
with the library's code on the device), a call allocates nothing: neither the library's
pool nor the device's free memory moves."""

import ctypes
import math

import numpy as np
import pytest

import kyto_b200 as K
from kyto_b200 import synthetic
from tests.conftest import load_golden

pytestmark = pytest.mark.gpu

MAX_VALUES = 1 << 20
MAX_GENES = 1 << 16


def _device(a: np.ndarray):
    import torch

    view = {np.dtype(np.uint64): np.int64, np.dtype(np.uint32): np.int32}.get(a.dtype)
    arr = np.ascontiguousarray(a).view(view) if view else np.ascontiguousarray(a)
    return torch.from_numpy(arr).cuda()


def _moments(fn, ctx, indptr, indices, values, dtype, n_genes, target_sum=1e4, log1p=1):
    n_rows = int(indptr.numel() if hasattr(indptr, "numel") else len(indptr)) - 1
    sums = np.full(n_genes, np.nan)
    squares = np.full(n_genes, np.nan)
    positives = np.zeros(n_genes, dtype=np.uint64)
    status = fn(ctx.handle, K._ptr(indptr), K._ptr(indices), K._ptr(values), dtype, n_rows,
                n_genes, target_sum, log1p, K._ptr(sums), K._ptr(squares), K._ptr(positives))
    return status, sums, squares, positives


def _blocks():
    g = load_golden("synthetic_counts")
    golden = (g["indptr"], g["indices"], g["counts"], K.KG_U32, int(g["n_genes"][0]))
    b = synthetic.counts_csr(3000, 4000, 150.0, 4, 100, seed=7, device="cpu")
    counts = (b.indptr, b.indices, b.values, K.KG_U32, b.n_genes)
    x = synthetic.log1p_csr(1500, 2500, 90.0, 3, 50, seed=8, device="cpu")
    f32 = (x.indptr, x.indices, x.values.astype(np.float32), K.KG_F32, x.n_genes)
    return [golden, counts, f32]


def test_noalloc_matches_the_allocating_pass_on_consecutive_calls():
    import torch

    ctx = K.Context(0)
    L = K.library()
    blocks = _blocks()
    staged = [([_device(indptr), _device(indices), _device(values)], dtype, n_genes)
              for indptr, indices, values, dtype, n_genes in blocks]
    for indptr, *_ in blocks:
        assert int(indptr[-1]) <= MAX_VALUES
    # Two passes over the blocks: every call after the first reuses the same scratch.
    for round_no in range(2):
        for d, dtype, n_genes in staged:
            target = math.nan if dtype == K.KG_F32 else 1e4
            log1p = 0 if dtype == K.KG_F32 else 1
            torch.cuda.synchronize()
            pool = K.pool_usage(0, reset_high=True)
            free_before = torch.cuda.mem_get_info()[0]
            st, s0, q0, p0 = _moments(L.kg_hvg_moments_noalloc, ctx, *d, dtype, n_genes,
                                      target, log1p)
            K._check(st)
            torch.cuda.synchronize()
            if round_no or d is not staged[0][0]:
                # Past the first call: nothing taken from the library's pool, nothing from
                # the device.
                assert K.pool_usage(0)["used_high"] == pool["used"]
                assert torch.cuda.mem_get_info()[0] == free_before
            st, s1, q1, p1 = _moments(L.kg_hvg_moments, ctx, *d, dtype, n_genes, target, log1p)
            K._check(st)
            assert np.array_equal(s0.view(np.uint64), s1.view(np.uint64))
            assert np.array_equal(q0.view(np.uint64), q1.view(np.uint64))
            assert np.array_equal(p0, p1)
    ctx.close()


def test_noalloc_rejects_blocks_beyond_its_limits():
    ctx = K.Context(0)
    L = K.library()
    indices = _device(np.zeros(4, dtype=np.uint32))
    values = _device(np.ones(4, dtype=np.uint32))
    # More stored values than the scratch holds: refused before any launch.
    big = _device(np.array([0, MAX_VALUES + 1], dtype=np.uint64))
    st, *_ = _moments(L.kg_hvg_moments_noalloc, ctx, big, indices, values, K.KG_U32, 10)
    assert st == K.KG_ERR_INVALID
    small = _device(np.array([0, 4], dtype=np.uint64))
    st, *_ = _moments(L.kg_hvg_moments_noalloc, ctx, small, indices, values, K.KG_U32,
                      MAX_GENES + 1)
    assert st == K.KG_ERR_INVALID
    # Host inputs would need staging buffers: refused too.
    host = np.array([0, 4], dtype=np.uint64)
    st, *_ = _moments(L.kg_hvg_moments_noalloc, ctx, host, indices, values, K.KG_U32, 10)
    assert st == K.KG_ERR_INVALID
    buf = ctypes.create_string_buffer(512)
    L.kg_last_error(None, buf, len(buf))
    assert b"device memory" in buf.value
    # A refused call leaves the entry point usable.
    st, s, q, p = _moments(L.kg_hvg_moments_noalloc, ctx, small, indices, values, K.KG_U32, 10)
    K._check(st)
    assert p[0] == 4 and s[0] > 0
    ctx.close()
