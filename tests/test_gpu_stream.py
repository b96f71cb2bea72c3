"""The asynchronous push (kg_pca_push_block_async): blocks queued from pinned host memory
without waiting give the same bits as synchronous pushes; a gene index out of range is
refused when the run starts; a session pushed asynchronously while another session's
search runs gives its own results unchanged (the copies on one session's stream, the
search on the context's)."""

import numpy as np
import pytest

import kyto_b200 as K
from kyto_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return K.Context(0)


@pytest.fixture(scope="module")
def cells():
    return synthetic.counts_csr(40_000, 2000, 300.0, 10, 100, seed=12)


def _pinned(a):
    import torch

    view = {np.dtype(np.uint64): np.int64, np.dtype(np.uint32): np.int32}.get(a.dtype)
    return torch.from_numpy(np.ascontiguousarray(a).view(view) if view else a).pin_memory()


def _blocks(x, step):
    for a in range(0, x.n_cells, step):
        b = min(x.n_cells, a + step)
        e0, e1 = int(x.indptr[a]), int(x.indptr[b])
        yield (x.indptr[a:b + 1] - x.indptr[a]).astype(np.uint64), x.indices[e0:e1], x.values[e0:e1]


def test_async_push_gives_the_same_bits(ctx, cells):
    ref = K.PcaSession(30, 2000, target_sum=1e4, log1p=True, ctx=ctx)
    for ip, ix, v in _blocks(cells, 8192):
        ref.push(ip, ix, v)
    ref.run()
    want = ref.results()
    ref.close()
    sess = K.PcaSession(30, 2000, target_sum=1e4, log1p=True, ctx=ctx)
    for ip, ix, v in _blocks(cells, 8192):
        sess.push(_pinned(ip), _pinned(ix), _pinned(v), wait=False)
    sess.run()
    got = sess.results()
    sess.close()
    assert np.array_equal(got.embedding.view(np.uint32), want.embedding.view(np.uint32))
    assert np.array_equal(got.variance, want.variance)


def test_async_push_refuses_a_bad_index_at_run(ctx, cells):
    ip, ix, v = next(_blocks(cells, 1000))
    ix = ix.copy()
    ix[17] = 2000  # one past the genes
    sess = K.PcaSession(10, 2000, target_sum=1e4, log1p=True, ctx=ctx)
    sess.push(_pinned(ip), _pinned(ix), _pinned(v), wait=False)
    with pytest.raises(K.KytoError) as e:
        sess.run()
    assert e.value.status == K.KG_ERR_INVALID and "gene index" in str(e.value)
    sess.close()
    # The synchronous push refuses it at once.
    sess = K.PcaSession(10, 2000, target_sum=1e4, log1p=True, ctx=ctx)
    with pytest.raises(K.KytoError):
        sess.push(ip, ix, v)
    sess.close()


def test_push_beside_a_search(ctx, cells):
    import torch

    pts = torch.randn((300_000, 30), generator=torch.Generator().manual_seed(3)).cuda()
    alone = K.neighbors(pts.cpu().numpy(), 15, ctx=ctx)
    ref = K.pca(cells.indptr, cells.indices, cells.values, 2000, 30, target_sum=1e4,
                log1p=True, ctx=ctx)
    sess = K.PcaSession(30, 2000, target_sum=1e4, log1p=True, ctx=ctx)
    sess.push(_pinned(cells.indptr), _pinned(cells.indices), _pinned(cells.values), wait=False)
    beside = K.neighbors(pts.cpu().numpy(), 15, ctx=ctx)  # while the push's copies run
    sess.run()
    got = sess.results()
    sess.close()
    assert np.array_equal(got.embedding.view(np.uint32), ref.embedding.view(np.uint32))
    assert np.array_equal(beside.indices, alone.indices)
    assert np.array_equal(beside.distances.view(np.uint32), alone.distances.view(np.uint32))


@pytest.mark.gpu
def test_pca_results_exported_through_dlpack():
    """kg_pca_result_dlpack: the embedding and loadings reach torch as kDLCUDA tensors with
    the results' bits, outlive the session, and are freed by their deleter once torch
    drops them; a result nobody took is given back by close()."""
    import gc

    import torch

    ctx = K.Context(0)
    x = synthetic.counts_csr(3000, 800, 80, 5, 40, seed=2, device="cpu")
    sess = K.PcaSession(15, 800, seed=0, target_sum=1e4, log1p=True, ctx=ctx)
    sess.push(x.indptr, x.indices, x.values)
    sess.run()
    res = sess.results()
    live = K.dlpack_live()
    emb = torch.from_dlpack(sess.result_dlpack("embedding"))
    load = torch.from_dlpack(sess.result_dlpack("loadings"))
    assert K.dlpack_live() == live + 2
    unused = sess.result_dlpack("embedding")
    assert unused.__dlpack_device__() == (2, 0)
    assert K.dlpack_live() == live + 3
    unused.close()
    assert K.dlpack_live() == live + 2
    with pytest.raises(BufferError):
        unused.__dlpack__()
    sess.close()
    assert emb.is_cuda and emb.dtype == torch.float32 and tuple(emb.shape) == (3000, 15)
    assert emb.device.index == 0
    assert np.array_equal(emb.cpu().numpy().view(np.uint32), res.embedding.view(np.uint32))
    assert np.array_equal(load.cpu().numpy().view(np.uint32), res.loadings.view(np.uint32))
    # A device consumer uses it in place: the row norms on the GPU.
    assert torch.allclose((emb * emb).sum(1).cpu(),
                          torch.from_numpy((res.embedding.astype(np.float64) ** 2).sum(1)).float(),
                          rtol=1e-5, atol=1e-6)
    del emb, load
    gc.collect()
    torch.cuda.synchronize()
    assert K.dlpack_live() == live
