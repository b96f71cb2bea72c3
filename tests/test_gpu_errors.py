"""The error paths of the C ABI, made to happen without faulting or stalling a GPU
(kyto: RunControl::check -> KY-E503, crates/kyto-exec/src/run_control.rs:66-80, and its
tests in crates/kyto-exec/tests/it/run_control.rs; device failures -> KY-E505):

- cancel: a host thread sets the cancel flag once the call's progress shows it running
  (mid-PCA after two passes, mid-kNN once the search has started); the call returns
  KG_CANCELLED (KY-E503) and the context serves the next call with the same results;
- out of memory: allocation failures injected on the host (kg_diag_fail_allocations) at
  many points of a PCA and of a kNN search; each call returns KG_ERR_OOM with kyto's
  memory_limit hint, frees what it allocated (the library pool's bytes in use return to
  where they were) and the next call succeeds;
- progress: kg_progress counts the PCA's passes (cells x passes) while it runs;
- wait limit: a call whose host wait runs past kg_set_wait_limit returns KG_ERR_TIMEOUT
  while its queued device work finishes on its own; the context works afterwards.
The device kernels' own bounded waits (mbarrier polls with an iteration limit) are not
made to run out here: that would need a stalled pipeline on the GPU."""

import gc
import threading
import time

import numpy as np
import pytest

import kyto_b200 as K
from kyto_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = K.Context(0)
    yield c
    c.set_cancel_flag(None)
    K.fail_allocations(None)


@pytest.fixture(scope="module")
def cells():
    return synthetic.counts_csr(300_000, 2000, 600.0, 20, 100, seed=4)


@pytest.fixture(scope="module")
def points():
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    return torch.randn((1_000_000, 50), generator=g, device="cuda")


def _pca(ctx, x, k=30):
    return K.pca(x.indptr, x.indices, x.values, x.n_genes, k, seed=0, target_sum=1e4,
                 log1p=True, ctx=ctx)


def _knn(ctx, pts):
    import torch

    n = pts.shape[0]
    out = (torch.empty(n + 1, dtype=torch.int64, device="cuda"),
           torch.empty(n * 14, dtype=torch.int32, device="cuda"),
           torch.empty(n * 14, dtype=torch.float32, device="cuda"))
    K._check(K.library().kg_knn_exact(ctx.handle, K._ptr(pts), n, 50, 0, 15, K._ptr(out[0]),
                                      K._ptr(out[1]), K._ptr(out[2]), None))
    torch.cuda.synchronize()
    return out


class _Watcher(threading.Thread):
    """Polls kg_progress; sets the cancel flag once `ready(done, total)` holds."""

    def __init__(self, ctx, flag, ready):
        super().__init__(daemon=True)
        self.ctx, self.flag, self.ready = ctx, flag, ready
        self.seen = []
        self.stop = False

    def run(self):
        t0 = time.monotonic()
        while not self.stop and time.monotonic() - t0 < 60:
            done, total = self.ctx.progress()
            self.seen.append((done, total))
            if self.flag is not None and self.ready(done, total):
                self.flag[0] = 1
                return
            time.sleep(0.0001)


def test_cancel_mid_pca_then_the_context_works(ctx, cells):
    before = _pca(ctx, cells)
    n = cells.n_cells
    flag = np.zeros(1, dtype=np.int32)
    ctx.set_cancel_flag(flag)
    try:
        # Armed by this run only: the previous run left done == total == 11 n.
        w = _Watcher(ctx, flag, lambda d, t: t == 11 * n and 2 * n <= d < 11 * n)
        w.start()
        with pytest.raises(K.KytoError) as e:
            _pca(ctx, cells)
        w.stop = True
        w.join()
        assert e.value.status == K.KG_CANCELLED and e.value.code == "KY-E503"
        # The captured traceback holds the cancelled call's session (its held input) in
        # a cycle through this frame: let it go now, not at some later collection.
        del e
        gc.collect()
        done, total = ctx.progress()
        assert 2 * n <= done < total == 11 * n
    finally:
        flag[0] = 0
        ctx.set_cancel_flag(None)
    after = _pca(ctx, cells)
    assert np.array_equal(after.embedding.view(np.uint32), before.embedding.view(np.uint32))
    assert np.array_equal(after.variance, before.variance)


def test_cancel_mid_knn_then_the_context_works(ctx, points):
    n = points.shape[0]
    before = _knn(ctx, points)
    flag = np.zeros(1, dtype=np.int32)
    ctx.set_cancel_flag(flag)
    try:
        # A finished search leaves done == total == n; a started one has done < n.
        w = _Watcher(ctx, flag, lambda d, t: t == n and d < n)
        w.start()
        with pytest.raises(K.KytoError) as e:
            _knn(ctx, points)
        w.stop = True
        w.join()
        assert e.value.status == K.KG_CANCELLED and e.value.code == "KY-E503"
        del e
        gc.collect()
    finally:
        flag[0] = 0
        ctx.set_cancel_flag(None)
    after = _knn(ctx, points)
    for a, b in zip(after, before):
        assert bool((a == b).all())


def test_progress_counts_the_pca_passes(ctx, cells):
    n = cells.n_cells
    w = _Watcher(ctx, None, lambda d, t: False)
    w.start()
    res = _pca(ctx, cells)
    w.stop = True
    w.join()
    assert ctx.progress() == (11 * n, 11 * n)
    assert res.passes_run == 11
    during = sorted({d for d, t in w.seen if t == 11 * n and 0 < d < 11 * n})
    assert during and all(d % n == 0 for d in during)


@pytest.mark.parametrize("after", [0, 1, 3, 8, 20, 60])
def test_injected_oom_frees_what_it_allocated(ctx, cells, points, after):
    import torch

    _pca(ctx, cells, k=10)
    _knn(ctx, points)
    # Objects awaiting the cyclic collector (an earlier test's failed call kept alive by
    # its traceback) still hold pool memory: collect them before taking the baseline.
    gc.collect()
    torch.cuda.synchronize()
    base = K.pool_usage(0)["used"]
    for call in (lambda: _pca(ctx, cells, k=10), lambda: _knn(ctx, points)):
        K.fail_allocations(after)
        failed = None
        try:
            call()
        except K.KytoError as e:
            # Only what the error says: the exception's traceback would keep the failed
            # call's session (and its buffers) alive.
            failed = (e.status, e.code, str(e))
        finally:
            K.fail_allocations(None)
        gc.collect()
        torch.cuda.synchronize()
        if failed is not None:
            assert failed[0] == K.KG_ERR_OOM and failed[1] == "KY-E505"
            assert "memory_limit" in failed[2]
        assert K.pool_usage(0)["used"] == base
        if after == 0:
            assert failed is not None  # the call's first allocation failed
    ok = _pca(ctx, cells, k=10)
    assert np.all(np.isfinite(ok.variance))


def test_wait_limit_returns_timeout_and_the_context_works(ctx, cells):
    import torch

    before = _pca(ctx, cells)
    sess = K.PcaSession(30, cells.n_genes, seed=0, target_sum=1e4, log1p=True, ctx=ctx)
    sess.push(cells.indptr, cells.indices, cells.values)
    # The run's last wait (after the embedding pass is queued) finds work still running.
    ctx.set_wait_limit(1e-9)
    try:
        st = K.library().kg_pca_run(sess._h)
    finally:
        ctx.set_wait_limit(900.0)
    assert st == K.KG_ERR_TIMEOUT
    sess.close()  # waits for the session's queued work
    torch.cuda.synchronize()
    after = _pca(ctx, cells)
    assert np.array_equal(after.embedding.view(np.uint32), before.embedding.view(np.uint32))
