"""GPU tests of the serving loop (qld_srv_*): results are the same alone and
in the mix, admission is by output memory, summaries match the r^2 blocks."""
import time

import numpy as np
import pytest
import torch

import oracle
from conftest import assert_r2_close, lower_mask
from qld_b200 import api, synth

pytestmark = pytest.mark.gpu

M, N = 3000, 5000


@pytest.fixture(scope="module")
def table():
    f = synth.beta_freqs(M, 0.1, 1.0, 91, clip_min=1.0 / N)
    t = synth.copying_table(M, N, 20, 50, 300, 0.01, f, 91)
    A = t.numpy().view(np.uint64)
    return A, oracle.bitcounts(A)


def _queries(seed, count, max_side):
    rng = np.random.default_rng(seed)
    qs = []
    for k in range(count):
        la = int(rng.integers(1, max_side))
        a0 = int(rng.integers(0, M - la + 1))
        if k % 3 == 0:                       # single region
            qs.append((a0, a0 + la, a0, a0 + la))
        else:
            lb = int(rng.integers(1, max_side))
            b0 = int(rng.integers(0, M - lb + 1))
            qs.append((a0, a0 + la, b0, b0 + lb))
    return qs


def _wait_all(srv, ids, timeout_s=120, release=False):
    got = {}
    t0 = time.time()
    while len(got) < len(ids) and time.time() - t0 < timeout_s:
        for r in srv.poll(wait_ms=200):
            got[r.id] = r
            if release:
                srv.release(r.id)
    assert len(got) == len(ids), f"{len(ids) - len(got)} queries never finished"
    return got


def _summary(block, sym, thr):
    n, m = block.shape
    mask = (np.arange(m)[None, :] > np.arange(n)[:, None]) if sym else np.ones((n, m), bool)
    v = block[mask]
    v = v[v < 100]
    return int((v >= thr).sum()), float(v.astype(np.float64).sum()), float(v.max()) if v.size else 0.0


def test_same_alone_and_in_the_mix(table):
    A, bc = table
    qs = _queries(5, 24, 1200)
    ctx = api.Context(0)
    bufs_alone = [ctx.pinned_empty((b1 - b0, a1 - a0), np.float32) for (a0, a1, b0, b1) in qs]
    bufs_mix = [ctx.pinned_empty((b1 - b0, a1 - a0), np.float32) for (a0, a1, b0, b1) in qs]
    with api.Server(0, pool_bytes=1 << 30, max_inflight=3) as srv:
        tid = srv.add_table(A, bc, N)
        alone = []
        for q, buf in zip(qs, bufs_alone):       # one at a time
            qid = srv.submit(tid, *q, threshold=0.1, host_r2=buf)
            alone.append(_wait_all(srv, [qid])[qid])
        ids = [srv.submit(tid, *q, threshold=0.1, host_r2=buf) for q, buf in zip(qs, bufs_mix)]
        mix = _wait_all(srv, ids)
    for (a0, a1, b0, b1), ba, bm, ra, qid in zip(qs, bufs_alone, bufs_mix, alone, ids):
        sym = (a0, a1) == (b0, b1)
        mask = lower_mask(b1 - b0, a1 - a0) if sym else np.ones((b1 - b0, a1 - a0), bool)
        assert ra.status == api.OK and mix[qid].status == api.OK
        assert np.array_equal(ba[mask].view(np.uint32), bm[mask].view(np.uint32))
        assert (ra.n_above, ra.pairs) == (mix[qid].n_above, mix[qid].pairs)
        # against the oracle
        Aq, Bq = A[a0:a1], A[b0:b1]
        want_c = oracle.counts(Aq, Bq)
        assert_r2_close(bm, oracle.r2_exact(bc[a0:a1], bc[b0:b1], want_c, N), mask=mask)
        n_above, s, mx = _summary(bm, sym, 0.1)
        assert mix[qid].n_above == n_above
        assert abs(mix[qid].sum_r2 - s) <= 1e-6 * max(1.0, s)
        assert mix[qid].max_r2 == pytest.approx(mx, rel=0, abs=0)
    ctx.close()


def test_admission_by_output_memory(table):
    A, bc = table
    side = 1500                                # 9 MB of r^2 per query
    with api.Server(0, pool_bytes=20 << 20, max_inflight=4) as srv:   # room for two
        tid = srv.add_table(A, bc, N)
        ids = [srv.submit(tid, 0, side, side, 2 * side) for _ in range(8)]
        # results stay on the device until released: releasing them as they
        # arrive is what lets the waiting queries in
        got = _wait_all(srv, ids, release=True)
        assert all(r.status == api.OK for r in got.values())
        with pytest.raises(api.QldError) as e:
            srv.submit(tid, 0, M, 0, M)         # 36 MB alone exceeds the pool
        assert e.value.code == api.ERR_BUSY


def test_fetch_and_release(table):
    A, bc = table
    with api.Server(0, pool_bytes=256 << 20, max_inflight=2) as srv:
        tid = srv.add_table(A, bc, N)
        qid = srv.submit(tid, 100, 900, 1500, 2100, threshold=0.05)
        res = _wait_all(srv, [qid])[qid]
        out = np.empty((600, 800), np.float32)
        srv.fetch(qid, out)
        want_c = oracle.counts(A[100:900], A[1500:2100])
        assert_r2_close(out, oracle.r2_exact(bc[100:900], bc[1500:2100], want_c, N))
        assert res.n_above == _summary(out, False, 0.05)[0]
        srv.release(qid)
        with pytest.raises(api.QldError):
            srv.fetch(qid, out)


def test_destroy_with_work_pending(table):
    A, bc = table
    srv = api.Server(0, pool_bytes=64 << 20, max_inflight=2)
    tid = srv.add_table(A, bc, N)
    for k in range(40):
        srv.submit(tid, 0, 2000, 1000, 3000)
    t0 = time.time()
    srv.close()                                 # cancels pending, waits for running batches
    assert time.time() - t0 < 60


def test_bad_queries_rejected(table):
    A, bc = table
    with api.Server(0, pool_bytes=64 << 20, max_inflight=1) as srv:
        tid = srv.add_table(A, bc, N)
        with pytest.raises(api.QldError) as e:
            srv.submit(tid, 10, 5, 0, 3)
        assert e.value.code == api.ERR_INVALID
        with pytest.raises(api.QldError) as e:
            srv.submit(tid + 1, 0, 3, 0, 3)
        assert e.value.code == api.ERR_INVALID
        with pytest.raises(api.QldError) as e:   # pageable host buffer
            srv.submit(tid, 0, 3, 0, 3, host_r2=np.empty((3, 3), np.float32))
        assert e.value.code == api.ERR_INVALID


def test_device_table_same_as_host_table(table):
    """A table added from device memory (odd K: it goes through the device
    staging copy and the re-pitching kernel) gives the same r^2 blocks and
    summaries as the same table added from host memory."""
    A, bc = table
    assert A.shape[1] % 2 == 1
    dA = torch.from_numpy(A.view(np.int64).copy()).cuda()
    dbc = torch.from_numpy(bc.view(np.int32).copy()).cuda()
    ctx = api.Context(0)
    qs = [(0, 1800, 0, 1800), (100, 2900, 2000, 3000)]
    outs = {}
    try:
        for name, (tA, tbc) in {"host": (A, bc), "device": (dA, dbc)}.items():
            with api.Server(0, pool_bytes=256 << 20, max_inflight=2) as srv:
                tid = srv.add_table(tA, tbc, N)
                bufs = [ctx.pinned_empty((b1 - b0, a1 - a0), np.float32) for (a0, a1, b0, b1) in qs]
                ids = [srv.submit(tid, *q, host_r2=buf) for q, buf in zip(qs, bufs)]
                got = _wait_all(srv, ids, release=True)
                outs[name] = ([b.copy() for b in bufs],
                              [(got[i].n_above, got[i].sum_r2, got[i].max_r2) for i in ids])
    finally:
        ctx.close()
    for h, d in zip(outs["host"][0], outs["device"][0]):
        assert np.array_equal(h.view(np.uint32), d.view(np.uint32))
    assert outs["host"][1] == outs["device"][1] or all(
        hn == dn and abs(hs - ds) <= 1e-9 * max(1.0, hs) and hm == dm
        for (hn, hs, hm), (dn, ds, dm) in zip(outs["host"][1], outs["device"][1]))
