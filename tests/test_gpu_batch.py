"""GPU parity of the batched launch (qld_cuda_ld_batch): heterogeneous tasks
in one persistent launch give each task the same r^2 and counts as running it
alone, and the oracle's counts."""
import numpy as np
import pytest
import torch

import oracle
from conftest import assert_r2_close, lower_mask
from qld_b200 import api, synth

pytestmark = pytest.mark.gpu


def _make_jobs(seed, count, max_rows, max_samples, dev):
    rng = np.random.default_rng(seed)
    jobs, host = [], []
    shared = None
    for j in range(count):
        sym = bool(rng.integers(0, 2))
        m = int(rng.integers(1, max_rows))
        n = m if sym else int(rng.integers(1, max_rows))
        N = int(rng.integers(1, max_samples))
        if j % 7 == 3:
            m = 0 if sym else m            # an empty task
            n = m if sym else 0
        t, _ = synth.all_pairs_workload(m=max(1, m) + (0 if sym else max(1, n)), n=N,
                                        seed=seed * 1000 + j)
        T = t.numpy().view(np.uint64)
        K = T.shape[1]
        lda = K + (K & 1)
        A = np.ascontiguousarray(T[:m])
        B = A if sym else np.ascontiguousarray(T[max(1, m):max(1, m) + n])
        if j == 5 and shared is not None:  # two tasks reading the same table
            A, N, K, lda = shared
            m = A.shape[0]
            sym, B, n = True, A, A.shape[0]
        if j == 2:
            shared = (A, N, K, lda)
        dA = torch.zeros(max(1, m), lda, dtype=torch.int64, device=dev)
        dB = torch.zeros(max(1, n), lda, dtype=torch.int64, device=dev)
        if m:
            dA[:m, :K] = torch.from_numpy(A.view(np.int64)).to(dev)
        if n and not sym:
            dB[:n, :K] = torch.from_numpy(B.view(np.int64)).to(dev)
        bcA = oracle.bitcounts(A) if m else np.zeros(0, np.uint32)
        bcB = bcA if sym else (oracle.bitcounts(B) if n else np.zeros(0, np.uint32))
        dbcA = torch.from_numpy(bcA.view(np.int32).copy()).to(dev) if m else \
            torch.zeros(1, dtype=torch.int32, device=dev)
        dbcB = dbcA if sym else (torch.from_numpy(bcB.view(np.int32).copy()).to(dev) if n else
                                 torch.zeros(1, dtype=torch.int32, device=dev))
        r2 = torch.full((max(1, n), max(1, m)), -5.0, dtype=torch.float32, device=dev)
        cnt = torch.zeros((max(1, n), max(1, m)), dtype=torch.int32, device=dev)
        jobs.append(dict(A=dA, bcA=dbcA, m=m, lda=lda, B=dA if sym else dB, bcB=dbcB, n=n,
                         ldb=lda, K=K, S=N, symmetric=sym, r2=r2, ldr=max(1, m), counts=cnt,
                         ldc=max(1, m)))
        host.append((A, B, bcA, bcB, N, sym))
    return jobs, host


@pytest.mark.parametrize("mode", [api.R2_EXACT, api.R2_REFERENCE])
def test_batch_matches_single_tasks_and_oracle(gpu_ctx, mode):
    dev = torch.device("cuda", 0)
    jobs, host = _make_jobs(7, 40, 700, 9000, dev)
    gpu_ctx.set_option(api.OPT_R2_MODE, mode)
    st = torch.cuda.current_stream()
    try:
        gpu_ctx.ld_batch(jobs, stream=st)
        gpu_ctx.sync(stream=st)
        batch_r2 = [j["r2"].clone() for j in jobs]
        batch_cnt = [j["counts"].clone() for j in jobs]
        # the single-task 4-bit kernel does the batch's arithmetic (F32 counts,
        # the same r^2 evaluation), so the r^2 bits must agree
        gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_FP4)
        for j in jobs:
            j["r2"].fill_(-5.0)
            if j["m"] and j["n"]:
                gpu_ctx.ld_device(j["A"], j["bcA"], j["m"], j["lda"], j["B"], j["bcB"], j["n"],
                                  j["ldb"], j["K"], j["S"], j["symmetric"], j["r2"], j["ldr"],
                                  stream=st)
        gpu_ctx.sync(stream=st)
    finally:
        gpu_ctx.set_option(api.OPT_R2_MODE, api.R2_EXACT)
        gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_AUTO)
    for j, (A, B, bcA, bcB, N, sym), r2b, cb in zip(jobs, host, batch_r2, batch_cnt):
        m, n = j["m"], j["n"]
        if not (m and n):
            assert torch.all(r2b == -5.0), "an empty task wrote output"
            continue
        mask = lower_mask(n, m) if sym else np.ones((n, m), bool)
        single = j["r2"][:n, :m].cpu().numpy()
        got = r2b[:n, :m].cpu().numpy()
        assert np.array_equal(got[mask].view(np.uint32), single[mask].view(np.uint32))
        want_c = oracle.counts(A, B)
        assert np.array_equal(cb[:n, :m].cpu().numpy().view(np.uint32)[mask], want_c[mask])
        if mode == api.R2_EXACT:
            assert_r2_close(got, oracle.r2_exact(bcA, bcB, want_c, N), mask=mask)
        else:
            want = oracle.r2_reference(bcA, bcB, want_c, N, fma_contract=False)
            assert np.array_equal(got[mask].view(np.uint32), want[mask].view(np.uint32))


def test_batch_many_small_tasks(gpu_ctx):
    """More tasks than SMs and ring slots: the queue must hand out every item."""
    dev = torch.device("cuda", 0)
    jobs, host = _make_jobs(11, 400, 300, 3000, dev)
    st = torch.cuda.current_stream()
    gpu_ctx.ld_batch(jobs, stream=st)
    gpu_ctx.sync(stream=st)
    for j, (A, B, bcA, bcB, N, sym) in zip(jobs, host):
        m, n = j["m"], j["n"]
        if not (m and n):
            continue
        mask = lower_mask(n, m) if sym else np.ones((n, m), bool)
        want_c = oracle.counts(A, B)
        assert np.array_equal(j["counts"][:n, :m].cpu().numpy().view(np.uint32)[mask],
                              want_c[mask])


def test_batch_rejects_bad_job(gpu_ctx):
    dev = torch.device("cuda", 0)
    jobs, _ = _make_jobs(13, 3, 100, 500, dev)
    jobs[1] = dict(jobs[1], lda=jobs[1]["K"] - 1)
    with pytest.raises(api.QldError) as e:
        gpu_ctx.ld_batch(jobs)
    assert e.value.code == api.ERR_INVALID


def test_batch_past_the_int8_limit(gpu_ctx):
    """Tasks of 140,000 and 200,000 samples (past 131,071, the int8 kernels'
    exact range) in one batch: counts exact, r^2 within the FP64 bar."""
    dev = torch.device("cuda", 0)
    jobs, host = [], []
    for seed, (m, N, sym) in enumerate([(300, 140_000, True), (130, 200_000, False)]):
        t, _ = synth.all_pairs_workload(m=m + (0 if sym else 90), n=N, seed=60 + seed)
        T = t.numpy().view(np.uint64)
        K = T.shape[1]
        lda = K + (K & 1)
        A, B = T[:m], (T[:m] if sym else T[m:])
        dA = torch.zeros(m, lda, dtype=torch.int64, device=dev)
        dA[:, :K] = torch.from_numpy(A.view(np.int64)).to(dev)
        dB = dA
        if not sym:
            dB = torch.zeros(B.shape[0], lda, dtype=torch.int64, device=dev)
            dB[:, :K] = torch.from_numpy(np.ascontiguousarray(B).view(np.int64)).to(dev)
        bcA, bcB = oracle.bitcounts(A), oracle.bitcounts(B)
        n = B.shape[0]
        r2 = torch.full((n, m), -5.0, dtype=torch.float32, device=dev)
        cnt = torch.zeros((n, m), dtype=torch.int32, device=dev)
        jobs.append(dict(A=dA, bcA=torch.from_numpy(bcA.view(np.int32).copy()).to(dev), m=m,
                         lda=lda, B=dB, bcB=torch.from_numpy(bcB.view(np.int32).copy()).to(dev),
                         n=n, ldb=lda, K=K, S=N, symmetric=sym, r2=r2, ldr=m, counts=cnt, ldc=m))
        host.append((A, B, bcA, bcB, N, sym))
    st = torch.cuda.current_stream()
    gpu_ctx.ld_batch(jobs, stream=st)
    gpu_ctx.sync(stream=st)
    for j, (A, B, bcA, bcB, N, sym) in zip(jobs, host):
        n, m = j["n"], j["m"]
        mask = lower_mask(n, m) if sym else np.ones((n, m), bool)
        want_c = oracle.counts(A, B)
        assert np.array_equal(j["counts"].cpu().numpy().view(np.uint32)[mask], want_c[mask])
        assert_r2_close(j["r2"].cpu().numpy(), oracle.r2_exact(bcA, bcB, want_c, N), mask=mask)


def _device_job(A, B, N, sym, dev):
    """One task's device buffers from host tables (rows padded to an even pitch)."""
    K = A.shape[1]
    lda = K + (K & 1)
    m, n = A.shape[0], B.shape[0]
    dA = torch.zeros(m, lda, dtype=torch.int64, device=dev)
    dA[:, :K] = torch.from_numpy(np.ascontiguousarray(A).view(np.int64)).to(dev)
    dB = dA
    if not sym:
        dB = torch.zeros(n, lda, dtype=torch.int64, device=dev)
        dB[:, :K] = torch.from_numpy(np.ascontiguousarray(B).view(np.int64)).to(dev)
    bcA, bcB = oracle.bitcounts(A), oracle.bitcounts(B)
    return dict(A=dA, bcA=torch.from_numpy(bcA.view(np.int32).copy()).to(dev), m=m, lda=lda,
                B=dB, bcB=torch.from_numpy(bcB.view(np.int32).copy()).to(dev), n=n, ldb=lda,
                K=K, S=N, symmetric=sym,
                r2=torch.full((n, m), -5.0, dtype=torch.float32, device=dev), ldr=m,
                counts=torch.zeros((n, m), dtype=torch.int32, device=dev), ldc=m)


def _check_job(j, A, B, N, sym):
    n, m = j["n"], j["m"]
    mask = lower_mask(n, m) if sym else np.ones((n, m), bool)
    want_c = oracle.counts(A, B)
    assert np.array_equal(j["counts"].cpu().numpy().view(np.uint32)[mask], want_c[mask])
    assert_r2_close(j["r2"].cpu().numpy(), oracle.r2_exact(oracle.bitcounts(A),
                                                           oracle.bitcounts(B), want_c, N),
                    mask=mask)


def test_batch_routes_past_2_24_samples_to_popcount(gpu_ctx):
    """K * 64 > 2^24: the 4-bit path's F32 accumulators would round, so that
    task runs on the popcount kernel after the persistent launch, beside 4-bit
    tasks in the same call; every task matches the oracle."""
    dev = torch.device("cuda", 0)
    specs = [(40, (1 << 24) + 200, True, 90), (30, (1 << 24) + 64 * 7, False, 91),
             (500, 3000, True, 92), (300, 7000, False, 93)]
    jobs, host = [], []
    for m, N, sym, seed in specs:
        t, _ = synth.all_pairs_workload(m=m + (0 if sym else 25), n=N, seed=seed)
        T = t.numpy().view(np.uint64)
        A, B = T[:m], (T[:m] if sym else T[m:])
        jobs.append(_device_job(A, B, N, sym, dev))
        host.append((A, B, N, sym))
    st = torch.cuda.current_stream()
    gpu_ctx.stats(reset=True)
    gpu_ctx.ld_batch(jobs, stream=st)
    gpu_ctx.sync(stream=st)
    stats = gpu_ctx.stats(reset=True)
    assert stats.counts_launches >= 3          # the persistent launch + two popcount launches
    for j, (A, B, N, sym) in zip(jobs, host):
        _check_job(j, A, B, N, sym)


def test_batch_follows_the_autotuner_per_job(tmp_path):
    """A tuned class that prefers the popcount kernel takes its jobs out of the
    persistent launch; the other jobs stay in it; results match the oracle."""
    dev = torch.device("cuda", 0)
    path = tmp_path / "tune.txt"
    path.write_text("qld-tune 1\n9 9 5 1 1 0 0.9\n")   # 512-1023 SNPs, 32-63 words, single
    jobs, host = [], []
    for m, N, sym, seed in [(700, 2500, True, 94), (700, 2500, False, 95),
                            (200, 2500, True, 96)]:
        t, _ = synth.all_pairs_workload(m=m + (0 if sym else 100), n=N, seed=seed)
        T = t.numpy().view(np.uint64)
        A, B = T[:m], (T[:m] if sym else T[m:])
        jobs.append(_device_job(A, B, N, sym, dev))
        host.append((A, B, N, sym))
    with api.Context(0) as ctx:                      # its own tuning table
        ctx.tune_load(str(path))
        st = torch.cuda.current_stream()
        ctx.ld_batch(jobs, stream=st)
        ctx.sync(stream=st)
        stats = ctx.stats(reset=True)
    assert stats.counts_launches == 2               # the persistent launch + one popcount launch
    assert stats.last_kernel == api.KERNEL_POPC
    for j, (A, B, N, sym) in zip(jobs, host):
        _check_job(j, A, B, N, sym)


def test_batch_rejects_a_forced_kernel_that_is_not_exact(gpu_ctx):
    """A forced 4-bit kernel past 2^24 samples: refused before anything runs."""
    dev = torch.device("cuda", 0)
    K = (1 << 24) // 64 + 2
    A = torch.zeros(2, K, dtype=torch.int64, device=dev)
    bc = torch.zeros(2, dtype=torch.int32, device=dev)
    r2 = torch.zeros(2, 2, dtype=torch.float32, device=dev)
    job = dict(A=A, bcA=bc, m=2, lda=K, B=A, bcB=bc, n=2, ldb=K, K=K, S=K * 64, symmetric=True,
               r2=r2, ldr=2, counts=None, ldc=2)
    gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_FP4)
    try:
        with pytest.raises(api.QldError) as e:
            gpu_ctx.ld_batch([job])
    finally:
        gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_AUTO)
    assert e.value.code == api.ERR_UNSUPPORTED
