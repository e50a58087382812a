"""GPU tests of the graph-captured batched call (qld_cuda_batch_plan /
qld_cuda_batch_run): a replay gives every task the same r^2 bits and counts
as the direct batched call and the oracle's counts, reads the tables as they
are at replay time, keeps the options the plan was made with, and replays of
one plan on different streams run one after another."""
import numpy as np
import pytest
import torch

import oracle
from conftest import assert_r2_close, lower_mask
from qld_b200 import api, synth
from test_gpu_batch import _check_job, _device_job, _make_jobs

pytestmark = pytest.mark.gpu


def _outputs(jobs):
    return [(j["r2"].clone(), j["counts"].clone()) for j in jobs]


def _reset(jobs):
    for j in jobs:
        j["r2"].fill_(-5.0)
        j["counts"].zero_()


def _same(jobs, ref):
    for j, (r2, cnt) in zip(jobs, ref):
        assert torch.equal(j["r2"].view(torch.int32), r2.view(torch.int32))
        assert torch.equal(j["counts"], cnt)


def test_replay_matches_direct_call_and_oracle(gpu_ctx):
    dev = torch.device("cuda", 0)
    jobs, host = _make_jobs(17, 60, 700, 9000, dev)
    st = torch.cuda.current_stream()
    gpu_ctx.ld_batch(jobs, stream=st)
    gpu_ctx.sync(stream=st)
    direct = _outputs(jobs)
    _reset(jobs)
    with gpu_ctx.batch_plan(jobs) as plan:
        gpu_ctx.sync(stream=st)
        assert all(torch.all(j["r2"] == -5.0) for j in jobs), "making a plan ran work"
        gpu_ctx.stats(reset=True)
        for _ in range(2):                      # every replay recomputes every task
            _reset(jobs)
            plan.run(stream=st)
            gpu_ctx.sync(stream=st)
            _same(jobs, direct)
        stats = gpu_ctx.stats(reset=True)
    assert stats.counts_launches == 2           # one persistent launch per replay
    for j, (A, B, bcA, bcB, N, sym) in list(zip(jobs, host))[:12]:
        m, n = j["m"], j["n"]
        if not (m and n):
            continue
        mask = lower_mask(n, m) if sym else np.ones((n, m), bool)
        want_c = oracle.counts(A, B)
        assert np.array_equal(j["counts"][:n, :m].cpu().numpy().view(np.uint32)[mask],
                              want_c[mask])
        assert_r2_close(j["r2"][:n, :m].cpu().numpy(), oracle.r2_exact(bcA, bcB, want_c, N),
                        mask=mask)


def test_replay_reads_the_tables_as_they_are_then(gpu_ctx):
    """Tables rewritten in place (new haplotypes, same shapes) between
    replays: the second replay gives the new tables' results."""
    dev = torch.device("cuda", 0)
    specs = [(600, 5000, True), (300, 7000, False), (250, 3000, True)]
    jobs, tables = [], []
    for i, (m, N, sym) in enumerate(specs):
        t, _ = synth.all_pairs_workload(m=m + (0 if sym else 200), n=N, seed=300 + i)
        T = t.numpy().view(np.uint64)
        A, B = T[:m], (T[:m] if sym else T[m:])
        jobs.append(_device_job(A, B, N, sym, dev))
        tables.append((A, B, N, sym))
    st = torch.cuda.current_stream()
    with gpu_ctx.batch_plan(jobs) as plan:
        plan.run(stream=st)
        gpu_ctx.sync(stream=st)
        for j, (A, B, N, sym) in zip(jobs, tables):
            _check_job(j, A, B, N, sym)
        new = []
        for i, (j, (A, B, N, sym)) in enumerate(zip(jobs, tables)):
            t, _ = synth.all_pairs_workload(m=A.shape[0] + (0 if sym else B.shape[0]), n=N,
                                            seed=400 + i)
            T = t.numpy().view(np.uint64)
            A2, B2 = T[:A.shape[0]], (T[:A.shape[0]] if sym else T[A.shape[0]:])
            K = A2.shape[1]
            j["A"][:, :K] = torch.from_numpy(np.ascontiguousarray(A2).view(np.int64)).to(dev)
            j["bcA"].copy_(torch.from_numpy(oracle.bitcounts(A2).view(np.int32).copy()))
            if not sym:
                j["B"][:, :K] = torch.from_numpy(np.ascontiguousarray(B2).view(np.int64)).to(dev)
                j["bcB"].copy_(torch.from_numpy(oracle.bitcounts(B2).view(np.int32).copy()))
            new.append((A2, B2, N, sym))
        _reset(jobs)
        plan.run(stream=st)
        gpu_ctx.sync(stream=st)
    for j, (A, B, N, sym) in zip(jobs, new):
        _check_job(j, A, B, N, sym)


def test_plan_keeps_its_r2_mode(gpu_ctx):
    """Made in reference mode, replayed after the context went back to exact
    mode: the r^2 bits are the reference sequence's."""
    dev = torch.device("cuda", 0)
    jobs, host = _make_jobs(19, 16, 500, 6000, dev)
    st = torch.cuda.current_stream()
    gpu_ctx.set_option(api.OPT_R2_MODE, api.R2_REFERENCE)
    try:
        plan = gpu_ctx.batch_plan(jobs)
    finally:
        gpu_ctx.set_option(api.OPT_R2_MODE, api.R2_EXACT)
    with plan:
        plan.run(stream=st)
        gpu_ctx.sync(stream=st)
    for j, (A, B, bcA, bcB, N, sym) in zip(jobs, host):
        m, n = j["m"], j["n"]
        if not (m and n):
            continue
        mask = lower_mask(n, m) if sym else np.ones((n, m), bool)
        want = oracle.r2_reference(bcA, bcB, oracle.counts(A, B), N, fma_contract=False)
        got = j["r2"][:n, :m].cpu().numpy()
        assert np.array_equal(got[mask].view(np.uint32), want[mask].view(np.uint32))


def test_plan_with_routed_tasks(tmp_path):
    """A tuned class that prefers the popcount kernel: its tasks are routed
    launches inside the captured graph, the others stay in the persistent
    launch; a replay counts both and matches the oracle."""
    dev = torch.device("cuda", 0)
    path = tmp_path / "tune.txt"
    path.write_text("qld-tune 1\n9 9 5 1 1 0 0.9\n")   # 512-1023 SNPs, 32-63 words, single
    jobs, host = [], []
    for m, N, sym, seed in [(700, 2500, True, 194), (700, 2500, False, 195),
                            (200, 2500, True, 196), (800, 2600, True, 197)]:
        t, _ = synth.all_pairs_workload(m=m + (0 if sym else 100), n=N, seed=seed)
        T = t.numpy().view(np.uint64)
        A, B = T[:m], (T[:m] if sym else T[m:])
        jobs.append(_device_job(A, B, N, sym, dev))
        host.append((A, B, N, sym))
    with api.Context(0) as ctx:
        ctx.tune_load(str(path))
        st = torch.cuda.current_stream()
        plan = ctx.batch_plan(jobs)
        ctx.stats(reset=True)
        plan.run(stream=st)
        ctx.sync(stream=st)
        stats = ctx.stats(reset=True)
        plan.close()
    assert stats.counts_launches == 3       # the persistent launch + two popcount launches
    for j, (A, B, N, sym) in zip(jobs, host):
        _check_job(j, A, B, N, sym)


def test_replays_on_two_streams_run_in_turn(gpu_ctx):
    """Two replays of one plan on different streams, back to back: they share
    the plan's ticket counter, so the second must wait for the first."""
    dev = torch.device("cuda", 0)
    jobs, host = _make_jobs(23, 30, 600, 8000, dev)
    st = torch.cuda.current_stream()
    gpu_ctx.ld_batch(jobs, stream=st)
    gpu_ctx.sync(stream=st)
    direct = _outputs(jobs)
    _reset(jobs)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    s1.wait_stream(st)
    s2.wait_stream(st)
    with gpu_ctx.batch_plan(jobs) as plan:
        plan.run(stream=s1)
        plan.run(stream=s2)
        gpu_ctx.sync(stream=s1)
        gpu_ctx.sync(stream=s2)
    _same(jobs, direct)


def test_plan_errors_and_empty_plans(gpu_ctx):
    dev = torch.device("cuda", 0)
    jobs, _ = _make_jobs(29, 3, 100, 500, dev)
    bad = list(jobs)
    bad[1] = dict(bad[1], lda=bad[1]["K"] - 1)
    with pytest.raises(api.QldError) as e:
        gpu_ctx.batch_plan(bad)
    assert e.value.code == api.ERR_INVALID
    st = torch.cuda.current_stream()
    empty = [dict(jobs[0], m=0, n=0)]
    for js in ([], empty):                   # no work: a replay does nothing
        with gpu_ctx.batch_plan(js) as plan:
            plan.run(stream=st)
            gpu_ctx.sync(stream=st)
    # a plan left alive is freed with its context; using it then is refused
    with api.Context(0) as ctx:
        plan = ctx.batch_plan(jobs)
    with pytest.raises(api.QldError):
        plan.run()
    plan.close()
