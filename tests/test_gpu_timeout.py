"""GPU test of the kernels' bounded waits, without a fault.

Every wait inside a counts kernel gives up after a cycle budget
(QLD_OPT_WAIT_CYCLES), records the cause in the context's status word and
ends the kernel early, after draining its own copies and MMAs; the host turns
the status into QLD_ERR_TIMEOUT.  With a budget of one cycle the epilogue's
first wait for a tile's accumulators (one tile of 100,000 samples takes
~0.1 ms of MMAs) runs out, so the call must fail with that code, and the
same context, back on the default budget, must then compute the task
exactly: the context stays usable."""
import numpy as np
import pytest
import torch

import oracle
from conftest import assert_r2_close, lower_mask
from qld_b200 import api, synth

pytestmark = pytest.mark.gpu

N = 100_000          # 1,563 words per SNP


@pytest.fixture(scope="module")
def table():
    t, _ = synth.all_pairs_workload(m=600, n=N, seed=41)
    A = t.numpy().view(np.uint64)
    return A, oracle.bitcounts(A), oracle.counts(A)


def test_host_call_times_out_then_recovers(table):
    A, bc, want = table
    c = api.Context(0)
    try:
        c.set_option(api.OPT_WAIT_CYCLES, 1)
        with pytest.raises(api.QldError) as e:
            c.ld(A, bc, S=N)
        assert e.value.code == api.ERR_TIMEOUT
        c.set_option(api.OPT_WAIT_CYCLES, 0)
        r2, cnt = c.ld(A, bc, S=N, counts=True)
        mask = lower_mask(*want.shape)
        assert np.array_equal(cnt[mask], want[mask])
        assert_r2_close(r2, oracle.r2_exact(bc, bc, want, N), mask=mask)
        with pytest.raises(api.QldError) as e:
            c.set_option(api.OPT_WAIT_CYCLES, -5)
        assert e.value.code == api.ERR_INVALID
    finally:
        c.close()


def test_batched_launch_times_out_then_recovers(table):
    A, bc, want = table
    dev = torch.device("cuda", 0)
    K = A.shape[1]
    lda = K + (K & 1)
    m = A.shape[0]
    dA = torch.zeros(m, lda, dtype=torch.int64, device=dev)
    dA[:, :K] = torch.from_numpy(A.view(np.int64)).to(dev)
    dbc = torch.from_numpy(bc.view(np.int32).copy()).to(dev)
    r2 = torch.zeros(m, m, dtype=torch.float32, device=dev)
    cnt = torch.zeros(m, m, dtype=torch.int32, device=dev)
    job = dict(A=dA, bcA=dbc, m=m, lda=lda, B=dA, bcB=dbc, n=m, ldb=lda, K=K, S=N,
               symmetric=True, r2=r2, ldr=m, counts=cnt, ldc=m)
    c = api.Context(0)
    st = torch.cuda.current_stream()
    try:
        c.set_option(api.OPT_WAIT_CYCLES, 1)
        c.ld_batch([job], stream=st)
        with pytest.raises(api.QldError) as e:
            c.sync(stream=st)
        assert e.value.code == api.ERR_TIMEOUT
        c.set_option(api.OPT_WAIT_CYCLES, 0)
        c.ld_batch([job], stream=st)
        c.sync(stream=st)
        mask = lower_mask(m, m)
        assert np.array_equal(cnt.cpu().numpy().view(np.uint32)[mask], want[mask])
    finally:
        c.close()
