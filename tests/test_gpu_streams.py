"""Stream ordering between torch and the library, through the Python binding.

torch's default stream is the legacy NULL stream, while the C ABI reads a
NULL stream as the context's own (non-blocking) stream.  The binding passes
torch's default stream as cudaStreamLegacy, so a call is ordered after the
torch work that writes its inputs; Server.add_table waits for the streams
that write a device table.  Each test delays that torch work with a spin
kernel (torch.cuda._sleep, a bounded loop of clock cycles) so that an
unordered call would read the stale inputs."""
import numpy as np
import pytest
import torch

import oracle
from conftest import assert_r2_close, lower_mask
from qld_b200 import api, synth

pytestmark = pytest.mark.gpu

SPIN = 200_000_000          # ~0.1 s of GPU clock cycles


def _task(seed):
    t, n = synth.all_pairs_workload(m=1500, n=3000, seed=seed)
    A = t.numpy().view(np.uint64)
    return A, oracle.bitcounts(A), n


def test_device_call_on_torch_default_stream_follows_torch_work(gpu_ctx):
    A, bc, N = _task(31)
    m, K = A.shape
    dev = torch.device("cuda", 0)
    lda = K + (K & 1)
    dA = torch.zeros(m, lda, dtype=torch.int64, device=dev)
    dbc = torch.full((m,), 7, dtype=torch.int32, device=dev)       # stale bit counts
    out = torch.full((m, m), -3.0, dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream(dev)
    assert st.cuda_stream == 0                                     # the legacy stream
    hA = torch.from_numpy(A.view(np.int64).copy()).pin_memory()
    hbc = torch.from_numpy(bc.view(np.int32).copy()).pin_memory()
    torch.cuda._sleep(SPIN)                                        # the host does not wait
    dA[:, :K].copy_(hA, non_blocking=True)
    dbc.copy_(hbc, non_blocking=True)
    gpu_ctx.ld_device(dA, dbc, m, lda, dA, dbc, m, lda, K, N, True, out, m, stream=st)
    gpu_ctx.sync(stream=st)
    want = oracle.r2_exact(bc, bc, oracle.counts(A), N)
    assert_r2_close(out.cpu().numpy(), want, mask=lower_mask(m, m))


def test_server_table_from_a_side_stream(tmp_path):
    A, bc, N = _task(32)
    m, K = A.shape
    dev = torch.device("cuda", 0)
    side = torch.cuda.Stream(device=dev)
    dA = torch.zeros(m, K, dtype=torch.int64, device=dev)
    dbc = torch.zeros(m, dtype=torch.int32, device=dev)
    hA = torch.from_numpy(A.view(np.int64).copy()).pin_memory()
    hbc = torch.from_numpy(bc.view(np.int32).copy()).pin_memory()
    with torch.cuda.stream(side):
        torch.cuda._sleep(SPIN)
        dA.copy_(hA, non_blocking=True)
        dbc.copy_(hbc, non_blocking=True)
        with api.Server(0, pool_bytes=256 << 20, max_inflight=2) as srv:
            tid = srv.add_table(dA, dbc, N)
            qid = srv.submit(tid, 100, 900, 300, 1400, threshold=0.2)
            got = {}
            while qid not in got:
                for r in srv.poll(wait_ms=200):
                    got[r.id] = r
            assert got[qid].status == api.OK
            blk = np.empty((1100, 800), np.float32)
            srv.fetch(qid, blk)
    want = oracle.r2_exact(bc[100:900], bc[300:1400], oracle.counts(A[100:900], A[300:1400]), N)
    assert_r2_close(blk, want)
