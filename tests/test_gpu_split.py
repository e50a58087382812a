"""GPU test of one task split over GPUs (qld_cuda_ld_device_part): the parts,
computed here one after another on one GPU (each part is independent: no
exchange between GPUs), give bit for bit the r^2 and counts of the whole
task, for each kernel and both task kinds; empty trailing parts launch
nothing."""
import numpy as np
import pytest
import torch

import oracle
from conftest import lower_mask
from qld_b200 import api, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernel", [api.KERNEL_AUTO, api.KERNEL_POPC, api.KERNEL_MMA])
@pytest.mark.parametrize("m,n,N,sym,nparts", [(3000, 3000, 4096, True, 3),
                                              (1700, 900, 2500, False, 4),
                                              (300, 300, 1000, True, 5)])
def test_parts_equal_the_whole_task(gpu_ctx, kernel, m, n, N, sym, nparts):
    dev = torch.device("cuda", 0)
    t, _ = synth.all_pairs_workload(m=m + (0 if sym else n), n=N, seed=m + n)
    T = t.numpy().view(np.uint64)
    K = T.shape[1]
    lda = K + (K & 1)
    rows = m if sym else m + n
    dT = torch.zeros(rows, lda, dtype=torch.int64, device=dev)
    dT[:, :K] = torch.from_numpy(T.view(np.int64)).to(dev)
    bc = torch.from_numpy(oracle.bitcounts(T).view(np.int32).copy()).to(dev)
    A, bcA = dT[:m], bc[:m]
    B, bcB = (A, bcA) if sym else (dT[m:], bc[m:])
    gpu_ctx.set_option(api.OPT_KERNEL, kernel)
    st = torch.cuda.current_stream()
    whole = torch.full((n, m), -2.0, dtype=torch.float32, device=dev)
    wcnt = torch.zeros((n, m), dtype=torch.int32, device=dev)
    gpu_ctx.ld_device(A, bcA, m, lda, B, bcB, n, lda, K, N, sym, whole, m, counts=wcnt, ldc=m,
                      stream=st)
    split = torch.full((n, m), -2.0, dtype=torch.float32, device=dev)
    scnt = torch.zeros((n, m), dtype=torch.int32, device=dev)
    covered = 0
    for p in range(nparts):
        gpu_ctx.stats(reset=True)
        r0, r1 = gpu_ctx.ld_device_part(A, bcA, m, lda, B, bcB, n, lda, K, N, sym,
                                        split[covered:], m, p, nparts, counts=scnt[covered:],
                                        ldc=m, stream=st)
        gpu_ctx.sync(stream=st)
        assert r0 == covered and r1 >= r0
        if r1 == r0:
            assert gpu_ctx.stats().counts_launches == 0
        covered = r1
    assert covered == n
    mask = lower_mask(n, m) if sym else np.ones((n, m), bool)
    w, s_ = whole.cpu().numpy(), split.cpu().numpy()
    assert np.array_equal(w[mask].view(np.uint32), s_[mask].view(np.uint32))
    assert np.array_equal(wcnt.cpu().numpy()[mask], scnt.cpu().numpy()[mask])
    want = oracle.counts(T[:m], None if sym else T[m:])
    assert np.array_equal(scnt.cpu().numpy().view(np.uint32)[mask], want[mask])


def test_bench_split_path_runs_at_one_gpu():
    """bench.py --split at N = 1 runs the split path (qld_cuda_ld_device_part,
    one part) over the whole region and reports it as such."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--split", "--snps",
                          "4096", "--steps", "2", "--warmup", "1", "--no-e2e", "--no-cpu",
                          "--no-parity", "--sections", "none"],
                         capture_output=True, text=True, timeout=600, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1])
    assert line["split_rows"] == [0, 4096]
    assert line["scaling"] == "strong" and line["value"] > 0
    assert line["config"]["parallelism"].startswith("tile-row split x1")
    assert line["gpu_launches"] >= 2
