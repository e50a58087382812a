"""GPU parity of the windowed (band) LD entry points: r^2 and counts for
pairs (i, i+1+d), d < band, against the oracle's full single-region result."""
import numpy as np
import pytest
import torch

import oracle
from conftest import assert_r2_close
from qld_b200 import api, synth
from test_gpu_parity import KERNELS, set_kernel

pytestmark = pytest.mark.gpu


def band_view(full, band):
    """(m, band) array of full[i, i+1+d] (B row i, A row i+1+d); NaN off the end."""
    m = full.shape[0]
    out = np.full((m, band), np.nan, dtype=np.float64)
    valid = np.zeros((m, band), bool)
    for d in range(band):
        i = np.arange(m - 1 - d) if m - 1 - d > 0 else np.arange(0)
        out[i, d] = full[i, i + 1 + d]
        valid[i, d] = True
    return out, valid


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("m,N,band", [(1500, 3000, 300), (700, 130, 1), (400, 4096, 1000),
                                      (2100, 9000, 517)])
def test_band_host_streaming(gpu_ctx, kernel, m, N, band):
    set_kernel(gpu_ctx, kernel)
    gpu_ctx.set_option(api.OPT_BAND_ROWS, 512)        # several streamed blocks
    try:
        t, _ = synth.all_pairs_workload(m=m, n=N, seed=m + band)
        A = t.numpy().view(np.uint64)
        bc = oracle.bitcounts(A)
        r2, cnt = gpu_ctx.ld_band(A, bc, S=N, band=band, counts=True)
    finally:
        gpu_ctx.set_option(api.OPT_BAND_ROWS, 4096)
    full_c = oracle.counts(A)
    want_c, valid = band_view(full_c.astype(np.float64), band)
    assert np.array_equal(cnt[valid].astype(np.float64), want_c[valid])
    want_r2, _ = band_view(oracle.r2_exact(bc, bc, full_c, N), band)
    got = np.where(valid, r2, 0).astype(np.float64)
    assert_r2_close(got, np.where(valid, want_r2, 0))


@pytest.mark.parametrize("kernel", KERNELS)
def test_band_device_padded_rows(gpu_ctx, kernel):
    set_kernel(gpu_ctx, kernel)
    m, N, band = 1300, 2500, 250
    t, _ = synth.all_pairs_workload(m=m, n=N, seed=77)
    A = t.numpy().view(np.uint64)
    K = A.shape[1]
    lda = K + 2 + (K & 1)
    dev = torch.device("cuda", 0)
    dA = torch.zeros(m, lda, dtype=torch.int64, device=dev)
    dA[:, :K] = t.to(dev)
    bc = oracle.bitcounts(A)
    dbc = torch.from_numpy(bc.view(np.int32).copy()).to(dev)
    ldr = band + 11
    r2 = torch.full((m, ldr), -3.0, dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream()
    gpu_ctx.ld_band_device(dA, dbc, m, lda, K, N, band, r2, ldr, stream=st)
    gpu_ctx.sync(stream=st)
    got = r2.cpu().numpy()
    assert np.all(got[:, band:] == -3.0), "wrote outside the band columns"
    want, valid = band_view(oracle.r2_exact(bc, bc, oracle.counts(A), N), band)
    assert np.all(got[:, :band][~valid] == -3.0), "wrote past the last SNP"
    assert_r2_close(np.where(valid, got[:, :band], 0).astype(np.float64), np.where(valid, want, 0))


def test_band_reference_mode_bit_exact(gpu_ctx):
    set_kernel(gpu_ctx, "mma256")
    gpu_ctx.set_option(api.OPT_R2_MODE, api.R2_REFERENCE)
    try:
        m, N, band = 900, 1200, 200
        t, _ = synth.all_pairs_workload(m=m, n=N, seed=5)
        A = t.numpy().view(np.uint64)
        bc = oracle.bitcounts(A)
        r2 = gpu_ctx.ld_band(A, bc, S=N, band=band)
    finally:
        gpu_ctx.set_option(api.OPT_R2_MODE, api.R2_EXACT)
    full = oracle.r2_reference(bc, bc, oracle.counts(A), N, fma_contract=False)
    want, valid = band_view(full.astype(np.float64), band)
    assert np.array_equal(r2[valid].astype(np.float32).view(np.uint32),
                          want[valid].astype(np.float32).view(np.uint32))
