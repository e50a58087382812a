"""GPU test of qld_cuda_ld_noalloc(), the entry point for callers that cannot
allocate device memory (their GPU memory is owned by another component).

It is checked through the C ABI against the regular entry point,
qld_cuda_ld(), on the same inputs: r^2 within the suite's tolerance (1e-6
relative; special values exact), on two calls in a row, because every call
reuses the same static scratch array and must not see the previous call's
contents.  The file is named to be collected last.
"""
import ctypes as ct

import numpy as np
import pytest

import oracle
from conftest import assert_r2_close, lower_mask
from qld_b200 import api, synth

pytestmark = pytest.mark.gpu

ERR_TOO_LARGE = -8


def _lib():
    lib = api.load_library()
    vp, i = ct.c_void_p, ct.c_int
    lib.qld_cuda_ld_noalloc.argtypes = [vp, vp, i, vp, vp, i, i, i, i, vp, vp]
    lib.qld_cuda_ld_noalloc.restype = i
    return lib


def _noalloc(lib, A, bcA, B, bcB, S, symmetric):
    m, K = A.shape
    n = m if symmetric else B.shape[0]
    out = np.full((n, m), np.nan, np.float32)
    rc = lib.qld_cuda_ld_noalloc(A.ctypes.data, bcA.ctypes.data, m,
                                 None if symmetric else B.ctypes.data,
                                 None if symmetric else bcB.ctypes.data, n, K, int(S),
                                 int(symmetric), out.ctypes.data, None)
    return rc, out


@pytest.mark.parametrize("m,n,N,sym", [
    (2048, 2048, 4096, True),    # the all-pairs workload
    (3000, 3000, 4096, True),    # several output bands through the scratch
    (700, 450, 9000, False),     # two regions (K = 141: rows padded on the device)
    (1500, 1500, 2049, True),    # single region, K = 33
])
def test_noalloc_matches_regular_entry_point_twice(m, n, N, sym):
    lib = _lib()
    t, _ = synth.all_pairs_workload(m=m + (0 if sym else n), n=N, seed=m + 3 * n)
    T = t.numpy().view(np.uint64)
    A = np.ascontiguousarray(T[:m])
    B = None if sym else np.ascontiguousarray(T[m:])
    bcA = oracle.bitcounts(A)
    bcB = bcA if sym else oracle.bitcounts(B)
    with api.Context(0) as ctx:
        ctx.set_option(api.OPT_R2_MODE, api.R2_EXACT)
        want = ctx.ld(A, bcA, B, bcB, S=N, symmetric=sym)
    mask = lower_mask(n, m) if sym else None
    for _ in range(2):
        rc, got = _noalloc(lib, A, bcA, B, bcB, N, sym)
        assert rc == api.OK
        assert_r2_close(got, want.astype(np.float64), mask=mask)


def test_noalloc_rejects_tasks_beyond_its_scratch():
    lib = _lib()
    m, N = 20_000, 16_622          # 20,000 x 260 words = 41.6 MB of table > 16 MiB
    A = np.zeros((m, (N + 63) // 64), np.uint64)
    bc = np.zeros(m, np.uint32)
    out = np.zeros((1, 1), np.float32)
    rc = lib.qld_cuda_ld_noalloc(A.ctypes.data, bc.ctypes.data, m, None, None, m, A.shape[1], N,
                                 1, out.ctypes.data, None)
    assert rc == ERR_TOO_LARGE
