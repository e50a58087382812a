"""GPU test of qld_cuda_ld_noalloc(), the entry point for callers that cannot
allocate device memory (their GPU memory is owned by another component).

It is checked through the C ABI against the oracle (counts from
oracle.counts, r^2 from oracle.r2_exact: within the suite's tolerance of
1e-6 relative, special values exact) and against the regular entry point,
qld_cuda_ld(), on the same inputs.  Every call reuses the same static
scratch array, so each task is run twice with a call on a different task
(other m, K and S, odd K so the r^2 band area serves as the staging area)
in between: the second call must not depend on what the previous call left
there.  The cases cover several output bands for one and two regions, and
an odd-K table too large for the band area, which goes up row by row.  The
file is named to be collected last.
"""
import ctypes as ct

import numpy as np
import pytest

import oracle
from conftest import assert_r2_close, lower_mask
from qld_b200 import api, synth

pytestmark = pytest.mark.gpu

ERR_TOO_LARGE = -8
SCRATCH = 16 << 20


def _lib():
    lib = api.load_library()
    vp, i = ct.c_void_p, ct.c_int
    lib.qld_cuda_ld_noalloc.argtypes = [vp, vp, i, vp, vp, i, i, i, i, vp, vp]
    lib.qld_cuda_ld_noalloc.restype = i
    return lib


def _task(m, n, N, sym, seed):
    t, _ = synth.all_pairs_workload(m=m + (0 if sym else n), n=N, seed=seed)
    T = t.numpy().view(np.uint64)
    A = np.ascontiguousarray(T[:m])
    B = A if sym else np.ascontiguousarray(T[m:])
    bcA = oracle.bitcounts(A)
    bcB = bcA if sym else oracle.bitcounts(B)
    want = oracle.r2_exact(bcA, bcB, oracle.counts(A, None if sym else B), N)
    return dict(A=A, B=B, bcA=bcA, bcB=bcB, m=m, n=n, N=N, sym=sym, want=want,
                mask=lower_mask(n, m) if sym else None)


def _noalloc(lib, t):
    m, K = t["A"].shape
    out = np.full((t["n"], m), np.nan, np.float32)
    rc = lib.qld_cuda_ld_noalloc(t["A"].ctypes.data, t["bcA"].ctypes.data, m,
                                 None if t["sym"] else t["B"].ctypes.data,
                                 None if t["sym"] else t["bcB"].ctypes.data, t["n"], K,
                                 int(t["N"]), int(t["sym"]), out.ctypes.data, None)
    return rc, out


def _bands(m, n, N, sym):
    """Output bands the entry point uses for this task (its scratch layout)."""
    K = (N + 63) // 64
    Kp = K + (K & 1)
    a = lambda x: (x + 255) & ~255  # noqa: E731
    off = a(256 + m * 4)
    if not sym:
        off = a(off + n * 4)
    off = a(off + m * Kp * 8)
    if not sym:
        off = a(off + n * Kp * 8)
    fit = (SCRATCH - off) // (m * 4)
    band = n if fit >= n else fit // 256 * 256
    return -(-n // band), SCRATCH - off


@pytest.mark.parametrize("m,n,N,sym", [
    (2048, 2048, 4096, True),    # the all-pairs workload
    (3000, 3000, 4096, True),    # single region, several output bands
    (3000, 2000, 4096, False),   # two regions, several output bands
    (700, 450, 9000, False),     # two regions, K = 141: rows padded on the device
    (4000, 4000, 16_800, True),  # K = 263: table larger than the band area
])
def test_noalloc_matches_oracle_and_regular_entry_point(m, n, N, sym):
    lib = _lib()
    t = _task(m, n, N, sym, seed=m + 3 * n + N)
    other = _task(900, 900, 2049, True, seed=7)        # K = 33, staged through the band area
    with api.Context(0) as ctx:
        ctx.set_option(api.OPT_R2_MODE, api.R2_EXACT)
        regular = ctx.ld(t["A"], t["bcA"], None if sym else t["B"], None if sym else t["bcB"],
                         S=N, symmetric=sym)
    assert_r2_close(regular, t["want"], mask=t["mask"])
    for _ in range(2):
        rc, got = _noalloc(lib, t)
        assert rc == api.OK
        assert_r2_close(got, t["want"], mask=t["mask"])
        assert_r2_close(got, regular, mask=t["mask"])
        rc, got_other = _noalloc(lib, other)
        assert rc == api.OK
        assert_r2_close(got_other, other["want"], mask=other["mask"])


def test_case_shapes_reach_the_paths_they_name():
    """The parameters above reach what their comments say (scratch layout
    restated): several bands, and a table past the band area."""
    assert _bands(3000, 3000, 4096, True)[0] > 1
    assert _bands(3000, 2000, 4096, False)[0] > 1
    bands, area = _bands(4000, 4000, 16_800, True)
    assert bands > 1 and 4000 * 263 * 8 > area


def test_noalloc_rejects_tasks_beyond_its_scratch():
    lib = _lib()
    m, N = 20_000, 16_622          # 20,000 x 260 words = 41.6 MB of table > 16 MiB
    A = np.zeros((m, (N + 63) // 64), np.uint64)
    bc = np.zeros(m, np.uint32)
    out = np.zeros((1, 1), np.float32)
    rc = lib.qld_cuda_ld_noalloc(A.ctypes.data, bc.ctypes.data, m, None, None, m, A.shape[1], N,
                                 1, out.ctypes.data, None)
    assert rc == ERR_TOO_LARGE
