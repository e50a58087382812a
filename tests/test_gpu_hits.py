"""GPU tests of qld_cuda_ld_hits: the report's pairs filtered on the device
are exactly the dense r^2 array's pairs under qLD's rule (r2limit <= r^2 <
100, j > i for a triangle), bit for bit, over block boundaries and ragged
widths; the callback can stop a task and the context stays usable."""
import numpy as np
import pytest

import oracle
from qld_b200 import api, host_api, synth

pytestmark = pytest.mark.gpu


def _table(m, N, seed):
    f = synth.beta_freqs(m, 0.1, 1.0, seed, clip_min=1.0 / N)
    t = synth.copying_table(m, N, 12, 30, 200, 0.01, f, seed)
    A = t.numpy().view(np.uint64)
    return A, oracle.bitcounts(A)


def _want(ctx, A, bcA, B, bcB, N, lim, symmetric, triangle):
    r2 = ctx.ld(A, bcA, None if symmetric else B, None if symmetric else bcB, S=N,
                symmetric=symmetric)
    return host_api.hits_from_dense(r2, lim, triangle)


@pytest.mark.parametrize("mode", [api.R2_EXACT, api.R2_REFERENCE])
@pytest.mark.parametrize("lim", [0.0, 0.05, 0.4, 2.0])
@pytest.mark.parametrize("form", ["single", "two", "split"])
def test_hits_equal_dense(gpu_ctx, mode, lim, form):
    gpu_ctx.set_option(api.OPT_R2_MODE, mode)
    gpu_ctx.set_option(api.OPT_BAND_ROWS, 256)          # several blocks
    try:
        N = 1500
        T, bc = _table(1400, N, 17)
        if form == "single":
            A, bcA, B, bcB, sym, tri = T[:1000], bc[:1000], None, None, True, True
        else:
            A, bcA, B, bcB = T[:700], bc[:700], T[100:1400], bc[100:1400]
            sym, tri = False, form == "split"
        got = gpu_ctx.ld_hits(A, bcA, B, bcB, S=N, r2limit=lim, symmetric=sym, triangle=tri)
        want = _want(gpu_ctx, A, bcA, B, bcB, N, lim, sym, tri)
        assert np.array_equal(got[0], want[0]), "mask differs"
        assert np.array_equal(got[1], want[1]), "row offsets differ"
        assert np.array_equal(got[2].view(np.uint32), want[2].view(np.uint32)), "values differ"
    finally:
        gpu_ctx.set_option(api.OPT_BAND_ROWS, 4096)
        gpu_ctx.set_option(api.OPT_R2_MODE, api.R2_EXACT)


@pytest.mark.parametrize("m,n", [(1, 1), (33, 5), (129, 300), (257, 1), (640, 1025)])
@pytest.mark.parametrize("kernel", [api.KERNEL_POPC, api.KERNEL_MMA, api.KERNEL_FP4])
def test_hits_ragged_shapes(gpu_ctx, m, n, kernel):
    gpu_ctx.set_option(api.OPT_KERNEL, kernel)
    try:
        N = 700
        T, bc = _table(m + n, N, 23)
        A, bcA, B, bcB = T[:m], bc[:m], T[m:], bc[m:]
        for tri in (False, True):
            got = gpu_ctx.ld_hits(A, bcA, B, bcB, S=N, r2limit=0.01, symmetric=False,
                                  triangle=tri)
            want = _want(gpu_ctx, A, bcA, B, bcB, N, 0.01, False, tri)
            assert np.array_equal(got[0], want[0])
            assert np.array_equal(got[1], want[1])
            assert np.array_equal(got[2].view(np.uint32), want[2].view(np.uint32))
        got = gpu_ctx.ld_hits(A, bcA, S=N, r2limit=0.0)
        want = _want(gpu_ctx, A, bcA, None, None, N, 0.0, True, True)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[2], want[2])
    finally:
        gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_AUTO)


def test_hits_values_against_oracle(gpu_ctx):
    N = 2000
    T, bc = _table(900, N, 29)
    mask, off, val = gpu_ctx.ld_hits(T, bc, S=N, r2limit=0.02)
    e = oracle.r2_exact(bc, bc, oracle.counts(T), N)
    keep = (e >= 0.02) & (e < 100) & (np.arange(900)[None, :] > np.arange(900)[:, None])
    # entries within one FP32 ulp of the limit may fall either side
    near = np.abs(e - 0.02) <= 2e-6 * 0.02
    bits = np.unpackbits(mask.view(np.uint8), bitorder="little").reshape(900, -1)[:, :900]
    assert np.all(bits[~near] == keep[~near])
    rel = np.abs(val.astype(np.float64) - e[bits.astype(bool)]) / e[bits.astype(bool)]
    assert rel.max() <= 1e-6


def test_callback_stops_and_context_recovers(gpu_ctx):
    gpu_ctx.set_option(api.OPT_BAND_ROWS, 256)
    try:
        N = 1000
        T, bc = _table(1200, N, 31)
        seen = []

        def stop_second(b):
            seen.append((b.row0, b.rows))
            return 7 if len(seen) == 2 else 0

        rc = gpu_ctx.ld_hits(T, bc, S=N, r2limit=0.1, on_block=stop_second)
        # blocks are QLD_OPT_BAND_ROWS rounded down to whole tile rows of the
        # kernel (256, or 240 for the 4-bit kernel)
        rows = seen[0][1]
        assert rc == 7 and rows in (240, 256) and seen == [(0, rows), (rows, rows)]
        got = gpu_ctx.ld_hits(T, bc, S=N, r2limit=0.1)
        want = _want(gpu_ctx, T, bc, None, None, N, 0.1, True, True)
        assert np.array_equal(got[2], want[2])
        st = gpu_ctx.stats(reset=True)
        assert st.hits_rows >= 1200 and st.hits_pairs >= len(want[2])
    finally:
        gpu_ctx.set_option(api.OPT_BAND_ROWS, 4096)


def test_hits_report_equals_dense_report(gpu_ctx, tmp_path):
    """Device-filtered blocks through the streamed writer give the dense
    writer's report bytes (reference-semantics r^2)."""
    gpu_ctx.set_option(api.OPT_R2_MODE, api.R2_REFERENCE)
    gpu_ctx.set_option(api.OPT_BAND_ROWS, 512)
    try:
        N = 2500
        T, bc = _table(1800, N, 37)
        pos = (1000 + 10 * np.arange(1800)).astype(np.uint32)
        tab = host_api.Table(T, bc, pos, [f"rs{i}" for i in range(1800)])
        blocks = []

        def keep(b):
            rows, W = b.rows, b.words
            mk = np.ctypeslib.as_array(b.mask, (rows * W,)).reshape(rows, W).copy()
            of = np.ctypeslib.as_array(b.row_off, (rows + 1,)).copy()
            tot = int(of[rows])
            v = np.ctypeslib.as_array(b.val, (tot,)).copy() if tot else np.zeros(0, np.float32)
            blocks.append((b.row0, mk, of, v))
            return 0

        assert gpu_ctx.ld_hits(T, bc, S=N, r2limit=0.01, on_block=keep) == 0
        hits = tmp_path / "hits.txt"
        host_api.write_report_hits(str(hits), tab, tab, blocks, N, threads=4)
        r2 = gpu_ctx.ld(T, bc, S=N)
        dense = tmp_path / "dense.txt"
        host_api.write_report(str(dense), tab, tab, r2, N, 0.01, True, threads=4)
        assert hits.read_bytes() == dense.read_bytes()
        assert hits.read_bytes().count(b"\n") > 1000
    finally:
        gpu_ctx.set_option(api.OPT_BAND_ROWS, 4096)
        gpu_ctx.set_option(api.OPT_R2_MODE, api.R2_EXACT)
