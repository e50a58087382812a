"""GPU parity of the counts kernels + fused r^2 epilogue against the oracle
and the reference's golden vectors, through the C ABI.

Bars: counts bit-exact; r^2 in QLD_R2_REFERENCE mode bit-identical to the
reference's get_pairwise_ld_score(); r^2 in QLD_R2_EXACT mode within 1e-6
relative of the FP64 oracle (special values exact).
"""
import numpy as np
import pytest
import torch

import oracle
from conftest import assert_r2_close, golden_names, load_golden, lower_mask
from qld_b200 import api, synth

pytestmark = pytest.mark.gpu

KERNELS = ["popc", "mma128", "mma256", "fp4", "fp4pair"]


def set_kernel(ctx, name):
    """fp4: the 4-bit kernel on one SM per tile; fp4pair: on a cluster of two."""
    ctx.set_option(api.OPT_KERNEL, {"popc": api.KERNEL_POPC, "mma128": api.KERNEL_MMA,
                                    "mma256": api.KERNEL_MMA, "fp4": api.KERNEL_FP4,
                                    "fp4pair": api.KERNEL_FP4}[name])
    ctx.set_option(api.OPT_MMA_TILE, {"mma128": 128, "mma256": 256}.get(name, 0))
    ctx.set_option(api.OPT_SM_PAIR, {"fp4": 1, "fp4pair": 2}.get(name, 0))
    assert ctx.stats(reset=True) is not None


def _check_task(ctx, A, B, S, symmetric, kernel):
    set_kernel(ctx, kernel)
    bcA = oracle.bitcounts(A)
    Bx = A if symmetric else B
    bcB = oracle.bitcounts(Bx)
    want_c = oracle.counts(A, Bx)
    mask = lower_mask(*want_c.shape) if symmetric else None
    sel = (lambda x: x[mask]) if symmetric else (lambda x: x)

    ctx.set_option(api.OPT_R2_MODE, api.R2_EXACT)
    r2, cnt = ctx.ld(A, bcA, None if symmetric else B, None if symmetric else bcB, S=S,
                     symmetric=symmetric, counts=True)
    assert np.array_equal(sel(cnt), sel(want_c)), "counts differ"
    want64 = oracle.r2_exact(bcA, bcB, want_c, S)
    err = assert_r2_close(r2, want64, mask=mask)

    ctx.set_option(api.OPT_R2_MODE, api.R2_REFERENCE)
    r2r = ctx.ld(A, bcA, None if symmetric else B, None if symmetric else bcB, S=S,
                 symmetric=symmetric)
    want_ref = oracle.r2_reference(bcA, bcB, want_c, S, fma_contract=False)
    assert np.array_equal(sel(r2r).view(np.uint32), sel(want_ref).view(np.uint32)), \
        "reference-mode r2 not bit-identical"
    ctx.set_option(api.OPT_R2_MODE, api.R2_EXACT)
    return err


SHAPES = [
    # m, n, samples, symmetric
    (1, 1, 1, False),
    (5, 3, 64, False),
    (129, 77, 450, False),
    (300, 200, 1000, False),
    (257, 257, 16622, True),
    (1000, 1000, 4096, True),
    (640, 1300, 130, False),
    (130, 130, 2049, True),
    (2048, 2048, 4096, True),       # the all-pairs workload's size
]


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("m,n,N,sym", SHAPES)
def test_random_shapes(gpu_ctx, kernel, m, n, N, sym):
    t, _ = synth.all_pairs_workload(m=m + (0 if sym else n), n=N, seed=m * 7 + n)
    T = t.numpy().view(np.uint64)
    A = T[:m]
    B = None if sym else T[m:]
    _check_task(gpu_ctx, A, B, N, sym, kernel)


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("name", golden_names())
def test_golden(gpu_ctx, kernel, name):
    g = load_golden(name)
    set_kernel(gpu_ctx, kernel)
    sym = g["symmetric"]
    mask = lower_mask(*g["counts"].shape) if sym else np.ones(g["counts"].shape, bool)
    gpu_ctx.set_option(api.OPT_R2_MODE, api.R2_REFERENCE)
    r2, cnt = gpu_ctx.ld(g["A"], g["bcA"], None if sym else g["B"], None if sym else g["bcB"],
                         S=g["S"], symmetric=sym, counts=True)
    gpu_ctx.set_option(api.OPT_R2_MODE, api.R2_EXACT)
    assert np.array_equal(cnt[mask], g["counts"][mask])
    assert np.array_equal(r2[mask].view(np.uint32), g["r2_ref"][mask].view(np.uint32))
    # the report written from the GPU results is the reference's, byte for byte
    if sym:
        r2 = np.where(mask, r2, g["r2_ref"])
    rep = oracle.write_results(g["posA"], g["idA"], g["bcA"], g["posB"], g["idB"], g["bcB"],
                               g["S"], r2, g["r2limit"], 0 if sym else 1)
    assert rep == g["report"]


@pytest.mark.parametrize("kernel", KERNELS)
def test_device_resident_call(gpu_ctx, kernel):
    """qld_cuda_ld_device on torch buffers with padded pitches."""
    set_kernel(gpu_ctx, kernel)
    m, n, N = 700, 300, 3000
    t, _ = synth.all_pairs_workload(m=m + n, n=N, seed=4)
    K = t.shape[1]
    lda = K + 6 + (K & 1)   # even pitch (16-byte aligned rows), padded
    dev = torch.device("cuda", 0)
    At = torch.zeros(m, lda, dtype=torch.int64, device=dev)
    Bt = torch.zeros(n, lda, dtype=torch.int64, device=dev)
    At[:, :K] = t[:m].to(dev)
    Bt[:, :K] = t[m:].to(dev)
    At[:, K:] = -1   # words past K must never be read
    Bt[:, K:] = -1
    A = t[:m].numpy().view(np.uint64)
    B = t[m:].numpy().view(np.uint64)
    bcA = torch.from_numpy(oracle.bitcounts(A).view(np.int32)).to(dev)
    bcB = torch.from_numpy(oracle.bitcounts(B).view(np.int32)).to(dev)
    ldr = m + 13
    r2 = torch.full((n, ldr), -7.0, dtype=torch.float32, device=dev)
    cnt = torch.zeros((n, ldr), dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream()
    gpu_ctx.ld_device(At, bcA, m, lda, Bt, bcB, n, lda, K, N, False, r2, ldr, cnt, ldr, stream=st)
    gpu_ctx.sync(stream=st)
    want_c = oracle.counts(A, B)
    got_c = cnt[:, :m].cpu().numpy().view(np.uint32)
    assert np.array_equal(got_c, want_c)
    assert torch.all(r2[:, m:] == -7.0), "wrote past m in a padded row"
    assert_r2_close(r2[:, :m].cpu().numpy(), oracle.r2_exact(oracle.bitcounts(A), oracle.bitcounts(B), want_c, N))


@pytest.mark.parametrize("kernel", KERNELS)
def test_streamed_bands(gpu_ctx, kernel):
    """Host-buffer call with several output bands (band rows < n)."""
    set_kernel(gpu_ctx, kernel)
    gpu_ctx.set_option(api.OPT_BAND_ROWS, 256)
    try:
        T1 = synth.all_pairs_workload(m=1100, n=1500, seed=9)[0].numpy().view(np.uint64)
        err = _check_task(gpu_ctx, T1, None, 1500, True, kernel)
        t, _ = synth.all_pairs_workload(m=1700, n=777, seed=10)
        T = t.numpy().view(np.uint64)
        _check_task(gpu_ctx, T[:600], T[600:], 777, False, kernel)
    finally:
        gpu_ctx.set_option(api.OPT_BAND_ROWS, 4096)
    assert err[0] <= 1e-6


def test_pinned_buffers(gpu_ctx):
    set_kernel(gpu_ctx, "mma128")
    m, N = 900, 5000
    t, _ = synth.all_pairs_workload(m=m, n=N, seed=21)
    A = gpu_ctx.pinned_empty(t.shape, np.uint64)
    A[:] = t.numpy().view(np.uint64)
    bc = gpu_ctx.pinned_empty((m,), np.uint32)
    bc[:] = oracle.bitcounts(A)
    out = gpu_ctx.pinned_empty((m, m), np.float32)
    gpu_ctx.ld(A, bc, S=N, r2_out=out)
    want = oracle.r2_exact(bc, bc, oracle.counts(A), N)
    assert_r2_close(out, want, mask=lower_mask(m, m))


def test_invalid_arguments_return_codes(gpu_ctx):
    A = np.zeros((4, 2), np.uint64)
    bc = np.zeros(4, np.uint32)
    with pytest.raises(api.QldError) as e:
        gpu_ctx.ld(A, bc, S=0)
    assert e.value.code == api.ERR_INVALID
    with pytest.raises(api.QldError) as e:
        gpu_ctx.set_option(api.OPT_KERNEL, 99)
    assert e.value.code == api.ERR_INVALID
    with pytest.raises(api.QldError) as e:
        gpu_ctx.set_option(api.OPT_MMA_TILE, 64)
    assert e.value.code == api.ERR_INVALID


def test_tensor_core_limits(gpu_ctx):
    """Each tensor-core kernel refuses tasks past its exact range with
    UNSUPPORTED; AUTO takes the 4-bit kernel up to 2^24 samples and the
    popcount kernel beyond."""
    gpu_ctx.set_option(api.OPT_MMA_TILE, 0)
    try:
        N = 131_200                          # past the i8 kernels' 131,071
        t, _ = synth.all_pairs_workload(m=40, n=N, seed=31)
        A = t.numpy().view(np.uint64)
        bc = oracle.bitcounts(A)
        gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_AUTO)
        gpu_ctx.stats(reset=True)
        r2, cnt = gpu_ctx.ld(A, bc, S=N, counts=True)
        assert gpu_ctx.stats().last_kernel == api.KERNEL_FP4
        mask = lower_mask(40, 40)
        assert np.array_equal(cnt[mask], oracle.counts(A)[mask])
        gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_MMA)
        with pytest.raises(api.QldError) as e:
            gpu_ctx.ld(A, bc, S=N)
        assert e.value.code == api.ERR_UNSUPPORTED
        # past 2^24 samples: the F32 accumulators would round
        K = (1 << 24) // 64 + 1
        rng = np.random.default_rng(32)
        A = rng.integers(0, 2**63, size=(20, K), dtype=np.uint64)
        bc = oracle.bitcounts(A)
        gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_AUTO)
        gpu_ctx.stats(reset=True)
        r2, cnt = gpu_ctx.ld(A, bc, S=K * 64, counts=True)
        assert gpu_ctx.stats().last_kernel == api.KERNEL_POPC
        mask = lower_mask(20, 20)
        assert np.array_equal(cnt[mask], oracle.counts(A)[mask])
        gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_FP4)
        with pytest.raises(api.QldError) as e:
            gpu_ctx.ld(A, bc, S=K * 64)
        assert e.value.code == api.ERR_UNSUPPORTED
    finally:
        gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_AUTO)


def test_fp4_past_the_int8_limit(gpu_ctx):
    """The 4-bit kernel's F32 accumulators stay exact far past the i8
    kernels' 131,071-sample limit (up to 2^24): 200,000 samples here."""
    N = 200_000
    t, _ = synth.all_pairs_workload(m=300, n=N, seed=33)
    A = t.numpy().view(np.uint64)
    bc = oracle.bitcounts(A)
    want = oracle.counts(A[:130], A[130:])
    try:
        for name in ("fp4", "fp4pair"):
            set_kernel(gpu_ctx, name)
            r2, cnt = gpu_ctx.ld(A[:130], bc[:130], A[130:], bc[130:], S=N, counts=True)
            assert np.array_equal(cnt, want), name
            assert_r2_close(r2, oracle.r2_exact(bc[:130], bc[130:], want, N))
            assert gpu_ctx.stats().last_kernel == api.KERNEL_FP4
    finally:
        gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_AUTO)
        gpu_ctx.set_option(api.OPT_SM_PAIR, 0)


# (count, bcA, bcB) with S = 1000 whose FP64 r^2 lies around the 1.0001
# sentinel threshold: bit counts that do not match the rows (a caller's error
# the reference does not check) are the only way past r^2 = 1.
THRESHOLD_CASES = [
    (297, 299, 295),   # 1.0000918: kept (the 4-bit kernels re-evaluate in FP64)
    (666, 624, 718),   # 1.0000909: kept
    (512, 409, 702),   # 1.0001041: 123.456
    (628, 745, 552),   # 1.0001030: 123.456
    (476, 817, 779),   # 1.0000890: kept
    (501, 850, 767),   # 1.0000110
    (297, 470, 920),   # 0.9999673
    (900, 100, 100),   # far above: 123.456
    (300, 1000, 250),  # cA = S, D != 0: inf -> 123.456
    (250, 1000, 250),  # cA = S, D = 0: NaN
    (10, 0, 250),      # cA = 0: 0
]


@pytest.mark.parametrize("kernel", KERNELS)
def test_threshold_with_inconsistent_bitcounts(gpu_ctx, kernel):
    """Every kernel classifies r^2 against the 1.0001 sentinel exactly as the
    FP64 oracle does, including the 4-bit kernels' FP32 evaluation."""
    S, K = 1000, 16
    n = len(THRESHOLD_CASES)
    bits = np.zeros((n, K * 64), np.uint8)
    for i, (c, _, _) in enumerate(THRESHOLD_CASES):
        bits[i, :c] = 1
    rows = np.packbits(bits, axis=1).reshape(n, K, 8)
    rows = rows.view(">u8").reshape(n, K).astype(np.uint64)   # bit 0 = MSB of word 0
    bcA = np.array([t[1] for t in THRESHOLD_CASES], np.uint32)
    bcB = np.array([t[2] for t in THRESHOLD_CASES], np.uint32)
    set_kernel(gpu_ctx, kernel)
    try:
        r2, cnt = gpu_ctx.ld(rows, bcA, rows.copy(), bcB, S=S, counts=True)
    finally:
        gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_AUTO)
        gpu_ctx.set_option(api.OPT_SM_PAIR, 0)
    want_c = oracle.counts(rows, rows)
    assert np.array_equal(cnt, want_c)
    want = oracle.r2_exact(bcA, bcB, want_c, S)
    d = np.diag(want)
    assert (d == 123.456).sum() == 4 and np.isnan(d).sum() == 1 and (d == 0).sum() == 1
    assert_r2_close(r2, want)


@pytest.mark.parametrize("kernel", KERNELS)
def test_reference_mode_edge_pairs_bit_identical(gpu_ctx, kernel):
    """Reference-mode r^2 bit for bit against the reference's operation
    sequence on the pairs its special cases and the kernels' rounding tests
    single out: the sentinel threshold, fixed SNPs (x/0 -> 123.456 and 0/0 ->
    the reference build's NaN), monomorphic SNPs, and a small sample count
    (S = 50) whose simple fractions often sit near FP32 rounding midpoints."""
    S, K = 1000, 16
    # plus bit counts above S: den is -0 (x / -0 = -inf, kept) or negative
    cases = THRESHOLD_CASES + [(250, 1010, 1000), (600, 1020, 990)]
    n = len(cases)
    bits = np.zeros((n, K * 64), np.uint8)
    for i, (c, _, _) in enumerate(cases):
        bits[i, :c] = 1
    rows = np.packbits(bits, axis=1).reshape(n, K, 8).view(">u8").reshape(n, K)
    rows = rows.astype(np.uint64)
    bcA = np.array([t[1] for t in cases], np.uint32)
    bcB = np.array([t[2] for t in cases], np.uint32)
    rng = np.random.default_rng(7)
    S2 = 50
    small = np.zeros((300, 64), np.uint8)
    for i in range(300):
        small[i, :S2] = rng.random(S2) < rng.uniform(0.0, 1.0)
    small[0, :S2] = 1            # fixed SNP
    small[1, :] = 0              # monomorphic
    srows = np.packbits(small, axis=1).reshape(300, 1, 8).view(">u8").reshape(300, 1)
    srows = srows.astype(np.uint64)
    sbc = oracle.bitcounts(srows)
    set_kernel(gpu_ctx, kernel)
    gpu_ctx.set_option(api.OPT_R2_MODE, api.R2_REFERENCE)
    try:
        r2 = gpu_ctx.ld(rows, bcA, rows.copy(), bcB, S=S)
        r2s = gpu_ctx.ld(srows, sbc, S=S2)
    finally:
        gpu_ctx.set_option(api.OPT_R2_MODE, api.R2_EXACT)
        gpu_ctx.set_option(api.OPT_KERNEL, api.KERNEL_AUTO)
        gpu_ctx.set_option(api.OPT_SM_PAIR, 0)
    want = oracle.r2_reference(bcA, bcB, oracle.counts(rows, rows), S, fma_contract=False)
    assert np.isnan(np.diag(want)).sum() == 1 and np.isneginf(want).any()
    assert np.array_equal(r2.view(np.uint32), want.view(np.uint32))
    wants = oracle.r2_reference(sbc, sbc, oracle.counts(srows), S2, fma_contract=False)
    mask = lower_mask(300, 300)
    assert np.isnan(wants[mask]).any()
    assert np.array_equal(r2s[mask].view(np.uint32), wants[mask].view(np.uint32))
