"""CPU tests: the oracle against the reference's golden vectors (and against
the reference library itself when it is built)."""
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, golden_names, load_golden, lower_mask


@pytest.mark.parametrize("name", golden_names())
def test_counts_match_golden(name):
    g = load_golden(name)
    C = oracle.counts(g["A"], g["B"])
    assert np.array_equal(C, g["counts"])


@pytest.mark.parametrize("name", golden_names())
def test_bitcounts_match_golden(name):
    g = load_golden(name)
    assert np.array_equal(oracle.bitcounts(g["A"]), g["bcA"])


@pytest.mark.parametrize("name", golden_names())
def test_r2_reference_semantics_bit_exact(name):
    g = load_golden(name)
    r = oracle.r2_reference(g["bcA"], g["bcB"], g["counts"], g["S"], fma_contract=False)
    assert np.array_equal(r.view(np.uint32), g["r2_ref"].view(np.uint32))


@pytest.mark.parametrize("name", golden_names())
def test_report_bytes_match_golden(name):
    g = load_golden(name)
    rep = oracle.write_results(g["posA"], g["idA"], g["bcA"], g["posB"], g["idB"], g["bcB"],
                               g["S"], g["r2_ref"], g["r2limit"], 0 if g["symmetric"] else 1)
    assert rep == g["report"]


@pytest.mark.parametrize("name", golden_names())
def test_exact_oracle_agrees_where_reference_is_well_conditioned(name):
    """The FP64 oracle and the reference agree to float precision wherever the
    reference's FP32 numerator does not cancel (r^2 > 1e-2)."""
    g = load_golden(name)
    e = oracle.r2_exact(g["bcA"], g["bcB"], g["counts"], g["S"])
    r = g["r2_ref"].astype(np.float64)
    sel = np.isfinite(e) & (e > 1e-2) & (e < 100)
    if g["symmetric"]:
        sel &= lower_mask(*e.shape)
    if sel.any():
        rel = np.abs(r[sel] - e[sel]) / e[sel]
        assert rel.max() < 1e-3


def test_fprint_f_truncates_like_reference():
    assert oracle.fprint_f(0.0) == "0."
    assert oracle.fprint_f(1.0) == "1."
    assert oracle.fprint_f(0.5) == "0.500000000"
    assert oracle.fprint_f(0.25) == "0.250000000"
    # float32(0.1) * 1e9 in float -> 100000000 exactly -> "0.100000000"
    assert oracle.fprint_f(0.1) == "0.100000000"
    # float32(1/3) * 1e9 rounds to 333333344 in float before truncation
    assert oracle.fprint_f(1.0 / 3.0) == "0.333333344"
    assert oracle.fprint_f(123.456).startswith("123.")


def test_symmetric_counts_lower_triangle():
    rng = np.random.default_rng(3)
    A = rng.integers(0, 2**63, size=(40, 5), dtype=np.uint64)
    full = oracle.counts(A)
    low = oracle.counts(A, lower_only=True)
    mask = lower_mask(40, 40)
    assert np.array_equal(full[mask], low[mask])
    assert np.all(low[~mask] == 0)
    assert np.array_equal(full, full.T)


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_restatement_matches_reference_library_random():
    rng = np.random.default_rng(5)
    for (m, n, K) in [(1, 1, 1), (17, 9, 3), (150, 131, 7)]:
        A = rng.integers(0, 2**64 - 1, size=(m, K), dtype=np.uint64)
        B = rng.integers(0, 2**64 - 1, size=(n, K), dtype=np.uint64)
        C = oracle.counts(A, B)
        assert np.array_equal(C.astype(np.uint64), oracle.ref_counts_gemm(A, B))
        assert np.array_equal(C.astype(np.uint64), oracle.ref_counts_ukr(A, B, threads=2))
        S = 64 * K
        bcA, bcB = oracle.bitcounts(A), oracle.bitcounts(B)
        r_ref = oracle.ref_ld_score(bcA, bcB, C.astype(np.uint64), S)
        r_me = oracle.r2_reference(bcA, bcB, C, S, fma_contract=False)
        assert np.array_equal(r_ref.view(np.uint32), r_me.view(np.uint32))


def _states_cases():
    d = os.path.join(GOLDEN, "states")
    return sorted(f[:-4] for f in os.listdir(d) if f.endswith(".npz")) if os.path.isdir(d) else []


def load_states_golden(name):
    """A COUNTSTATES golden case: the table, its A/B windows (rows by
    position, as qLD's window rule keeps them) and the reference's report."""
    z = np.load(os.path.join(GOLDEN, "states", f"{name}.npz"))
    flags = [str(f) for f in z["flags"]]
    t, pos = z["table"], z["positions"]
    win = dict(zip(flags[::2], (int(v) for v in flags[1::2])))
    single = "-posWmin2" not in win
    lo1, hi1 = win.get("-posWmin1", int(pos[0])), win.get("-posWmax1", int(pos[-1]))
    a = (pos >= lo1) & (pos <= hi1)
    b = a if single else (pos >= win["-posWmin2"]) & (pos <= win["-posWmax2"])
    ids = np.array([f"rs{i + 1}" for i in range(len(pos))])
    with open(os.path.join(GOLDEN, "states", f"{name}.report.txt"), "rb") as f:
        report = f.read()
    return dict(z=z, flags=flags, single=single, A=t[a], posA=pos[a], idA=list(ids[a]),
                B=t[b], posB=pos[b], idB=list(ids[b]), report=report)


@pytest.mark.parametrize("name", _states_cases())
def test_count_states_report_matches_golden(name):
    g = load_states_golden(name)
    st = oracle.count_states(g["A"], g["B"])
    rep = oracle.write_states(g["posA"], g["idA"], g["posB"], g["idB"], st,
                              0 if g["single"] else 1)
    assert rep == g["report"]


def test_count_states_small_python_restatement():
    """The C loop against a literal Python transcription on a small case."""
    rng = np.random.default_rng(5)
    A = rng.integers(0, 2**63, (6, 2), dtype=np.uint64)
    A[0] = 0
    A[1, 1] = 0
    B = rng.integers(0, 2**63, (4, 2), dtype=np.uint64) & np.uint64(0xF0F0F0F0F0F0F0F0)

    def states(a, b):
        s = 0
        for k in range(len(a)):
            for p in range(64):
                if s == 15:
                    break
                s |= 1 << (((int(a[k]) >> p) & 1) * 2 + ((int(b[k]) >> p) & 1))
            s = bin(s).count("1")
        return s

    want = np.array([[states(A[j], B[i]) for j in range(6)] for i in range(4)], np.uint8)
    assert np.array_equal(oracle.count_states(A, B), want)


@pytest.mark.skipif(not oracle.blis_available(), reason="BLIS build of the reference absent")
@pytest.mark.parametrize("m,n,N", [(700, None, 4096), (513, 300, 1000), (257, None, 130)])
def test_stock_blis_path_matches_the_oracle(m, n, N):
    """The reference's -blis path (BLIS dsyrk / dgemm with bin_gemm_2x2, then
    get_pairwise_ld_score) as the CPU baseline times it: counts equal the
    restatement's (SYRK fills the lower triangle only), r^2 bit-identical to
    the reference-semantics restatement."""
    rng = np.random.default_rng(m)
    K = (N + 63) // 64
    A = rng.integers(0, 2 ** 63, (m, K), dtype=np.uint64)
    A[:, -1] &= np.uint64(((1 << 64) - 1) ^ ((1 << (K * 64 - N)) - 1))
    bcA = oracle.bitcounts(A)
    if n is None:
        C, R, _, _ = oracle.ref_blis_counts_ld(A, bcA, N)
        want = oracle.counts(A)
        low = np.arange(m)[None, :] >= np.arange(m)[:, None]
        assert np.array_equal(C[low].astype(np.uint32), want[low])
        ref = oracle.r2_reference(bcA, bcA, want, N, fma_contract=False)
        assert np.array_equal(R[low].view(np.uint32), ref[low].view(np.uint32))
    else:
        B = rng.integers(0, 2 ** 63, (n, K), dtype=np.uint64)
        bcB = oracle.bitcounts(B)
        C, R, _, _ = oracle.ref_blis_counts_ld(A, bcA, N, B=B, bcB=bcB)
        want = oracle.counts(A, B)
        assert np.array_equal(C.astype(np.uint32), want)
        ref = oracle.r2_reference(bcA, bcB, want, N, fma_contract=False)
        assert np.array_equal(R.view(np.uint32), ref.view(np.uint32))
