"""CPU oracle for the qLD LD hot path -- TEST INFRASTRUCTURE ONLY.

Thin ctypes/numpy layer over two libraries:

* ``libqld_oracle.so`` -- the C restatement in ``qld_oracle.c`` (counts, the
  reference-semantics r^2, the FP64 r^2 oracle, the text report).
* ``_ref/libqldref.so`` -- the reference's own functions compiled from the qLD
  sources (``gemm()``/``mlt()``/``get_pairwise_ld_score()``/``writeResults()``
  /``correlate()`` and the BLIS ``bin_gemm_2x2`` micro-kernel), see Makefile.
* ``_ref/libqldref_blis.so`` -- the reference's stock ``-blis`` path:
  ``blis_gemm()`` on BLIS 0.1.8 ``binary_gemm`` built from its sources, then
  ``get_pairwise_ld_score()`` (``ref_blis_counts_ld``).

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.  The library under test never does.

Array conventions (as in qLD's gemm_cpu.c): a SNP table is row-major
``(rows, K)`` uint64; counts are column-major m x n, held here as a numpy
``(n, m)`` array so ``counts[b, a]`` is the reference's ``C[a + b*m]``; r^2 is
``(n, m)`` B-major like the reference's ``results[i*m + j]``.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lock = threading.Lock()
_libs: dict[str, ct.CDLL] = {}

_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build_oracle(with_reference: bool = True) -> None:
    """Compile the restatement, and the reference when its sources exist."""
    subprocess.run(["make", "-s", "-C", _HERE, "libqld_oracle.so"], check=True)
    # The qLD source tree: $QLD_REFERENCE, else the Makefile's REF default.
    ref = os.environ.get("QLD_REFERENCE") or subprocess.run(
        ["make", "-s", "--no-print-directory", "-C", _HERE, "ref-dir"], check=True,
        capture_output=True, text=True).stdout.strip()
    if with_reference and ref and os.path.isdir(os.path.join(ref, "src", "correlator")):
        subprocess.run(["make", "-s", f"-j{os.cpu_count() or 1}", "-C", _HERE, f"REF={ref}",
                        "ref"], check=True)


def _lib(name: str) -> ct.CDLL:
    with _lock:
        if name in _libs:
            return _libs[name]
        if name == "oracle":
            path = os.path.join(_HERE, "libqld_oracle.so")
            if not os.path.exists(path):
                subprocess.run(["make", "-s", "-C", _HERE, "libqld_oracle.so"], check=True)
            lib = ct.CDLL(path)
            lib.qo_counts.argtypes = [_u64p, ct.c_int, _u64p, ct.c_int, ct.c_int, ct.c_int, _u32p]
            lib.qo_bitcounts.argtypes = [_u64p, ct.c_int, ct.c_int, _u32p]
            lib.qo_r2_reference.argtypes = [_u32p, ct.c_int, _u32p, ct.c_int, _u32p, ct.c_int,
                                            ct.c_int, _f32p]
            lib.qo_r2_exact.argtypes = [_u32p, ct.c_int, _u32p, ct.c_int, _u32p, ct.c_int,
                                        ct.c_void_p, ct.c_void_p]
            lib.qo_fprint_f.argtypes = [ct.c_char_p, ct.c_size_t, ct.c_float, ct.c_int]
            lib.qo_fprint_f.restype = ct.c_size_t
            lib.qo_write_results.argtypes = [
                ct.c_char_p, ct.c_size_t, ct.c_int,
                _u32p, ct.POINTER(ct.c_char_p), _u32p, ct.c_int,
                _u32p, ct.POINTER(ct.c_char_p), _u32p, ct.c_int, ct.c_int,
                _f32p, ct.c_float, ct.c_int]
            lib.qo_write_results.restype = ct.c_size_t
            lib.qo_count_states.argtypes = [_u64p, ct.c_int, _u64p, ct.c_int, ct.c_int,
                                            ct.c_void_p]
            lib.qo_write_states.argtypes = [
                ct.c_char_p, ct.c_size_t, _u32p, ct.POINTER(ct.c_char_p), ct.c_int,
                _u32p, ct.POINTER(ct.c_char_p), ct.c_int, ct.c_void_p, ct.c_int]
            lib.qo_write_states.restype = ct.c_size_t
            lib.qo_srand.argtypes = [ct.c_uint]
            lib.qo_vcf_pack.argtypes = [ct.c_char_p, ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int,
                                        ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                        ct.c_void_p, ct.POINTER(ct.c_char_p)]
            lib.qo_vcf_pack.restype = ct.c_int
        elif name == "ref":
            path = os.path.join(_HERE, "_ref", "libqldref.so")
            if not os.path.exists(path):
                raise FileNotFoundError(
                    f"{path} is not built (make -C oracle ref needs the qLD sources)")
            lib = ct.CDLL(path)
            lib.ref_counts_gemm.argtypes = [ct.c_int, ct.c_int, ct.c_int, _u64p, _u64p, _u64p]
            lib.ref_counts_ukr.argtypes = [ct.c_int, ct.c_int, ct.c_int, _u64p, _u64p, _u64p,
                                           ct.c_int, ct.c_int]
            lib.ref_ld_score.argtypes = [_u32p, _u32p, _u64p, ct.c_int, ct.c_int, ct.c_int,
                                         ct.c_int, _f32p]
            lib.ref_ld_score_mt.argtypes = [_u32p, _u32p, _u64p, ct.c_int, ct.c_int, ct.c_int,
                                            _f32p, ct.c_int]
            lib.ref_write_report.argtypes = [
                ct.c_char_p, _u32p, ct.POINTER(ct.c_char_p), _u32p, ct.c_int,
                _u32p, ct.POINTER(ct.c_char_p), _u32p, ct.c_int, ct.c_int,
                _f32p, ct.c_float, ct.c_int]
            lib.ref_correlate.argtypes = [
                ct.c_char_p, ct.c_char_p,
                _u64p, _u32p, ct.POINTER(ct.c_char_p), _u32p, ct.c_int,
                _u64p, _u32p, ct.POINTER(ct.c_char_p), _u32p, ct.c_int,
                ct.c_int, ct.c_int, ct.c_int, ct.c_float]
        elif name == "ref_blis":
            lib = ct.CDLL(os.path.join(_HERE, "_ref", "libqldref_blis.so"))
            lib.refb_counts_ld.argtypes = [ct.c_int, ct.c_int, ct.c_int, _u64p, _u64p, _u32p,
                                           _u32p, ct.c_int, ct.c_int, _u64p, _f32p,
                                           ct.c_void_p, ct.c_void_p]
            lib.refb_counts_ld.restype = ct.c_int
        else:
            raise KeyError(name)
        _libs[name] = lib
        return lib


def reference_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libqldref.so"))


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _ids(ids):
    arr = (ct.c_char_p * len(ids))()
    arr[:] = [s.encode() if isinstance(s, str) else s for s in ids]
    return arr


# ------------------------------------------------------------- restatement --

def counts(A, B=None, lower_only=False) -> np.ndarray:
    """Pairwise AND+popcount counts, (n, m) uint32 with [b, a] = C[a + b*m]."""
    A = _c(A, np.uint64)
    B = A if B is None else _c(B, np.uint64)
    m, K = A.shape
    n = B.shape[0]
    out = np.empty((n, m), np.uint32)
    _lib("oracle").qo_counts(A, m, B, n, K, int(lower_only), out)
    return out


def bitcounts(A) -> np.ndarray:
    A = _c(A, np.uint64)
    out = np.empty(A.shape[0], np.uint32)
    _lib("oracle").qo_bitcounts(A, A.shape[0], A.shape[1], out)
    return out


def r2_reference(bcA, bcB, C, S, fma_contract=True) -> np.ndarray:
    bcA, bcB, C = _c(bcA, np.uint32), _c(bcB, np.uint32), _c(C, np.uint32)
    n, m = C.shape
    out = np.empty((n, m), np.float32)
    _lib("oracle").qo_r2_reference(bcA, m, bcB, n, C, int(S), int(fma_contract), out)
    return out


def r2_exact(bcA, bcB, C, S) -> np.ndarray:
    """FP64 r^2 oracle (exact integer D), (n, m) float64."""
    bcA, bcB, C = _c(bcA, np.uint32), _c(bcB, np.uint32), _c(C, np.uint32)
    n, m = C.shape
    out = np.empty((n, m), np.float64)
    _lib("oracle").qo_r2_exact(bcA, m, bcB, n, C, int(S), out.ctypes.data, None)
    return out


def fprint_f(val: float, precision: int = 9) -> str:
    buf = ct.create_string_buffer(64)
    k = _lib("oracle").qo_fprint_f(buf, 64, float(val), precision)
    return buf.raw[:k].decode()


def write_results(posA, idA, bcA, posB, idB, bcB, S, results, r2limit, posWset2,
                  with_header=True) -> bytes:
    posA, bcA = _c(posA, np.uint32), _c(bcA, np.uint32)
    posB, bcB = _c(posB, np.uint32), _c(bcB, np.uint32)
    results = _c(results, np.float32)
    m, n = len(posA), len(posB)
    lib = _lib("oracle")
    ia, ib = _ids(idA), _ids(idB)
    args = (int(with_header), posA, ia, bcA, m, posB, ib, bcB, n, int(S), results,
            float(r2limit), int(posWset2))
    need = lib.qo_write_results(None, 0, *args)
    buf = ct.create_string_buffer(need + 1)
    lib.qo_write_results(buf, need + 1, *args)
    return buf.raw[:need]


def count_states(A, B=None) -> np.ndarray:
    """countStates_mode()'s state counts, (n, m) uint8 (B-major)."""
    A = _c(A, np.uint64)
    B = A if B is None else _c(B, np.uint64)
    m, K = A.shape
    n = B.shape[0]
    out = np.empty((n, m), np.uint8)
    _lib("oracle").qo_count_states(A, m, B, n, K, out.ctypes.data)
    return out


def write_states(posA, idA, posB, idB, states, posWset2) -> bytes:
    """writeStateCount()'s report bytes."""
    posA, posB = _c(posA, np.uint32), _c(posB, np.uint32)
    states = _c(states, np.uint8)
    m, n = len(posA), len(posB)
    lib = _lib("oracle")
    args = (posA, _ids(idA), m, posB, _ids(idB), n, states.ctypes.data, int(posWset2))
    need = lib.qo_write_states(None, 0, *args)
    buf = ct.create_string_buffer(need + 1)
    lib.qo_write_states(buf, need + 1, *args)
    return buf.raw[:need]


VCF_SITE = np.dtype([("off", np.int64), ("len", np.int32), ("gt_pos", np.int32),
                     ("n_states", np.int32), ("states", "S4")], align=True)


def vcf_seed(seed: int) -> None:
    """srand() of the C library the oracle calls rand() from."""
    _lib("oracle").qo_srand(int(seed))


def vcf_pack(text: bytes, sites: np.ndarray, valid, ploidy: int, K: int):
    """qLD-parse-2MDF's per-site processing of `sites` (VCF_SITE records over
    `text`): (words (n, K) uint64, bc, snip_len, keep), or raises ValueError
    naming the first site qLD stops on."""
    sites = np.ascontiguousarray(sites, VCF_SITE)
    valid = np.ascontiguousarray(valid, np.uint8)
    n = len(sites)
    words = np.zeros((max(n, 1), K), np.uint64)
    bc = np.zeros(max(n, 1), np.uint32)
    ln = np.zeros(max(n, 1), np.int32)
    keep = np.zeros(max(n, 1), np.uint8)
    what = ct.c_char_p()
    fail = _lib("oracle").qo_vcf_pack(text, sites.ctypes.data, n, valid.ctypes.data, len(valid),
                                      int(ploidy), int(K), words.ctypes.data, bc.ctypes.data,
                                      ln.ctypes.data, keep.ctypes.data, ct.byref(what))
    if fail >= 0:
        raise ValueError(f"site {fail}: {what.value.decode()}")
    return words[:n], bc[:n], ln[:n], keep[:n]


# --------------------------------------------------------------- reference --

def ref_counts_gemm(A, B=None) -> np.ndarray:
    """The reference's own fallback gemm(): full m x n counts as (n, m) uint64."""
    A = _c(A, np.uint64)
    B = A if B is None else _c(B, np.uint64)
    m, K = A.shape
    n = B.shape[0]
    out = np.empty((n, m), np.uint64)
    if _lib("ref").ref_counts_gemm(m, n, K, A, B, out) != 0:
        raise MemoryError("ref_counts_gemm")
    return out


def ref_counts_ukr(A, B=None, lower_only=False, threads=1) -> np.ndarray:
    """BLIS-style loop around the reference micro-kernel bin_gemm_2x2."""
    A = _c(A, np.uint64)
    B = A if B is None else _c(B, np.uint64)
    m, K = A.shape
    n = B.shape[0]
    out = np.empty((n, m), np.uint64)
    if _lib("ref").ref_counts_ukr(m, n, K, A, B, out, int(lower_only), int(threads)) != 0:
        raise MemoryError("ref_counts_ukr")
    return out


def ref_ld_score(bcA, bcB, C64, S, threads=1) -> np.ndarray:
    """The reference's get_pairwise_ld_score(), (n, m) float32."""
    bcA, bcB, C64 = _c(bcA, np.uint32), _c(bcB, np.uint32), _c(C64, np.uint64)
    n, m = C64.shape
    out = np.empty((n, m), np.float32)
    _lib("ref").ref_ld_score_mt(bcA, bcB, C64, m, n, int(S), out, int(threads))
    return out


def blis_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libqldref_blis.so"))


def ref_blis_counts_ld(A, bc, S, B=None, bcB=None, C=None, results=None):
    """The reference's stock -blis path on one task (ref_blis.c): BLIS
    cblas_dsyrk (single region, lower triangle of C) or cblas_dgemm (two
    regions), then get_pairwise_ld_score() on one thread.  BLIS threading
    comes from BLIS_JC_NT / BLIS_IC_NT / ... in the environment.  Returns
    (counts (n, m) uint64, results (n, m) float32, gemm seconds, ld seconds);
    C / results may be preallocated (n, m) buffers."""
    lib = _lib("ref_blis")
    A = _c(A, np.uint64)
    bc = _c(bc, np.uint32)
    single = B is None
    B = A if single else _c(B, np.uint64)
    bcB = bc if single else _c(bcB, np.uint32)
    m, K = A.shape
    n = B.shape[0]
    C = np.empty((n, m), np.uint64) if C is None else C
    results = np.empty((n, m), np.float32) if results is None else results
    tg, tl = ct.c_double(), ct.c_double()
    lib.refb_counts_ld(m, n, K, A, B, bc, bcB, int(S), 0 if single else 1, C, results,
                       ct.byref(tg), ct.byref(tl))
    return C, results, tg.value, tl.value


def ref_write_report(path, posA, idA, bcA, posB, idB, bcB, S, results, r2limit,
                     posWset2) -> None:
    posA, bcA = _c(posA, np.uint32), _c(bcA, np.uint32)
    posB, bcB = _c(posB, np.uint32), _c(bcB, np.uint32)
    results = _c(results, np.float32)
    rc = _lib("ref").ref_write_report(
        os.fsencode(path), posA, _ids(idA), bcA, len(posA), posB, _ids(idB), bcB,
        len(posB), int(S), results, float(r2limit), int(posWset2))
    if rc != 0:
        raise OSError(f"ref_write_report({path})")


def ref_correlate(out_path, log_path, A, posA, idA, bcA, B, posB, idB, bcB, S,
                  posWset2, r2limit) -> None:
    """The reference's whole correlate() for one task (fallback counts path)."""
    A, B = _c(A, np.uint64), _c(B, np.uint64)
    posA, bcA = _c(posA, np.uint32), _c(bcA, np.uint32)
    posB, bcB = _c(posB, np.uint32), _c(bcB, np.uint32)
    rc = _lib("ref").ref_correlate(
        os.fsencode(out_path), os.fsencode(log_path), A, posA, _ids(idA), bcA, A.shape[0],
        B, posB, _ids(idB), bcB, B.shape[0], A.shape[1], int(S), int(posWset2),
        float(r2limit))
    if rc != 0:
        raise OSError("ref_correlate")


# ------------------------------------------------- sampled checks of large --

def r2_errors(got, want64):
    """Compare FP32 r^2 with the FP64 oracle value by value.  Returns
    (specials_ok, max_rel, mean_rel, compared): NaN, exact zeros and the
    123.456 sentinel must match exactly; the relative error is taken over the
    other values."""
    got = np.asarray(got).astype(np.float64).ravel()
    want = np.asarray(want64).astype(np.float64).ravel()
    nan_w = np.isnan(want)
    ok = bool(np.array_equal(nan_w, np.isnan(got)))
    g, w = got[~nan_w], want[~nan_w]
    sent = w == 123.456
    ok &= bool(np.all(np.abs(g[sent] - 123.456) < 1e-4))
    g, w = g[~sent], w[~sent]
    zero = w == 0
    ok &= bool(np.all(g[zero] == 0))
    g, w = g[~zero], w[~zero]
    if not g.size:
        return ok, 0.0, 0.0, 0
    rel = np.abs(g - w) / np.abs(w)
    return ok, float(rel.max()), float(rel.mean()), int(rel.size)


def _group_values(g, mode):
    """Oracle values for one group: (counts, FP64 r^2, reference r^2 or None)."""
    C = counts(g["A"], g["B"])
    want64 = r2_exact(g["bcA"], g["bcB"], C, g["S"])
    ref = r2_reference(g["bcA"], g["bcB"], C, g["S"], fma_contract=False) \
        if mode == "reference" else None
    return C, want64, ref


def check_groups(groups, mode="exact", rtol=1e-6, workers=None):
    """Check r^2 (and counts) of sampled outputs against the oracle.

    Each group is a dict: A (w, K) and B (r, K) packed rows with their bit
    counts bcA / bcB, S, `got` -- the library's (r, w) r^2 for those rows in
    its B-major layout --, `valid` (r, w) marking the entries the task
    defines, and optionally `counts` (r, w).  Groups are evaluated on a
    thread pool (the C oracle releases the GIL).  Counts must be bit-exact.
    In "exact" mode r^2 must be within `rtol` relative of the FP64 oracle
    (NaN, zeros and the 123.456 sentinel exactly); in "reference" mode
    bit-identical to the reference's float/double sequence.  The max and
    mean relative error against FP64 are reported in both modes.
    """
    from concurrent.futures import ThreadPoolExecutor
    workers = workers or min(32, os.cpu_count() or 1)
    with ThreadPoolExecutor(workers) as ex:
        vals = list(ex.map(lambda g: _group_values(g, mode), groups))
    got, w64, ref, cnt_ok, rows, pairs = [], [], [], True, 0, 0
    for g, (C, want64, r) in zip(groups, vals):
        v = np.asarray(g["valid"], bool)
        gg = np.asarray(g["got"], np.float32)
        got.append(gg[v])
        w64.append(want64[v])
        if r is not None:
            ref.append(r[v])
        if g.get("counts") is not None:
            cnt_ok &= bool(np.array_equal(np.asarray(g["counts"])[v].astype(np.uint32), C[v]))
        rows += gg.shape[0]
        pairs += int(v.sum())
    got = np.concatenate(got) if got else np.zeros(0, np.float32)
    w64 = np.concatenate(w64) if w64 else np.zeros(0)
    specials, max_rel, mean_rel, n_rel = r2_errors(got, w64)
    res = {"rows_checked": rows, "pairs_checked": pairs, "r2_max_rel": max_rel,
           "r2_mean_rel": mean_rel, "r2_rel_count": n_rel, "r2_mode": mode}
    has_counts = any(g.get("counts") is not None for g in groups)
    if has_counts:
        res["counts_exact"] = cnt_ok
    if mode == "reference":
        ref = np.concatenate(ref) if ref else np.zeros(0, np.float32)
        res["r2_bit_identical"] = bool(np.array_equal(got.view(np.uint32), ref.view(np.uint32)))
        res["ok"] = res["r2_bit_identical"]
    else:
        res["r2_within_tol"] = bool(specials and max_rel <= rtol)
        res["rtol"] = rtol
        res["ok"] = res["r2_within_tol"]
    if has_counts:
        res["ok"] = res["ok"] and cnt_ok
    return res


def check_rows(A, bcA, Brows, bcBrows, S, got_r2, valid, got_counts=None, mode="exact",
               rtol=1e-6):
    """check_groups() for sampled B rows against every row of A, the row set
    split into groups so the thread pool shares the work."""
    r = Brows.shape[0]
    step = max(1, -(-r // 64))
    groups = []
    for k in range(0, r, step):
        sl = slice(k, min(r, k + step))
        groups.append(dict(A=A, bcA=bcA, B=Brows[sl], bcB=bcBrows[sl], S=S,
                           got=np.asarray(got_r2)[sl], valid=np.asarray(valid)[sl],
                           counts=None if got_counts is None else np.asarray(got_counts)[sl]))
    return check_groups(groups, mode=mode, rtol=rtol)


def tile_row_samples(n, block, per_block, rng, extra=()):
    """Sorted distinct B rows: `per_block` random rows from every block of
    `block` rows (so every output tile row is sampled), plus `extra`."""
    rows = set(int(x) for x in extra if 0 <= x < n)
    for b0 in range(0, n, block):
        b1 = min(n, b0 + block)
        k = min(per_block, b1 - b0)
        rows.update(int(x) for x in rng.choice(np.arange(b0, b1), k, replace=False))
    return np.array(sorted(rows), np.int64)
