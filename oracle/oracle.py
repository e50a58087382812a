"""CPU oracle for the qLD LD hot path -- TEST INFRASTRUCTURE ONLY.

Thin ctypes/numpy layer over two libraries:

* ``libqld_oracle.so`` -- the C restatement in ``qld_oracle.c`` (counts, the
  reference-semantics r^2, the FP64 r^2 oracle, the text report).
* ``_ref/libqldref.so`` -- the reference's own functions compiled from the qLD
  sources (``gemm()``/``mlt()``/``get_pairwise_ld_score()``/``writeResults()``
  /``correlate()`` and the BLIS ``bin_gemm_2x2`` micro-kernel), see Makefile.

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
    ref = os.environ.get("QLD_REFERENCE", "/root/reference")
    if with_reference and os.path.isdir(os.path.join(ref, "src", "correlator")):
        subprocess.run(["make", "-s", "-C", _HERE, f"REF={ref}", "ref"], check=True)


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
