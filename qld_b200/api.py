"""Python binding of libqld_cuda's C ABI (include/qld_cuda.h).

This is the host-side mirror of qLD-compute's compute entry point for the
tests and the benchmark: ``Context.ld`` takes the same arguments as the
reference's ``correlate()`` compute part (src/correlator/include/gemm_cpu.h:24-38:
table A + bit counts + size, table B + bit counts + size, compressed snip size
K, snip size S, posWset2) and returns its ``results`` array.  Errors surface as
``QldError`` carrying the library's status code and message -- the library
never exits the process.

The library must be built (``python -m qld_b200.build``); there is no fallback
path: loading fails loudly when the CUDA library is missing.
"""
from __future__ import annotations

import ctypes as ct
import os
import weakref
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libqld_cuda.so")

OK = 0
ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_NODEVICE, ERR_TIMEOUT, ERR_BUSY, ERR_UNSUPPORTED = (
    -1, -2, -3, -4, -5, -6, -7)
R2_EXACT, R2_REFERENCE = 0, 1
KERNEL_AUTO, KERNEL_POPC, KERNEL_MMA, KERNEL_FP4 = 0, 1, 2, 3
OPT_KERNEL, OPT_R2_MODE, OPT_PROFILE, OPT_BAND_ROWS, OPT_MMA_TILE, OPT_SM_PAIR = 1, 2, 3, 4, 5, 6
OPT_WAIT_CYCLES, OPT_MEM_CAP = 7, 8

EXPORTED = (
    "qld_cuda_init", "qld_cuda_release", "qld_cuda_last_error", "qld_cuda_set_option",
    "qld_cuda_ld", "qld_cuda_ld_device", "qld_cuda_ld_hits", "qld_cuda_ld_batch",
    "qld_cuda_batch_plan", "qld_cuda_batch_run", "qld_cuda_batch_free",
    "qld_cuda_ld_device_part", "qld_cuda_split_rows",
    "qld_cuda_count_states", "qld_cuda_count_states_device", "qld_cuda_vcf_pack",
    "qld_cuda_ld_band",
    "qld_cuda_ld_band_device", "qld_cuda_sync",
    "qld_cuda_host_alloc",
    "qld_cuda_host_free", "qld_cuda_get_stats", "qld_cuda_measure_popc_peak",
    "qld_cuda_measure_mma_peak", "qld_cuda_autotune", "qld_cuda_tune_save", "qld_cuda_tune_load",
    "qld_srv_create", "qld_srv_add_table", "qld_srv_submit", "qld_srv_poll", "qld_srv_fetch",
    "qld_srv_release", "qld_srv_destroy", "qld_srv_last_error",
)


class QldError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class _LdArgs(ct.Structure):
    _fields_ = [
        ("A", ct.c_void_p), ("bcA", ct.c_void_p), ("m", ct.c_int), ("lda", ct.c_longlong),
        ("B", ct.c_void_p), ("bcB", ct.c_void_p), ("n", ct.c_int), ("ldb", ct.c_longlong),
        ("K", ct.c_int), ("S", ct.c_int), ("symmetric", ct.c_int),
        ("r2", ct.c_void_p), ("ldr", ct.c_longlong),
        ("counts", ct.c_void_p), ("ldc", ct.c_longlong),
    ]


class _Stats(ct.Structure):
    _fields_ = [("counts_launches", ct.c_longlong), ("kernel_launches", ct.c_longlong),
                ("counts_kernel_ms", ct.c_double), ("last_kernel", ct.c_int),
                ("hits_rows", ct.c_longlong), ("hits_pairs", ct.c_longlong)]


@dataclass
class Stats:
    counts_launches: int
    kernel_launches: int
    counts_kernel_ms: float
    last_kernel: int
    hits_rows: int = 0
    hits_pairs: int = 0


class HitsBlock(ct.Structure):
    """qld_hits_block: one block of B rows of qld_cuda_ld_hits."""
    _fields_ = [("row0", ct.c_int), ("rows", ct.c_int), ("m", ct.c_int), ("words", ct.c_int),
                ("mask", ct.POINTER(ct.c_uint32)), ("row_off", ct.POINTER(ct.c_longlong)),
                ("val", ct.POINTER(ct.c_float))]


HITS_FN = ct.CFUNCTYPE(ct.c_int, ct.c_void_p, ct.POINTER(HitsBlock))
RAND_FN = ct.CFUNCTYPE(ct.c_uint, ct.c_void_p)


class _Query(ct.Structure):
    _fields_ = [("table", ct.c_int), ("a0", ct.c_int), ("a1", ct.c_int), ("b0", ct.c_int),
                ("b1", ct.c_int), ("threshold", ct.c_float), ("host_r2", ct.c_void_p)]


class _QueryResult(ct.Structure):
    _fields_ = [("id", ct.c_longlong), ("status", ct.c_int), ("latency_ms", ct.c_double),
                ("pairs", ct.c_longlong), ("n_above", ct.c_longlong), ("sum_r2", ct.c_double),
                ("max_r2", ct.c_float)]


_lib = None


def load_library(path: str = LIB_PATH) -> ct.CDLL:
    """Load libqld_cuda.so (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built; run `python -m qld_b200.build`")
    lib = ct.CDLL(path)
    vp, i, ll = ct.c_void_p, ct.c_int, ct.c_longlong
    lib.qld_cuda_init.argtypes = [i, ct.POINTER(vp)]
    lib.qld_cuda_release.argtypes = [vp]
    lib.qld_cuda_last_error.argtypes = [vp]
    lib.qld_cuda_last_error.restype = ct.c_char_p
    lib.qld_cuda_set_option.argtypes = [vp, i, ll]
    lib.qld_cuda_ld.argtypes = [vp, vp, vp, i, vp, vp, i, i, i, i, vp, vp]
    lib.qld_cuda_ld_device.argtypes = [vp, ct.POINTER(_LdArgs), vp]
    lib.qld_cuda_ld_batch.argtypes = [vp, ct.POINTER(_LdArgs), i, vp]
    lib.qld_cuda_batch_plan.argtypes = [vp, ct.POINTER(_LdArgs), i, ct.POINTER(vp)]
    lib.qld_cuda_batch_run.argtypes = [vp, vp]
    lib.qld_cuda_batch_free.argtypes = [vp]
    lib.qld_cuda_ld_device_part.argtypes = [vp, ct.POINTER(_LdArgs), i, i, ct.POINTER(i),
                                            ct.POINTER(i), vp]
    lib.qld_cuda_split_rows.argtypes = [i, i, i, i, i, i, i, ct.POINTER(i), ct.POINTER(i)]
    lib.qld_cuda_count_states.argtypes = [vp, vp, i, vp, i, i, i, vp]
    lib.qld_cuda_vcf_pack.argtypes = [vp, ct.c_char_p, ct.c_size_t, vp, i, vp, i, i, i, RAND_FN,
                                      vp, vp, vp, vp, vp, ct.POINTER(i)]
    lib.qld_cuda_count_states_device.argtypes = [vp, vp, i, ll, vp, i, ll, i, i, vp, ll, vp]
    lib.qld_cuda_ld_hits.argtypes = [vp, vp, vp, i, vp, vp, i, i, i, i, i, ct.c_float, HITS_FN, vp]
    lib.qld_cuda_ld_band.argtypes = [vp, vp, vp, i, i, i, i, vp, vp]
    lib.qld_cuda_ld_band_device.argtypes = [vp, vp, vp, i, ll, i, i, i, vp, ll, vp, ll, vp]
    lib.qld_cuda_sync.argtypes = [vp, vp]
    lib.qld_cuda_host_alloc.argtypes = [vp, ct.c_size_t, ct.POINTER(vp)]
    lib.qld_cuda_host_free.argtypes = [vp, vp]
    lib.qld_cuda_get_stats.argtypes = [vp, ct.POINTER(_Stats), i]
    lib.qld_cuda_measure_popc_peak.argtypes = [vp, ct.POINTER(ct.c_double)]
    lib.qld_cuda_measure_mma_peak.argtypes = [vp, i, ct.POINTER(ct.c_double)]
    ip = ct.POINTER(ct.c_int)
    lib.qld_cuda_autotune.argtypes = [vp, i, i, i, i, ip, ip, ct.POINTER(ct.c_float)]
    lib.qld_cuda_tune_save.argtypes = [vp, ct.c_char_p]
    lib.qld_cuda_tune_load.argtypes = [vp, ct.c_char_p]
    lib.qld_srv_create.argtypes = [i, ct.c_size_t, i, ct.POINTER(vp)]
    lib.qld_srv_add_table.argtypes = [vp, vp, vp, i, i, i, ct.POINTER(i)]
    lib.qld_srv_submit.argtypes = [vp, ct.POINTER(_Query), ct.POINTER(ll)]
    lib.qld_srv_poll.argtypes = [vp, ct.POINTER(_QueryResult), i, ct.POINTER(i), i]
    lib.qld_srv_fetch.argtypes = [vp, ll, vp]
    lib.qld_srv_release.argtypes = [vp, ll]
    lib.qld_srv_destroy.argtypes = [vp]
    lib.qld_srv_last_error.argtypes = [vp]
    lib.qld_srv_last_error.restype = ct.c_char_p
    _lib = lib
    return lib


def _ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # torch tensor


class Context:
    """One libqld_cuda context (one per host thread), bound to a device."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ct.c_void_p()
        rc = self.lib.qld_cuda_init(int(device), ct.byref(h))
        if rc != OK:
            raise QldError(rc, f"qld_cuda_init(device={device}) failed")
        self.h = h
        self.device = device
        self._pinned: dict[int, int] = {}
        self._plans: weakref.WeakSet = weakref.WeakSet()

    def close(self):
        if getattr(self, "h", None):
            for plan in list(self._plans):   # qld_cuda_release frees them
                plan.h = None
            self._plans.clear()
            for p in list(self._pinned):
                self.lib.qld_cuda_host_free(self.h, ct.c_void_p(p))
            self._pinned.clear()
            self.lib.qld_cuda_release(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != OK:
            raise QldError(rc, self.lib.qld_cuda_last_error(self.h).decode(errors="replace"))

    def set_option(self, option: int, value: int):
        self._check(self.lib.qld_cuda_set_option(self.h, option, int(value)))

    def stats(self, reset: bool = False) -> Stats:
        s = _Stats()
        self._check(self.lib.qld_cuda_get_stats(self.h, ct.byref(s), int(reset)))
        return Stats(s.counts_launches, s.kernel_launches, s.counts_kernel_ms, s.last_kernel,
                     s.hits_rows, s.hits_pairs)

    def measure_popc_peak(self) -> float:
        """Measured popcount-pipe peak in bit-ops/s."""
        v = ct.c_double()
        self._check(self.lib.qld_cuda_measure_popc_peak(self.h, ct.byref(v)))
        return v.value

    def autotune(self, m: int, n: int, K: int, symmetric: bool = True):
        """Time every exact counts kernel on a synthetic m x n x K task and make
        the fastest the automatic choice for its shape class; returns
        (kernel, option, ms per launch)."""
        k, o, t = ct.c_int(), ct.c_int(), ct.c_float()
        self._check(self.lib.qld_cuda_autotune(self.h, int(m), int(n), int(K),
                                               int(bool(symmetric)), ct.byref(k), ct.byref(o),
                                               ct.byref(t)))
        return k.value, o.value, t.value

    def tune_save(self, path: str):
        self._check(self.lib.qld_cuda_tune_save(self.h, str(path).encode()))

    def tune_load(self, path: str):
        self._check(self.lib.qld_cuda_tune_load(self.h, str(path).encode()))

    def measure_mma_peak(self, kernel: int) -> float:
        """Measured dense tensor-pipe rate in ops/s (2 per multiply-accumulate)
        for KERNEL_MMA (kind::i8) or KERNEL_FP4 (kind::mxf4)."""
        v = ct.c_double()
        self._check(self.lib.qld_cuda_measure_mma_peak(self.h, int(kernel), ct.byref(v)))
        return v.value

    # -------------------------------------------------------------- host --
    def pinned_empty(self, shape, dtype) -> np.ndarray:
        """numpy array in pinned host memory owned by this context."""
        dtype = np.dtype(dtype)
        nbytes = int(np.prod(shape)) * dtype.itemsize
        p = ct.c_void_p()
        self._check(self.lib.qld_cuda_host_alloc(self.h, max(nbytes, 1), ct.byref(p)))
        self._pinned[p.value] = nbytes
        buf = (ct.c_byte * max(nbytes, 1)).from_address(p.value)
        return np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

    def ld(self, A, bcA, B=None, bcB=None, *, S: int, symmetric: bool | None = None,
           r2_out=None, counts: bool | np.ndarray = False):
        """One LD task from host arrays; returns r2 (n, m) [and counts (n, m)].

        A, B: (rows, K) uint64 (or int64 bit patterns); bcA, bcB: uint32.
        symmetric defaults to B is None (single region).
        """
        if symmetric is None:
            symmetric = B is None
        A = np.ascontiguousarray(A).view(np.uint64) if A.dtype != np.uint64 else np.ascontiguousarray(A)
        bcA = np.ascontiguousarray(bcA, dtype=np.uint32)
        m, K = A.shape
        if symmetric:
            B, bcB, n = A, bcA, m
        else:
            B = np.ascontiguousarray(B).view(np.uint64) if B.dtype != np.uint64 else np.ascontiguousarray(B)
            bcB = np.ascontiguousarray(bcB, dtype=np.uint32)
            n = B.shape[0]
            if B.shape[1] != K:
                raise ValueError("A and B must have the same number of words per row")
        if r2_out is None:
            r2_out = np.empty((n, m), np.float32)
        cnt = None
        if isinstance(counts, np.ndarray):
            cnt = counts
        elif counts:
            cnt = np.empty((n, m), np.uint32)
        self._check(self.lib.qld_cuda_ld(self.h, _ptr(A), _ptr(bcA), m, _ptr(B), _ptr(bcB), n,
                                         K, int(S), int(bool(symmetric)), _ptr(r2_out), _ptr(cnt)))
        return (r2_out, cnt) if cnt is not None else r2_out

    def ld_hits(self, A, bcA, B=None, bcB=None, *, S: int, r2limit: float,
                symmetric: bool | None = None, triangle: bool | None = None,
                on_block=None):
        """The report's pairs of one task, filtered on the GPU.

        Without `on_block`: returns (mask (n, ceil(m/32)) uint32, row_off (n+1,)
        int64, val (total,) float32) for the whole task.  With `on_block`, it
        is called with each HitsBlock (valid during the call) and may return a
        nonzero int to stop.  triangle defaults to symmetric."""
        if symmetric is None:
            symmetric = B is None
        if triangle is None:
            triangle = symmetric
        A = np.ascontiguousarray(A).view(np.uint64)
        bcA = np.ascontiguousarray(bcA, dtype=np.uint32)
        m, K = A.shape
        if symmetric:
            B, bcB, n = A, bcA, m
        else:
            B = np.ascontiguousarray(B).view(np.uint64)
            bcB = np.ascontiguousarray(bcB, dtype=np.uint32)
            n = B.shape[0]
        W = (m + 31) // 32
        masks, offs, vals = [], [np.zeros(1, np.int64)], []
        err: list = []

        def cb(_user, bp):
            try:
                b = bp.contents
                if on_block is not None:
                    return int(on_block(b) or 0)
                mk = np.ctypeslib.as_array(b.mask, (b.rows * b.words,)).reshape(b.rows, b.words)
                of = np.ctypeslib.as_array(b.row_off, (b.rows + 1,))
                tot = int(of[b.rows])
                masks.append(mk.copy())
                offs.append(of[1:] + offs[-1][-1])
                vals.append(np.ctypeslib.as_array(b.val, (tot,)).copy() if tot else
                            np.zeros(0, np.float32))
                return 0
            except Exception as e:   # surface Python errors after the call
                err.append(e)
                return -100

        fn = HITS_FN(cb)
        rc = self.lib.qld_cuda_ld_hits(self.h, _ptr(A), _ptr(bcA), m, _ptr(B), _ptr(bcB), n, K,
                                       int(S), int(bool(symmetric)), int(bool(triangle)),
                                       float(r2limit), fn, None)
        if err:
            raise err[0]
        if on_block is not None and rc > 0:
            return rc
        self._check(rc)
        if on_block is not None:
            return 0
        mask = np.concatenate(masks) if masks else np.zeros((0, W), np.uint32)
        row_off = np.concatenate(offs)
        val = np.concatenate(vals) if vals else np.zeros(0, np.float32)
        return mask, row_off, val

    def count_states(self, A, B=None, *, symmetric: bool | None = None, out=None):
        """COUNTSTATES: (n, m) uint8 state values (qld_cuda_count_states)."""
        if symmetric is None:
            symmetric = B is None
        A = np.ascontiguousarray(A).view(np.uint64)
        m, K = A.shape
        if symmetric:
            B, n = A, m
        else:
            B = np.ascontiguousarray(B).view(np.uint64)
            n = B.shape[0]
            if B.shape[1] != K:
                raise ValueError("A and B must have the same number of words per row")
        if out is None:
            out = np.empty((n, m), np.uint8)
        self._check(self.lib.qld_cuda_count_states(self.h, _ptr(A), m, _ptr(B), n, K,
                                                   int(bool(symmetric)), _ptr(out)))
        return out

    def vcf_pack(self, text: bytes, sites: np.ndarray, valid, ploidy: int, K: int,
                 seed: int | None = 1):
        """qld_cuda_vcf_pack over qld_vcf_site records `sites` (a numpy array of
        host_api.VCF_SITE): returns (words (n, K) uint64, bc, snip_len, keep).
        Unphased genotypes draw from libc rand() after srand(seed), as
        qLD-parse-2MDF does; seed None leaves the generator unseeded."""
        sites = np.ascontiguousarray(sites)
        valid = np.ascontiguousarray(valid, np.uint8)
        n = len(sites)
        words = np.zeros((max(n, 1), K), np.uint64)
        bc = np.zeros(max(n, 1), np.uint32)
        ln = np.zeros(max(n, 1), np.int32)
        keep = np.zeros(max(n, 1), np.uint8)
        libc = ct.CDLL(None)
        libc.rand.restype = ct.c_int
        seeded = [seed is None]

        def draw(_user):
            if not seeded[0]:
                libc.srand(ct.c_uint(seed))
                seeded[0] = True
            return libc.rand()

        fn = RAND_FN(draw)
        bad = ct.c_int(-1)
        self._check(self.lib.qld_cuda_vcf_pack(self.h, text, len(text), sites.ctypes.data, n,
                                               valid.ctypes.data, len(valid), int(ploidy), int(K),
                                               fn, None, words.ctypes.data, bc.ctypes.data,
                                               ln.ctypes.data, keep.ctypes.data, ct.byref(bad)))
        return words[:n], bc[:n], ln[:n], keep[:n]

    def count_states_device(self, A, m, lda, B, n, ldb, K, symmetric, out, lds, stream=None):
        self._check(self.lib.qld_cuda_count_states_device(
            self.h, _p(A), int(m), int(lda), _p(B), int(n), int(ldb), int(K),
            int(bool(symmetric)), _p(out), int(lds), _stream(stream)))

    # ------------------------------------------------------------ device --
    def ld_device(self, A, bcA, m, lda, B, bcB, n, ldb, K, S, symmetric, r2, ldr,
                  counts=None, ldc=0, stream=None):
        """Enqueue one task on device buffers (torch tensors or raw pointers)."""
        a = _LdArgs(_p(A), _p(bcA), int(m), int(lda), _p(B), _p(bcB), int(n), int(ldb), int(K),
                    int(S), int(bool(symmetric)), _p(r2), int(ldr), _p(counts), int(ldc))
        self._check(self.lib.qld_cuda_ld_device(self.h, ct.byref(a), _stream(stream)))

    def ld_device_part(self, A, bcA, m, lda, B, bcB, n, ldb, K, S, symmetric, r2, ldr, part,
                       nparts, counts=None, ldc=0, stream=None):
        """Part `part` of `nparts` of a task split over GPUs: enqueues B rows
        [row0, row1) into r2 (row 0 = B row row0); returns (row0, row1)."""
        a = _LdArgs(_p(A), _p(bcA), int(m), int(lda), _p(B), _p(bcB), int(n), int(ldb), int(K),
                    int(S), int(bool(symmetric)), _p(r2), int(ldr), _p(counts), int(ldc))
        r0, r1 = ct.c_int(), ct.c_int()
        self._check(self.lib.qld_cuda_ld_device_part(self.h, ct.byref(a), int(part), int(nparts),
                                                     ct.byref(r0), ct.byref(r1), _stream(stream)))
        return r0.value, r1.value

    @staticmethod
    def _ld_args(jobs):
        arr = (_LdArgs * len(jobs))()
        for i, j in enumerate(jobs):
            arr[i] = _LdArgs(_p(j["A"]), _p(j["bcA"]), int(j["m"]), int(j["lda"]),
                             _p(j.get("B")), _p(j.get("bcB")), int(j.get("n", j["m"])),
                             int(j.get("ldb", j["lda"])), int(j["K"]), int(j["S"]),
                             int(bool(j["symmetric"])), _p(j["r2"]), int(j["ldr"]),
                             _p(j.get("counts")), int(j.get("ldc", 0)))
        return arr

    def ld_batch(self, jobs, stream=None):
        """Enqueue many tasks in one launch.  `jobs`: sequence of dicts with
        the ld_device keyword names (A, bcA, m, lda, B, bcB, n, ldb, K, S,
        symmetric, r2, ldr, counts=None, ldc=0)."""
        arr = self._ld_args(jobs)
        self._check(self.lib.qld_cuda_ld_batch(self.h, arr, len(jobs), _stream(stream)))

    def batch_plan(self, jobs) -> "BatchPlan":
        """qld_cuda_batch_plan: the batched call over `jobs` (as ld_batch)
        captured once as a CUDA graph; BatchPlan.run() replays it.  The jobs'
        device tensors must outlive the plan."""
        arr = self._ld_args(jobs)
        h = ct.c_void_p()
        self._check(self.lib.qld_cuda_batch_plan(self.h, arr, len(jobs), ct.byref(h)))
        plan = BatchPlan(self, h)
        self._plans.add(plan)
        return plan

    def ld_band(self, A, bcA, *, S: int, band: int, r2_out=None, counts=False):
        """Windowed LD from host arrays: r2 (m, band), r2[i, d] = r^2(i, i+1+d)."""
        A = np.ascontiguousarray(A).view(np.uint64) if A.dtype != np.uint64 else np.ascontiguousarray(A)
        bcA = np.ascontiguousarray(bcA, dtype=np.uint32)
        m, K = A.shape
        if r2_out is None:
            r2_out = np.empty((m, band), np.float32)
        cnt = None
        if isinstance(counts, np.ndarray):
            cnt = counts
        elif counts:
            cnt = np.empty((m, band), np.uint32)
        self._check(self.lib.qld_cuda_ld_band(self.h, _ptr(A), _ptr(bcA), m, K, int(S), int(band),
                                              _ptr(r2_out), _ptr(cnt)))
        return (r2_out, cnt) if cnt is not None else r2_out

    def ld_band_device(self, A, bcA, m, lda, K, S, band, r2, ldr, counts=None, ldc=0,
                       stream=None):
        self._check(self.lib.qld_cuda_ld_band_device(
            self.h, _p(A), _p(bcA), int(m), int(lda), int(K), int(S), int(band), _p(r2),
            int(ldr), _p(counts), int(ldc), _stream(stream)))

    def sync(self, stream=None):
        self._check(self.lib.qld_cuda_sync(self.h, _stream(stream)))


class BatchPlan:
    """A batched call captured as a CUDA graph (qld_cuda_batch_plan)."""

    def __init__(self, ctx: Context, h):
        self.ctx = ctx
        self.h = h

    def run(self, stream=None):
        """Replay on `stream` (asynchronous: Context.sync collects it)."""
        if not self.h:
            raise QldError(ERR_INVALID, "batch plan is closed")
        self.ctx._check(self.ctx.lib.qld_cuda_batch_run(self.h, _stream(stream)))

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.qld_cuda_batch_free(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def split_rows(m, n, K, symmetric, kernel, part, nparts):
    """(row0, row1) of part `part` of `nparts` (qld_cuda_split_rows; no GPU
    needed)."""
    lib = load_library()
    r0, r1 = ct.c_int(), ct.c_int()
    rc = lib.qld_cuda_split_rows(int(m), int(n), int(K), int(bool(symmetric)), int(kernel),
                                 int(part), int(nparts), ct.byref(r0), ct.byref(r1))
    if rc != OK:
        raise QldError(rc, "qld_cuda_split_rows: bad arguments")
    return r0.value, r1.value


def _p(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return _ptr(x)


CUDA_STREAM_LEGACY = 1   # cudaStreamLegacy: the legacy default stream's handle


def _stream(s):
    """A cudaStream_t for the C ABI.  None (or 0) keeps the C meaning: the
    context's own stream.  A torch stream object is passed as itself; torch's
    default stream is the legacy NULL stream, which the C ABI would read as
    the context's stream (not ordered with torch's work), so it goes as
    cudaStreamLegacy instead."""
    if s is None:
        return None
    if isinstance(s, int):
        return s
    h = s.cuda_stream  # torch.cuda.Stream
    return h if h else CUDA_STREAM_LEGACY


@dataclass
class QueryResult:
    id: int
    status: int
    latency_ms: float
    pairs: int
    n_above: int
    sum_r2: float
    max_r2: float


class Server:
    """The serving loop (qld_srv_*): resident tables, queries admitted by
    output memory and batched continuously on the device."""

    def __init__(self, device: int = 0, pool_bytes: int = 8 << 30, max_inflight: int = 3):
        self.lib = load_library()
        h = ct.c_void_p()
        rc = self.lib.qld_srv_create(int(device), int(pool_bytes), int(max_inflight), ct.byref(h))
        if rc != OK:
            raise QldError(rc, "qld_srv_create failed")
        self.h = h

    def _check(self, rc):
        if rc != OK:
            raise QldError(rc, self.lib.qld_srv_last_error(self.h).decode(errors="replace"))

    def add_table(self, A, bc, S) -> int:
        """A: (m, K) uint64 numpy array or contiguous int64 torch tensor (host
        or device); bc: its row bit counts.  The copy does not wait for work
        on other streams, so torch's current stream on a device tensor's
        device is synchronized first (a table written on another stream must
        be complete before the call)."""
        if isinstance(A, np.ndarray):
            A = np.ascontiguousarray(A).view(np.uint64)
            bc = np.ascontiguousarray(bc, dtype=np.uint32)
        else:
            import torch
            for t in (A, bc):
                if isinstance(t, torch.Tensor) and t.is_cuda:
                    torch.cuda.current_stream(t.device).synchronize()
        tid = ct.c_int()
        self._check(self.lib.qld_srv_add_table(self.h, _ptr(A), _ptr(bc), A.shape[0], A.shape[1],
                                               int(S), ct.byref(tid)))
        return tid.value

    def submit(self, table, a0, a1, b0, b1, threshold=0.2, host_r2=None) -> int:
        q = _Query(int(table), int(a0), int(a1), int(b0), int(b1), float(threshold),
                   _ptr(host_r2))
        qid = ct.c_longlong()
        self._check(self.lib.qld_srv_submit(self.h, ct.byref(q), ct.byref(qid)))
        return qid.value

    def poll(self, max_results=256, wait_ms=100):
        arr = (_QueryResult * max_results)()
        n = ct.c_int()
        self._check(self.lib.qld_srv_poll(self.h, arr, max_results, ct.byref(n), int(wait_ms)))
        return [QueryResult(r.id, r.status, r.latency_ms, r.pairs, r.n_above, r.sum_r2, r.max_r2)
                for r in arr[:n.value]]

    def fetch(self, qid, out: np.ndarray):
        self._check(self.lib.qld_srv_fetch(self.h, int(qid), _ptr(out)))
        return out

    def release(self, qid):
        self._check(self.lib.qld_srv_release(self.h, int(qid)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.qld_srv_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
