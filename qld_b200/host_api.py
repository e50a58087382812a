"""ctypes binding of libqld_host.so (include/qld_host.h): MDF loading and
qLD's text report from Python.

    hdr = host_api.read_header(path)
    tab = host_api.load_mdf(path, pos_min, pos_max, K, threads=8, ctx=None)
    host_api.write_report(out_path, tab_a, tab_b, r2, snip_size, r2limit,
                          single_region, threads=8)
    host_api.write_report_hits(out_path, tab_a, tab_b, blocks, snip_size)

``load_mdf`` returns a ``Table`` (numpy copies of words, BC, POS and IDs) and
releases the C-side buffers; with a ``api.Context`` the C side assembles in
pinned memory, with ``ctx=None`` in pageable memory (no GPU needed).
"""
from __future__ import annotations

import ctypes as ct
import os
from dataclasses import dataclass

import numpy as np

from . import api

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libqld_host.so")
CLI_PATH = os.path.join(_PKG, "qld-ld")


class _Header(ct.Structure):
    _fields_ = [("id", ct.c_char * 256), ("snips_per_file", ct.c_int), ("snip_size", ct.c_int),
                ("total_snips", ct.c_int), ("pos_min", ct.c_int), ("pos_max", ct.c_int),
                ("samples", ct.c_int)]


class _Table(ct.Structure):
    _fields_ = [("words", ct.POINTER(ct.c_uint64)), ("bc", ct.POINTER(ct.c_uint32)),
                ("pos", ct.POINTER(ct.c_uint32)), ("ids", ct.POINTER(ct.c_char_p)),
                ("id_pool", ct.c_char_p), ("rows", ct.c_int), ("K", ct.c_int),
                ("pinned", ct.c_int)]


@dataclass
class Header:
    id: str
    snips_per_file: int
    snip_size: int
    total_snips: int
    pos_min: int
    pos_max: int
    samples: int


@dataclass
class Table:
    words: np.ndarray      # (rows, K) uint64
    bc: np.ndarray         # (rows,) uint32
    pos: np.ndarray        # (rows,) uint32
    ids: list

    @property
    def rows(self) -> int:
        return self.words.shape[0]


_lib = None


def lib() -> ct.CDLL:
    global _lib
    if _lib is None:
        api.load_library()   # libqld_cuda.so first: libqld_host.so resolves against it
        if not os.path.exists(LIB_PATH):
            raise api.QldError(api.ERR_INVALID, f"{LIB_PATH} not built (python -m qld_b200.build)")
        L = ct.CDLL(LIB_PATH)
        L.qld_mdf_read_header.argtypes = [ct.c_char_p, ct.POINTER(_Header)]
        L.qld_mdf_read_header.restype = ct.c_int
        L.qld_mdf_listed_samples.argtypes = [ct.c_char_p, ct.POINTER(ct.c_char_p), ct.c_int,
                                             ct.POINTER(ct.c_int)]
        L.qld_mdf_listed_samples.restype = ct.c_int
        L.qld_mdf_load.argtypes = [ct.c_void_p, ct.c_char_p, ct.c_int, ct.c_int, ct.c_int, ct.c_int,
                                   ct.POINTER(_Table)]
        L.qld_mdf_load.restype = ct.c_int
        L.qld_table_free.argtypes = [ct.c_void_p, ct.POINTER(_Table)]
        L.qld_table_free.restype = None
        L.qld_report_write.argtypes = [ct.c_void_p, ct.POINTER(_Table), ct.POINTER(_Table),
                                       ct.c_void_p, ct.c_int, ct.c_float, ct.c_int, ct.c_int]
        L.qld_report_write.restype = ct.c_int
        L.qld_report_open.argtypes = [ct.POINTER(ct.c_void_p), ct.c_void_p, ct.POINTER(_Table),
                                      ct.POINTER(_Table), ct.c_int, ct.c_int]
        L.qld_report_open.restype = ct.c_int
        L.qld_report_hits.argtypes = [ct.c_void_p, ct.POINTER(api.HitsBlock)]
        L.qld_report_hits.restype = ct.c_int
        L.qld_report_close.argtypes = [ct.c_void_p]
        L.qld_report_close.restype = ct.c_int
        L.qld_report_states.argtypes = [ct.c_void_p, ct.POINTER(_Table), ct.POINTER(_Table),
                                        ct.c_void_p, ct.c_int, ct.c_int]
        L.qld_report_states.restype = ct.c_int
        L.qld_host_last_error.argtypes = []
        L.qld_host_last_error.restype = ct.c_char_p
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != api.OK:
        msg = lib().qld_host_last_error()
        raise api.QldError(rc, msg.decode() if msg else "")


def read_header(path: str) -> Header:
    h = _Header()
    _check(lib().qld_mdf_read_header(os.fsencode(path), ct.byref(h)))
    return Header(h.id.decode(), h.snips_per_file, h.snip_size, h.total_snips, h.pos_min,
                  h.pos_max, h.samples)


def listed_samples(path: str, names=None) -> int:
    """Sample names of the dataset's #CHROM line that `names` holds (all of
    them for None): the count qLD-compute's -sampleList gives
    (qld_mdf_listed_samples)."""
    names = list(names or [])
    arr = (ct.c_char_p * max(1, len(names)))(*[n.encode() for n in names])
    out = ct.c_int()
    _check(lib().qld_mdf_listed_samples(os.fsencode(path), arr, len(names), ct.byref(out)))
    return out.value


def load_mdf(path: str, pos_min: int, pos_max: int, K: int, threads: int = 1,
             ctx: "api.Context | None" = None) -> Table:
    t = _Table()
    handle = ctx.h if ctx is not None else None
    _check(lib().qld_mdf_load(handle, os.fsencode(path), int(pos_min), int(pos_max), int(K),
                              int(threads), ct.byref(t)))
    try:
        n = t.rows
        words = np.ctypeslib.as_array(t.words, (max(n, 1), K))[:n].copy() if n else \
            np.zeros((0, K), np.uint64)
        bc = np.ctypeslib.as_array(t.bc, (n,)).copy() if n else np.zeros(0, np.uint32)
        pos = np.ctypeslib.as_array(t.pos, (n,)).copy() if n else np.zeros(0, np.uint32)
        ids = [t.ids[i].decode() for i in range(n)]
    finally:
        lib().qld_table_free(handle, ct.byref(t))
    return Table(words, bc, pos, ids)


def _as_c_table(tab: Table, keep: list) -> _Table:
    t = _Table()
    n = len(tab.pos)
    bc = np.ascontiguousarray(tab.bc, np.uint32)
    pos = np.ascontiguousarray(tab.pos, np.uint32)
    ids = (ct.c_char_p * max(n, 1))()
    ids[:n] = [s.encode() for s in tab.ids]
    keep += [bc, pos, ids]
    t.words = None
    t.bc = bc.ctypes.data_as(ct.POINTER(ct.c_uint32))
    t.pos = pos.ctypes.data_as(ct.POINTER(ct.c_uint32))
    t.ids = ct.cast(ids, ct.POINTER(ct.c_char_p))
    t.rows = n
    t.K = 0
    return t


def _libc():
    libc = ct.CDLL(None)
    libc.fopen.argtypes = [ct.c_char_p, ct.c_char_p]
    libc.fopen.restype = ct.c_void_p
    libc.fclose.argtypes = [ct.c_void_p]
    libc.fclose.restype = ct.c_int
    return libc


def hits_from_dense(r2: np.ndarray, r2limit: float, triangle: bool, row0: int = 0):
    """(mask, row_off, val) of a dense (rows, m) r^2 block under qLD's report
    rule -- the host-side statement of what qld_cuda_ld_hits delivers."""
    r2 = np.asarray(r2, np.float32)
    rows, m = r2.shape
    keep = (r2 >= np.float32(r2limit)) & (r2 < 100)
    if triangle:
        keep &= np.arange(m)[None, :] > (row0 + np.arange(rows))[:, None]
    W = (m + 31) // 32
    bits = np.zeros((rows, W * 32), bool)
    bits[:, :m] = keep
    mask = (bits.reshape(rows, W, 32).astype(np.uint64) << np.arange(32, dtype=np.uint64)).sum(
        axis=2).astype(np.uint32)
    row_off = np.zeros(rows + 1, np.int64)
    row_off[1:] = np.cumsum(keep.sum(axis=1))
    return mask, row_off, r2[keep].astype(np.float32)


def write_report_hits(path: str, A: Table, B: Table, blocks, snip_size: int,
                      threads: int = 1) -> None:
    """qLD's report from filtered blocks: `blocks` yields (row0, mask, row_off,
    val) in B-row order (qld_report_open / qld_report_hits / qld_report_close)."""
    libc = _libc()
    keep: list = []
    ta = _as_c_table(A, keep)
    tb = ta if B is A else _as_c_table(B, keep)
    fp = libc.fopen(os.fsencode(path), b"wb")
    if not fp:
        raise OSError(f"cannot open {path}")
    rep = ct.c_void_p()
    try:
        _check(lib().qld_report_open(ct.byref(rep), fp, ct.byref(ta), ct.byref(tb),
                                     int(snip_size), int(threads)))
        try:
            for row0, mask, row_off, val in blocks:
                mask = np.ascontiguousarray(mask, np.uint32)
                row_off = np.ascontiguousarray(row_off, np.int64)
                val = np.ascontiguousarray(val, np.float32)
                b = api.HitsBlock(int(row0), mask.shape[0], len(A.pos), mask.shape[1],
                                  mask.ctypes.data_as(ct.POINTER(ct.c_uint32)),
                                  row_off.ctypes.data_as(ct.POINTER(ct.c_longlong)),
                                  val.ctypes.data_as(ct.POINTER(ct.c_float)))
                _check(lib().qld_report_hits(rep, ct.byref(b)))
        finally:
            lib().qld_report_close(rep)
    finally:
        if libc.fclose(fp) != 0:
            raise OSError(f"cannot close {path}")


def write_report(path: str, A: Table, B: Table, r2: np.ndarray, snip_size: int,
                 r2limit: float, single_region: bool, threads: int = 1) -> None:
    """qLD's report of one task; r2 is (B rows, A rows) float32."""
    r2 = np.ascontiguousarray(r2, np.float32)
    if r2.shape != (len(B.pos), len(A.pos)):
        raise ValueError(f"r2 is {r2.shape}, expected {(len(B.pos), len(A.pos))}")
    libc = _libc()
    keep: list = []
    ta = _as_c_table(A, keep)
    tb = ta if B is A else _as_c_table(B, keep)
    fp = libc.fopen(os.fsencode(path), b"wb")
    if not fp:
        raise OSError(f"cannot open {path}")
    try:
        rc = lib().qld_report_write(fp, ct.byref(ta), ct.byref(tb), r2.ctypes.data,
                                    int(snip_size), float(r2limit), int(bool(single_region)),
                                    int(threads))
    finally:
        if libc.fclose(fp) != 0:
            raise OSError(f"cannot close {path}")
    _check(rc)


def write_states_report(path: str, A: Table, B: Table, states: np.ndarray,
                        single_region: bool, threads: int = 1) -> None:
    """qLD's COUNTSTATES report (writeStateCount); states is (B rows, A rows) uint8."""
    states = np.ascontiguousarray(states, np.uint8)
    if states.shape != (len(B.pos), len(A.pos)):
        raise ValueError(f"states is {states.shape}, expected {(len(B.pos), len(A.pos))}")
    libc = _libc()
    keep: list = []
    ta = _as_c_table(A, keep)
    tb = ta if B is A else _as_c_table(B, keep)
    fp = libc.fopen(os.fsencode(path), b"wb")
    if not fp:
        raise OSError(f"cannot open {path}")
    try:
        rc = lib().qld_report_states(fp, ct.byref(ta), ct.byref(tb), states.ctypes.data,
                                     int(bool(single_region)), int(threads))
    finally:
        if libc.fclose(fp) != 0:
            raise OSError(f"cannot close {path}")
    _check(rc)


# ------------------------------------------------------------- VCF -> MDF --

class _VcfHeader(ct.Structure):
    _fields_ = [("id", ct.c_char * 256), ("path", ct.c_char * 4096), ("line1", ct.c_char_p),
                ("line2", ct.c_char_p), ("nsamples", ct.c_int), ("valid", ct.POINTER(ct.c_uint8)),
                ("valid_count", ct.c_int), ("snips_per_file", ct.c_int), ("snip_size", ct.c_int),
                ("total_snips", ct.c_int)]


class _VcfPart(ct.Structure):
    _fields_ = [("text", ct.c_void_p), ("bytes", ct.c_size_t), ("pinned", ct.c_int),
                ("lines", ct.c_int), ("skipped", ct.c_int), ("nsites", ct.c_int),
                ("sites", ct.c_void_p), ("pos", ct.POINTER(ct.c_uint32)),
                ("ids", ct.POINTER(ct.c_size_t)), ("id_pool", ct.c_void_p)]


# one qld_vcf_site record (include/qld_cuda.h)
VCF_SITE = np.dtype([("off", np.int64), ("len", np.int32), ("gt_pos", np.int32),
                     ("n_states", np.int32), ("states", "S4")], align=True)


def _vcf_lib() -> ct.CDLL:
    L = lib()
    if not hasattr(L, "_vcf_bound"):
        L.qld_vcf_read_header.argtypes = [ct.c_char_p, ct.c_int, ct.POINTER(ct.c_char_p), ct.c_int,
                                          ct.POINTER(_VcfHeader)]
        L.qld_vcf_read_header.restype = ct.c_int
        L.qld_vcf_header_free.argtypes = [ct.POINTER(_VcfHeader)]
        L.qld_vcf_header_free.restype = None
        L.qld_vcf_list_parts.argtypes = [ct.c_char_p, ct.POINTER(_VcfHeader),
                                         ct.POINTER(ct.POINTER(ct.c_char_p)), ct.POINTER(ct.c_int)]
        L.qld_vcf_list_parts.restype = ct.c_int
        L.qld_vcf_list_free.argtypes = [ct.POINTER(ct.c_char_p), ct.c_int]
        L.qld_vcf_list_free.restype = None
        L.qld_vcf_load_part.argtypes = [ct.c_void_p, ct.c_char_p, ct.POINTER(_VcfHeader),
                                        ct.POINTER(_VcfPart)]
        L.qld_vcf_load_part.restype = ct.c_int
        L.qld_vcf_part_free.argtypes = [ct.c_void_p, ct.POINTER(_VcfPart)]
        L.qld_vcf_part_free.restype = None
        L.qld_vcf_site_id.argtypes = [ct.POINTER(_VcfPart), ct.c_int]
        L.qld_vcf_site_id.restype = ct.c_char_p
        L.qld_mdf_part_path.argtypes = [ct.c_char_p, ct.c_char_p, ct.c_char_p, ct.c_size_t]
        L.qld_mdf_part_path.restype = ct.c_int
        L.qld_mdf_write_part.argtypes = [ct.c_char_p, ct.c_char_p, ct.POINTER(_VcfPart), ct.c_int,
                                         ct.c_void_p, ct.c_void_p, ct.c_void_p]
        L.qld_mdf_write_part.restype = ct.c_int
        L._vcf_bound = True
    return L


class VcfHeader:
    """A qLD-parse-VCF dataset's header (qld_vcf_read_header)."""

    def __init__(self, path: str, ploidy: int, sample_list=None):
        names = list(sample_list or [])
        arr = (ct.c_char_p * max(len(names), 1))(*[n.encode() for n in names])
        self._h = _VcfHeader()
        _check(_vcf_lib().qld_vcf_read_header(os.fsencode(path), int(ploidy), arr, len(names),
                                              ct.byref(self._h)))
        h = self._h
        self.id = h.id.decode()
        self.path = h.path.decode()
        self.nsamples = h.nsamples
        self.valid = np.ctypeslib.as_array(h.valid, (h.nsamples,)).copy()
        self.valid_count = h.valid_count
        self.K = (h.valid_count + 63) // 64
        self.snip_size = h.snip_size

    def parts(self, path: str) -> list[str]:
        pp = ct.POINTER(ct.c_char_p)()
        n = ct.c_int()
        _check(_vcf_lib().qld_vcf_list_parts(os.fsencode(path), ct.byref(self._h), ct.byref(pp),
                                             ct.byref(n)))
        out = [pp[i].decode() for i in range(n.value)]
        _vcf_lib().qld_vcf_list_free(pp, n.value)
        return out

    def close(self):
        if getattr(self, "_h", None) is not None:
            _vcf_lib().qld_vcf_header_free(ct.byref(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class VcfPart:
    """One part file read and filtered on its fixed fields (qld_vcf_load_part)."""

    def __init__(self, path: str, header: VcfHeader):
        self.path = path
        self._p = _VcfPart()
        _check(_vcf_lib().qld_vcf_load_part(None, os.fsencode(path), ct.byref(header._h),
                                            ct.byref(self._p)))
        p = self._p
        self.text = ct.string_at(p.text, p.bytes)
        self.lines, self.skipped, self.nsites = p.lines, p.skipped, p.nsites
        n = p.nsites
        self.sites = (np.frombuffer(ct.string_at(p.sites, n * VCF_SITE.itemsize), VCF_SITE).copy()
                      if n else np.zeros(0, VCF_SITE))
        self.pos = np.ctypeslib.as_array(p.pos, (n,)).copy() if n else np.zeros(0, np.uint32)
        self.ids = [_vcf_lib().qld_vcf_site_id(ct.byref(p), i).decode() for i in range(n)]

    def write_mdf(self, out_dir: str, header: VcfHeader, words, bc, keep) -> str:
        """The part's MDF file in out_dir (qld_mdf_write_part); returns its path."""
        buf = ct.create_string_buffer(8192)
        _check(_vcf_lib().qld_mdf_part_path(os.fsencode(out_dir), os.fsencode(self.path), buf,
                                            8192))
        words = np.ascontiguousarray(words, np.uint64)
        bc = np.ascontiguousarray(bc, np.uint32)
        keep = np.ascontiguousarray(keep, np.uint8)
        _check(_vcf_lib().qld_mdf_write_part(buf.value, header.id.encode(), ct.byref(self._p),
                                             int(header.K), words.ctypes.data, bc.ctypes.data,
                                             keep.ctypes.data))
        return buf.value.decode()

    def close(self):
        if getattr(self, "_p", None) is not None:
            _vcf_lib().qld_vcf_part_free(None, ct.byref(self._p))
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


VCF2MDF_PATH = os.path.join(_PKG, "qld-vcf2mdf")
