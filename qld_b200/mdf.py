"""qLD MDF datasets: a directory with a header and part files.

Layout (what qLD-compute's -mdf mode reads):

* ``<id>_header.vcf.gz`` -- gzip text: a first line, the VCF ``#CHROM ...
  FORMAT s1 ... sN`` line (its N sample names set the valid-sample count),
  then ``<id> snipsPerFile snipSize totalSnips posMin posMax``
  (readHeaderFile, src/correlator/src/correlate_IO.c:79-259; written by
  qLD-parse-VCF, src/parser/src/parse_vcf_output.c:20-71).
* ``<id>_<i0>_<i1>_<pos0>_<pos1>.mdf`` -- SNPs i0..i1 (1-based) at positions
  pos0..pos1; every part holds snipsPerFile SNPs except the last
  (findFiles, correlate_IO.c:294-376).  Body: ``##fileformat=MDFv0.1``,
  ``##SNPs:<n>``, ``#CHROM\\tPOS\\tID\\tBC\\tcompSNP_0...``, then one row per
  SNP ``CHROM\\tPOS\\tID\\tBC\\tw0\\tw1...`` with the packed 64-bit words in
  decimal and no newline after the last row (qLD-parse-2MDF,
  src/mdf_extension/src/process_data.c:447-460; read by writeMDF_x64,
  correlate_IOx64.c:27-122).

``write_dataset`` builds such a directory from a packed table (tests and
benchmarks run the reference's own qLD-compute on it); ``read_region`` parses
one back with qLD-compute's window rule (keep rows with posWmin <= POS <=
posWmax, correlate_IOx64.c:423-425).
"""
from __future__ import annotations

import glob
import gzip
import os
import re

import numpy as np


def write_dataset(path: str, table: np.ndarray, n_samples: int, positions=None, ids=None,
                  alignment_id: str = "chr1", snps_per_file: int = 1000) -> str:
    """Write a packed (rows, K) uint64 table as an MDF dataset; returns the
    directory path with its trailing slash (qLD-compute concatenates file
    names to it)."""
    table = np.ascontiguousarray(table).view(np.uint64)
    m, K = table.shape
    os.makedirs(path, exist_ok=True)
    if positions is None:
        positions = 1000 + 10 * np.arange(m, dtype=np.int64)
    positions = np.asarray(positions, dtype=np.int64)
    if np.any(np.diff(positions) <= 0):
        raise ValueError("positions must increase")
    if ids is None:
        ids = [f"rs{i + 1}" for i in range(m)]
    bc = np.zeros(m, np.int64)
    tbl8 = table.view(np.uint8).reshape(m, K * 8)
    pop8 = np.array([bin(i).count("1") for i in range(256)], np.int64)
    bc = pop8[tbl8].sum(axis=1)
    samples = "\t".join(f"s{i + 1}" for i in range(n_samples))
    with gzip.open(os.path.join(path, f"{alignment_id}_header.vcf.gz"), "wt") as f:
        f.write("##fileformat=VCFv4.2\n")
        f.write("#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\t" + samples + "\n")
        f.write(f"{alignment_id} {snps_per_file} {n_samples} {m} {int(positions[0])} "
                f"{int(positions[-1])}\n")
    colhdr = "#CHROM\tPOS\tID\tBC" + "".join(f"\tcompSNP_{k}" for k in range(K))
    for s0 in range(0, m, snps_per_file):
        s1 = min(m, s0 + snps_per_file)
        name = f"{alignment_id}_{s0 + 1}_{s1}_{int(positions[s0])}_{int(positions[s1 - 1])}.mdf"
        lines = [f"##fileformat=MDFv0.1\n##SNPs:{s1 - s0}\n{colhdr}"]
        for r in range(s0, s1):
            words = "\t".join(str(int(w)) for w in table[r])
            lines.append(f"\n{alignment_id}\t{int(positions[r])}\t{ids[r]}\t{int(bc[r])}\t{words}")
        with open(os.path.join(path, name), "w") as f:
            f.write("".join(lines))
    return path.rstrip("/") + "/"


_PART = re.compile(r"^(?P<id>[^_]+)_(?P<i0>\d+)_(?P<i1>\d+)_(?P<p0>-?\d+)_(?P<p1>-?\d+)\.mdf$")


def read_header(path: str):
    """(alignment_id, sample names, snipsPerFile, snipSize, totalSnips, posMin, posMax)."""
    hdr = sorted(glob.glob(os.path.join(path, "*header*")))
    if not hdr:
        raise FileNotFoundError(f"no header file in {path}")
    aid = os.path.basename(hdr[0]).split("_")[0]
    samples = None
    info = None
    with gzip.open(hdr[0], "rt") as f:
        lines = f.read().split("\n")
    for i, ln in enumerate(lines):
        if ln.startswith("#CHROM"):
            samples = ln.split("\t")[9:]
            info = lines[i + 1].split()
            break
    if info is None:
        raise ValueError("header has no #CHROM line")
    if info[0] != aid:
        raise ValueError("header id differs from its file name")
    return (aid, samples, int(info[1]), int(info[2]), int(info[3]), int(info[4]), int(info[5]))


def read_region(path: str, pos_min=None, pos_max=None):
    """Rows with pos_min <= POS <= pos_max as (table, bc, pos, ids)."""
    aid, samples, spf, snip_size, total, pmin, pmax = read_header(path)
    pos_min = pmin if pos_min is None else pos_min
    pos_max = pmax if pos_max is None else pos_max
    K = (len(samples) + 63) // 64
    parts = []
    for fn in os.listdir(path):
        mt = _PART.match(fn)
        if mt and mt.group("id") == aid:
            parts.append((int(mt.group("i0")), fn))
    rows, bcs, poss, ids = [], [], [], []
    for _, fn in sorted(parts):
        with open(os.path.join(path, fn)) as f:
            for ln in f.read().split("\n")[3:]:
                fields = ln.split("\t")
                if len(fields) < 4:
                    continue
                pos = int(fields[1])
                if pos_min <= pos <= pos_max:
                    words = [int(w) for w in fields[4:4 + K]]   # words past K: ignored
                    rows.append(words + [0] * (K - len(words)))
                    bcs.append(int(fields[3]))
                    poss.append(pos)
                    ids.append(fields[2])
    table = np.array(rows, dtype=np.uint64).reshape(len(rows), K)
    return table, np.array(bcs, np.uint32), np.array(poss, np.uint32), ids, snip_size
