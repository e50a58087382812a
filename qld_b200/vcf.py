"""qLD-parse-VCF datasets: a header file plus gzip parts of VCF data lines.

Layout (what qLD-parse-VCF writes and qLD-parse-2MDF reads):

* ``<id>_header.vcf.gz`` -- the VCF's meta lines, its ``#CHROM ... FORMAT
  s1 ... sN`` line, then ``<id> snipsPerFile snipSize totalSnips posMin
  posMax`` (src/parser/src/parse_vcf_output.c; read by readHeaderFile,
  src/mdf_extension/src/io.c:148-333).
* ``<id>_<i0>_<i1>_<pos0>_<pos1>.vcf.gz`` -- the first meta line, the
  ``#CHROM`` line, then data lines, each ending in a newline.

``write_dataset`` builds such a directory from data lines; ``site_lines``
makes seeded genotype lines (haploid, phased or unphased diploid, with
missing calls) mixed with lines qLD-parse-2MDF skips or drops, for tests and
benchmarks.
"""
from __future__ import annotations

import gzip
import os

import numpy as np

META = "##fileformat=VCFv4.1"
FIXED = "#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT"


def write_dataset(path: str, lines: list[str], samples: list[str], alignment_id: str = "1",
                  snps_per_file: int = 100, positions=None, level: int = 1) -> str:
    """Write data lines (without newlines) as a qLD-parse-VCF dataset; returns
    the directory with a trailing slash."""
    os.makedirs(path, exist_ok=True)
    chrom = "\t".join([FIXED, *samples])
    if positions is None:
        positions = [int(ln.split(None, 2)[1]) for ln in lines]
    n = len(lines)
    pmin = min(positions) if n else 0
    pmax = max(positions) if n else 0
    with gzip.open(os.path.join(path, f"{alignment_id}_header.vcf.gz"), "wt",
                   compresslevel=level) as f:
        f.write(f"{META}\n##FORMAT=<ID=GT,Number=1,Type=String,Description=\"Genotype\">\n")
        f.write(chrom + "\n")
        f.write(f"{alignment_id} {snps_per_file} {len(samples)} {n} {pmin} {pmax}\n")
    for s0 in range(0, n, snps_per_file):
        s1 = min(n, s0 + snps_per_file)
        name = f"{alignment_id}_{s0 + 1}_{s1}_{positions[s0]}_{positions[s1 - 1]}.vcf.gz"
        with gzip.open(os.path.join(path, name), "wt", compresslevel=level) as f:
            f.write(META + "\n" + chrom + "\n")
            f.write("".join(ln + "\n" for ln in lines[s0:s1]))
    return path.rstrip("/") + "/"


def site_lines(n_sites: int, n_samples: int, seed: int, ploidy: int = 1, phased: bool = True,
               missing: float = 0.0, oddities: bool = True, first_pos: int = 100):
    """Seeded VCF data lines: biallelic SNPs whose genotypes follow per-site
    allele frequencies; with `oddities`, a share of lines that qLD-parse-2MDF
    skips (multi-base REF/ALT, symbolic ALT, failed FILTER, AF=0/1, VT=INDEL,
    no GT in FORMAT) or drops as monomorphic, and INFO/FORMAT variants it
    accepts (AF lists, VT=SNP, GT not first in FORMAT is avoided: qLD mangles
    it)."""
    rng = np.random.default_rng(seed)
    bases = np.array(list("ACGT"))
    lines = []
    pos = first_pos
    for i in range(n_sites):
        pos += int(rng.integers(1, 30))
        ref, alt = rng.choice(bases, 2, replace=False)
        p = float(rng.beta(0.4, 1.2))
        info, filt, fmt = ".", ".", "GT"
        kind = rng.random() if oddities else 1.0
        if kind < 0.03:
            ref = ref + "T"                              # multi-base REF: skipped
        elif kind < 0.05:
            alt = "<DEL>"                                # symbolic: skipped
        elif kind < 0.07:
            filt = "q10"                                 # failed FILTER: skipped
        elif kind < 0.09:
            info = "AF=0;DP=10" if rng.random() < 0.5 else "DP=3;AF=1.0"   # skipped
        elif kind < 0.11:
            info = "VT=INDEL"                            # skipped
        elif kind < 0.13:
            fmt = "DP"                                   # no GT: skipped
        elif kind < 0.16:
            p = 0.0                                      # monomorphic: dropped
        elif kind < 0.20:
            info = f"AF={p:.4f};VT=SNP" if rng.random() < 0.5 else f"DP=7;AF=0,{p:.3f}"
            filt = "PASS"
        elif kind < 0.22:
            fmt = "GT:DP"
        alleles = (rng.random((n_samples, ploidy)) < p).astype(int)
        miss = rng.random((n_samples, ploidy)) < missing
        sep = "|" if phased else "/"
        gts = []
        for s in range(n_samples):
            a = ["." if miss[s, k] else str(alleles[s, k]) for k in range(ploidy)]
            g = sep.join(a)
            if fmt == "GT:DP":
                g += f":{int(rng.integers(1, 60))}"
            elif fmt == "DP":
                g = str(int(rng.integers(1, 60)))
            gts.append(g)
        lines.append("\t".join(["1", str(pos), f"rs{i + 1}", ref, alt, ".", filt, info, fmt,
                                *gts]))
    return lines
