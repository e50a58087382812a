"""Seeded synthetic SNP x haplotype tables in qLD's packed MDF layout.

Layout (qLD ``table_x64``, src/correlator/include/correlate_MEM.h:66-75, packed
by compressSnip_x64, src/correlator/src/snip_processing.c:783-815): one row per
SNP of ``K = ceil(N/64)`` 64-bit words, MSB-first -- sample ``s`` is bit
``63 - s % 64`` of word ``s // 64`` -- with the tail of the last word zero.
The row's popcount is the MDF "BC" field.

The generators stand in for the public datasets the workloads are quoted on
(none ship with qLD beyond one small VCF): they reproduce the shapes, sizes and
allele-frequency distributions of each workload.  Everything is torch so the
large tables are generated directly in device memory; rows are int64 tensors
holding the uint64 bit patterns (``.numpy().view(np.uint64)`` on the host).

* ``iid_table``      independent Bernoulli genotypes, per-SNP frequency drawn
                     from a given distribution (all-pairs workload, batched jobs).
* ``copying_table``  haplotype-copying model: founder haplotypes, recombination
                     blocks inside which every sample copies one founder, and
                     per-site mutation noise (single-region, windowed and
                     resident-chromosome workloads).
"""
from __future__ import annotations

import math

import numpy as np
import torch

def words_for(n_samples: int) -> int:
    return (n_samples + 63) // 64


def pack_bits(bits: torch.Tensor) -> torch.Tensor:
    """(rows, N) bool/uint8 -> (rows, K) int64, MSB-first, zero tail."""
    rows, n = bits.shape
    K = words_for(n)
    dev = bits.device
    if n != K * 64:
        bits = torch.cat([bits.to(torch.uint8),
                          torch.zeros(rows, K * 64 - n, dtype=torch.uint8, device=dev)], 1)
    b = bits.to(torch.int64).view(rows, K, 64)
    shifts = torch.arange(63, -1, -1, device=dev, dtype=torch.int64)
    return (b << shifts).sum(dim=2)  # disjoint bits: sum == OR (wraps into the sign bit)


def unpack_bits(table: torch.Tensor, n: int) -> torch.Tensor:
    rows, K = table.shape
    shifts = torch.arange(63, -1, -1, device=table.device, dtype=torch.int64)
    return ((table.unsqueeze(2) >> shifts) & 1).view(rows, K * 64)[:, :n].to(torch.uint8)


_POP8 = None


def popcount_rows(table: torch.Tensor) -> torch.Tensor:
    """Row popcounts (the BC field) as int64."""
    global _POP8
    if _POP8 is None or _POP8.device != table.device:
        _POP8 = torch.tensor([bin(i).count("1") for i in range(256)], dtype=torch.int64,
                             device=table.device)
    by = table.contiguous().view(torch.uint8).view(table.shape[0], -1).to(torch.int64)
    return _POP8[by].sum(dim=1)


def tail_mask(n: int) -> int:
    """Valid-bit mask of the last word (as a signed int64 value)."""
    r = n % 64
    if r == 0:
        return -1
    v = ((1 << r) - 1) << (64 - r)
    return v - (1 << 64) if v >= (1 << 63) else v


def _rand_words(shape, gen, device) -> torch.Tensor:
    lo = torch.randint(0, 1 << 32, shape, generator=gen, device=device, dtype=torch.int64)
    hi = torch.randint(0, 1 << 32, shape, generator=gen, device=device, dtype=torch.int64)
    return lo | (hi << 32)


def biased_words(shape, p: float, gen, device, digits: int = 10) -> torch.Tensor:
    """Random words whose bits are 1 with probability round(p*2^digits)/2^digits.

    Binary-expansion method: fold random words from the least significant
    digit of p up, OR for a 1 digit and AND for a 0 digit.
    """
    q = int(round(p * (1 << digits)))
    out = torch.zeros(shape, dtype=torch.int64, device=device)
    for i in range(digits):  # digit i (LSB first) of q / 2^digits
        r = _rand_words(shape, gen, device)
        out = (out | r) if (q >> i) & 1 else (out & r)
    return out


def _apply_tail(table: torch.Tensor, n: int) -> torch.Tensor:
    tm = tail_mask(n)
    if tm != -1:
        table[:, -1] &= tm
    return table


def iid_table(m: int, n: int, freq: torch.Tensor, seed: int, device="cpu",
              chunk: int = 4096) -> torch.Tensor:
    """m SNPs x n samples, SNP i Bernoulli(freq[i]) iid over samples."""
    gen = torch.Generator(device=device).manual_seed(seed)
    freq = freq.to(device=device, dtype=torch.float32)
    out = torch.empty(m, words_for(n), dtype=torch.int64, device=device)
    for r0 in range(0, m, chunk):
        r1 = min(m, r0 + chunk)
        u = torch.rand(r1 - r0, n, generator=gen, device=device)
        out[r0:r1] = pack_bits(u < freq[r0:r1, None])
    return out


def uniform_freqs(m, lo, hi, seed, device="cpu"):
    rng = np.random.default_rng(seed + 7919)
    return torch.from_numpy(rng.uniform(lo, hi, m).astype(np.float32)).to(device)


def beta_freqs(m, a, b, seed, device="cpu", clip_min=0.0):
    rng = np.random.default_rng(seed + 104729)
    p = np.clip(rng.beta(a, b, m), clip_min, 1.0).astype(np.float32)
    return torch.from_numpy(p).to(device)


def copying_table(m: int, n: int, founders: int, block_min: int, block_max: int,
                  mut_p: float, freq: torch.Tensor, seed: int, device="cpu") -> torch.Tensor:
    """Haplotype-copying model in packed form.

    SNPs are cut into recombination blocks of block_min..block_max SNPs.  In
    each block every sample copies one founder chosen uniformly; founder f
    carries the ALT allele at SNP s with probability freq[s].  Each bit is
    then flipped with probability mut_p (per-site mutation noise).
    Because each sample copies exactly one founder, the per-founder sample
    masks are disjoint and a row is the SUM of the masks of the founders that
    carry the allele, computed as an exact float64 matmul on 16-bit chunks.
    """
    gen = torch.Generator(device=device).manual_seed(seed)
    K = words_for(n)
    out = torch.empty(m, K, dtype=torch.int64, device=device)
    freq = freq.to(device=device, dtype=torch.float32)
    cuts = []
    s = 0
    while s < m:
        ln = int(torch.randint(block_min, block_max + 1, (1,), generator=gen, device=device))
        cuts.append((s, min(m, s + ln)))
        s += ln
    chunk16 = torch.tensor([0xFFFF], dtype=torch.int64, device=device)
    for (b0, b1) in cuts:
        choice = torch.randint(0, founders, (n,), generator=gen, device=device)
        onehot = choice[None, :] == torch.arange(founders, device=device)[:, None]
        masks = pack_bits(onehot)                                   # (F, K) int64
        m16 = torch.stack([(masks >> (16 * c)) & chunk16 for c in range(4)], dim=2)
        m16 = m16.view(founders, K * 4).to(torch.float64)
        fa = (torch.rand(b1 - b0, founders, generator=gen, device=device)
              < freq[b0:b1, None]).to(torch.float64)
        rows16 = (fa @ m16).round().to(torch.int64).view(b1 - b0, K, 4)
        rows = rows16[..., 0] | (rows16[..., 1] << 16) | (rows16[..., 2] << 32) | (rows16[..., 3] << 48)
        if mut_p > 0:
            rows ^= biased_words(rows.shape, mut_p, gen, device)
        out[b0:b1] = rows
    return _apply_tail(out, n)


# ------------------------------------------------------------ workloads ----

def all_pairs_workload(device="cpu", m=2048, n=4096, seed=1):
    """All-pairs r^2, one region: 2,048 SNPs x 4,096 haploid samples, iid
    Bernoulli genotypes with per-SNP frequency ~ Uniform(0.05, 0.5)."""
    f = uniform_freqs(m, 0.05, 0.5, seed, device)
    return iid_table(m, n, f, seed, device), n


def single_region_workload(device="cpu", m=29_817, n=16_622, seed=2, founders=20):
    """Dataset-shaped single region: 29,817 SNPs x 16,622 haploid sequences,
    frequencies ~ Beta(0.1, 1) clipped to >= 1/16,622, copying model with 20
    founders, blocks of 50-500 SNPs and 1% per-site mutation noise."""
    f = beta_freqs(m, 0.1, 1.0, seed, device, clip_min=1.0 / n)
    return copying_table(m, n, founders, 50, 500, 0.01, f, seed, device), n


def windowed_workload(device="cpu", m=200_000, n=100_000, seed=3, founders=100):
    """Large windowed LD: 200,000 SNPs x 100,000 haplotypes, copying model with
    100 founders (band of 5,000 SNPs is applied by the caller)."""
    f = beta_freqs(m, 0.1, 1.0, seed, device, clip_min=1.0 / n)
    return copying_table(m, n, founders, 50, 500, 0.01, f, seed, device), n


def log_uniform_ints(count, lo, hi, rng):
    u = rng.uniform(0.0, 1.0, count)
    return np.rint(np.exp(math.log(lo) + u * (math.log(hi) - math.log(lo)))).astype(np.int64)
