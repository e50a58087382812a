"""Generate the golden vectors in this directory from the qLD reference itself.

    make -C oracle ref          # builds oracle/_ref/libqldref.so from the qLD sources
    python tests/golden/make_golden.py

qLD ships no known-answer tests, so the golden vectors are the reference's own
outputs on seeded synthetic tables: for every case the counts come from the
reference's gemm() (src/correlator/src/gemm_cpu.c:280-341, after mlt()), r^2
from its get_pairwise_ld_score() (:343-404) and the report text from its
writeResultsHeader()/writeResults() (correlate_IO.c:378-429).  The whole
correlate() task (gemm_cpu.c:420-623) is also run and must write the same
report bytes.  Each case is saved as <name>.npz plus <name>.report.txt.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from qld_b200 import synth  # noqa: E402


def _np(t):
    return t.numpy().view(np.uint64)


def edge_table(n_samples: int) -> np.ndarray:
    """Rows that exercise the epilogue's special cases."""
    rng = np.random.default_rng(99)
    K = synth.words_for(n_samples)
    bits = (rng.random((64, n_samples)) < rng.uniform(0.05, 0.6, (64, 1))).astype(np.uint8)
    bits[0] = 0                      # monomorphic REF: r^2 = 0 by the zero-count rule
    bits[1] = 1                      # monomorphic ALT: 0/0 -> NaN, or inf -> 123.456
    bits[2] = 0
    bits[2, 7] = 1                   # a single ALT sample
    bits[3] = bits[4]                # duplicated rows: r^2 = 1
    bits[5] = 1 - bits[6]            # complementary rows: r^2 = 1
    bits[7] = 1
    bits[7, -1] = 0                  # all but one sample
    t = synth.pack_bits(__import__("torch").from_numpy(bits)).numpy().view(np.uint64)
    assert t.shape == (64, K)
    return t


def cases():
    import torch  # noqa: F401
    t, n = synth.all_pairs_workload(m=500, n=450, seed=11)
    yield "trans_iid", _np(t[:300]), _np(t[300:]), n, 0.02
    t, n = synth.all_pairs_workload(m=257, n=1000, seed=12)
    yield "cis_iid", _np(t), None, n, 0.02
    t, n = synth.all_pairs_workload(m=8, n=64, seed=13)
    yield "tiny", _np(t[:5]), _np(t[5:]), n, 0.0
    yield "edge", edge_table(130), None, 130, 0.0
    f = synth.beta_freqs(96, 0.1, 1.0, 14, clip_min=1.0 / 16622)
    t = synth.copying_table(96, 16622, 20, 50, 500, 0.01, f, 14)
    yield "copying_rare", _np(t), None, 16622, 0.2


def main():
    if not oracle.reference_available():
        raise SystemExit("oracle/_ref/libqldref.so missing: run `make -C oracle ref` first")
    for name, A, B, S, r2limit in cases():
        sym = B is None
        Bx = A if sym else B
        m, n = A.shape[0], Bx.shape[0]
        bcA = oracle.bitcounts(A)
        bcB = oracle.bitcounts(Bx)
        counts = oracle.ref_counts_gemm(A, Bx)                  # (n, m) uint64
        r2 = oracle.ref_ld_score(bcA, bcB, counts, S)           # (n, m) float32
        posA = (np.arange(m, dtype=np.uint32) * 37 + 1001)
        posB = posA if sym else (np.arange(n, dtype=np.uint32) * 53 + 2003)
        idA = [f"rsA{i}" for i in range(m)]
        idB = idA if sym else [f"rsB{i}" for i in range(n)]
        with tempfile.TemporaryDirectory() as td:
            rep = os.path.join(td, "w.txt")
            oracle.ref_write_report(rep, posA, idA, bcA, posB, idB, bcB, S, r2, r2limit,
                                    0 if sym else 1)
            report = open(rep, "rb").read()
            full = os.path.join(td, "c.txt")
            oracle.ref_correlate(full, os.path.join(td, "log"), A, posA, idA, bcA, Bx, posB,
                                 idB, bcB, S, 0 if sym else 1, r2limit)
            if open(full, "rb").read() != report:
                raise SystemExit(f"{name}: correlate() report differs from writeResults()")
        out = dict(A=A, bcA=bcA, posA=posA, S=np.int64(S), r2limit=np.float32(r2limit),
                   symmetric=np.int64(sym), counts=counts.astype(np.uint32), r2_ref=r2)
        if not sym:
            out.update(B=B, bcB=bcB, posB=posB)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        with open(os.path.join(HERE, f"{name}.report.txt"), "wb") as f:
            f.write(report)
        print(f"{name}: m={m} n={n} K={A.shape[1]} S={S} report={len(report)} B")


if __name__ == "__main__":
    main()
