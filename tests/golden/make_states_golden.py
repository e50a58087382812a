"""Generate the COUNTSTATES golden reports in tests/golden/states/ from the
qLD reference itself.

    make -C oracle ref          # builds oracle/_ref/qLD-compute-cstates
    python tests/golden/make_states_golden.py

qLD-compute built with -DCOUNTSTATES (src/correlator/Makefile:63) replaces the
r^2 task by countStates_mode() (src/correlator/src/correlate_IO.c:472-516) and
writes writeStateCount()'s report (:430-470).  Each case is an MDF dataset
written from a seeded synthetic table (saved as <name>.npz: the packed table,
positions, sample count, part size and the window flags) and the report the
reference writes for it (<name>.report.txt).
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "states")
sys.path.insert(0, ROOT)

from qld_b200 import mdf, synth  # noqa: E402

BIN = os.path.join(ROOT, "oracle", "_ref", "qLD-compute-cstates")


def table(m: int, n_samples: int, seed: int) -> np.ndarray:
    """Copying-model rows with rare and monomorphic SNPs mixed in, so pairs
    see every number of joint states."""
    f = synth.beta_freqs(m, 0.1, 1.0, seed, clip_min=1.0 / n_samples)
    t = synth.copying_table(m, n_samples, 8, 10, 60, 0.02, f, seed).numpy().view(np.uint64)
    t = t.copy()
    K = t.shape[1]
    rng = np.random.default_rng(seed)
    tail = n_samples % 64
    full = np.uint64(0xFFFFFFFFFFFFFFFF)
    last = full if tail == 0 else np.uint64(((1 << tail) - 1) << (64 - tail))
    t[3] = 0                                        # monomorphic REF
    t[4] = full
    t[4, K - 1] = last                              # monomorphic ALT
    t[5] = 0
    t[5, rng.integers(K)] = np.uint64(1) << np.uint64(63 - rng.integers(min(64, n_samples)))
    return t


CASES = [
    ("states_single", 160, 300, 31, []),
    ("states_windows", 160, 300, 31, ["-posWmin1", "1000", "-posWmax1", "1990",
                                      "-posWmin2", "1500", "-posWmax2", "2590"]),
    ("states_k1", 90, 50, 32, []),
]


def main() -> None:
    os.makedirs(OUT, exist_ok=True)
    for name, m, n_samples, seed, flags in CASES:
        t = table(m, n_samples, seed)
        pos = 1000 + 10 * np.arange(m)
        with tempfile.TemporaryDirectory() as tmp:
            d = mdf.write_dataset(os.path.join(tmp, "d"), t, n_samples, positions=pos,
                                  snps_per_file=40)
            out = os.path.join(tmp, "out.txt")
            subprocess.run([BIN, "-input", d, "-ploidy", "haploid", "-mdf", *flags,
                            "-output", out], cwd=tmp, check=True, capture_output=True)
            report = open(out, "rb").read()
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), table=t, positions=pos,
                            n_samples=n_samples, snps_per_file=40, flags=np.array(flags))
        with open(os.path.join(OUT, f"{name}.report.txt"), "wb") as f:
            f.write(report)
        print(name, len(report), "bytes")


if __name__ == "__main__":
    main()
