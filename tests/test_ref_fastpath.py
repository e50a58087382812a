"""CPU check of the reference-mode r^2 fast path's arithmetic (the steps of
qld_b200/csrc/epilogue.cuh: ref_factors and r2_reference_ff, restated in C)
against the reference's operation sequence, bit for bit, over 4 million
random pairs.  The GPU parity tests check the device code itself."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "fastpath", "ref_fastpath_check.c")


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_fast_path_matches_reference_sequence(tmp_path):
    exe = str(tmp_path / "ref_fastpath_check")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", exe, SRC, "-lm"], check=True)
    out = subprocess.run([exe, "4000000"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "mismatches 0" in out.stdout
