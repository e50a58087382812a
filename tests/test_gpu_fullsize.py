"""Parity at the benchmarked sizes, through the same code bench.py times.

The benchmark's workloads run at their full sizes and their outputs are
checked on samples against the oracle (bench.py's parity helpers):

* single region, 29,817 SNPs x 16,622 haplotypes (K = 260 words, 7,419
  256x240 tiles per launch, about 100 tiles per CTA pair): ~2 B rows from
  every 120-row block, so every output tile -- including the last tiles each
  CTA (pair) walks, through both accumulator buffers and the resumed tile
  list -- is checked, against all 29,817 A rows; counts bit-exact, r^2 within
  1e-6 relative of FP64 (exact mode) or bit-identical to the reference's
  float/double sequence (reference mode); both 4-bit kernels in both modes;
* windowed, 200,000 SNPs x 100,000 haplotypes, band 5,000: one band row per
  240-row block, all its pairs, counts and r^2, in both r^2 modes;
* batched, the 4,096-task mix in one persistent launch: two B rows of every
  task against all its A rows, in both r^2 modes;
* served, the 22 resident chromosomes: a short stream, then sampled queries'
  blocks (three B rows each) and their device summaries.
"""
import pytest
import torch

import bench
from qld_b200 import synth

pytestmark = pytest.mark.gpu


def _args(*extra):
    return bench.parse(["--steps", "1", "--warmup", "1", "--no-e2e", *extra])


@pytest.fixture(scope="module")
def region():
    dev = torch.device("cuda", 0)
    T, S = synth.single_region_workload(device=dev, seed=2)
    Tp, lda = bench.padded(T, dev)
    bc = synth.popcount_rows(T).to(torch.int32)
    out = torch.empty(T.shape[0], T.shape[0], dtype=torch.float32, device=dev)
    yield Tp, lda, bc, T.shape[0], T.shape[1], S, out
    del out, Tp, bc
    torch.cuda.empty_cache()


@pytest.mark.parametrize("mode,sm_pair", [("exact", 0), ("reference", 0), ("exact", 1),
                                          ("reference", 1)])
def test_single_region_full_size(region, mode, sm_pair):
    Tp, lda, bc, m, K, S, out = region
    assert (m, K, S) == (29_817, 260, 16_622)
    args = _args("--r2-mode", mode, "--sm-pair", str(sm_pair))
    ctx = bench.new_context(0, args)
    st = torch.cuda.current_stream()
    try:
        out.fill_(-7.0)
        ctx.ld_device(Tp, bc, m, lda, Tp, bc, m, lda, K, S, True, out, m, stream=st)
        ctx.sync(stream=st)
        assert ctx.stats().last_kernel == 3          # the 4-bit kernel
        res = bench.region_parity(ctx, Tp, bc, m, lda, K, S, out, st, mode, seed=sm_pair)
    finally:
        ctx.close()
    assert res["rows_checked"] >= 490
    assert res["counts_exact"], res
    assert res["rerun_bit_identical"], res
    if mode == "exact":
        assert res["r2_within_tol"] and res["r2_max_rel"] <= 1e-6, res
    else:
        assert res["r2_bit_identical"], res
    assert res["ok"]


@pytest.mark.parametrize("mode", ["exact", "reference"])
def test_windowed_full_size(mode):
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    res = bench.section_windowed(_args("--r2-mode", mode), 0, flush)
    par = res["parity"]
    assert res["config"]["snps"] == 200_000 and res["config"]["haplotypes"] == 100_000
    assert par["rows_checked"] >= 830 and par["counts_exact"], par
    if mode == "exact":
        assert par["r2_max_rel"] <= 1e-6 and par["ok"], par
    else:
        assert par["r2_bit_identical"] and par["ok"], par


@pytest.mark.parametrize("mode", ["exact", "reference"])
def test_batched_full_size(mode):
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    res = bench.section_batched(_args("--r2-mode", mode), 0, flush)
    par = res["parity"]
    assert par["rows_checked"] >= 2 * 4096 - 64, par
    if mode == "exact":
        assert par["r2_max_rel"] <= 1e-6 and par["ok"], par
    else:
        assert par["r2_bit_identical"] and par["ok"], par


def test_served_full_size():
    res = bench.section_served(_args("--queries", "200"), 0)
    assert res["completed"] == 200 and res["failed"] == 0
    par = res["parity"]
    assert par["summaries_match_blocks"] and par["ok"], par
    assert par["r2_max_rel"] <= 1e-6
