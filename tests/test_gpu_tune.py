"""GPU tests of the autotuner (qld_cuda_autotune, qld_cuda_tune_save/load):
it picks a kernel that is exact for the shape, the automatic choice then uses
that kernel for tasks of the shape class with unchanged results, and the
persisted table round-trips.  Each test uses contexts of its own, so the
tuning table never reaches the other tests' shared context."""
import numpy as np
import pytest

import oracle
from conftest import assert_r2_close, lower_mask
from qld_b200 import api, synth

pytestmark = pytest.mark.gpu


@pytest.fixture
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def _task(m, N, seed):
    t, _ = synth.all_pairs_workload(m=m, n=N, seed=seed)
    A = t.numpy().view(np.uint64)
    return A, oracle.bitcounts(A)


def _check_auto(c, A, bc, N, want_kernel):
    r2, cnt = c.ld(A, bc, S=N, counts=True)
    assert c.stats().last_kernel == want_kernel
    want = oracle.counts(A)
    mask = lower_mask(*want.shape)
    assert np.array_equal(cnt[mask], want[mask])
    assert_r2_close(r2, oracle.r2_exact(bc, bc, want, N), mask=mask)


def test_autotune_choice_is_used_by_auto(ctx):
    st0 = ctx.stats(reset=False)
    k, opt, ms = ctx.autotune(1024, 1024, 64, True)
    assert k in (api.KERNEL_POPC, api.KERNEL_MMA, api.KERNEL_FP4) and ms > 0
    assert opt in {api.KERNEL_POPC: (0,), api.KERNEL_MMA: (128, 256), api.KERNEL_FP4: (1, 2)}[k]
    # the tuner's own launches do not show in the caller's statistics
    assert ctx.stats().counts_launches == st0.counts_launches
    A, bc = _task(1100, 4200, 5)          # K = 66 words: same shape class as (1024, 64)
    _check_auto(ctx, A, bc, 4200, k)


def test_autotune_past_the_int8_limit(ctx):
    k, opt, ms = ctx.autotune(600, 500, 2100, False)   # 134,400 samples: no int8 candidate
    assert k in (api.KERNEL_POPC, api.KERNEL_FP4) and ms > 0


def test_table_round_trip_and_forced_entries(ctx, tmp_path):
    # log2 700 = 9, log2 40 = 5, single region: first the int8 kernel, 128-row tiles
    path = tmp_path / "tune.txt"
    path.write_text("qld-tune 1\n9 9 5 1 2 128 0.5\n")
    ctx.tune_load(str(path))
    A, bc = _task(700, 2500, 7)            # K = 40 words
    _check_auto(ctx, A, bc, 2500, api.KERNEL_MMA)
    # a later load overrides the entry; untuned classes keep the built-in rule
    path.write_text("qld-tune 1\n9 9 5 1 1 0 0.9\n")
    ctx.tune_load(str(path))
    _check_auto(ctx, A, bc, 2500, api.KERNEL_POPC)
    A2, bc2 = _task(300, 2500, 8)
    _check_auto(ctx, A2, bc2, 2500, api.KERNEL_FP4)
    # save, then load into a fresh context
    out = tmp_path / "saved.txt"
    ctx.tune_save(str(out))
    lines = out.read_text().split("\n")
    assert lines[0] == "qld-tune 1" and lines[1].startswith("9 9 5 1 1 0 ")
    c2 = api.Context(0)
    try:
        c2.tune_load(str(out))
        _check_auto(c2, A, bc, 2500, api.KERNEL_POPC)
    finally:
        c2.close()


def test_bad_table_is_rejected_and_changes_nothing(ctx, tmp_path):
    bad = tmp_path / "bad.txt"
    bad.write_text("qld-tune 1\n9 9 5 1 1 0 0.9\n9 9 5 1 7 0 0.9\n")   # kernel 7 does not exist
    with pytest.raises(api.QldError) as e:
        ctx.tune_load(str(bad))
    assert e.value.code == api.ERR_INVALID
    A, bc = _task(700, 2500, 7)
    _check_auto(ctx, A, bc, 2500, api.KERNEL_FP4)
    bad.write_text("not a table\n")
    with pytest.raises(api.QldError):
        ctx.tune_load(str(bad))


def test_entries_are_per_r2_mode(ctx, tmp_path):
    """An entry tuned in reference mode steers only reference-mode calls."""
    path = tmp_path / "tune.txt"
    path.write_text("qld-tune 1\n9 9 5 5 1 0 0.9\n")      # kind 1 + 4: reference mode
    ctx.tune_load(str(path))
    A, bc = _task(700, 2500, 7)
    _check_auto(ctx, A, bc, 2500, api.KERNEL_FP4)         # exact mode: untuned
    ctx.set_option(api.OPT_R2_MODE, api.R2_REFERENCE)
    try:
        r2, cnt = ctx.ld(A, bc, S=2500, counts=True)
        assert ctx.stats().last_kernel == api.KERNEL_POPC
        want = oracle.counts(A)
        mask = lower_mask(*want.shape)
        assert np.array_equal(cnt[mask], want[mask])
        ref = oracle.r2_reference(bc, bc, want, 2500, fma_contract=False)
        assert np.array_equal(r2[mask].view(np.uint32), ref[mask].view(np.uint32))
    finally:
        ctx.set_option(api.OPT_R2_MODE, api.R2_EXACT)
