"""GPU tests of the host-table uploads of the host-buffer calls: tables with
an odd word count K go up through a staging buffer, 8,192 rows at a time,
and a kernel re-pitches them to the devices' even row pitch.  Tables larger
than one staging chunk, in both region forms and through the band and
report-filter calls, must give the oracle's counts exactly."""
import numpy as np
import pytest

import oracle
from conftest import lower_mask
from qld_b200 import api, synth

pytestmark = pytest.mark.gpu

S_ODD = 130            # K = 3 words per row


def _table(m, seed):
    t, _ = synth.all_pairs_workload(m=m, n=S_ODD, seed=seed)
    A = t.numpy().view(np.uint64)
    assert A.shape[1] % 2 == 1
    return A, oracle.bitcounts(A)


def test_single_region_past_one_staging_chunk():
    A, bc = _table(9000, 61)
    c = api.Context(0)
    try:
        _, cnt = c.ld(A, bc, S=S_ODD, counts=True)
    finally:
        c.close()
    want = oracle.counts(A)
    mask = lower_mask(*want.shape)
    assert np.array_equal(cnt[mask], want[mask])


def test_two_regions_past_one_staging_chunk():
    A, bcA = _table(8500, 62)
    B, bcB = _table(300, 63)
    c = api.Context(0)
    try:
        _, cnt = c.ld(A, bcA, B, bcB, S=S_ODD, counts=True)
    finally:
        c.close()
    assert np.array_equal(cnt, oracle.counts(A, B))


def test_band_past_one_staging_chunk():
    A, bc = _table(8300, 64)
    band = 40
    c = api.Context(0)
    try:
        _, cnt = c.ld_band(A, bc, S=S_ODD, band=band, counts=True)
    finally:
        c.close()
    full = oracle.counts(A)
    m = A.shape[0]
    for d in (0, 17, band - 1):
        i = np.arange(m - 1 - d)
        assert np.array_equal(cnt[i, d], full[i + 1 + d, i])


def test_report_filter_past_one_staging_chunk():
    A, bc = _table(8400, 65)
    c = api.Context(0)
    try:
        dense = c.ld(A, bc, S=S_ODD)
        mask, off, val = c.ld_hits(A, bc, S=S_ODD, r2limit=0.3)
    finally:
        c.close()
    n, m = dense.shape
    keep = (np.arange(m)[None, :] > np.arange(n)[:, None]) & (dense >= 0.3) & (dense < 100)
    assert off[-1] == int(keep.sum())
    assert np.array_equal(val, dense[keep])
