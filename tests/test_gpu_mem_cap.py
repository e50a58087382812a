"""GPU test of an allocation failure, injected through the context's device
memory cap (QLD_OPT_MEM_CAP): a call that would grow the context's buffers
past the cap fails with QLD_ERR_NOMEM before launching anything, and the
same context, with the cap lifted, then computes the task exactly."""
import numpy as np
import pytest

import oracle
from conftest import assert_r2_close, lower_mask
from qld_b200 import api, synth

pytestmark = pytest.mark.gpu


def test_cap_refuses_then_context_recovers():
    t, _ = synth.all_pairs_workload(m=2048, n=4096, seed=51)
    A = t.numpy().view(np.uint64)
    bc = oracle.bitcounts(A)
    c = api.Context(0)
    try:
        c.set_option(api.OPT_MEM_CAP, 4 << 20)        # the r^2 band alone needs 16 MiB
        with pytest.raises(api.QldError) as e:
            c.ld(A, bc, S=4096)
        assert e.value.code == api.ERR_NOMEM and "cap" in str(e.value)
        assert c.stats().counts_launches == 0         # refused before any launch
        c.set_option(api.OPT_MEM_CAP, 0)
        r2, cnt = c.ld(A, bc, S=4096, counts=True)
        want = oracle.counts(A)
        mask = lower_mask(*want.shape)
        assert np.array_equal(cnt[mask], want[mask])
        assert_r2_close(r2, oracle.r2_exact(bc, bc, want, 4096), mask=mask)
        # a cap the held buffers already fit leaves the next call unaffected
        c.set_option(api.OPT_MEM_CAP, 64 << 20)
        r2b = c.ld(A, bc, S=4096)
        assert np.array_equal(r2b[mask].view(np.uint32), r2[mask].view(np.uint32))
        with pytest.raises(api.QldError) as e:
            c.set_option(api.OPT_MEM_CAP, -1)
        assert e.value.code == api.ERR_INVALID
    finally:
        c.close()
