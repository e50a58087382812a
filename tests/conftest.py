import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built CUDA library")
    config.addinivalue_line("markers", "slow: full-size workload")
    # A NaN or garbage value reaching a numeric comparison is a test bug.
    config.addinivalue_line("filterwarnings", "error::RuntimeWarning")


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    g = {k: z[k] for k in z.files}
    g["symmetric"] = bool(g["symmetric"])
    g["S"] = int(g["S"])
    g["r2limit"] = float(g["r2limit"])
    if g["symmetric"]:
        g["B"], g["bcB"], g["posB"] = g["A"], g["bcA"], g["posA"]
    with open(os.path.join(GOLDEN, f"{name}.report.txt"), "rb") as f:
        g["report"] = f.read()
    g["idA"] = [f"rsA{i}" for i in range(g["A"].shape[0])]
    g["idB"] = g["idA"] if g["symmetric"] else [f"rsB{i}" for i in range(g["B"].shape[0])]
    return g


def lower_mask(n, m):
    """Entries (i over B, j over A) with j >= i: the single-region triangle."""
    i = np.arange(n)[:, None]
    j = np.arange(m)[None, :]
    return j >= i


def assert_r2_close(got, want64, rtol=1e-6, mask=None):
    """FP32 r^2 against the FP64 oracle: relative tolerance 1e-6, special
    values (0, NaN, the 123.456 sentinel) exactly.  Entries outside `mask`
    are unspecified (the single-region triangle's other half holds whatever
    the output buffer held) and are dropped before any arithmetic.
    Returns (max, mean) relative error over the compared nonzero values."""
    got = np.asarray(got)
    want = np.asarray(want64)
    if mask is not None:
        got, want = got[mask], want[mask]
    got = got.astype(np.float64)
    want = want.astype(np.float64)
    nan_w = np.isnan(want)
    assert np.array_equal(nan_w, np.isnan(got)), "NaN pattern differs"
    g, w = got[~nan_w], want[~nan_w]
    sent = w == 123.456
    assert np.all(np.abs(g[sent] - 123.456) < 1e-4), "sentinel differs"
    g, w = g[~sent], w[~sent]
    zero = w == 0
    assert np.all(g[zero] == 0), "exact zeros differ"
    rel = np.abs(g[~zero] - w[~zero]) / np.abs(w[~zero])
    if rel.size:
        assert rel.max() <= rtol, f"max relative error {rel.max():.3e} > {rtol}"
    return float(rel.max()) if rel.size else 0.0, float(rel.mean()) if rel.size else 0.0


@pytest.fixture(scope="session")
def gpu_ctx():
    from qld_b200 import api
    ctx = api.Context(0)
    yield ctx
    ctx.close()


@pytest.fixture(autouse=True)
def _reset_gpu_ctx_options(request):
    """Tests share one context: each starts from its default options, whatever
    the previous test set (kernel, tiles, SM pairs, r^2 mode, band rows)."""
    if "gpu_ctx" in request.fixturenames:
        from qld_b200 import api
        ctx = request.getfixturevalue("gpu_ctx")
        for opt, val in ((api.OPT_KERNEL, api.KERNEL_AUTO), (api.OPT_MMA_TILE, 0),
                         (api.OPT_SM_PAIR, 0), (api.OPT_R2_MODE, api.R2_EXACT),
                         (api.OPT_BAND_ROWS, 4096)):
            ctx.set_option(opt, val)
    yield
