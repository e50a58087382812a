"""GPU tests of the COUNTSTATES mode: the kernel's state values equal the
oracle's restatement of countStates_mode() byte for byte, and qld-ld
-countstates writes the reference's COUNTSTATES reports."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT
from qld_b200 import api, host_api, mdf, synth
from test_oracle import _states_cases, load_states_golden

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref", "qLD-compute-cstates")


def _table(m, n_samples, seed, sparse=False):
    f = synth.beta_freqs(m, 0.1, 1.0, seed, clip_min=1.0 / n_samples)
    t = synth.copying_table(m, n_samples, 8, 10, 60, 0.02, f, seed).numpy().view(np.uint64).copy()
    if sparse:   # mostly-zero words: the fold then sees few states per word
        t &= np.uint64(0x8000000100000001)
    return t


@pytest.mark.parametrize("n_samples", [40, 64, 300, 1024, 1090, 2110])
@pytest.mark.parametrize("sym", [True, False])
def test_states_equal_oracle(gpu_ctx, n_samples, sym):
    T = _table(400, n_samples, 3 + n_samples, sparse=n_samples == 1090)
    if sym:
        A, B = T[:260], None
    else:
        A, B = T[:130], T[130:400]
    got = gpu_ctx.count_states(A, B)
    want = oracle.count_states(A, B)
    if sym:
        keep = np.arange(A.shape[0])[None, :] >= np.arange(A.shape[0])[:, None]
        assert np.array_equal(got[keep], want[keep])
    else:
        assert np.array_equal(got, want)
    assert set(np.unique(want)) <= {1, 2, 3, 4}


@pytest.mark.parametrize("m,n", [(1, 1), (129, 3), (3, 257), (300, 700)])
def test_states_ragged_and_streamed(gpu_ctx, m, n):
    gpu_ctx.set_option(api.OPT_BAND_ROWS, 256)
    try:
        T = _table(m + n, 777, 11)
        A, B = T[:m], T[m:]
        assert np.array_equal(gpu_ctx.count_states(A, B), oracle.count_states(A, B))
    finally:
        gpu_ctx.set_option(api.OPT_BAND_ROWS, 4096)


def test_states_device_form(gpu_ctx):
    import torch
    T = _table(500, 900, 13)
    m, K = T.shape
    lda = K + (K & 1)
    dev = torch.zeros((m, lda), dtype=torch.int64, device="cuda")
    dev[:, :K] = torch.from_numpy(T.view(np.int64)).cuda()
    out = torch.full((m, m + 16), 255, dtype=torch.uint8, device="cuda")
    gpu_ctx.count_states_device(dev, m, lda, dev, m, lda, K, True, out, m + 16)
    gpu_ctx.sync()
    got = out.cpu().numpy()[:, :m]
    want = oracle.count_states(T)
    keep = np.arange(m)[None, :] >= np.arange(m)[:, None]
    assert np.array_equal(got[keep], want[keep])
    assert np.all(out.cpu().numpy()[:, m:] == 255)        # nothing past lds's used part


def _run(args, cwd, binary=None):
    os.makedirs(cwd, exist_ok=True)
    r = subprocess.run([binary or host_api.CLI_PATH, *args], cwd=cwd, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.parametrize("name", _states_cases())
def test_cli_states_match_golden(tmp_path, name):
    if not os.path.exists(host_api.CLI_PATH):
        pytest.skip("qld-ld not built")
    g = load_states_golden(name)
    z = g["z"]
    d = mdf.write_dataset(str(tmp_path / "d"), z["table"], int(z["n_samples"]),
                          positions=z["positions"], snps_per_file=int(z["snps_per_file"]))
    out = tmp_path / "out.txt"
    _run(["-input", d, "-ploidy", "haploid", "-mdf", "-countstates", "-threads", "3",
          *g["flags"], "-output", str(out)], str(tmp_path))
    assert out.read_bytes() == g["report"]


def test_cli_states_match_reference_two_inputs(tmp_path):
    if not (os.path.exists(REF) and os.path.exists(host_api.CLI_PATH)):
        pytest.skip("qLD-compute-cstates or qld-ld not built")
    T = _table(700, 500, 17)
    d1 = mdf.write_dataset(str(tmp_path / "d1"), T[:400], 500, snps_per_file=90)
    d2 = mdf.write_dataset(str(tmp_path / "d2"), T[400:], 500,
                           positions=50_000 + 3 * np.arange(300), snps_per_file=70,
                           alignment_id="chr9")
    args = ["-input", d1, "-input2", d2, "-ploidy", "haploid", "-mdf", "-posWmin1", "1500",
            "-posWmax1", "4990", "-posWmin2", "50000", "-posWmax2", "50897"]
    outs = []
    for tag, binary, extra in (("ref", REF, []), ("qld", None, ["-countstates"])):
        o = tmp_path / f"{tag}.txt"
        _run([*args, *extra, "-output", str(o)], str(tmp_path / tag), binary)
        outs.append(o.read_bytes())
    assert outs[0] == outs[1] and outs[0].count(b"\n") > 10_000
