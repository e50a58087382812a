"""The drop-in, end to end: qLD-compute's own CLI, MDF reader, task queue,
threads and report writer, with correlate() computed on the B200.

oracle/_ref/qLD-compute is the reference built from its sources (fallback
counts path); oracle/_ref/qLD-compute-cuda is the same objects with
correlate() routed to correlate_cuda() (qld_b200/host/correlate_cuda.c) when
QLD_CUDA is set.  Both run on the same MDF datasets; the reports must be
byte-identical (reference-semantics r^2, the default of correlate_cuda()).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from qld_b200 import mdf, synth

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref", "qLD-compute")
CUDA = os.path.join(ROOT, "oracle", "_ref", "qLD-compute-cuda")


def _run(binary, args, cwd, cuda):
    env = dict(os.environ)
    env.pop("QLD_CUDA", None)
    if cuda:
        env["QLD_CUDA"] = "1"
    os.makedirs(cwd, exist_ok=True)
    r = subprocess.run([binary, *args], cwd=cwd, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r


def _reports(tmp, name, args):
    outs = []
    for tag, binary, cuda in (("ref", REF, False), ("cuda", CUDA, True)):
        d = os.path.join(tmp, f"{name}_{tag}")
        _run(binary, [*args, "-output", os.path.join(d, "out.txt")], d, cuda)
        files = sorted(f for f in os.listdir(d) if f.startswith("out"))
        outs.append({f: open(os.path.join(d, f), "rb").read() for f in files})
    return outs


@pytest.fixture(scope="module")
def dataset(tmp_path_factory):
    if not (os.path.exists(REF) and os.path.exists(CUDA)):
        pytest.skip("oracle/_ref binaries not built")
    tmp = str(tmp_path_factory.mktemp("mdf"))
    f = synth.beta_freqs(1500, 0.1, 1.0, 41, clip_min=1.0 / 2500)
    t = synth.copying_table(1500, 2500, 20, 50, 300, 0.01, f, 41)
    T = t.numpy().view(np.uint64)
    d1 = mdf.write_dataset(os.path.join(tmp, "d1"), T[:900], 2500, snps_per_file=200)
    pos2 = 100_000 + 7 * np.arange(600)
    d2 = mdf.write_dataset(os.path.join(tmp, "d2"), T[900:], 2500, positions=pos2,
                           snps_per_file=250, alignment_id="chr2")
    # same positions as d1's first 600 SNPs, different genotypes
    d3 = mdf.write_dataset(os.path.join(tmp, "d3"), T[900:], 2500, snps_per_file=150,
                           alignment_id="chr3")
    return tmp, d1, d2, d3


def test_single_region_report_identical(dataset):
    tmp, d1, _, _ = dataset
    ref, cuda = _reports(tmp, "single", ["-input", d1, "-ploidy", "haploid", "-mdf",
                                         "-r2limit", "0"])
    assert ref and ref == cuda
    assert sum(len(v) for v in ref.values()) > 100_000


def test_two_windows_report_identical(dataset):
    tmp, d1, _, _ = dataset
    ref, cuda = _reports(tmp, "windows", ["-input", d1, "-ploidy", "haploid", "-mdf",
                                          "-posWmin1", "1000", "-posWmax1", "4000",
                                          "-posWmin2", "3000", "-posWmax2", "9000",
                                          "-r2limit", "0.01"])
    assert ref and ref == cuda


def test_two_inputs_report_identical(dataset):
    """Two inputs need explicit windows: without them qLD-compute searches
    the second input over the first header's positions and never stops
    (findFiles, correlate_IO.c:312-375)."""
    tmp, d1, d2, _ = dataset
    ref, cuda = _reports(tmp, "inputs", ["-input", d1, "-input2", d2, "-ploidy", "haploid",
                                         "-mdf", "-posWmin1", "1000", "-posWmax1", "9990",
                                         "-posWmin2", "100000", "-posWmax2", "104193",
                                         "-r2limit", "0.005"])
    assert ref and ref == cuda


def test_split_file_inputs_report_identical(dataset):
    """Two inputs over the same window: qLD sets posWset2 = 0 with a
    different table B (load_balancer.c:262-268), which readTable_x64() then
    reads only up to each part's column-name line (correlate_IOx64.c:444):
    correlate() gets an empty table B and both reports are the header alone."""
    tmp, d1, _, d3 = dataset
    ref, cuda = _reports(tmp, "split", ["-input", d1, "-input2", d3, "-ploidy", "haploid",
                                        "-mdf", "-posWmin1", "1000", "-posWmax1", "6990",
                                        "-posWmin2", "1000", "-posWmax2", "6990",
                                        "-r2limit", "0"])
    assert ref and ref == cuda


def test_threads_and_input_list_identical(dataset):
    tmp, d1, _, _ = dataset
    lst = os.path.join(tmp, "list.csv")
    with open(lst, "w") as f:
        f.write(f"{d1},1000,3000,{d1},1000,3000\n")
        f.write(f"{d1},1000,5000,{d1},6000,9990\n")
        f.write(f"{d1},2000,4000,{d1},2000,6000\n")
    ref, cuda = _reports(tmp, "list", ["-inputList", lst, "-ploidy", "haploid", "-mdf",
                                       "-threads", "2", "-competing", "-r2limit", "0.01"])
    assert len(ref) >= 3 and ref == cuda
