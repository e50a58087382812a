"""qld-ld end to end on the B200: MDF datasets in, qLD's report out.

The reports must be byte-identical to those of qLD-compute built from its
sources (oracle/_ref/qLD-compute, counts fallback path) on the same
datasets and flags; -r2mode exact is checked value by value against the
FP64 oracle."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT
from qld_b200 import host_api, mdf, synth

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref", "qLD-compute")


def _run(args, cwd, binary):
    os.makedirs(cwd, exist_ok=True)
    env = dict(os.environ)
    env.pop("QLD_CUDA", None)
    r = subprocess.run([binary, *args], cwd=cwd, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r


def _reports(tmp, name, args, threads=4):
    outs = []
    for tag, binary, extra in (("ref", REF, []), ("qld", host_api.CLI_PATH,
                                                  ["-threads", str(threads)])):
        d = os.path.join(tmp, f"{name}_{tag}")
        _run([*args, *extra, "-output", os.path.join(d, "out.txt")], d, binary)
        files = sorted(f for f in os.listdir(d) if f.startswith("out"))
        outs.append({f: open(os.path.join(d, f), "rb").read() for f in files})
    return outs


@pytest.fixture(scope="module")
def dataset(tmp_path_factory):
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/qLD-compute not built")
    if not os.path.exists(host_api.CLI_PATH):
        pytest.skip("qld-ld not built")
    tmp = str(tmp_path_factory.mktemp("cli"))
    f = synth.beta_freqs(1500, 0.1, 1.0, 43, clip_min=1.0 / 2500)
    t = synth.copying_table(1500, 2500, 20, 50, 300, 0.01, f, 43)
    T = t.numpy().view(np.uint64)
    d1 = mdf.write_dataset(os.path.join(tmp, "d1"), T[:900], 2500, snps_per_file=200)
    pos2 = 100_000 + 7 * np.arange(600)
    d2 = mdf.write_dataset(os.path.join(tmp, "d2"), T[900:], 2500, positions=pos2,
                           snps_per_file=250, alignment_id="chr2")
    d3 = mdf.write_dataset(os.path.join(tmp, "d3"), T[900:], 2500, snps_per_file=150,
                           alignment_id="chr3")
    return tmp, d1, d2, d3, T


def test_single_region(dataset):
    tmp, d1, _, _, _ = dataset
    ref, qld = _reports(tmp, "single", ["-input", d1, "-ploidy", "haploid", "-mdf",
                                        "-r2limit", "0"])
    assert ref and ref == qld
    assert sum(len(v) for v in ref.values()) > 100_000


def test_default_limit_and_windows(dataset):
    tmp, d1, _, _, _ = dataset
    ref, qld = _reports(tmp, "windows", ["-input", d1, "-ploidy", "haploid", "-mdf",
                                         "-posWmin1", "1000", "-posWmax1", "4000",
                                         "-posWmin2", "3000", "-posWmax2", "9000"])
    assert ref and ref == qld


def test_out_of_range_windows_clamp(dataset):
    tmp, d1, _, _, _ = dataset
    ref, qld = _reports(tmp, "clamp", ["-input", d1, "-ploidy", "haploid", "-mdf",
                                       "-posWmin1", "-5", "-posWmax1", "5000",
                                       "-posWmin2", "7000", "-posWmax2", "99999999",
                                       "-r2limit", "0.02"])
    assert ref and ref == qld


def test_two_inputs(dataset):
    tmp, d1, d2, _, _ = dataset
    ref, qld = _reports(tmp, "inputs", ["-input", d1, "-input2", d2, "-ploidy", "haploid",
                                        "-mdf", "-posWmin1", "1000", "-posWmax1", "9990",
                                        "-posWmin2", "100000", "-posWmax2", "104193",
                                        "-r2limit", "0.005"])
    assert ref and ref == qld


def test_split_file_rule(dataset):
    """Two inputs over one window: qLD sets posWset2 = 0 (load_balancer.c:262-268)
    and then reads table B only up to each part's column-name line
    (correlate_IOx64.c:444), so its report is the header line alone."""
    tmp, d1, _, d3, _ = dataset
    ref, qld = _reports(tmp, "split", ["-input", d1, "-input2", d3, "-ploidy", "haploid",
                                       "-mdf", "-posWmin1", "1000", "-posWmax1", "6990",
                                       "-posWmin2", "1000", "-posWmax2", "6990",
                                       "-r2limit", "0"])
    assert ref and ref == qld
    assert ref["out.txt"].count(b"\n") == 1


@pytest.fixture(scope="module")
def list_reports(dataset):
    tmp, d1, d2, _, _ = dataset
    lst = os.path.join(tmp, "list2.csv")
    with open(lst, "w") as f:
        f.write(f"{d1},1000,3000,{d1},1000,3000\n")
        f.write("not,a,valid,line\n")
        f.write(f"{d1},1000,5000,{d1},6000,9990\n")
        f.write(f"{d1},2000,4000,{d2},100000,103000\n")
        f.write(f"{d1},5000,4000,{d1},2000,6000\n")
    outs = []
    for tag, binary, extra in (("ref", REF, ["-threads", "2", "-competing"]),
                               ("qld", host_api.CLI_PATH, ["-threads", "3", "-competing"])):
        d = os.path.join(tmp, f"list2_{tag}")
        _run(["-inputList", lst, "-ploidy", "haploid", "-mdf", "-r2limit", "0.01", *extra,
              "-output", os.path.join(d, "out.txt")], d, binary)
        outs.append({f: open(os.path.join(d, f), "rb").read()
                     for f in sorted(os.listdir(d)) if f.startswith("out")})
    return outs


def test_input_list_identical(list_reports):
    ref, qld = list_reports
    assert sorted(ref) == ["out_1.txt", "out_3.txt", "out_4.txt"]
    assert ref == qld


def test_host_filter_matches(dataset):
    """-filter host (dense r^2 back, filtered by report.c) writes the same bytes."""
    tmp, d1, d2, _, _ = dataset
    for name, args in (("hf1", ["-input", d1, "-r2limit", "0.01"]),
                       ("hf2", ["-input", d1, "-input2", d2, "-posWmin1", "1000",
                                "-posWmax1", "9990", "-posWmin2", "100000",
                                "-posWmax2", "104193", "-r2limit", "0.005"])):
        outs = []
        for flt in ("gpu", "host"):
            d = os.path.join(tmp, f"{name}_{flt}")
            _run([*args, "-ploidy", "haploid", "-mdf", "-filter", flt, "-threads", "3",
                  "-output", os.path.join(d, "out.txt")], d, host_api.CLI_PATH)
            outs.append(open(os.path.join(d, "out.txt"), "rb").read())
        assert outs[0] == outs[1] and outs[0].count(b"\n") > 100


def test_exact_mode_against_oracle(dataset, tmp_path):
    tmp, d1, _, _, T = dataset
    out = tmp_path / "exact.txt"
    _run(["-input", d1, "-ploidy", "haploid", "-mdf", "-r2limit", "0", "-r2mode", "exact",
          "-posWmin1", "1000", "-posWmax1", "3990", "-posWmin2", "2000", "-posWmax2", "8990",
          "-output", str(out)], str(tmp_path), host_api.CLI_PATH)
    A = T[:300]                      # positions 1000 + 10 i
    B = T[100:800]
    bcA, bcB = oracle.bitcounts(A), oracle.bitcounts(B)
    want = oracle.r2_exact(bcA, bcB, oracle.counts(A, B), 2500)
    lines = out.read_text().split("\n")[1:-1]
    got = np.full(want.shape, np.nan)
    for ln in lines:
        p2, p1, _, _, _, _, v = ln.split("\t")
        got[(int(p2) - 2000) // 10, (int(p1) - 1000) // 10] = float(v)
    sel = (want < 100) & np.isfinite(want)
    assert np.count_nonzero(~np.isnan(got)) == np.count_nonzero(sel)
    # the report truncates to 9 decimals: 1e-9 absolute on top of 1e-6 relative
    g, w = got[sel], want[sel]
    assert np.all(np.abs(g - w) <= 1e-6 * w + 1.1e-9)


def test_sample_lists(dataset):
    """-sampleList / -sampleList2 with MDF input: qLD-compute sizes the rows
    from the listed names (K = ceil(listed x ploidy / 64)) and keeps each
    row's first K words; qld-ld writes the same bytes.  One region, two
    windows, and two inputs whose lists give the same K."""
    tmp, d1, d2, _, _ = dataset
    l1 = os.path.join(tmp, "samples1.txt")
    l2 = os.path.join(tmp, "samples2.txt")
    with open(l1, "w") as f:                      # 1,300 of 2,500 names: K 40 -> 21
        f.write("\n".join(f"s{i}" for i in range(1, 2501, 2)))
        f.write("\n" + " ".join(f"s{i}" for i in range(2, 102, 2)) + "\nnot_a_sample\n")
    with open(l2, "w") as f:                      # 1,290 names: K 21 as well
        f.write("\n".join(f"s{i}" for i in range(1211, 2501)) + "\n")
    cases = {
        "sl_single": ["-input", d1, "-sampleList", l1, "-r2limit", "0"],
        "sl_windows": ["-input", d1, "-sampleList", l1, "-sampleList2", l2,
                       "-posWmin1", "1000", "-posWmax1", "4000", "-posWmin2", "3000",
                       "-posWmax2", "9000", "-r2limit", "0.01"],
        "sl_inputs": ["-input", d1, "-input2", d2, "-sampleList", l1, "-sampleList2", l2,
                      "-posWmin1", "1000", "-posWmax1", "9990", "-posWmin2", "100000",
                      "-posWmax2", "104193", "-r2limit", "0.005"],
    }
    for name, args in cases.items():
        ref, qld = _reports(tmp, name, [*args, "-ploidy", "haploid", "-mdf"])
        assert ref and ref == qld, name
        assert ref["out.txt"].count(b"\n") > 10, name
