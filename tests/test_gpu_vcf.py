"""GPU tests of VCF -> MDF conversion: qld_cuda_vcf_pack against the oracle's
restatement of qLD-parse-2MDF's per-site processing, and the qld-vcf2mdf
command against qLD-parse-2MDF itself (oracle/_ref, run on the host cores)."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT
from qld_b200 import api, host_api, vcf

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref", "qLD-parse-2MDF")
SAMPLES = [f"s{i}" for i in range(700)]


def messy(lines, seed):
    """Runs of separators and CR line ends, which qLD's word splitter absorbs."""
    rng = np.random.default_rng(seed)
    out = []
    for ln in lines:
        r = rng.random()
        if r < 0.1:
            ln = ln.replace("\t", " \t", 5)
        elif r < 0.15:
            ln = ln + "\r"
        out.append(ln)
    return out


CASES = [
    ("haploid", dict(ploidy=1, missing=0.01), 1, None),
    ("phased", dict(ploidy=2, phased=True, missing=0.03), 2, None),
    ("unphased", dict(ploidy=2, phased=False, missing=0.03), 2, None),
    ("unphased_seed", dict(ploidy=2, phased=False), 2, 23),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
def test_pack_equals_oracle(gpu_ctx, tmp_path, case):
    name, kw, ploidy, seed = case
    lines = messy(vcf.site_lines(500, len(SAMPLES), 31, **kw), 3)
    d = vcf.write_dataset(str(tmp_path / "in"), lines, SAMPLES, snps_per_file=150)
    h = host_api.VcfHeader(d, ploidy)
    parts = [host_api.VcfPart(p, h) for p in h.parts(d)]
    # both sides draw from the one libc generator: all oracle parts first,
    # then all GPU parts from the same seed (later parts continue the sequence)
    oracle.vcf_seed(seed or 1)
    want = [oracle.vcf_pack(q.text, q.sites, h.valid, ploidy, h.K) for q in parts]
    got = [gpu_ctx.vcf_pack(q.text, q.sites, h.valid, ploidy, h.K,
                            seed=(seed or 1) if i == 0 else None) for i, q in enumerate(parts)]
    for g, w in zip(got, want):
        for x, y in zip(g, w):
            assert np.array_equal(x, y)
        assert w[3].sum() > 0


def test_pack_reports_first_bad_site(gpu_ctx, tmp_path):
    lines = vcf.site_lines(60, 30, 7, ploidy=2, oddities=False)
    d = vcf.write_dataset(str(tmp_path / "in"), lines, SAMPLES[:30], snps_per_file=60)
    h = host_api.VcfHeader(d, 1)
    part = host_api.VcfPart(h.parts(d)[0], h)
    with pytest.raises(api.QldError) as e:
        gpu_ctx.vcf_pack(part.text, part.sites, h.valid, 1, h.K)
    assert e.value.code == api.ERR_INVALID and "site 0" in str(e.value)
    # the context still works
    h2 = host_api.VcfHeader(d, 2)
    got = gpu_ctx.vcf_pack(part.text, part.sites, h2.valid, 2, h2.K)
    want = oracle.vcf_pack(part.text, part.sites, h2.valid, 2, h2.K)
    assert np.array_equal(got[0], want[0])


def _cli(args):
    return subprocess.run(args, capture_output=True, text=True, timeout=900)


def _same_dirs(a, b):
    fa = sorted(f for f in os.listdir(a) if f.endswith(".mdf") or "header" in f)
    fb = sorted(f for f in os.listdir(b) if f.endswith(".mdf") or "header" in f)
    assert fa == fb and len(fa) > 1
    for f in fa:
        assert open(os.path.join(a, f), "rb").read() == open(os.path.join(b, f), "rb").read(), f


@pytest.mark.parametrize("case", [
    ("haploid", dict(ploidy=1, missing=0.01), ["-ploidy", "haploid"]),
    ("phased", dict(ploidy=2, phased=True, missing=0.02), ["-ploidy", "phased_diploid"]),
    ("unphased", dict(ploidy=2, phased=False, missing=0.02), ["-ploidy", "unphased_diploid"]),
    ("unphased_seed", dict(ploidy=2, phased=False), ["-ploidy", "unphased_diploid", "-seed",
                                                     "5"]),
], ids=lambda c: c[0])
def test_cli_matches_reference(tmp_path, case):
    if not (os.path.exists(REF) and os.path.exists(host_api.VCF2MDF_PATH)):
        pytest.skip("qLD-parse-2MDF or qld-vcf2mdf not built")
    name, kw, flags = case
    lines = messy(vcf.site_lines(900, len(SAMPLES), 41, **kw), 9)
    d = vcf.write_dataset(str(tmp_path / "in"), lines, SAMPLES, snps_per_file=200)
    r = _cli([REF, "-input", d, "-output", str(tmp_path / "ref"), *flags])
    assert r.returncode == 0, r.stderr[-500:]
    q = _cli([host_api.VCF2MDF_PATH, "-input", d, "-output", str(tmp_path / "qld"), "-threads",
              "3", *flags])
    assert q.returncode == 0, q.stderr[-2000:]
    _same_dirs(str(tmp_path / "ref"), str(tmp_path / "qld"))
    assert sorted(os.path.basename(x) for x in q.stdout.split()) == \
        sorted(f for f in os.listdir(tmp_path / "qld") if f.endswith(".mdf"))


def test_cli_sample_list_and_errors(tmp_path):
    if not (os.path.exists(REF) and os.path.exists(host_api.VCF2MDF_PATH)):
        pytest.skip("qLD-parse-2MDF or qld-vcf2mdf not built")
    lines = vcf.site_lines(300, len(SAMPLES), 43, ploidy=1)
    d = vcf.write_dataset(str(tmp_path / "in"), lines, SAMPLES, snps_per_file=100)
    lst = tmp_path / "list.txt"
    lst.write_text("\n".join(SAMPLES[1::4]))
    r = _cli([REF, "-input", d, "-output", str(tmp_path / "ref"), "-ploidy", "haploid",
              "-sampleList", str(lst)])
    assert r.returncode == 0
    q = _cli([host_api.VCF2MDF_PATH, "-input", d, "-output", str(tmp_path / "qld"), "-ploidy",
              "haploid", "-sampleList", str(lst)])
    assert q.returncode == 0, q.stderr[-2000:]
    _same_dirs(str(tmp_path / "ref"), str(tmp_path / "qld"))
    # diploid genotypes read as haploid: both stop with an error
    lines = vcf.site_lines(50, 40, 44, ploidy=2, oddities=False)
    d2 = vcf.write_dataset(str(tmp_path / "in2"), lines, SAMPLES[:40], snps_per_file=50)
    assert _cli([REF, "-input", d2, "-output", str(tmp_path / "r2"), "-ploidy",
                 "haploid"]).returncode != 0
    q = _cli([host_api.VCF2MDF_PATH, "-input", d2, "-output", str(tmp_path / "q2"), "-ploidy",
              "haploid"])
    assert q.returncode != 0 and "ploidy" in q.stderr
    assert _cli([host_api.VCF2MDF_PATH, "-input", d2, "-output", str(tmp_path / "q3"),
                 "-impute"]).returncode != 0
