"""CPU tests of VCF -> MDF conversion: the host half (libqld_host.so: header,
part list, fixed-field filtering, MDF writer) with the oracle's restatement of
qLD-parse-2MDF's per-site processing, against qLD-parse-2MDF itself built from
its sources (oracle/_ref/qLD-parse-2MDF) on seeded synthetic datasets."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT
from qld_b200 import host_api, vcf

REF = os.path.join(ROOT, "oracle", "_ref", "qLD-parse-2MDF")
SAMPLES = [f"s{i}" for i in range(130)]


def convert_with_oracle(d, out, ploidy, seed=1, names=None):
    h = host_api.VcfHeader(d, ploidy, names)
    oracle.vcf_seed(seed)
    os.makedirs(out, exist_ok=True)
    for p in h.parts(d):
        part = host_api.VcfPart(p, h)
        w, bc, ln, keep = oracle.vcf_pack(part.text, part.sites, h.valid, ploidy, h.K)
        part.write_mdf(out, h, w, bc, keep)
    return h


def reference(d, out, flags):
    r = subprocess.run([REF, "-input", d, "-output", out, *flags], capture_output=True,
                       text=True, timeout=600)
    return r.returncode


def mdf_rows(path, data_words=None):
    """MDF lines; with data_words, row words past it are dropped (qLD leaves
    them uninitialised)."""
    lines = open(path).read().split("\n")
    if data_words is None:
        return lines
    return lines[:3] + ["\t".join(ln.split("\t")[:4 + data_words]) for ln in lines[3:]]


def same_outputs(a, b, data_words=None):
    fa = sorted(f for f in os.listdir(a) if f.endswith(".mdf"))
    fb = sorted(f for f in os.listdir(b) if f.endswith(".mdf"))
    assert fa == fb and fa
    for f in fa:
        assert mdf_rows(os.path.join(a, f), data_words) == mdf_rows(os.path.join(b, f),
                                                                   data_words), f


needs_ref = pytest.mark.skipif(not os.path.exists(REF), reason="qLD-parse-2MDF not built")


@needs_ref
@pytest.mark.parametrize("case", [
    ("haploid", dict(ploidy=1, missing=0.01), ["-ploidy", "haploid"], 1, None),
    ("phased", dict(ploidy=2, phased=True, missing=0.02), ["-ploidy", "phased_diploid"], 2,
     None),
    ("unphased", dict(ploidy=2, phased=False, missing=0.02), ["-ploidy", "unphased_diploid"], 2,
     None),
    ("unphased_seed", dict(ploidy=2, phased=False), ["-ploidy", "unphased_diploid", "-seed",
                                                     "17"], 2, 17),
], ids=lambda c: c[0])
def test_oracle_pipeline_matches_reference(tmp_path, case):
    name, kw, flags, ploidy, seed = case
    lines = vcf.site_lines(300, len(SAMPLES), 11, **kw)
    d = vcf.write_dataset(str(tmp_path / "in"), lines, SAMPLES, snps_per_file=70)
    assert reference(d, str(tmp_path / "ref"), flags) == 0
    convert_with_oracle(d, str(tmp_path / "ours"), ploidy, seed if seed is not None else 1)
    same_outputs(str(tmp_path / "ref"), str(tmp_path / "ours"))
    # the header file is copied next to the parts
    assert os.path.exists(tmp_path / "ref" / "1_header.vcf.gz")


@needs_ref
def test_sample_list(tmp_path):
    lines = vcf.site_lines(200, len(SAMPLES), 12, ploidy=1)
    d = vcf.write_dataset(str(tmp_path / "in"), lines, SAMPLES, snps_per_file=64)
    names = SAMPLES[::3] + ["not_a_sample"]
    lst = tmp_path / "list.txt"
    lst.write_text("\n".join(names) + "\n")
    assert reference(d, str(tmp_path / "ref"), ["-ploidy", "haploid", "-sampleList",
                                                 str(lst)]) == 0
    h = convert_with_oracle(d, str(tmp_path / "ours"), 1, names=names)
    assert h.valid.sum() == len(SAMPLES[::3])
    same_outputs(str(tmp_path / "ref"), str(tmp_path / "ours"))


@needs_ref
def test_haploid_data_at_default_ploidy(tmp_path):
    """qLD-parse-2MDF's default ploidy is 2: haploid rows get twice the words,
    the extra ones uninitialised in qLD (zero here); the data words match."""
    lines = vcf.site_lines(250, len(SAMPLES), 13, ploidy=1)
    d = vcf.write_dataset(str(tmp_path / "in"), lines, SAMPLES, snps_per_file=80)
    assert reference(d, str(tmp_path / "ref"), []) == 0
    h = convert_with_oracle(d, str(tmp_path / "ours"), 2)
    data_words = (len(SAMPLES) + 63) // 64
    assert h.K == (2 * len(SAMPLES) + 63) // 64 > data_words
    same_outputs(str(tmp_path / "ref"), str(tmp_path / "ours"), data_words)
    for f in os.listdir(tmp_path / "ours"):
        if f.endswith(".mdf"):
            for ln in open(tmp_path / "ours" / f).read().split("\n")[3:]:
                assert all(w == "0" for w in ln.split("\t")[4 + data_words:])


def test_fixed_field_filter():
    """Lines qLD-parse-2MDF skips on their fixed fields never become sites."""
    base = ["1", "", "rsX", "A", "G", ".", ".", ".", "GT"] + ["0", "1", "1"]
    variants = {
        "keep": {},
        "multi_ref": {3: "AT"},
        "multi_alt": {4: "G,T"},
        "symbolic": {4: "<DEL>"},
        "filter": {6: "LowQual"},
        "filter_pass": {6: "PASS"},
        "af0": {7: "DP=4;AF=0"},
        "af1": {7: "AF=1.0000000001"},            # read to 9 characters: 1.0000000
        "af_list": {7: "AF=0,0.25"},
        "vt_indel": {7: "AF=0.5;VT=INDEL"},
        "vt_snp": {7: "VT=SNP"},
        "no_gt": {8: "DP:GQ"},
        "gt_second": {8: "DP:GT"},
    }
    want_kept = {"keep", "filter_pass", "af_list", "vt_snp", "gt_second"}
    lines = []
    for k, (name, ch) in enumerate(variants.items()):
        f = list(base)
        f[1] = str(100 + k)
        f[2] = name
        for i, v in ch.items():
            f[i] = v
        lines.append("\t".join(f))
    import tempfile
    with tempfile.TemporaryDirectory() as tmp:
        d = vcf.write_dataset(os.path.join(tmp, "in"), lines, ["a", "b", "c"], snps_per_file=100)
        h = host_api.VcfHeader(d, 1)
        part = host_api.VcfPart(h.parts(d)[0], h)
        assert set(part.ids) == want_kept
        assert part.skipped == len(variants) - len(want_kept)
        gts = {i: int(part.sites[j]["gt_pos"]) for j, i in enumerate(part.ids)}
        assert gts["gt_second"] == 1 and gts["keep"] == 0


@needs_ref
def test_errors_where_reference_stops(tmp_path):
    """Diploid genotypes with -ploidy haploid: qLD-parse-2MDF exits; the
    restatement names the site."""
    lines = vcf.site_lines(40, 20, 5, ploidy=2, oddities=False)
    d = vcf.write_dataset(str(tmp_path / "in"), lines, SAMPLES[:20], snps_per_file=40)
    assert reference(d, str(tmp_path / "ref"), ["-ploidy", "haploid"]) != 0
    h = host_api.VcfHeader(d, 1)
    part = host_api.VcfPart(h.parts(d)[0], h)
    with pytest.raises(ValueError, match="ploidy"):
        oracle.vcf_pack(part.text, part.sites, h.valid, 1, h.K)
