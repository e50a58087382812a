"""CPU tests of the C host layer (libqld_host.so): the MDF loader against the
Python reader, the report writer against the reference's golden reports and
the oracle's writeResults restatement, and qld-ld's argument handling."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import golden_names, load_golden
from qld_b200 import api, host_api, mdf, synth


@pytest.fixture(scope="module")
def dataset(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("host")
    rng = np.random.default_rng(3)
    n_samples = 300                                   # K = 5, 44 bits used in the last word
    T = rng.integers(0, 2**63, size=(700, 5), dtype=np.uint64)
    T[:, -1] &= np.uint64(((1 << 44) - 1) << 20)
    pos = 5000 + np.cumsum(rng.integers(1, 40, size=700))
    ids = [f"rs{i}_{rng.integers(1e6)}" for i in range(700)]
    path = mdf.write_dataset(str(tmp / "d"), T, n_samples, positions=pos, ids=ids,
                             snps_per_file=97, alignment_id="chr7")
    return path, T, pos


@pytest.mark.parametrize("window", [None, (5000, 9000), (9001, 9001), (0, 4000), (7000, 10**9)])
@pytest.mark.parametrize("threads", [1, 5])
def test_loader_matches_reader(dataset, window, threads):
    path, T, pos = dataset
    h = host_api.read_header(path)
    lo, hi = window if window else (h.pos_min, h.pos_max)
    got = host_api.load_mdf(path, lo, hi, 5, threads=threads)
    want = mdf.read_region(path, lo, hi)
    assert got.rows == want[0].shape[0]
    assert np.array_equal(got.words, want[0])
    assert np.array_equal(got.bc, want[1])
    assert np.array_equal(got.pos, want[2])
    assert got.ids == want[3]


def test_header(dataset):
    path, T, pos = dataset
    h = host_api.read_header(path)
    assert (h.id, h.snips_per_file, h.snip_size, h.total_snips, h.samples) == \
        ("chr7", 97, 300, 700, 300)
    assert (h.pos_min, h.pos_max) == (int(pos[0]), int(pos[-1]))


def test_loader_ignores_words_past_k(tmp_path):
    """qLD-parse-2MDF pads haploid rows to its diploid default width with
    words it never initialises; qLD-compute ignores them, and so does the
    loader."""
    T = np.zeros((10, 2), np.uint64)
    T[:, 0] = np.arange(10, dtype=np.uint64)
    T[4, 1] = 7                                      # a word the 64 samples do not need
    path = mdf.write_dataset(str(tmp_path / "p"), T, 64, snps_per_file=4)
    got = host_api.load_mdf(path, 0, 10**9, 1)
    assert got.rows == 10 and np.array_equal(got.words[:, 0], T[:, 0])


def test_loader_rejects_short_rows_and_missing_header(tmp_path):
    T = np.ones((6, 3), np.uint64)
    path = mdf.write_dataset(str(tmp_path / "s"), T, 192, snps_per_file=6)
    with pytest.raises(api.QldError) as e:
        host_api.load_mdf(path, 0, 10**9, 4)            # 4 words asked, 3 on each row
    assert "words" in str(e.value)
    os.makedirs(tmp_path / "empty")
    with pytest.raises(api.QldError) as e:
        host_api.read_header(str(tmp_path / "empty"))
    assert "no header" in str(e.value)


def _tables(g):
    A = host_api.Table(g["A"], g["bcA"], g["posA"], g["idA"])
    if g["symmetric"]:
        return A, A
    return A, host_api.Table(g["B"], g["bcB"], g["posB"], g["idB"])


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("threads", [1, 3])
def test_report_matches_golden(tmp_path, name, threads):
    g = load_golden(name)
    A, B = _tables(g)
    out = tmp_path / "r.txt"
    host_api.write_report(str(out), A, B, g["r2_ref"], g["S"], g["r2limit"], g["symmetric"],
                          threads=threads)
    assert out.read_bytes() == g["report"]


@pytest.mark.parametrize("single", [True, False])
def test_report_many_blocks_special_values(tmp_path, single):
    """Enough rows for several write-out rounds of 64-row blocks; NaN, the
    123.456 sentinel, exact limits, 0, 1 and values just under 100."""
    rng = np.random.default_rng(9)
    m, n = 900, (900 if single else 1300)
    r2 = rng.random((n, m), dtype=np.float32) ** 3
    specials = np.array([np.nan, 123.456, 0.05, 0.0, 1.0, 99.99, 100.0, np.inf, 0.0499999],
                        np.float32)
    idx = rng.integers(0, r2.size, 4000)
    r2.flat[idx] = specials[rng.integers(0, len(specials), idx.size)]
    S = 1234
    posA = np.sort(rng.choice(10**7, m, replace=False)).astype(np.uint32)
    bcA = rng.integers(0, S + 1, m).astype(np.uint32)
    idA = [f"snp{i}" for i in range(m)]
    A = host_api.Table(np.zeros((m, 1), np.uint64), bcA, posA, idA)
    if single:
        B = A
    else:
        posB = np.sort(rng.choice(10**7, n, replace=False)).astype(np.uint32)
        B = host_api.Table(np.zeros((n, 1), np.uint64), rng.integers(0, S + 1, n).astype(np.uint32),
                           posB, [f"b{i}" for i in range(n)])
    want = oracle.write_results(A.pos, A.ids, A.bc, B.pos, B.ids, B.bc, S, r2, 0.05,
                                0 if single else 1)
    for threads in (1, 4, 7):
        out = tmp_path / f"r{threads}.txt"
        host_api.write_report(str(out), A, B, r2, S, 0.05, single, threads=threads)
        assert out.read_bytes() == want
    if oracle.reference_available():
        ref = tmp_path / "ref.txt"
        oracle.ref_write_report(str(ref), A.pos, A.ids, A.bc, B.pos, B.ids, B.bc, S, r2, 0.05,
                                0 if single else 1)
        assert ref.read_bytes() == want


def test_report_rectangle_with_triangle_rule(tmp_path):
    """qLD's split-file case: two different tables with posWset2 == 0 print
    j > i over the rectangle (correlate_IO.c:403-406)."""
    rng = np.random.default_rng(2)
    m, n = 150, 260
    r2 = rng.random((n, m), dtype=np.float32)
    A = host_api.Table(np.zeros((m, 1), np.uint64), rng.integers(0, 99, m).astype(np.uint32),
                       np.arange(m, dtype=np.uint32) + 10, [f"a{i}" for i in range(m)])
    B = host_api.Table(np.zeros((n, 1), np.uint64), rng.integers(0, 99, n).astype(np.uint32),
                       np.arange(n, dtype=np.uint32) + 10, [f"b{i}" for i in range(n)])
    want = oracle.write_results(A.pos, A.ids, A.bc, B.pos, B.ids, B.bc, 99, r2, 0.0, 0)
    out = tmp_path / "t.txt"
    host_api.write_report(str(out), A, B, r2, 99, 0.0, True, threads=3)
    assert out.read_bytes() == want


@pytest.mark.parametrize("single,block_rows", [(True, 64), (True, 1000), (False, 77)])
def test_report_from_hit_blocks_matches_dense(tmp_path, single, block_rows):
    """The streamed writer fed with filtered blocks (mask + packed values, the
    form qld_cuda_ld_hits delivers) writes the dense writer's bytes."""
    rng = np.random.default_rng(4)
    m, n = 700, (700 if single else 450)
    r2 = (rng.random((n, m), dtype=np.float32) ** 4).astype(np.float32)
    r2.flat[rng.integers(0, r2.size, 500)] = np.float32(np.nan)
    r2.flat[rng.integers(0, r2.size, 500)] = np.float32(123.456)
    S = 999
    A = host_api.Table(np.zeros((m, 1), np.uint64), rng.integers(0, S, m).astype(np.uint32),
                       np.arange(m, dtype=np.uint32) * 3 + 1, [f"a{i}" for i in range(m)])
    B = A if single else host_api.Table(
        np.zeros((n, 1), np.uint64), rng.integers(0, S, n).astype(np.uint32),
        np.arange(n, dtype=np.uint32) * 5 + 2, [f"b{i}" for i in range(n)])
    dense = tmp_path / "dense.txt"
    host_api.write_report(str(dense), A, B, r2, S, 0.03, single, threads=2)

    def blocks():
        for r0 in range(0, n, block_rows):
            mask, off, val = host_api.hits_from_dense(r2[r0:r0 + block_rows], 0.03, single, r0)
            yield r0, mask, off, val

    hits = tmp_path / "hits.txt"
    host_api.write_report_hits(str(hits), A, B, blocks(), S, threads=3)
    assert hits.read_bytes() == dense.read_bytes()


def test_report_hits_rejects_foreign_block(tmp_path):
    A = host_api.Table(np.zeros((40, 1), np.uint64), np.ones(40, np.uint32),
                       np.arange(40, dtype=np.uint32), [f"a{i}" for i in range(40)])
    mask, off, val = host_api.hits_from_dense(np.ones((10, 40), np.float32) * 0.5, 0.1, False)
    with pytest.raises(api.QldError):          # rows 35..44 of a 40-row table B
        host_api.write_report_hits(str(tmp_path / "x.txt"), A, A, [(35, mask, off, val)], 10)


@pytest.mark.parametrize("threads", [1, 4])
def test_states_report_matches_golden(tmp_path, threads):
    """The C states writer with the oracle's states against the reference's
    COUNTSTATES reports (tests/golden/states)."""
    from test_oracle import _states_cases, load_states_golden
    for name in _states_cases():
        g = load_states_golden(name)
        st = oracle.count_states(g["A"], g["B"])
        A = host_api.Table(g["A"], np.zeros(len(g["posA"]), np.uint32), g["posA"], g["idA"])
        B = A if g["single"] else host_api.Table(g["B"], np.zeros(len(g["posB"]), np.uint32),
                                                 g["posB"], g["idB"])
        out = tmp_path / f"{name}.txt"
        host_api.write_states_report(str(out), A, B, st, g["single"], threads=threads)
        assert out.read_bytes() == g["report"], name


def _cli(*args, timeout=60):
    return subprocess.run([host_api.CLI_PATH, *args], capture_output=True, text=True,
                          timeout=timeout)


def test_cli_argument_errors(dataset, tmp_path):
    path, _, _ = dataset
    if not os.path.exists(host_api.CLI_PATH):
        pytest.skip("qld-ld not built")
    r = _cli("-input", path, "-output", str(tmp_path / "o.txt"), "-mdf")
    assert r.returncode == 1 and "ploidy" in r.stderr
    r = _cli("-input", path, "-output", str(tmp_path / "o.txt"), "-ploidy", "haploid")
    assert r.returncode == 1 and "-mdf" in r.stderr
    r = _cli("-input", path, "-output", str(tmp_path / "o.txt"), "-ploidy", "triploid", "-mdf")
    assert r.returncode == 1
    r = _cli("-input", path, "-ploidy", "haploid", "-mdf", "-bogus", "1")
    assert r.returncode == 1 and "not a valid" in r.stderr
    r = _cli("-input", path, "-ploidy", "haploid", "-mdf", "-seed", "3")
    assert r.returncode == 1 and "not a valid" in r.stderr
    r = _cli("-help")
    assert r.returncode == 0 and "usage" in r.stdout


def test_listed_samples(dataset, tmp_path):
    """-sampleList's valid count: the #CHROM names the list holds (every name
    without a list); unknown and repeated list entries count once or not at
    all (sample_isValid, correlate_IO.c:60-76)."""
    path, _, _ = dataset
    assert host_api.listed_samples(path) == 300
    assert host_api.listed_samples(path, ["s1", "s2", "s300", "s2", "nobody"]) == 3
    assert host_api.listed_samples(path, [f"s{i}" for i in range(1, 301, 2)]) == 150
    assert host_api.listed_samples(path, ["nobody"]) == 0


def test_cli_sample_list_errors(dataset, tmp_path):
    path, _, _ = dataset
    if not os.path.exists(host_api.CLI_PATH):
        pytest.skip("qld-ld not built")
    r = _cli("-input", path, "-output", str(tmp_path / "o.txt"), "-ploidy", "haploid", "-mdf",
             "-sampleList", str(tmp_path / "missing.txt"))
    assert r.returncode == 1 and "sample list" in r.stderr
