"""CPU tests of bench.py's bookkeeping: the measured peaks it divides by and
the ncu capture it takes each kernel's DRAM traffic from."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

WORKLOAD = "single_region_29817x16622_lower_triangle"


def test_measured_peaks_read_from_the_pool_file():
    mp = bench.measured_peaks()
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            assert mp == {"hbm_gbs": float(json.load(f)["hbm_gbs"]),
                          "source": "MEASURED_PEAKS.json"}
    else:
        assert mp == {"hbm_gbs": 6650.0, "source": "fallback"}


def _profile_value(name):
    with open(os.path.join(ROOT, "profiles", name)) as f:
        for line in f:
            if line.startswith("traffic_bytes_per_launch_full:"):
                return int(line.split(":")[1])
    raise AssertionError(name)


def test_traffic_follows_the_kernel_the_mode_runs():
    pair = _profile_value("k_ld_mxf4_pair_traffic_16384.md")
    single = _profile_value("k_ld_mxf4_traffic_16384.md")
    fp4, mma = 3, 2
    assert bench.measured_traffic(fp4, WORKLOAD, 0, "exact") == pair
    assert bench.measured_traffic(fp4, WORKLOAD, 0, "reference") == pair
    assert bench.measured_traffic(fp4, WORKLOAD, 1, "exact") == single
    assert bench.measured_traffic(fp4, WORKLOAD, 2, "reference") == pair
    assert bench.measured_traffic(mma, WORKLOAD) == _profile_value(
        "k_ld_mma_wide_traffic_16384.md")
    assert bench.measured_traffic(fp4, "all_pairs_2048x4096_symmetric") is None
    assert bench.measured_traffic(0, WORKLOAD) is None


def test_both_arms_print_the_same_config():
    args = bench.parse(["--impl", "reference"])
    ours = bench.parse([])
    assert bench.arm_config(args, 2) == bench.arm_config(ours, 2)
    cfg = bench.arm_config(ours, 1)
    assert cfg["workload"] == WORKLOAD and "parallelism" in cfg and "l2" in cfg


def test_band_pair_count():
    assert bench.band_pairs(10, 3) == sum(min(3, 9 - i) for i in range(10))
    m, W = 200_000, 5000
    assert bench.band_pairs(m, W) == sum(min(W, m - 1 - i) for i in range(0, m))


def test_host_cpu_reports_cores():
    model, phys, logical = bench.host_cpu()
    assert 1 <= phys <= logical and isinstance(model, str)


def test_pair_tiles_and_shared_memory_roofline():
    # the kernel's tile list: 7,419 tiles on the 29,817-SNP region, 579 on 8,192
    assert bench.pair_tiles(29817, 29817, True) == 7419
    assert bench.pair_tiles(8192, 8192, True) == 579
    assert bench.pair_tiles(300, 500, False) == 2 * 3
    r = bench.smem_roofline(29817, 29817, 260, True, 2.415, 1965.0)
    assert r["bytes_per_launch"] == 2 * 7419 * 66 * 248 * 320
    assert abs(r["peak"] - 148 * 128 * 1965e6 / 1e12) < 1e-9
    assert 0.8 < r["frac"] < 0.9
    assert bench.smem_roofline(100, 100, 4, True, 0.0, 1965.0) is None


def test_sampled_cpu_baseline_runs_the_reference_path():
    import numpy as np
    rng = np.random.default_rng(3)
    T = rng.integers(0, 2 ** 63, size=(300, 5), dtype=np.int64).view(np.uint64)
    calls = []

    def tasks(size):
        calls.append(size)
        return [(T[:size], None, 300), (T[:size], T[size:2 * size], 300)], \
            size * (size - 1) // 2 + size * size, f"{size} rows"
    r = bench.cpu_sampled_baseline(tasks, (20, 100), seconds_target=0.01)
    assert calls[0] == 20 and 20 <= calls[1] <= 100
    assert r["kind"] == "reference" and r["value"] > 0 and r["cores"] >= 1
    assert r["sample"].startswith(f"{calls[1]} rows")
