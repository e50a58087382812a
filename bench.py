"""Benchmark of the LD hot path (AND+popcount counts + fused r^2) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload single_region|all_pairs|windowed|batched|served]
                    [--sections all_pairs,reference_mode,windowed,batched,served|none]

Headline workload (default): the dataset-shaped single region -- 29,817 SNPs x
16,622 haploid sequences (K = 260 words per SNP), allele frequencies
Beta(0.1, 1) clipped to >= 1/16,622, haplotype-copying model (20 founders,
recombination blocks of 50-500 SNPs, 1% per-site mutation), lower-triangular
FP32 r^2.  Seeded synthetic data of that shape stands in for the dataset.

A step is one pass of the hot path over the region: counts + r^2 for all
M(M-1)/2 SNP pairs (the kernel also fills the diagonal).  `value` is
SNP-pairs/s with the packed table resident in HBM (device-to-device call,
output to HBM), timed per step with CUDA events on the launching stream after
an L2 flush (a 512 MB write); `e2e` is the same metric through the host-buffer
C-ABI call (qld_cuda_ld): pinned host table -> device, counts + r^2, lower
triangle -> pinned host memory, all inside the timed region.  `parity` checks
the timed output after the timed region: about two B rows from every 120-row
block (so every output tile, including the last tiles each CTA pair walks) are
compared with the CPU oracle -- counts bit-exact (from one more launch of the
same kernel with the counts output on), r^2 within 1e-6 relative of FP64 --
and reports the maximum and mean relative error.

The same line carries one sub-object per other workload form (`--sections`),
each with its own timing, clocks and sampled parity:
  all_pairs       2,048 SNPs x 4,096 samples, iid, every row checked;
  reference_mode  the headline region with r^2 bit-identical to qLD-compute
                  (the drop-in's default mode);
  windowed        200,000 SNPs x 100,000 haplotypes, 5,000-SNP band;
  batched         4,096 tasks in one persistent launch, replayed from a CUDA
                  graph captured once (and as a direct call per step), vs
                  per-task launches;
  served          22 resident chromosomes, Poisson stream of 10,000 queries.

With --gpus N (torchrun) every rank processes its own region of the same shape
(no data-path collective; weak scaling); timing is the max over ranks, and the
sections run on rank 0's line only at N = 1.  `--impl reference` times the
reference's stock fast CPU path -- qLD-compute -blis: BLIS 0.1.8 `binary_gemm`
cblas_dsyrk with BLIS_IC_NT = physical cores, then get_pairwise_ld_score on
one thread, built from the qLD sources into oracle/_ref -- on a bounded sample
of the same region.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "r2 SNP-pairs/s (counts + fused r2 epilogue)"
SECTIONS = ("all_pairs", "reference_mode", "windowed", "batched", "served")


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="single_region",
                    choices=["single_region", "all_pairs", "batched", "windowed", "served",
                             "dropin"])
    ap.add_argument("--sections", default=",".join(SECTIONS),
                    help="sub-objects of the headline line (comma list, or 'none')")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the sampled oracle checks of the timed outputs")
    ap.add_argument("--queries", type=int, default=10000, help="served workload: query count")
    ap.add_argument("--load", type=float, default=0.8,
                    help="served workload: offered load as a fraction of measured capacity")
    ap.add_argument("--pool-gb", type=int, default=48, help="served workload: r^2 pool (GB)")
    ap.add_argument("--inflight", type=int, default=3,
                    help="served workload: batched launches in flight")
    ap.add_argument("--band", type=int, default=5000, help="windowed workload: band width")
    ap.add_argument("--jobs", type=int, default=4096, help="batched workload: number of tasks")
    ap.add_argument("--kernel", default="auto", choices=["auto", "popc", "mma", "fp4"])
    ap.add_argument("--sm-pair", type=int, default=0, choices=[0, 1, 2],
                    help="4-bit kernel: SMs per output tile (0 = automatic)")
    ap.add_argument("--r2-mode", default="exact", choices=["exact", "reference"],
                    help="r^2 evaluation: exact (FP64-accurate) or reference (bit-identical "
                         "to qLD-compute's float/double sequence)")
    ap.add_argument("--autotune", action="store_true",
                    help="run qld_cuda_autotune on the workload's shape first (AUTO then uses it)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--mma-tile", type=int, default=0, choices=[0, 128, 256],
                    help="tensor-core tile rows (0: per shape)")
    ap.add_argument("--snps", type=int, default=0,
                    help="use only the first N SNPs of the workload (profiling captures)")
    ap.add_argument("--split", action="store_true",
                    help="with --gpus N: the ranks split ONE region by tile rows "
                         "(qld_cuda_ld_device_part; strong scaling) instead of one region each")
    return ap.parse_args(argv)


def workload_config(name):
    if name == "single_region":
        return dict(workload="single_region_29817x16622_lower_triangle", snps=29_817,
                    haplotypes=16_622, words_per_snp=260, model="copying(20 founders)",
                    freq="Beta(0.1,1) clipped >= 1/16622", output="fp32 lower triangle")
    return dict(workload="all_pairs_2048x4096_symmetric", snps=2048, haplotypes=4096,
                words_per_snp=64, model="iid Bernoulli", freq="Uniform(0.05,0.5)",
                output="fp32 lower triangle")


def arm_config(args, world):
    """The `config` of the headline line; both arms print the same dict."""
    cfg = workload_config(args.workload)
    cfg["parallelism"] = (f"tile-row split x{world} (one region, no collective)"
                          if args.split else
                          f"replicas x{world} (independent regions, no collective)")
    cfg["l2"] = "512 MB flush write between timed steps"
    if args.snps:
        cfg["snps"] = args.snps
        cfg["workload"] += f"_first{args.snps}"
    if args.r2_mode != "exact":
        cfg["r2_mode"] = args.r2_mode
    return cfg


def make_table(name, device, seed_offset=0):
    from qld_b200 import synth
    if name == "single_region":
        return synth.single_region_workload(device=device, seed=2 + seed_offset)
    return synth.all_pairs_workload(device=device, seed=1 + seed_offset)


# ------------------------------------------------------------------ clocks --

class ClockSampler:
    """nvidia-smi samples every 50 ms from before warm-up to after the timed
    region; summary() keeps the samples whose timestamps fall inside
    [mark_start(), mark_end()] (all samples if none do)."""
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            deadline = time.time() + 10
            while time.time() < deadline and os.path.getsize(self.path) == 0:
                time.sleep(0.05)
        except FileNotFoundError:
            self.proc = None
        return self

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        import datetime
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 10:
                    rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def ts(r):
            try:
                return datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                return None
        inside = [r for r in rows if self.t0 and self.t1 and ts(r) is not None
                  and self.t0 - 0.05 <= ts(r) <= self.t1 + 0.05]
        use = inside or rows
        sm = [float(r[2]) for r in use if r[2].replace(".", "").isdigit()]
        smax = [float(r[3]) for r in use if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in use for k in range(4) if r[6 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(use),
                "window": "timed region" if inside else "whole run (no sample inside the region)"}


def measured_peaks():
    """HBM copy bandwidth measured on this pool's B200s (MEASURED_PEAKS.json
    beside this file), else an earlier measurement on the same pool
    (6.65 TB/s)."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return {"hbm_gbs": float(json.load(f)["hbm_gbs"]), "source": "MEASURED_PEAKS.json"}
    except (OSError, ValueError, KeyError):
        return {"hbm_gbs": 6650.0, "source": "fallback"}


def kernel_roofline(ctx, variant, bitops, kern_ms, dev, int8_context=True):
    """Roofline of the counts kernel against the measured rate of the pipe it
    runs on: the tensor pipe of its MMA kind (qld_cuda_measure_mma_peak,
    2 ops per bit-pair), or the popcount pipe (1 bit-op per bit-pair)."""
    import torch
    from qld_b200 import api
    if variant in (api.KERNEL_MMA, api.KERNEL_FP4):
        peak = ctx.measure_mma_peak(variant) / 1e12
        achieved = 2 * bitops / (kern_ms * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak,
                "unit": "TFLOPS (E2M1 dense)" if variant == api.KERNEL_FP4 else "TOPS (int8)",
                "frac": achieved / peak,
                "peak_source": "measured: qld_cuda_measure_mma_peak, back-to-back 128x256 "
                               + ("kind::mxf4 MMAs (K=64)" if variant == api.KERNEL_FP4
                                  else "kind::i8 MMAs (K=32)") + ", one CTA per SM"}
        if int8_context:
            # for context: the int8 rate a library GEMM reaches on this GPU
            a = torch.randint(-2, 2, (8192, 8192), dtype=torch.int8, device=dev)
            b = torch.randint(-2, 2, (8192, 8192), dtype=torch.int8, device=dev).t()
            for _ in range(3):
                torch._int_mm(a, b)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(10):
                torch._int_mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            roof["int8_gemm_torch_tops"] = 2 * 8192 ** 3 * 10 / (e0.elapsed_time(e1) * 1e-3) / 1e12
        return roof
    popc_peak = ctx.measure_popc_peak() / 1e12
    achieved = bitops / (kern_ms * 1e-3) / 1e12
    return {"bound": "popc", "achieved": achieved, "peak": popc_peak, "unit": "Tbit-op/s",
            "frac": achieved / popc_peak,
            "peak_source": "measured: qld_cuda_measure_popc_peak (register-only AND+POPC)"}


def pair_tiles(m, n, symmetric, bm=256, bn=240):
    """Output tiles of the SM-pair 4-bit kernel for one task (its tile list:
    every bm x bn tile of A rows x B rows, in a single region those holding a
    pair a >= b)."""
    ta, tb = -(-m // bm), -(-n // bn)
    if not symmetric:
        return ta * tb
    return sum(min((bm * a + bm - 1) // bn, tb - 1) + 1 for a in range(ta))


def smem_roofline(m, n, K, symmetric, kern_ms, sm_mhz, sms=148):
    """Shared-memory roofline of the SM-pair 4-bit kernel: per CTA and
    256-sample stage its 248 rows (128 A + 120 B) each take 32 B of TMA
    writes (packed words), 32 B of unpack reads, 128 B of E2M1 stores and
    128 B of tensor-core operand reads -- 320 B per row, the minimum of this
    layout -- over two CTAs per tile and 2 * ceil(K / 8) stages per tile;
    against 128 B per clock per SM at the sampled SM clock (nominal)."""
    if not kern_ms or not sm_mhz:
        return None
    stages = 2 * (-(-K // 8))
    nbytes = 2 * pair_tiles(m, n, symmetric) * stages * 248 * 320
    achieved = nbytes / (kern_ms * 1e-3) / 1e12
    peak = sms * 128 * sm_mhz * 1e6 / 1e12
    return {"bytes_per_launch": nbytes, "achieved": achieved, "peak": peak, "unit": "TB/s",
            "frac": achieved / peak,
            "peak_source": "nominal: 128 B/clk per SM x %d SMs at the sampled %.0f MHz" %
                           (sms, sm_mhz),
            "per_stage": "per CTA and 256-sample stage: 248 rows x (32 B TMA + 32 B unpack "
                         "read + 128 B E2M1 store + 128 B tensor-core read)"}


def measured_traffic(variant, workload, sm_pair=0, r2_mode="exact"):
    """DRAM bytes per launch of the counts kernel from the ncu capture
    summarised under profiles/ (None when no capture covers this case).
    sm_pair 0 is the automatic choice: SM pairs in both r^2 modes."""
    if sm_pair == 0:
        sm_pair = 2
    names = {2: "k_ld_mma_wide_traffic_16384.md",
             3: "k_ld_mxf4_traffic_16384.md" if sm_pair == 1 else "k_ld_mxf4_pair_traffic_16384.md"}
    if variant not in names or workload != "single_region_29817x16622_lower_triangle":
        return None
    path = os.path.join(ROOT, "profiles", names[variant])
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch_full:"):
                return int(line.split(":")[1])
    except OSError:
        pass
    return None


# ------------------------------------------------------------ reference CPU --

def host_cpu():
    """(model name, physical cores, logical cpus) of this host."""
    model, cores = "unknown", set()
    phys = core = None
    try:
        for line in open("/proc/cpuinfo"):
            k, _, v = line.partition(":")
            k, v = k.strip(), v.strip()
            if k == "model name":
                model = v
            elif k == "physical id":
                phys = v
            elif k == "core id":
                core = v
            elif not k and phys is not None and core is not None:
                cores.add((phys, core))
                phys = core = None
        if phys is not None and core is not None:
            cores.add((phys, core))
    except OSError:
        pass
    logical = os.cpu_count() or 1
    return model, (len(cores) or logical), logical


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def _blis_threads(jc, ic):
    os.environ["BLIS_JC_NT"] = str(jc)
    os.environ["BLIS_IC_NT"] = str(ic)
    os.environ["BLIS_JR_NT"] = "1"
    os.environ["BLIS_IR_NT"] = "1"
    os.environ["OMP_NUM_THREADS"] = str(jc * ic)


def cpu_reference_sample(T_np, S, ms, factoring=None):
    """One timed run of the reference's stock -blis path on the first `ms`
    SNPs of the table (single region): BLIS cblas_dsyrk counts (BLIS threads
    from `factoring` = (JC, IC) ways) + get_pairwise_ld_score on one thread,
    as correlate() runs them.  Without the BLIS build, the reference
    micro-kernel in a BLIS-style loop stands in (and says so).  Returns
    (seconds, counts seconds, epilogue seconds, threads, kind of path)."""
    import numpy as np
    oracle = _oracle()
    _, phys, logical = host_cpu()
    blis = oracle.blis_available()
    factoring = factoring or (1, phys)
    A = np.ascontiguousarray(T_np[:ms])
    bc = oracle.bitcounts(A)
    if blis:
        _blis_threads(*factoring)
        _, _, tg, tl = oracle.ref_blis_counts_ld(A, bc, S)
        kind = (f"qLD-compute -blis path: BLIS 0.1.8 binary_gemm cblas_dsyrk (BLIS_JC_NT="
                f"{factoring[0]}, BLIS_IC_NT={factoring[1]}) + get_pairwise_ld_score (1 thread)")
        return tg + tl, tg, tl, factoring[0] * factoring[1], kind
    t0 = time.perf_counter()
    C = oracle.ref_counts_ukr(A, None, lower_only=True, threads=logical)
    t1 = time.perf_counter()
    oracle.ref_ld_score(bc, bc, C, S, threads=1)
    t2 = time.perf_counter()
    kind = ("stand-in (BLIS not built): bin_gemm_2x2 in a BLIS-style loop + "
            "get_pairwise_ld_score (1 thread)")
    return t2 - t0, t1 - t0, t2 - t1, logical, kind


def size_reference_sample(T_np, S, seconds_target, factoring=None):
    """SNP count Ms whose single-region sample takes ~seconds_target, capped
    so its C / results buffers (12 bytes per entry) fit in a quarter of the
    host's free memory."""
    try:
        mem = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_AVPHYS_PAGES")
    except (ValueError, OSError):
        mem = 16 << 30
    m = min(T_np.shape[0], int((mem / 4 / 12) ** 0.5))
    ms = min(m, 1024)
    t = cpu_reference_sample(T_np, S, ms, factoring)[0]
    while t < seconds_target / 8 and ms < m:
        ms = min(m, ms * 2)
        t = cpu_reference_sample(T_np, S, ms, factoring)[0]
    if t < seconds_target / 2 and ms < m:
        ms = min(m, int(ms * (seconds_target / max(t, 1e-3)) ** 0.5))
    return ms


def cpu_reference_rate(T_np, S, seconds_target=8.0, factoring=None, ms=None):
    """Pairs/s of the reference's stock CPU path on a bounded sample of the
    region.  Returns (pairs/s, threads, sample description, path)."""
    model, phys, _ = host_cpu()
    ms = ms or size_reference_sample(T_np, S, seconds_target, factoring)
    t, tg, tl, threads, kind = cpu_reference_sample(T_np, S, ms, factoring)
    desc = (f"first {ms} SNPs of the region, all {ms * (ms - 1) // 2} pairs, {t:.2f} s "
            f"(counts {tg:.2f} s, epilogue {tl:.2f} s); {model}, {phys} physical cores")
    return ms * (ms - 1) / 2 / t, threads, desc, kind


_FACTORING = {}   # the headline's best (JC, IC) BLIS split, reused by the sections


def cpu_reference_tasks(tasks):
    """The reference's stock -blis path over `tasks`, each (A, B or None, S)
    host tables: per task BLIS cblas_dsyrk (B None: a single region) or
    cblas_dgemm counts, then get_pairwise_ld_score on one thread, one task
    after another as an -inputList run does.  Bit counts are made before the
    clock starts (qLD makes them while loading).  Returns (seconds, threads,
    path)."""
    oracle = _oracle()
    _, phys, logical = host_cpu()
    prepared = [(A, oracle.bitcounts(A), B, None if B is None else oracle.bitcounts(B), S)
                for A, B, S in tasks]
    total = 0.0
    if oracle.blis_available():
        jc, ic = _FACTORING.get("blis", (1, phys))
        _blis_threads(jc, ic)
        for A, bcA, B, bcB, S in prepared:
            _, _, tg, tl = oracle.ref_blis_counts_ld(A, bcA, S, B=B, bcB=bcB)
            total += tg + tl
        return total, jc * ic, (f"qLD-compute -blis path per task: BLIS 0.1.8 binary_gemm "
                                f"cblas_dsyrk / cblas_dgemm (BLIS_JC_NT={jc}, BLIS_IC_NT={ic}) + "
                                f"get_pairwise_ld_score (1 thread)")
    for A, bcA, B, bcB, S in prepared:
        t0 = time.perf_counter()
        C = oracle.ref_counts_ukr(A, B, lower_only=B is None, threads=logical)
        oracle.ref_ld_score(bcA, bcA if B is None else bcB, C, S, threads=1)
        total += time.perf_counter() - t0
    return total, logical, ("stand-in (BLIS not built): bin_gemm_2x2 in a BLIS-style loop + "
                            "get_pairwise_ld_score (1 thread)")


def cpu_sampled_baseline(make_tasks, sizes, seconds_target=6.0):
    """cpu_baseline of a section: make_tasks(size) -> (tasks, pairs, description)
    for a growing sample size; the first size is a probe whose time sets the
    final size (time taken as proportional to size, capped at sizes[1])."""
    model, phys, _ = host_cpu()
    probe, cap = sizes
    tasks, pairs, _ = make_tasks(probe)
    t, _, _ = cpu_reference_tasks(tasks)
    size = max(probe, min(cap, int(probe * seconds_target / max(t, 1e-3))))
    tasks, pairs, desc = make_tasks(size)
    t, threads, path = cpu_reference_tasks(tasks)
    return {"value": pairs / t, "unit": "pairs/s", "cores": threads, "kind": "reference",
            "path": path, "sample": f"{desc}: {pairs} pairs in {t:.2f} s; {model}, "
                                    f"{phys} physical cores"}


def best_blis_factoring(T_np, S):
    """The fastest (JC, IC) split of the host's physical cores for the counts,
    tried on a small sample (the reference's README leaves BLIS threading to
    the BLIS_*_NT variables)."""
    import numpy as np
    oracle = _oracle()
    _, phys, _ = host_cpu()
    if not oracle.blis_available():
        return None
    cands = sorted({(1, phys), (2, max(1, phys // 2)), (phys, 1)})
    ms = min(T_np.shape[0], 6144)
    A = np.ascontiguousarray(T_np[:ms])
    bc = oracle.bitcounts(A)
    C = np.empty((ms, ms), np.uint64)
    R = np.empty((ms, ms), np.float32)
    best = None
    for f in cands:
        _blis_threads(*f)
        oracle.ref_blis_counts_ld(A, bc, S, C=C, results=R)
        _, _, tg, _ = oracle.ref_blis_counts_ld(A, bc, S, C=C, results=R)
        if best is None or tg < best[0]:
            best = (tg, f)
    return best[1]


def reference_arm(args, rank, world):
    import numpy as np
    cfg = arm_config(args, world)
    if rank != 0:
        return
    T, S = make_table(args.workload, "cpu")
    T_np = T.numpy().view(np.uint64)
    if args.snps:
        T_np = T_np[:args.snps]
    fac = best_blis_factoring(T_np, S)
    ms = size_reference_sample(T_np, S, 4.0, fac)
    for _ in range(args.warmup):
        cpu_reference_rate(T_np, S, factoring=fac, ms=max(1024, ms // 2))
    vals = []
    desc = kind = ""
    cores = os.cpu_count()
    for _ in range(args.steps):
        v, cores, desc, kind = cpu_reference_rate(T_np, S, factoring=fac, ms=ms)
        vals.append(v)
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64 popcount / f32 r2", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": "reference",
                             "path": kind, "sample": desc},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ shared timing --

def lower_tri_d2h_bytes(m, band=3840, block=512):
    """Bytes qld_cuda_ld moves to the host for a single region of m SNPs:
    B rows in bands (the default 4,096 rows rounded to whole 240-row tiles of
    the 4-bit kernel), each band in 512-row 2-D blocks of columns [r0, m)."""
    total = 0
    for b0 in range(0, m, band):
        b1 = min(m, b0 + band)
        for r0 in range(b0, b1, block):
            total += (min(block, b1 - r0)) * (m - r0) * 4
    return total


def max_over_ranks(value, world, device):
    """The largest of the ranks' values; every rank calls it (a no-op at 1)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def timed_steps(step, st, steps, warmup, flush, gpu, world=1):
    """W warm-up steps, then K steps each after an L2-flushing write, timed
    with CUDA events on the launching stream `st`, with nvidia-smi clock
    samples over the timed region.  Returns (per-step ms, clocks)."""
    import torch
    import torch.distributed as dist
    for _ in range(warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(gpu) as clk:
        clk.mark_start()
        for i in range(steps):
            flush.zero_()
            ev[i][0].record(st)
            step()
            ev[i][1].record(st)
        torch.cuda.synchronize()
        clk.mark_end()
    if world > 1:
        dist.barrier()
    return [a.elapsed_time(b) for a, b in ev], clk.summary()


def new_context(local_rank, args, kernel=None, r2_mode=None):
    from qld_b200 import api
    ctx = api.Context(local_rank)
    kern = {"auto": api.KERNEL_AUTO, "popc": api.KERNEL_POPC, "mma": api.KERNEL_MMA,
            "fp4": api.KERNEL_FP4}[kernel or args.kernel]
    ctx.set_option(api.OPT_KERNEL, kern)
    ctx.set_option(api.OPT_MMA_TILE, args.mma_tile)
    ctx.set_option(api.OPT_SM_PAIR, args.sm_pair)
    mode = r2_mode or args.r2_mode
    ctx.set_option(api.OPT_R2_MODE, api.R2_REFERENCE if mode == "reference" else api.R2_EXACT)
    ctx.set_option(api.OPT_PROFILE, 1)
    return ctx


def padded(T, dev):
    """Device copy of a packed table with an even row pitch (16-byte rows)."""
    import torch
    m, K = T.shape
    lda = K + (K & 1)
    Tp = torch.zeros(m, lda, dtype=torch.int64, device=dev)
    Tp[:, :K] = T
    return Tp, lda


# ------------------------------------------------------------------ parity --

def region_parity(ctx, Tp, bc, m, lda, K, S, out, st, mode, seed=0, per_block=2, block=120):
    """Sampled oracle check of a single-region output `out` (m x m, B-major,
    entries j >= i defined) left by the timed launches: ~per_block B rows from
    every `block` rows plus the first and last rows, against every A row.
    Counts come from one more launch of the same call with the counts output
    on, which must also reproduce the checked r^2 rows bit for bit."""
    import numpy as np
    import torch
    oracle = _oracle()
    rng = np.random.default_rng(seed)
    rows = oracle.tile_row_samples(m, block, per_block, rng, extra=(0, m - 1))
    idx = torch.as_tensor(rows, device=out.device)
    got = out.index_select(0, idx).cpu().numpy()
    cnt = torch.empty(m, m, dtype=torch.int32, device=out.device)
    ctx.ld_device(Tp, bc, m, lda, Tp, bc, m, lda, K, S, True, out, m, counts=cnt, ldc=m,
                  stream=st)
    ctx.sync(stream=st)
    again = out.index_select(0, idx).cpu().numpy()
    got_c = cnt.index_select(0, idx).cpu().numpy().view(np.uint32)
    del cnt
    T_np = Tp[:, :K].contiguous().cpu().numpy().view(np.uint64)
    bc_np = bc.cpu().numpy().astype(np.uint32)
    valid = np.arange(m)[None, :] >= rows[:, None]
    res = oracle.check_rows(T_np, bc_np, T_np[rows], bc_np[rows], S, got, valid,
                            got_counts=got_c, mode=mode)
    res["rerun_bit_identical"] = bool(np.array_equal(got[valid].view(np.uint32),
                                                     again[valid].view(np.uint32)))
    res["ok"] = res["ok"] and res["rerun_bit_identical"]
    res["sample"] = f"{len(rows)} B rows (~{per_block} per {block}-row block) x all {m} A rows"
    return res


# -------------------------------------------------------------------- ours --

def ours_arm(args, rank, world, local_rank):
    import numpy as np
    import torch

    from qld_b200 import api, synth

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    cfg = arm_config(args, world)

    split = args.split   # at N = 1 a one-part split: the same path over the whole region
    T, S = make_table(args.workload, dev, seed_offset=0 if split else rank)
    if args.snps:
        T = T[:args.snps].contiguous()
    m, K = T.shape
    Tp, lda = padded(T, dev)
    bc = synth.popcount_rows(T).to(torch.int32)
    r0, r1 = 0, m
    if split:   # this rank's tile rows of the one region
        r0, r1 = api.split_rows(m, m, K, True, api.KERNEL_AUTO, rank, world)
    out = torch.empty(max(1, r1 - r0), m, dtype=torch.float32, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)

    ctx = new_context(local_rank, args)
    # A dedicated stream: torch's default stream is the legacy NULL stream,
    # which the C ABI reads as "the context's own stream".
    st = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(st)

    def step():
        if split:
            ctx.ld_device_part(Tp, bc, m, lda, Tp, bc, m, lda, K, S, True, out, m, rank, world,
                               stream=st)
        else:
            ctx.ld_device(Tp, bc, m, lda, Tp, bc, m, lda, K, S, True, out, m, stream=st)

    tuned = None
    if args.autotune and args.kernel == "auto":
        tk, topt, tms = ctx.autotune(m, m, K, True)
        tuned = {"kernel": tk, "option": topt, "ms_per_launch_tuned": tms,
                 "measured_at": f"{min(m, 16384)}x{min(m, 16384)}x{K} words"}

    for _ in range(args.warmup):
        flush.zero_()
        step()
    ctx.sync(stream=st)
    ctx.stats(reset=True)
    torch.cuda.nvtx.range_push("qld_timed")
    step_ms, clocks = timed_steps(step, st, args.steps, 0, flush, local_rank, world)
    torch.cuda.nvtx.range_pop()
    ctx.sync(stream=st)
    total_ms = sum(step_ms)
    stats = ctx.stats(reset=True)

    pairs = m * (m - 1) / 2
    total_ms_max = max_over_ranks(total_ms, world, dev)
    regions = 1 if split else world   # the split ranks share one region
    value = pairs * args.steps * regions / (total_ms_max * 1e-3)

    # roofline of the counts kernel
    kern_ms = stats.counts_kernel_ms / max(1, stats.counts_launches)
    bitops = pairs * 64 * K
    # this rank's pairs: B rows [r0, r1) of the triangle (all of it unless split)
    rank_pairs = sum(m - 1 - i for i in range(r0, r1)) if split else pairs
    variant = stats.last_kernel
    roof = kernel_roofline(ctx, variant, rank_pairs * 64 * K, kern_ms, dev)
    alg_bytes = m * K * 8 * 2 + rank_pairs * 4
    sm_pair = args.sm_pair
    if tuned is not None and tuned["kernel"] == 3 and sm_pair == 0:
        sm_pair = tuned["option"]
    roof["traffic"] = measured_traffic(variant, cfg["workload"], sm_pair, args.r2_mode)
    roof["algorithmic_bytes_per_launch"] = alg_bytes
    roof["kernel_ms"] = kern_ms
    mp = measured_peaks()
    roof["hbm_frac_of_measured"] = (alg_bytes / (kern_ms * 1e-3) / 1e9) / mp["hbm_gbs"]
    roof["hbm_peak_gbs"] = mp["hbm_gbs"]
    roof["hbm_peak_source"] = mp["source"]
    if variant == api.KERNEL_FP4 and sm_pair in (0, 2) and not split and K * 64 <= 1 << 24:
        roof["shared_memory"] = smem_roofline(m, m, K, True, kern_ms, clocks.get("sm_mhz"))

    line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps,
            "higher_is_better": True, "scaling": "strong" if split else "weak",
            "vs_baseline": None,
            "dtype": "u64 popcount / f32 r2", "data": "synthetic", "config": cfg,
            "bitops_per_s": bitops * args.steps * regions / (total_ms_max * 1e-3),
            "gpu_launches": stats.kernel_launches, "kernel_variant": variant,
            "roofline": roof, "clocks": clocks}
    if tuned is not None:
        line["autotune"] = tuned

    if split:
        line["split_rows"] = [r0, r1]
    # ---- sampled oracle check of the output the timed steps wrote
    if not args.no_parity and rank == 0 and not split:
        line["parity"] = region_parity(ctx, Tp, bc, m, lda, K, S, out, st, args.r2_mode,
                                       seed=11)

    # ---- e2e through the host-buffer C-ABI call
    if split and not args.no_e2e:
        line["e2e_note"] = "no host-buffer form of a split task: e2e is measured without --split"
    if not args.no_e2e and not split:
        Th = ctx.pinned_empty((m, K), np.uint64)
        Th[:] = T.cpu().numpy().view(np.uint64)
        bch = ctx.pinned_empty((m,), np.uint32)
        bch[:] = bc.cpu().numpy().view(np.uint32)
        outh = ctx.pinned_empty((m, m), np.float32)
        for _ in range(max(1, args.warmup)):
            ctx.ld(Th, bch, S=S, r2_out=outh)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        ts = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            ctx.ld(Th, bch, S=S, r2_out=outh)
            ts.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(sum(ts), world, dev)
        line["e2e"] = {"value": pairs * args.steps * world / e2e_s, "unit": "pairs/s",
                       "h2d_bytes_per_step": m * K * 8 + m * 4,
                       "d2h_bytes_per_step": lower_tri_d2h_bytes(m),
                       "api": "qld_cuda_ld (pinned host buffers)"}
        del Th, bch, outh

    if rank == 0 and world == 1 and not args.no_cpu:
        T_np = T.cpu().numpy().view(np.uint64)
        fac = best_blis_factoring(T_np, S)
        if fac:
            _FACTORING["blis"] = fac
        v, cores, desc, kind = cpu_reference_rate(T_np, S, factoring=fac)
        line["cpu_baseline"] = {"value": v, "unit": "pairs/s", "cores": cores, "kind": "reference",
                                "path": kind, "sample": desc}

    sections = [] if args.sections in ("", "none") else args.sections.split(",")
    if world == 1 and args.workload == "single_region" and not args.snps:
        if "reference_mode" in sections:
            line["reference_mode"] = section_reference_mode(args, Tp, bc, m, lda, K, S, out,
                                                            flush, st, local_rank)
    ctx.close()
    del out, Tp, T, bc
    torch.cuda.empty_cache()
    if world == 1 and args.workload == "single_region" and not args.snps:
        for name, fn in (("all_pairs", section_all_pairs), ("windowed", section_windowed),
                         ("batched", section_batched), ("served", section_served)):
            if name in sections:
                line[name] = fn(args, local_rank, flush)
                torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- sections --

def section_reference_mode(args, Tp, bc, m, lda, K, S, out, flush, st, local_rank):
    """The headline region with r^2 in QLD_R2_REFERENCE mode (bit-identical to
    qLD-compute's get_pairwise_ld_score; the drop-in's default), automatic
    kernel choice."""
    from qld_b200 import api
    ctx = new_context(local_rank, args, r2_mode="reference")

    def step():
        ctx.ld_device(Tp, bc, m, lda, Tp, bc, m, lda, K, S, True, out, m, stream=st)
    ctx.stats(reset=True)
    step_ms, clocks = timed_steps(step, st, args.steps, args.warmup, flush, local_rank)
    ctx.sync(stream=st)
    stats = ctx.stats(reset=True)
    pairs = m * (m - 1) / 2
    ms = sum(step_ms) / len(step_ms)
    kern_ms = stats.counts_kernel_ms / max(1, stats.counts_launches)
    res = {"value": pairs / (ms * 1e-3), "unit": "pairs/s", "ms_per_step": ms,
           "steps": args.steps, "kernel_variant": stats.last_kernel,
           "gpu_launches": stats.kernel_launches // (args.steps + args.warmup),
           "roofline": dict(kernel_roofline(ctx, stats.last_kernel, pairs * 64 * K, kern_ms,
                                            None, int8_context=False), kernel_ms=kern_ms),
           "clocks": clocks}
    if stats.last_kernel == api.KERNEL_FP4 and args.sm_pair in (0, 2):
        res["roofline"]["shared_memory"] = smem_roofline(m, m, K, True, kern_ms,
                                                         clocks.get("sm_mhz"))
    if not args.no_parity:
        res["parity"] = region_parity(ctx, Tp, bc, m, lda, K, S, out, st, "reference", seed=12)
    ctx.close()
    return res


def section_all_pairs(args, local_rank, flush):
    """All-pairs r^2, one region: 2,048 SNPs x 4,096 samples (iid, Uniform(0.05,
    0.5) frequencies), every B row checked against the oracle."""
    import torch

    from qld_b200 import synth
    dev = torch.device("cuda", local_rank)
    T, S = synth.all_pairs_workload(device=dev, seed=1)
    m, K = T.shape
    Tp, lda = padded(T, dev)
    bc = synth.popcount_rows(T).to(torch.int32)
    out = torch.empty(m, m, dtype=torch.float32, device=dev)
    ctx = new_context(local_rank, args, r2_mode="exact")
    st = torch.cuda.current_stream(dev)

    def step():
        ctx.ld_device(Tp, bc, m, lda, Tp, bc, m, lda, K, S, True, out, m, stream=st)
    ctx.stats(reset=True)
    step_ms, clocks = timed_steps(step, st, args.steps, args.warmup, flush, local_rank)
    ctx.sync(stream=st)
    stats = ctx.stats(reset=True)
    pairs = m * (m - 1) / 2
    ms = sum(step_ms) / len(step_ms)
    kern_ms = stats.counts_kernel_ms / max(1, stats.counts_launches)
    res = {"config": {"workload": "all_pairs_2048x4096_symmetric", "snps": m, "haplotypes": S,
                      "words_per_snp": K, "model": "iid Bernoulli", "freq": "Uniform(0.05,0.5)",
                      "l2": "512 MB flush write between timed steps"},
           "value": pairs / (ms * 1e-3), "unit": "pairs/s", "ms_per_step": ms,
           "steps": args.steps, "kernel_variant": stats.last_kernel, "kernel_ms": kern_ms,
           "gpu_launches": stats.kernel_launches // (args.steps + args.warmup),
           "clocks": clocks}
    if not args.no_parity:
        res["parity"] = region_parity(ctx, Tp, bc, m, lda, K, S, out, st, "exact", seed=13,
                                      per_block=120)
    ctx.close()
    return res


def band_pairs(m, W):
    return sum(min(W, m - 1 - i) for i in range(m)) if m < 50_000 else \
        W * (m - W) + W * (W - 1) // 2


def band_parity(T_np, bc_np, S, out_rows, rows, W, mode="exact", counts_rows=None):
    """Sampled oracle check of band rows: out_rows[k, d] = r^2(B row rows[k],
    A row rows[k]+1+d) for the d that stay inside the table."""
    import numpy as np
    oracle = _oracle()
    m = T_np.shape[0]
    groups = []
    for k, i in enumerate(rows):
        w = min(W, m - 1 - int(i))
        if w <= 0:
            continue
        groups.append(dict(A=T_np[i + 1:i + 1 + w], bcA=bc_np[i + 1:i + 1 + w],
                           B=T_np[i:i + 1], bcB=bc_np[i:i + 1], S=S,
                           got=out_rows[k:k + 1, :w], valid=np.ones((1, w), bool),
                           counts=None if counts_rows is None else counts_rows[k:k + 1, :w]))
    return oracle.check_groups(groups, mode=mode)


def section_windowed(args, local_rank, flush, m_full=None):
    """Windowed workload: 200,000 SNPs x 100,000 haplotypes (copying model,
    100 founders), r^2 for pairs within `band` SNPs, FP32 band array."""
    import numpy as np
    import torch

    from qld_b200 import api, synth
    oracle = _oracle()
    dev = torch.device("cuda", local_rank)
    T, S = synth.windowed_workload(device=dev, m=m_full or args.snps or 200_000, seed=3)
    m, K = T.shape
    W = args.band
    Tp, lda = padded(T, dev)
    bc = synth.popcount_rows(T).to(torch.int32)
    out = torch.empty(m, W, dtype=torch.float32, device=dev)
    pairs = band_pairs(m, W)
    ctx = new_context(local_rank, args)
    st = torch.cuda.current_stream(dev)

    def step():
        ctx.ld_band_device(Tp, bc, m, lda, K, S, W, out, W, stream=st)
    ctx.stats(reset=True)
    step_ms, clocks = timed_steps(step, st, args.steps, args.warmup, flush, local_rank)
    ctx.sync(stream=st)
    stats = ctx.stats(reset=True)
    ms = sum(step_ms) / len(step_ms)
    kern_ms = stats.counts_kernel_ms / max(1, stats.counts_launches)
    bitops = pairs * 64 * K
    res = {"config": {"workload": f"windowed_{m}x{S}_band{W}", "snps": m, "haplotypes": S,
                      "words_per_snp": K, "band": W, "model": "copying(100 founders)",
                      "pairs_per_step": pairs, "l2": "inputs (2.5 GB) and outputs larger than L2"},
           "value": pairs / (ms * 1e-3), "unit": "pairs/s", "ms_per_step": ms,
           "steps": args.steps, "bitops_per_s": bitops / (ms * 1e-3),
           "gpu_launches": stats.kernel_launches // (args.steps + args.warmup),
           "kernel_variant": stats.last_kernel,
           "roofline": dict(kernel_roofline(ctx, stats.last_kernel, bitops, kern_ms, dev,
                                            int8_context=False), kernel_ms=kern_ms),
           "clocks": clocks}
    T_np = None
    if not args.no_parity:
        rng = np.random.default_rng(14)
        rows = oracle.tile_row_samples(m, 240, 1, rng, extra=(0, m - W - 1, m - 2))
        idx = torch.as_tensor(rows, device=dev)
        got = out.index_select(0, idx).cpu().numpy()
        cnt = torch.empty(m, W, dtype=torch.int32, device=dev)
        ctx.ld_band_device(Tp, bc, m, lda, K, S, W, out, W, counts=cnt, ldc=W, stream=st)
        ctx.sync(stream=st)
        again = out.index_select(0, idx).cpu().numpy()
        got_c = cnt.index_select(0, idx).cpu().numpy().view(np.uint32)
        del cnt
        T_np = T.cpu().numpy().view(np.uint64)
        bc_np = bc.cpu().numpy().astype(np.uint32)
        par = band_parity(T_np, bc_np, S, got, rows, W, mode=args.r2_mode, counts_rows=got_c)
        inside = np.arange(W)[None, :] < (m - 1 - rows)[:, None]
        par["rerun_bit_identical"] = bool(np.array_equal(got[inside].view(np.uint32),
                                                         again[inside].view(np.uint32)))
        par["ok"] = par["ok"] and par["rerun_bit_identical"]
        par["sample"] = f"{len(rows)} band rows (one per 240-row block) x their {W} pairs"
        res["parity"] = par
    if not args.no_e2e:
        Th = ctx.pinned_empty((m, K), np.uint64)
        Th[:] = T_np if T_np is not None else T.cpu().numpy().view(np.uint64)
        bch = ctx.pinned_empty((m,), np.uint32)
        bch[:] = bc.cpu().numpy().view(np.uint32)
        outh = ctx.pinned_empty((m, W), np.float32)
        ctx.set_option(api.OPT_BAND_ROWS, 8192)
        for _ in range(max(1, args.warmup)):
            ctx.ld_band(Th, bch, S=S, band=W, r2_out=outh)
        ts = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            ctx.ld_band(Th, bch, S=S, band=W, r2_out=outh)
            ts.append(time.perf_counter() - t0)
        res["e2e"] = {"value": pairs * len(ts) / sum(ts), "unit": "pairs/s",
                      "h2d_bytes_per_step": m * K * 8 + m * 4,
                      "d2h_bytes_per_step": m * W * 4,
                      "api": "qld_cuda_ld_band (pinned host buffers, streamed)"}
        del Th, bch, outh
    if not args.no_cpu:
        b0 = (m // 2) // 256 * 256

        def tasks(nb):
            # one rectangle of a split_region-style tiling of the band: B rows
            # [b0, b0 + nb) against the A rows [b0 + 1, b0 + nb - 1 + W] their
            # band pairs need; nb * W band pairs
            A = T[b0 + 1:b0 + nb + W].cpu().numpy().view(np.uint64)
            B = T[b0:b0 + nb].cpu().numpy().view(np.uint64)
            return ([(A, B, S)], nb * W,
                    f"one band tile: B rows [{b0}, {b0 + nb}) x A rows [{b0 + 1}, "
                    f"{b0 + nb + W - 1}] (rectangle computed whole, band pairs counted)")
        res["cpu_baseline"] = cpu_sampled_baseline(tasks, (128, 8192))
    ctx.close()
    return res


def make_batched_jobs(njobs, dev, seed=0):
    """Batched workload: njobs independent tasks; SNPs per side log-uniform in
    [64, 8192], samples log-uniform in [1000, 50000], per-SNP frequencies
    Beta(0.5, 0.5), iid genotypes; even tasks single region (triangle), odd
    tasks two regions (rectangle)."""
    import numpy as np
    import torch

    from qld_b200 import synth
    rng = np.random.default_rng(seed)
    Ms = synth.log_uniform_ints(njobs, 64, 8192, rng)
    Ns = synth.log_uniform_ints(njobs, 64, 8192, rng)
    Ss = synth.log_uniform_ints(njobs, 1000, 50000, rng)
    jobs, pairs, bitops = [], 0, 0
    for j in range(njobs):
        sym = j % 2 == 0
        m = int(Ms[j])
        n = m if sym else int(Ns[j])
        S = int(Ss[j])
        rows = m if sym else m + n
        f = torch.from_numpy(rng.beta(0.5, 0.5, rows).astype(np.float32))
        T = synth.iid_table(rows, S, f, seed * 100003 + j, device=dev, chunk=2048)
        K = T.shape[1]
        Tp, lda = padded(T, dev)
        del T
        bc = synth.popcount_rows(Tp).to(torch.int32)
        A, bcA = Tp[:m], bc[:m]
        B, bcB = (A, bcA) if sym else (Tp[m:], bc[m:])
        r2 = torch.empty(n, m, dtype=torch.float32, device=dev)
        jobs.append(dict(A=A, bcA=bcA, m=m, lda=lda, B=B, bcB=bcB, n=n, ldb=lda, K=K, S=S,
                         symmetric=sym, r2=r2, ldr=m))
        p = m * (m - 1) // 2 if sym else m * n
        pairs += p
        bitops += p * 64 * K
    return jobs, pairs, bitops


def batch_parity(jobs, rows_per_job=2, seed=0, chunk=256, mode="exact"):
    """Every job of a batched call, a few B rows each (one random row and the
    last row, whose tile is among the last the queue hands out), checked
    against the oracle over all of the job's A rows."""
    import numpy as np
    import torch
    oracle = _oracle()
    rng = np.random.default_rng(seed)
    total = None
    for c0 in range(0, len(jobs), chunk):
        groups = []
        for j in jobs[c0:c0 + chunk]:
            m, n, K = j["m"], j["n"], j["K"]
            rows = sorted({int(rng.integers(0, n)), n - 1} if rows_per_job >= 2
                          else {n - 1})
            idx = torch.as_tensor(rows, device=j["r2"].device)
            got = j["r2"].index_select(0, idx).cpu().numpy()
            A = j["A"][:, :K].contiguous().cpu().numpy().view(np.uint64)
            B = j["B"].index_select(0, idx)[:, :K].contiguous().cpu().numpy().view(np.uint64)
            bcA = j["bcA"].cpu().numpy().astype(np.uint32)
            bcB = j["bcB"].index_select(0, idx).cpu().numpy().astype(np.uint32)
            r = np.array(rows)
            valid = (np.arange(m)[None, :] >= r[:, None]) if j["symmetric"] \
                else np.ones((len(rows), m), bool)
            groups.append(dict(A=A, bcA=bcA, B=B, bcB=bcB, S=j["S"], got=got, valid=valid))
        res = oracle.check_groups(groups, mode=mode)
        if total is None:
            total = res
        else:
            n0, n1 = total["r2_rel_count"], res["r2_rel_count"]
            if n0 + n1:
                total["r2_mean_rel"] = (total["r2_mean_rel"] * n0 + res["r2_mean_rel"] * n1) / (n0 + n1)
            for k in ("rows_checked", "pairs_checked", "r2_rel_count"):
                total[k] += res[k]
            total["r2_max_rel"] = max(total["r2_max_rel"], res["r2_max_rel"])
            for k in ("r2_within_tol", "r2_bit_identical"):
                if k in res:
                    total[k] = total[k] and res[k]
            total["ok"] = total["ok"] and res["ok"]
    total["sample"] = f"all {len(jobs)} jobs x {rows_per_job} B rows x all A rows"
    return total


def section_batched(args, local_rank, flush):
    """Batched workload: the same tasks as one persistent launch -- replayed
    from a CUDA graph captured once (the headline), and as a direct batched
    call per step -- and as per-task launches."""
    import torch

    from qld_b200 import api
    dev = torch.device("cuda", local_rank)
    jobs, pairs, bitops = make_batched_jobs(args.jobs, dev, seed=0)
    ctx = api.Context(local_rank)
    ctx.set_option(api.OPT_PROFILE, 1)
    ctx.set_option(api.OPT_R2_MODE,
                   api.R2_REFERENCE if args.r2_mode == "reference" else api.R2_EXACT)
    st = torch.cuda.current_stream(dev)

    def batched():
        ctx.ld_batch(jobs, stream=st)

    def plain():
        for j in jobs:
            ctx.ld_device(j["A"], j["bcA"], j["m"], j["lda"], j["B"], j["bcB"], j["n"],
                          j["ldb"], j["K"], j["S"], j["symmetric"], j["r2"], j["ldr"], stream=st)

    t0 = time.perf_counter()
    plan = ctx.batch_plan(jobs)
    plan_ms = (time.perf_counter() - t0) * 1e3

    def graph():
        plan.run(stream=st)

    res = {}
    calls = args.steps + args.warmup
    for name, fn in (("plain", plain), ("batched", batched), ("graph", graph)):
        ctx.stats(reset=True)
        torch.cuda.nvtx.range_push(f"qld_timed_{name}")
        step_ms, clocks = timed_steps(fn, st, args.steps, args.warmup, flush, local_rank)
        torch.cuda.nvtx.range_pop()
        ctx.sync(stream=st)
        res[name] = (sum(step_ms) / len(step_ms), ctx.stats(reset=True), clocks)
    plan.close()
    ms_b, st_b, clk_b = res["graph"]
    ms_d, st_d, clk_d = res["batched"]
    ms_p, st_p, clk_p = res["plain"]
    out = {"config": {"workload": f"batched_{args.jobs}_tasks", "snps_per_side": "logU(64,8192)",
                      "samples": "logU(1000,50000)", "freq": "Beta(0.5,0.5)",
                      "half": "single region (triangle) / two regions (rectangle)",
                      "pairs_per_step": pairs, "bitops_per_step": bitops,
                      "l2": "512 MB flush write between timed steps"},
           "form": "qld_cuda_batch_run: replay of the call captured once as a CUDA graph "
                   "(qld_cuda_batch_plan; tensor maps and job table built at plan time)",
           "value": pairs / (ms_b * 1e-3), "unit": "pairs/s", "ms_per_step": ms_b,
           "kernel_ms": st_b.counts_kernel_ms / calls,
           "steps": args.steps, "bitops_per_s": bitops / (ms_b * 1e-3),
           "gpu_launches": st_b.kernel_launches // calls,
           "clocks": clk_b, "plan_ms": plan_ms,
           "direct": {"form": "qld_cuda_ld_batch per step (tensor maps and job table built "
                              "per call)",
                      "value": pairs / (ms_d * 1e-3), "unit": "pairs/s", "ms_per_step": ms_d,
                      "kernel_ms": st_d.counts_kernel_ms / calls,
                      "gpu_launches": st_d.kernel_launches // calls, "clocks": clk_d,
                      "speedup_vs_plain": ms_p / ms_d},
           "plain": {"value": pairs / (ms_p * 1e-3), "unit": "pairs/s", "ms_per_step": ms_p,
                     "kernel_ms": st_p.counts_kernel_ms / calls,
                     "launches_per_step": st_p.kernel_launches // calls,
                     "clocks": clk_p},
           "speedup_vs_plain": ms_p / ms_b}
    if not args.no_parity:
        # the graph replay ran last: its outputs are what the jobs hold now
        out["parity"] = batch_parity(jobs, seed=15, mode=args.r2_mode)
    if not args.no_cpu:
        import numpy as np

        def host(t, rows, K):
            return np.ascontiguousarray(t[:rows, :K].cpu().numpy().view(np.uint64))

        def tasks(count):
            # every (njobs // count)-th job, as one -inputList task each
            stride = max(1, len(jobs) // count)
            picked = jobs[::stride]
            ts, p = [], 0
            for j in picked:
                A = host(j["A"], j["m"], j["K"])
                B = None if j["symmetric"] else host(j["B"], j["n"], j["K"])
                ts.append((A, B, j["S"]))
                p += j["m"] * (j["m"] - 1) // 2 if j["symmetric"] else j["m"] * j["n"]
            return ts, p, f"every {stride}th of the {len(jobs)} tasks ({len(picked)} tasks)"
        out["cpu_baseline"] = cpu_sampled_baseline(tasks, (16, len(jobs)))
    ctx.close()
    del jobs
    return out


def section_served(args, local_rank, flush=None, check_queries=12):
    """Served workload: 22 resident chromosomes (50,000-250,000 SNPs x 20,000
    haplotypes, copying model), a Poisson stream of region-vs-region queries
    (each side 100-20,000 SNPs, uniform placement), admitted by output memory.
    The arrival rate is `load` x the capacity measured by a saturated burst.
    Parity: `check_queries` more queries from the same distribution, their r^2
    blocks fetched and three B rows each checked against the oracle, and the
    device summary (count >= threshold, maximum) against the fetched block."""
    import threading

    import numpy as np
    import torch

    from qld_b200 import api, synth
    oracle = _oracle()
    dev = torch.device("cuda", local_rank)
    rng = np.random.default_rng(5)
    H = 20_000
    srv = api.Server(local_rank, pool_bytes=args.pool_gb << 30, max_inflight=args.inflight)
    sizes, tables = [], []
    for c in range(22):
        m = int(rng.integers(50_000, 250_001))
        f = synth.beta_freqs(m, 0.1, 1.0, 100 + c, device=dev, clip_min=1.0 / H)
        T = synth.copying_table(m, H, 50, 50, 500, 0.01, f, 100 + c, device=dev)
        bc = synth.popcount_rows(T).to(torch.int32)
        srv.add_table(T, bc, H)
        sizes.append(m)
        tables.append((T, bc))
    torch.cuda.synchronize()

    def draw(n):
        qs = []
        for _ in range(n):
            c = int(rng.integers(0, 22))
            la, lb = (int(x) for x in rng.integers(100, 20_001, 2))
            a0 = int(rng.integers(0, sizes[c] - la + 1))
            b0 = int(rng.integers(0, sizes[c] - lb + 1))
            qs.append((c, a0, a0 + la, b0, b0 + lb))
        return qs

    def run(qs, rate, keep=False):
        """Submit qs (Poisson arrivals at `rate` per second, all at once if
        rate is None); return results, the wall time to the last one, and the
        query ids in submission order."""
        results = {}
        lock = threading.Lock()
        done_evt = threading.Event()

        def collector():
            while len(results) < len(qs):
                for r in srv.poll(wait_ms=50):
                    with lock:
                        results[r.id] = r
                    if r.status == api.OK and not keep:
                        srv.release(r.id)
            done_evt.set()

        th = threading.Thread(target=collector, daemon=True)
        t0 = time.perf_counter()
        th.start()
        gaps = rng.exponential(1.0 / rate, len(qs)) if rate else np.zeros(len(qs))
        t_next = t0
        ids = []
        for q, g in zip(qs, gaps):
            t_next += g
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            ids.append(srv.submit(q[0], q[1], q[2], q[3], q[4], threshold=0.2))
        done_evt.wait(timeout=3600)
        return results, time.perf_counter() - t0, ids

    warm = draw(max(8, args.warmup * 8))
    run(warm, None)
    calib = draw(min(400, max(50, args.queries // 10)))
    res_c, t_c, _ = run(calib, None)
    pairs_c = sum(r.pairs for r in res_c.values())
    capacity_qps = len(calib) / t_c
    qs = draw(args.queries)
    with ClockSampler(local_rank) as clk:
        clk.mark_start()
        res, t, _ = run(qs, args.load * capacity_qps)
        clk.mark_end()
    lat = np.array([r.latency_ms for r in res.values()])
    pairs = sum(r.pairs for r in res.values())
    K = (H + 63) // 64
    out = {"config": {"workload": f"served_{args.queries}_queries", "chromosomes": 22,
                      "snps_per_chromosome": "U(50000,250000)", "haplotypes": H,
                      "query_side_snps": "U(100,20000)", "arrivals": "Poisson",
                      "offered_load": args.load, "pool_gb": args.pool_gb,
                      "max_inflight_batches": args.inflight,
                      "delivered": "per query: count of r2 >= 0.2 (< 100), sum, max; "
                                   "r2 blocks stay on the device until released"},
           "value": pairs / t, "unit": "pairs/s", "wall_s": t, "queries": len(qs),
           "bitops_per_s": pairs * 64 * K / t,
           "latency_ms": {"p50": float(np.percentile(lat, 50)),
                          "p99": float(np.percentile(lat, 99)),
                          "mean": float(lat.mean()), "max": float(lat.max())},
           "arrival_qps": args.load * capacity_qps, "completed": len(res),
           "failed": sum(1 for r in res.values() if r.status != api.OK),
           "saturated_burst": {"queries": len(calib), "pairs_per_s": pairs_c / t_c},
           "clocks": clk.summary(),
           "timing": "host wall clock from the first arrival to the last result"}
    if not args.no_parity and check_queries:
        cq = draw(check_queries)
        got, _, ids = run(cq, None, keep=True)
        groups, summary_ok = [], True
        for q, qid in zip(cq, ids):
            c, a0, a1, b0, b1 = q
            r = got[qid]
            if r.status != api.OK:
                summary_ok = False
                continue
            blk = np.empty((b1 - b0, a1 - a0), np.float32)
            srv.fetch(qid, blk)
            srv.release(qid)
            sym = (a0, a1) == (b0, b1)
            full = (np.arange(a1 - a0)[None, :] > np.arange(b1 - b0)[:, None]) if sym \
                else np.ones(blk.shape, bool)
            v = blk[full]
            v = v[v < 100]
            summary_ok &= int((v >= 0.2).sum()) == r.n_above
            summary_ok &= (float(v.max()) if v.size else 0.0) == r.max_r2
            rows = sorted({0, b1 - b0 - 1, int(rng.integers(0, b1 - b0))})
            T, bc = tables[c]
            Kc = T.shape[1]
            A = T[a0:a1].cpu().numpy().view(np.uint64)
            bcA = bc[a0:a1].cpu().numpy().astype(np.uint32)
            idx = torch.as_tensor([b0 + x for x in rows], device=dev)
            B = T.index_select(0, idx)[:, :Kc].contiguous().cpu().numpy().view(np.uint64)
            bcB = bc.index_select(0, idx).cpu().numpy().astype(np.uint32)
            rr = np.array(rows)
            valid = (np.arange(a1 - a0)[None, :] >= rr[:, None]) if sym \
                else np.ones((len(rows), a1 - a0), bool)
            groups.append(dict(A=A, bcA=bcA, B=B, bcB=bcB, S=H, got=blk[rows], valid=valid))
        par = oracle.check_groups(groups, mode="exact") if groups else {"ok": False}
        par["summaries_match_blocks"] = bool(summary_ok)
        par["ok"] = par["ok"] and bool(summary_ok)
        par["sample"] = (f"{check_queries} more queries from the same distribution: 3 B rows "
                         "of each r2 block x all its A rows; device summaries vs the block")
        out["parity"] = par
    if not args.no_cpu:
        qrng = np.random.default_rng(6)
        cpu_qs = []
        for _ in range(64):   # queries from the same distribution, their own draw
            c = int(qrng.integers(0, 22))
            la, lb = (int(x) for x in qrng.integers(100, 20_001, 2))
            a0 = int(qrng.integers(0, sizes[c] - la + 1))
            b0 = int(qrng.integers(0, sizes[c] - lb + 1))
            cpu_qs.append((c, a0, a0 + la, b0, b0 + lb))

        def tasks(count):
            ts, p = [], 0
            for c, a0, a1, b0, b1 in cpu_qs[:count]:
                T = tables[c][0]
                A = T[a0:a1].cpu().numpy().view(np.uint64)
                B = T[b0:b1].cpu().numpy().view(np.uint64)
                ts.append((A, B, H))
                p += (a1 - a0) * (b1 - b0)
            return ts, p, f"{count} queries of the same distribution, one task each"
        out["cpu_baseline"] = cpu_sampled_baseline(tasks, (2, 64))
    srv.close()
    del tables
    return out


def section_dropin(args, local_rank, flush=None, windows=8):
    """Drop-in arm: qLD-compute's own CLI on an MDF dataset of the headline
    region's shape (29,817 SNPs x 16,622 haplotypes, K = 260), three ways --
    the stock build with -blis (oracle/_ref/qLD-compute-blis: BLIS dsyrk /
    dgemm on BLIS_IC_NT = physical cores, single-threaded epilogue), the same
    CLI with correlate() routed to the GPU (oracle/_ref/qLD-compute-cuda,
    QLD_CUDA=1: correlate_cuda()), and qld-ld (this package's native CLI,
    GPU report filter) -- on one single-region task and on an -inputList of
    window pairs (`windows` equal windows, every pair i < j: two-region
    tasks).  Each figure is one process's wall time from start to exit:
    MDF parse, counts + r^2, and the report at -r2limit 2 (which prints no
    pair, so the text writer's cost is its scan alone)."""
    import shutil
    import numpy as np
    import torch

    from qld_b200 import host_api, mdf, synth
    ref_blis = os.path.join(ROOT, "oracle", "_ref", "qLD-compute-blis")
    ref_cuda = os.path.join(ROOT, "oracle", "_ref", "qLD-compute-cuda")
    if not (os.path.exists(ref_blis) and os.path.exists(ref_cuda)):
        return {"unavailable": "oracle/_ref/qLD-compute-blis or qLD-compute-cuda not built"}
    dev = torch.device("cuda", local_rank)
    T, S = synth.single_region_workload(device=dev, seed=2)
    T_np = T.cpu().numpy().view(np.uint64)
    m = T_np.shape[0]
    tmp = tempfile.mkdtemp(prefix="qld_dropin_")
    _, phys, _ = host_cpu()
    try:
        d = mdf.write_dataset(os.path.join(tmp, "region"), T_np, S, snps_per_file=1000)
        pos = 1000 + 10 * np.arange(m)
        edges = np.linspace(0, m, windows + 1).astype(int)
        lst = os.path.join(tmp, "tasks.csv")
        pairs_list = 0
        with open(lst, "w") as f:
            for i in range(windows):
                for j in range(i + 1, windows):
                    f.write(f"{d},{pos[edges[i]]},{pos[edges[i + 1] - 1]},"
                            f"{d},{pos[edges[j]]},{pos[edges[j + 1] - 1]}\n")
                    pairs_list += int(edges[i + 1] - edges[i]) * int(edges[j + 1] - edges[j])
        env = dict(os.environ, BLIS_JC_NT="1", BLIS_IC_NT=str(phys), BLIS_JR_NT="1",
                   BLIS_IR_NT="1", OMP_NUM_THREADS=str(phys))
        env.pop("QLD_CUDA", None)
        runs = {"reference_blis": (ref_blis, ["-blis"], env),
                "reference_cli_cuda": (ref_cuda, [], dict(env, QLD_CUDA="1")),
                "qld_ld": (host_api.CLI_PATH, ["-threads", str(phys)], env)}
        common = ["-ploidy", "haploid", "-mdf", "-r2limit", "2"]
        res = {"config": {"workload": "dropin_cli_29817x16622", "snps": m, "haplotypes": S,
                          "words_per_snp": T_np.shape[1], "tasks_list": windows * (windows - 1) // 2,
                          "pairs_single": m * (m - 1) // 2, "pairs_list": pairs_list,
                          "r2limit": 2, "host_cores": phys},
               "timing": "process wall clock, start to exit"}
        outs = {}
        for name, (exe, extra, e) in runs.items():
            row = {}
            for task, targs in (("single", ["-input", d]), ("list", ["-inputList", lst])):
                wd = os.path.join(tmp, f"{name}_{task}")
                os.makedirs(wd)
                t0 = time.perf_counter()
                r = subprocess.run([exe, *targs, *common, *extra, "-output",
                                    os.path.join(wd, "out.txt")], cwd=wd, env=e,
                                   capture_output=True, text=True, timeout=1800)
                dt = time.perf_counter() - t0
                if r.returncode != 0:
                    row[task] = {"failed": r.returncode, "stderr": r.stderr[-300:]}
                    continue
                pairs = m * (m - 1) // 2 if task == "single" else pairs_list
                row[task] = {"wall_s": dt, "pairs_per_s": pairs / dt}
                outs[(name, task)] = {f: open(os.path.join(wd, f), "rb").read()
                                      for f in sorted(os.listdir(wd)) if f.startswith("out")}
            res[name] = row
        res["reports_identical"] = all(
            outs.get(("reference_blis", t)) == outs.get((n, t))
            for n in ("reference_cli_cuda", "qld_ld") for t in ("single", "list"))
        for task in ("single", "list"):
            try:
                res[f"speedup_cli_cuda_{task}"] = (res["reference_blis"][task]["wall_s"] /
                                                   res["reference_cli_cuda"][task]["wall_s"])
                res[f"speedup_qld_ld_{task}"] = (res["reference_blis"][task]["wall_s"] /
                                                 res["qld_ld"][task]["wall_s"])
            except KeyError:
                pass
        return res
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def standalone(args, rank, world, local_rank):
    """--workload windowed|batched|served|dropin: that section alone, as its
    own line."""
    import torch
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    fn = {"windowed": section_windowed, "batched": section_batched,
          "served": section_served, "dropin": section_dropin}[args.workload]
    res = fn(args, local_rank, flush)
    suffix = {"windowed": ", windowed band", "batched": ", batched tasks",
              "served": ", served queries", "dropin": ", qLD-compute CLI drop-in"}[args.workload]
    line = {"metric": METRIC + suffix, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64 popcount / f32 r2", "data": "synthetic", **res}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.workload in ("single_region", "all_pairs"):
            ours_arm(args, rank, world, local_rank)
        else:
            standalone(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
