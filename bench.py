"""Benchmark of the LD hot path (AND+popcount counts + fused r^2) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload single_region|all_pairs] [--kernel auto|popc|mma|fp4]

Workload (default): the dataset-shaped single region -- 29,817 SNPs x 16,622
haploid sequences (K = 260 words per SNP), allele frequencies Beta(0.1, 1)
clipped to >= 1/16,622, haplotype-copying model (20 founders, recombination
blocks of 50-500 SNPs, 1% per-site mutation), lower-triangular FP32 r^2.
Seeded synthetic data of that shape stands in for the dataset.

A step is one pass of the hot path over the region: counts + r^2 for all
M(M-1)/2 SNP pairs (the kernel also fills the diagonal).  `value` is
SNP-pairs/s with the packed table resident in HBM (device-to-device call,
output to HBM), timed per step with CUDA events on the launching stream after
an L2 flush (a 512 MB write); `e2e` is the same metric through the host-buffer
C-ABI call (qld_cuda_ld): pinned host table -> device, counts + r^2, lower
triangle -> pinned host memory, all inside the timed region.

With --gpus N (torchrun) every rank processes its own region of the same shape
(no data-path collective; weak scaling); timing is the max over ranks.
`--impl reference` times the reference's CPU path (its bin_gemm_2x2
micro-kernel in a BLIS-style loop plus its get_pairwise_ld_score, built from
the qLD sources into oracle/_ref) with all host threads on a bounded sample.
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="single_region",
                    choices=["single_region", "all_pairs", "batched", "windowed", "served"])
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
    return ap.parse_args()


def workload_config(name):
    if name == "single_region":
        return dict(workload="single_region_29817x16622_lower_triangle", snps=29_817,
                    haplotypes=16_622, words_per_snp=260, model="copying(20 founders)",
                    freq="Beta(0.1,1) clipped >= 1/16622", output="fp32 lower triangle")
    return dict(workload="all_pairs_2048x4096_symmetric", snps=2048, haplotypes=4096,
                words_per_snp=64, model="iid Bernoulli", freq="Uniform(0.05,0.5)",
                output="fp32 lower triangle")


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


def kernel_roofline(ctx, variant, bitops, kern_ms, dev):
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


def measured_traffic(variant, workload, sm_pair=0, r2_mode="exact"):
    """DRAM bytes per launch of the counts kernel from the ncu capture
    summarised under profiles/ (None when no capture covers this case).
    sm_pair 0 is the automatic choice: SM pairs for exact r^2, single SMs
    for reference r^2."""
    if sm_pair == 0:
        sm_pair = 1 if r2_mode == "reference" else 2
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

def cpu_reference_rate(T_np, S, seconds_target=12.0, threads=None):
    """Reference CPU path (bin_gemm_2x2 loop + get_pairwise_ld_score) on the
    first Ms SNPs of the table, single region; Ms chosen so the timed sample
    takes ~seconds_target.  Returns (pairs/s, cores, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import oracle
    threads = threads or os.cpu_count()

    def run(ms):
        A = np.ascontiguousarray(T_np[:ms])
        bc = oracle.bitcounts(A)
        t0 = time.perf_counter()
        C = oracle.ref_counts_ukr(A, None, lower_only=True, threads=threads)
        oracle.ref_ld_score(bc, bc, C, S, threads=threads)
        return time.perf_counter() - t0

    m = T_np.shape[0]
    ms = min(m, 1024)
    t = run(ms)
    while t < seconds_target / 8 and ms < m:
        ms = min(m, ms * 2)
        t = run(ms)
    if t < seconds_target / 2 and ms < m:
        ms = min(m, int(ms * (seconds_target / max(t, 1e-3)) ** 0.5))
        t = run(ms)
    pairs = ms * (ms - 1) / 2
    return pairs / t, threads, f"first {ms} SNPs of the region, all {ms*(ms-1)//2} pairs, {t:.2f} s"


def reference_arm(args, rank, world):
    import numpy as np
    cfg = workload_config(args.workload)
    if rank != 0:
        return
    T, S = make_table(args.workload, "cpu")
    T_np = T.numpy().view(np.uint64)
    for _ in range(args.warmup):
        cpu_reference_rate(T_np, S, seconds_target=2.0)
    vals = []
    desc = ""
    cores = os.cpu_count()
    for _ in range(args.steps):
        v, cores, desc = cpu_reference_rate(T_np, S, seconds_target=6.0)
        vals.append(v)
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64 popcount / f32 r2", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": "reference",
                             "sample": desc},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------------- ours --

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


def ours_arm(args, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist

    from qld_b200 import api, synth

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    cfg = workload_config(args.workload)
    cfg["parallelism"] = f"replicas x{world} (independent regions, no collective)"
    cfg["l2"] = "512 MB flush write between timed steps"

    T, S = make_table(args.workload, dev, seed_offset=rank)
    if args.snps:
        T = T[:args.snps].contiguous()
        cfg["snps"] = T.shape[0]
        cfg["workload"] += f"_first{T.shape[0]}"
    m, K = T.shape
    lda = K + (K & 1)
    Tp = torch.zeros(m, lda, dtype=torch.int64, device=dev)
    Tp[:, :K] = T
    bc = synth.popcount_rows(T).to(torch.int32)
    out = torch.empty(m, m, dtype=torch.float32, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)

    ctx = api.Context(local_rank)
    kern = {"auto": api.KERNEL_AUTO, "popc": api.KERNEL_POPC, "mma": api.KERNEL_MMA,
            "fp4": api.KERNEL_FP4}[args.kernel]
    ctx.set_option(api.OPT_KERNEL, kern)
    ctx.set_option(api.OPT_MMA_TILE, args.mma_tile)
    ctx.set_option(api.OPT_SM_PAIR, args.sm_pair)
    ctx.set_option(api.OPT_R2_MODE,
                   api.R2_REFERENCE if args.r2_mode == "reference" else api.R2_EXACT)
    if args.r2_mode != "exact":
        cfg["r2_mode"] = args.r2_mode
    ctx.set_option(api.OPT_PROFILE, 1)
    # A dedicated stream: torch's default stream is the legacy NULL stream,
    # which the C ABI reads as "the context's own stream".
    st = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(st)

    def step():
        ctx.ld_device(Tp, bc, m, lda, Tp, bc, m, lda, K, S, True, out, m, stream=st)

    tuned = None
    if args.autotune and kern == api.KERNEL_AUTO:
        tk, topt, tms = ctx.autotune(m, m, K, True)
        tuned = {"kernel": tk, "option": topt, "ms_per_launch_tuned": tms,
                 "measured_at": f"{min(m, 16384)}x{min(m, 16384)}x{K} words"}

    for _ in range(args.warmup):
        flush.zero_()
        step()
    ctx.sync(stream=st)
    ctx.stats(reset=True)

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        clk.mark_start()
        torch.cuda.nvtx.range_push("qld_timed")
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(st)
            step()
            ev[i][1].record(st)
        torch.cuda.nvtx.range_pop()
        ctx.sync(stream=st)
        torch.cuda.synchronize()
        clk.mark_end()
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    stats = ctx.stats(reset=True)
    clocks = clk.summary()

    pairs = m * (m - 1) / 2
    total_ms_max = max_over_ranks(total_ms, world, dev)
    value = pairs * args.steps * world / (total_ms_max * 1e-3)

    # roofline of the counts kernel
    kern_ms = stats.counts_kernel_ms / max(1, stats.counts_launches)
    bitops = pairs * 64 * K
    variant = stats.last_kernel
    roof = kernel_roofline(ctx, variant, bitops, kern_ms, dev)
    alg_bytes = m * K * 8 * 2 + pairs * 4
    sm_pair = args.sm_pair
    if tuned is not None and tuned["kernel"] == api.KERNEL_FP4 and sm_pair == 0:
        sm_pair = tuned["option"]
    roof["traffic"] = measured_traffic(variant, cfg["workload"], sm_pair, args.r2_mode)
    roof["algorithmic_bytes_per_launch"] = alg_bytes
    roof["kernel_ms"] = kern_ms
    mp = measured_peaks()
    roof["hbm_frac_of_measured"] = (alg_bytes / (kern_ms * 1e-3) / 1e9) / mp["hbm_gbs"]
    roof["hbm_peak_gbs"] = mp["hbm_gbs"]
    roof["hbm_peak_source"] = mp["source"]

    line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64 popcount / f32 r2", "data": "synthetic", "config": cfg,
            "bitops_per_s": bitops * args.steps * world / (total_ms_max * 1e-3),
            "gpu_launches": stats.kernel_launches, "kernel_variant": variant,
            "roofline": roof, "clocks": clocks}
    if tuned is not None:
        line["autotune"] = tuned

    # ---- e2e through the host-buffer C-ABI call
    if not args.no_e2e:
        Th = ctx.pinned_empty((m, K), np.uint64)
        Th[:] = T.cpu().numpy().view(np.uint64)
        bch = ctx.pinned_empty((m,), np.uint32)
        bch[:] = bc.cpu().numpy().view(np.uint32)
        outh = ctx.pinned_empty((m, m), np.float32)
        for _ in range(max(1, args.warmup)):
            ctx.ld(Th, bch, S=S, r2_out=outh)
        if world > 1:
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

    if rank == 0 and world == 1 and not args.no_cpu:
        v, cores, desc = cpu_reference_rate(T.cpu().numpy().view(np.uint64), S)
        line["cpu_baseline"] = {"value": v, "unit": "pairs/s", "cores": cores, "kind": "reference",
                                "sample": desc}
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


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
        lda = K + (K & 1)
        Tp = torch.zeros(rows, lda, dtype=torch.int64, device=dev)
        Tp[:, :K] = T
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


def batched_arm(args, rank, world, local_rank):
    import numpy as np  # noqa: F401
    import torch

    from qld_b200 import api
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    jobs, pairs, bitops = make_batched_jobs(args.jobs, dev, seed=rank)
    ctx = api.Context(local_rank)
    ctx.set_option(api.OPT_PROFILE, 1)
    st = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(st)

    def batched():
        ctx.ld_batch(jobs, stream=st)

    def plain():
        for j in jobs:
            ctx.ld_device(j["A"], j["bcA"], j["m"], j["lda"], j["B"], j["bcB"], j["n"],
                          j["ldb"], j["K"], j["S"], j["symmetric"], j["r2"], j["ldr"], stream=st)

    res = {}
    for name, fn in (("batched", batched), ("plain", plain)):
        for _ in range(args.warmup):
            fn()
        ctx.sync(stream=st)
        ctx.stats(reset=True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push(f"qld_timed_{name}")
        e0.record(st)
        for _ in range(args.steps):
            fn()
        e1.record(st)
        torch.cuda.nvtx.range_pop()
        ctx.sync(stream=st)
        torch.cuda.synchronize()
        res[name] = (e0.elapsed_time(e1) / args.steps, ctx.stats(reset=True))
    ms_b, st_b = res["batched"]
    ms_p, st_p = res["plain"]
    line = {"metric": METRIC + ", batched tasks", "value": pairs / (ms_b * 1e-3),
            "unit": "pairs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_b, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64 popcount / f32 r2", "data": "synthetic",
            "config": {"workload": f"batched_{args.jobs}_tasks", "snps_per_side": "logU(64,8192)",
                       "samples": "logU(1000,50000)", "freq": "Beta(0.5,0.5)",
                       "half": "single region (triangle) / two regions (rectangle)",
                       "pairs_per_step": pairs, "bitops_per_step": bitops},
            "bitops_per_s": bitops / (ms_b * 1e-3),
            "gpu_launches": st_b.kernel_launches // max(1, args.steps),
            "plain": {"value": pairs / (ms_p * 1e-3), "unit": "pairs/s", "ms_per_step": ms_p,
                      "launches_per_step": st_p.kernel_launches // max(1, args.steps)},
            "speedup_vs_plain": ms_p / ms_b}
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def windowed_arm(args, rank, world, local_rank):
    """Windowed workload: 200,000 SNPs x 100,000 haplotypes (copying model,
    100 founders), r^2 for pairs within `band` SNPs, FP32 band array."""
    import numpy as np
    import torch

    from qld_b200 import api, synth
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    m_full = args.snps or 200_000
    T, S = synth.windowed_workload(device=dev, m=m_full, seed=3 + rank)
    m, K = T.shape
    W = args.band
    lda = K + (K & 1)
    Tp = torch.zeros(m, lda, dtype=torch.int64, device=dev)
    Tp[:, :K] = T
    bc = synth.popcount_rows(T).to(torch.int32)
    out = torch.empty(m, W, dtype=torch.float32, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    pairs = sum(min(W, m - 1 - i) for i in range(0, m)) if m < 50_000 else \
        W * (m - W) + W * (W - 1) // 2
    ctx = api.Context(local_rank)
    kern = {"auto": api.KERNEL_AUTO, "popc": api.KERNEL_POPC, "mma": api.KERNEL_MMA,
            "fp4": api.KERNEL_FP4}[args.kernel]
    ctx.set_option(api.OPT_KERNEL, kern)
    ctx.set_option(api.OPT_MMA_TILE, args.mma_tile)
    ctx.set_option(api.OPT_SM_PAIR, args.sm_pair)
    ctx.set_option(api.OPT_R2_MODE,
                   api.R2_REFERENCE if args.r2_mode == "reference" else api.R2_EXACT)
    ctx.set_option(api.OPT_PROFILE, 1)
    st = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(st)

    def step():
        ctx.ld_band_device(Tp, bc, m, lda, K, S, W, out, W, stream=st)

    for _ in range(args.warmup):
        flush.zero_()
        step()
    ctx.sync(stream=st)
    ctx.stats(reset=True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        clk.mark_start()
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(st)
            step()
            ev[i][1].record(st)
        ctx.sync(stream=st)
        torch.cuda.synchronize()
        clk.mark_end()
    total_ms = sum(a.elapsed_time(b) for a, b in ev)
    stats = ctx.stats(reset=True)
    kern_ms = stats.counts_kernel_ms / max(1, stats.counts_launches)
    bitops = pairs * 64 * K
    line = {"metric": METRIC + ", windowed band", "value": pairs * args.steps / (total_ms * 1e-3),
            "unit": "pairs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64 popcount / f32 r2", "data": "synthetic",
            "config": {"workload": f"windowed_{m}x{S}_band{W}", "snps": m, "haplotypes": S,
                       "words_per_snp": K, "band": W, "model": "copying(100 founders)",
                       "pairs_per_step": pairs, "l2": "512 MB flush write between timed steps"},
            "bitops_per_s": bitops * args.steps / (total_ms * 1e-3),
            "gpu_launches": stats.kernel_launches // max(1, args.steps),
            "kernel_variant": stats.last_kernel,
            "roofline": dict(kernel_roofline(ctx, stats.last_kernel, bitops, kern_ms, dev),
                             kernel_ms=kern_ms),
            "clocks": clk.summary()}
    if args.r2_mode != "exact":
        line["config"]["r2_mode"] = args.r2_mode
    if not args.no_e2e:
        Th = ctx.pinned_empty((m, K), np.uint64)
        Th[:] = T.cpu().numpy().view(np.uint64)
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
        line["e2e"] = {"value": pairs * len(ts) / sum(ts), "unit": "pairs/s",
                       "h2d_bytes_per_step": m * K * 8 + m * 4,
                       "d2h_bytes_per_step": m * W * 4,
                       "api": "qld_cuda_ld_band (pinned host buffers, streamed)"}
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def served_arm(args, rank, world, local_rank):
    """Served workload: 22 resident chromosomes (50,000-250,000 SNPs x 20,000
    haplotypes, copying model), a Poisson stream of region-vs-region queries
    (each side 100-20,000 SNPs, uniform placement), admitted by output memory.
    The arrival rate is `load` x the capacity measured by a saturated burst."""
    import threading

    import numpy as np
    import torch

    from qld_b200 import api, synth
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(5 + rank)
    H = 20_000
    srv = api.Server(local_rank, pool_bytes=args.pool_gb << 30, max_inflight=args.inflight)
    sizes = []
    for c in range(22):
        m = int(rng.integers(50_000, 250_001))
        f = synth.beta_freqs(m, 0.1, 1.0, 100 + c, device=dev, clip_min=1.0 / H)
        T = synth.copying_table(m, H, 50, 50, 500, 0.01, f, 100 + c, device=dev)
        bc = synth.popcount_rows(T).to(torch.int32)
        srv.add_table(T, bc, H)
        sizes.append(m)
        del T, bc
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

    def run(qs, rate):
        """Submit qs (Poisson arrivals at `rate` per second, all at once if
        rate is None); return results and the wall time to the last one."""
        results = {}
        lock = threading.Lock()
        done_evt = threading.Event()

        def collector():
            while len(results) < len(qs):
                for r in srv.poll(wait_ms=50):
                    with lock:
                        results[r.id] = r
                    if r.status == api.OK:
                        srv.release(r.id)
            done_evt.set()

        th = threading.Thread(target=collector, daemon=True)
        t0 = time.perf_counter()
        th.start()
        gaps = rng.exponential(1.0 / rate, len(qs)) if rate else np.zeros(len(qs))
        t_next = t0
        for q, g in zip(qs, gaps):
            t_next += g
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            srv.submit(q[0], q[1], q[2], q[3], q[4], threshold=0.2)
        done_evt.wait(timeout=3600)
        return results, time.perf_counter() - t0

    warm = draw(max(8, args.warmup * 8))
    run(warm, None)
    calib = draw(min(400, max(50, args.queries // 10)))
    res_c, t_c = run(calib, None)
    pairs_c = sum(r.pairs for r in res_c.values())
    capacity_qps = len(calib) / t_c
    qs = draw(args.queries)
    res, t = run(qs, args.load * capacity_qps)
    lat = np.array([r.latency_ms for r in res.values()])
    pairs = sum(r.pairs for r in res.values())
    K = (H + 63) // 64
    line = {"metric": METRIC + ", served queries", "value": pairs / t, "unit": "pairs/s",
            "n_gpus": world, "steps": 1, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64 popcount / f32 r2", "data": "synthetic",
            "config": {"workload": f"served_{args.queries}_queries", "chromosomes": 22,
                       "snps_per_chromosome": "U(50000,250000)", "haplotypes": H,
                       "query_side_snps": "U(100,20000)", "arrivals": "Poisson",
                       "offered_load": args.load, "pool_gb": args.pool_gb,
                       "max_inflight_batches": args.inflight,
                       "delivered": "per query: count of r2 >= 0.2 (< 100), sum, max; "
                                    "r2 blocks stay on the device until released"},
            "bitops_per_s": pairs * 64 * K / t,
            "latency_ms": {"p50": float(np.percentile(lat, 50)),
                           "p99": float(np.percentile(lat, 99)),
                           "mean": float(lat.mean()), "max": float(lat.max())},
            "arrival_qps": args.load * capacity_qps, "completed": len(res),
            "failed": sum(1 for r in res.values() if r.status != api.OK),
            "saturated_burst": {"queries": len(calib), "pairs_per_s": pairs_c / t_c}}
    srv.close()
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
        if args.workload == "batched":
            batched_arm(args, rank, world, local_rank)
        elif args.workload == "windowed":
            windowed_arm(args, rank, world, local_rank)
        elif args.workload == "served":
            served_arm(args, rank, world, local_rank)
        else:
            ours_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
