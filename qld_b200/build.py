"""Build the native libraries in-tree (cross-compiles without a GPU).

    python -m qld_b200.build [--verbose]

Every .cu file under csrc/ is compiled for ``-gencode arch=compute_100a,
code=sm_100a`` and linked into ``qld_b200/libqld_cuda.so`` (static CUDA
runtime, so the library carries its own runtime independent of torch's).
The C host layer (host/mdf_loader.c, host/report.c, host/vcf.c) becomes
``qld_b200/libqld_host.so``, host/qld_ld_main.c the ``qld_b200/qld-ld`` command
and host/vcf2mdf_main.c ``qld_b200/qld-vcf2mdf``, all linked against
libqld_cuda.so through an $ORIGIN rpath.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libqld_cuda.so")
HOST = os.path.join(PKG, "host")
HOST_LIB = os.path.join(PKG, "libqld_host.so")
CLI = os.path.join(PKG, "qld-ld")
VCF2MDF = os.path.join(PKG, "qld-vcf2mdf")
HOST_FLAGS = ["-O3", "-std=gnu11", "-Wall", "-Wextra", "-Wno-unused-parameter", "-fPIC"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    deps.append(os.path.join(ROOT, "include", "qld_cuda.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    tmp = LIB + ".tmp"
    cmd += ["-o", tmp, *sources()]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


def cc() -> str:
    for cand in (shutil.which("gcc"), "/usr/bin/gcc", shutil.which("cc")):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("gcc not found")


def build_host(force: bool = False) -> str:
    """libqld_host.so and qld-ld (needs libqld_cuda.so first)."""
    lib_srcs = [os.path.join(HOST, f) for f in ("mdf_loader.c", "report.c", "vcf.c")]
    mains = {CLI: os.path.join(HOST, "qld_ld_main.c"),
             VCF2MDF: os.path.join(HOST, "vcf2mdf_main.c")}
    deps = (lib_srcs + list(mains.values()) + [LIB]
            + glob.glob(os.path.join(ROOT, "include", "*.h")) + glob.glob(os.path.join(HOST, "*.h")))
    outs = [HOST_LIB, *mains]
    if (not force and all(os.path.exists(o) for o in outs)
            and all(os.path.getmtime(d) <= min(os.path.getmtime(o) for o in outs) for d in deps)):
        return CLI
    inc = ["-I", os.path.join(ROOT, "include")]
    link = ["-L", PKG, "-lqld_cuda", "-Wl,-rpath,$ORIGIN", "-lz", "-lpthread"]
    subprocess.run([cc(), *HOST_FLAGS, *inc, "-shared", "-o", HOST_LIB + ".tmp", *lib_srcs, *link],
                   check=True)
    os.replace(HOST_LIB + ".tmp", HOST_LIB)
    for exe, src in mains.items():
        subprocess.run([cc(), *HOST_FLAGS, *inc, "-o", exe + ".tmp", src, "-L", PKG, "-lqld_host",
                        *link], check=True)
        os.replace(exe + ".tmp", exe)
    return CLI


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    build_host(force=True)
    print(LIB)
    print(HOST_LIB)
    print(CLI)
    print(VCF2MDF)
