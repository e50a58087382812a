"""qld_b200 -- qLD-compute's LD hot path (AND+popcount counts + r^2) for B200.

The product is ``libqld_cuda.so`` (C ABI in include/qld_cuda.h, sources in
csrc/).  ``api`` binds it from Python; ``synth`` generates packed SNP tables.
"""
from . import api  # noqa: F401

__all__ = ["api"]
