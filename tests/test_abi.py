"""CPU tests of the C ABI: the library loads and exports every function
include/qld_cuda.h declares; init without a GPU fails with a status code."""
import ctypes as ct
import os
import re

import pytest

from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+[\s*]+(qld_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_functions():
    names = declared_functions()
    assert "qld_cuda_init" in names and "qld_cuda_ld" in names
    assert len(names) >= 10


def test_library_exports_every_declared_symbol():
    from qld_b200 import api, build
    build.build()
    lib = ct.CDLL(api.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    for n in api.EXPORTED:
        assert hasattr(lib, n)


def test_init_without_gpu_returns_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from qld_b200 import api
    lib = api.load_library()
    h = ct.c_void_p()
    rc = lib.qld_cuda_init(0, ct.byref(h))
    assert rc == api.ERR_NODEVICE
    assert not h.value


def test_null_context_is_rejected():
    from qld_b200 import api
    lib = api.load_library()
    assert lib.qld_cuda_set_option(None, api.OPT_KERNEL, 1) == api.ERR_INVALID
    assert lib.qld_cuda_release(None) == api.OK
