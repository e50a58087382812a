"""CPU tests of the C ABI: each library loads and exports every function its
header declares (include/qld_cuda.h -> libqld_cuda.so, include/qld_host.h ->
libqld_host.so); init without a GPU fails with a status code."""
import ctypes as ct
import os
import re

import pytest

from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


LIBS = {"qld_cuda.h": "libqld_cuda.so", "qld_host.h": "libqld_host.so"}


def declared_functions(headers=None):
    names = []
    for h in headers or HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+[\s*]+(qld_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_functions():
    names = declared_functions()
    assert "qld_cuda_init" in names and "qld_cuda_ld" in names
    assert len(names) >= 10


def test_every_header_has_its_library():
    assert sorted(os.path.basename(h) for h in HEADERS) == sorted(LIBS)


@pytest.mark.parametrize("header", sorted(LIBS))
def test_library_exports_every_declared_symbol(header):
    from qld_b200 import api, build
    build.build()
    build.build_host()
    api.load_library()                  # libqld_host.so resolves against libqld_cuda.so
    lib = ct.CDLL(os.path.join(ROOT, "qld_b200", LIBS[header]))
    names = declared_functions([os.path.join(ROOT, "include", header)])
    assert names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    if header == "qld_cuda.h":
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
