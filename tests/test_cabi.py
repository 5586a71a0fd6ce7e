"""The C-ABI library loads and exports every entry point declared in include/*.h."""
import ctypes
import os
import re

import pytest

from coupled_cluster_doubles_b200 import _native, build

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(REPO, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:ccdgpu|ccdhost)_[a-z0-9_]+)\s*\(", text)))


def test_gpu_library_exports_header_symbols():
    build.build_gpu()
    lib = ctypes.CDLL(os.path.join(REPO, "coupled_cluster_doubles_b200", "libccdgpu.so"))
    names = declared("ccdgpu.h")
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(_native.GPU_SYMBOLS) <= set(names)


def test_host_library_exports_header_symbols():
    lib = ctypes.CDLL(os.path.join(REPO, "coupled_cluster_doubles_b200", "libccdhost.so"))
    for n in declared("ccdhost.h"):
        assert hasattr(lib, n), n


def test_strerror_and_defaults():
    lib = _native.gpu_lib()
    assert lib.ccdgpu_strerror(0) == b"ok"
    assert lib.ccdgpu_strerror(-4).startswith(b"remap table")
    opt = _native.Options()
    lib.ccdgpu_default_options(ctypes.byref(opt))
    assert opt.precision == 0 and opt.path == 0 and opt.use_graph == 1


def test_create_rejects_null_problem():
    lib = _native.gpu_lib()
    h = ctypes.c_void_p()
    assert lib.ccdgpu_create(None, None, ctypes.byref(h)) == -1


def test_no_silent_cpu_path_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from coupled_cluster_doubles_b200 import CCDGPUError, CCDSolver, System
    with System.pairing(1.0, 0.5, 4, 4) as s:
        with pytest.raises(CCDGPUError) as ei:
            CCDSolver(s)
        assert ei.value.status == -6
