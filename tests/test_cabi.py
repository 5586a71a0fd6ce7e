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


class ChannelRule(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("qn_stride", ctypes.c_int32),
                ("qn", ctypes.POINTER(ctypes.c_int32)), ("n_sp", ctypes.c_uint64),
                ("n_particles", ctypes.c_uint64), ("n_channels", ctypes.c_uint64),
                ("nmax", ctypes.c_int32), ("chan_tz_max", ctypes.c_int32),
                ("mod_chan_tz_max", ctypes.c_int32), ("device", ctypes.c_int32)]


def test_build_channels_checks_arguments_before_touching_a_device():
    """Argument errors come back as status codes before any CUDA call (so also without a GPU)."""
    lib = _native.gpu_lib()
    qn = (ctypes.c_int32 * 32)()
    dims = (ctypes.c_uint64 * 12)()
    lists = (ctypes.c_void_p * 4)(*([ctypes.addressof(dims)] * 4))

    def call(**kw):
        r = ChannelRule(kind=1, qn_stride=2, qn=qn, n_sp=16, n_particles=8, n_channels=3,
                        nmax=0, chan_tz_max=0, mod_chan_tz_max=0, device=-1)
        for k, v in kw.items():
            setattr(r, k, v)
        return lib.ccdgpu_build_channels(ctypes.byref(r), dims, dims, lists, lists,
                                         None, None, None, None)
    assert lib.ccdgpu_build_channels(None, dims, dims, lists, lists, None, None, None, None) == -1
    assert call(n_particles=0) == -1           # no holes
    assert call(n_particles=16) == -1          # no particles
    assert call(kind=7) == -1                  # unknown model
    assert call(qn_stride=1) == -1             # pairing rows need (level, spin)
    assert call(n_sp=70000, n_particles=8) == -7  # pair codes must fit 32 bits


def test_reference_energy_rejects_null_arguments():
    lib = _native.gpu_lib()
    e = ctypes.c_double()
    assert lib.ccdgpu_reference_energy(None, None, ctypes.byref(e), None) == -1
