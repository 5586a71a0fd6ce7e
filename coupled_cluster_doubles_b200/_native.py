"""ctypes bindings for the two native libraries of the package.

libccdhost.so  — host problem builder (include/ccdhost.h)
libccdgpu.so   — B200 CCD iteration behind the C ABI (include/ccdgpu.h)

Both are built in-tree (coupled_cluster_doubles_b200/build.py) and loaded from this
directory.  Loading never falls back to anything else: a missing library raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))

c_u64 = ctypes.c_uint64
c_i64 = ctypes.c_int64
c_i32 = ctypes.c_int32
c_dbl = ctypes.c_double
P = ctypes.POINTER


class Pair(ctypes.Structure):
    _fields_ = [("p", c_u64), ("q", c_u64)]


class ChannelDims(ctypes.Structure):
    _fields_ = [("pp", c_u64), ("hh", c_u64), ("hp", c_u64), ("ph", c_u64)]


class ChannelMaps(ctypes.Structure):
    _fields_ = [("pp", P(Pair)), ("hh", P(Pair)), ("hp", P(Pair)), ("ph", P(Pair))]


class ThreeBodyDims(ctypes.Structure):
    _fields_ = [("phh", c_u64), ("hpp", c_u64)]


class ChainIndex(ctypes.Structure):
    _fields_ = [("channel", c_u64), ("row", c_u64), ("column", c_u64)]


class Model(ctypes.Structure):
    _fields_ = [("kind", c_i32), ("qn_stride", c_i32), ("qn", P(c_i32)),
                ("params", c_dbl * 8)]


class Problem(ctypes.Structure):
    _fields_ = [
        ("n_sp", c_u64), ("n_particles", c_u64), ("n_channels", c_u64),
        ("sp_energy", P(c_dbl)),
        ("chan_dims", P(ChannelDims)), ("chan_mod_dims", P(ChannelDims)),
        ("chan_maps", P(ChannelMaps)), ("chan_mod_maps", P(ChannelMaps)),
        ("three_body_dims", P(ThreeBodyDims)),
        ("v_hhhh", P(P(c_dbl))), ("v_hhpp", P(P(c_dbl))), ("v_pppp", P(P(c_dbl))),
        ("v_hpph_mod", P(P(c_dbl))), ("v_hphp_mod", P(P(c_dbl))),
        ("v_h_hpp", P(P(c_dbl))), ("v_phh_p", P(P(c_dbl))),
        ("maps", P(P(ChainIndex)) * 8),
        ("model", P(Model)),
    ]


class Options(ctypes.Structure):
    _fields_ = [("device", c_i32), ("precision", c_i32), ("v_mode", c_i32), ("path", c_i32),
                ("polish_threshold", c_dbl), ("use_graph", c_i32), ("device_loop", c_i32),
                ("reserved", c_i32 * 6)]


class Schedule(ctypes.Structure):
    _fields_ = [("thin_split_mul", c_i32), ("wide_split_mul", c_i32), ("tc_split_mul", c_i32),
                ("mid_split_mul", c_i32), ("reserved", c_i32 * 4)]


class Result(ctypes.Structure):
    _fields_ = [("e_corr", c_dbl), ("e_diff", c_dbl), ("iterations", c_i64),
                ("converged", c_i32), ("polish_iterations", c_i32), ("seconds", c_dbl)]


class Profile(ctypes.Structure):
    _fields_ = [("ms_ladder", c_dbl), ("ms_hh_ladder", c_dbl), ("ms_ring", c_dbl),
                ("ms_onebody", c_dbl), ("ms_assemble", c_dbl), ("ms_total", c_dbl),
                ("launches", c_i64), ("iterations", c_i64), ("ms_create", c_dbl * 5),
                ("ms_loop_graph", c_dbl)]


_host = None
_gpu = None


def host_lib():
    """Load libccdhost.so (problem builder)."""
    global _host
    if _host is None:
        path = os.path.join(_HERE, "libccdhost.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing; run coupled_cluster_doubles_b200.build.build_all()")
        lib = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        lib.ccdhost_build_pairing.argtypes = [c_dbl, c_dbl, c_u64, c_u64, c_i32, P(vp)]
        lib.ccdhost_build_inf_matter.argtypes = [c_dbl, c_i32, c_u64, c_u64, c_i32, P(vp)]
        lib.ccdhost_build_electron_gas.argtypes = [c_dbl, c_u64, c_u64, c_i32, P(vp)]
        for f in ("ccdhost_build_pairing", "ccdhost_build_inf_matter", "ccdhost_build_electron_gas"):
            getattr(lib, f).restype = ctypes.c_int
        lib.ccdhost_free.argtypes = [vp]
        lib.ccdhost_free.restype = None
        lib.ccdhost_problem.argtypes = [vp]
        lib.ccdhost_problem.restype = P(Problem)
        lib.ccdhost_reference_energy.argtypes = [vp]
        lib.ccdhost_reference_energy.restype = c_dbl
        lib.ccdhost_mbpt2.argtypes = [vp]
        lib.ccdhost_mbpt2.restype = c_dbl
        lib.ccdhost_array.argtypes = [vp, ctypes.c_char_p, P(vp), P(c_u64), P(c_i32)]
        lib.ccdhost_array.restype = ctypes.c_int
        _host = lib
    return _host


GPU_SYMBOLS = [
    "ccdgpu_default_options", "ccdgpu_create", "ccdgpu_destroy", "ccdgpu_strerror",
    "ccdgpu_reset", "ccdgpu_set_t2", "ccdgpu_get_t2", "ccdgpu_t2_size", "ccdgpu_step",
    "ccdgpu_solve", "ccdgpu_calc_t2diff_p2_p1hh", "ccdgpu_calc_t2diff_h2pp_h1",
    "ccdgpu_calc_t2diff_phhp", "ccdgpu_calc_t2diff_pphh", "ccdgpu_map_from_distributed",
    "ccdgpu_calc_t2_pphh", "ccdgpu_map_to_distributed", "ccdgpu_read_chain",
    "ccdgpu_get_profile", "ccdgpu_enable_profiling", "ccdgpu_work_per_iteration",
    "ccdgpu_energy_history", "ccdgpu_stream", "ccdgpu_calc_channel_t2diff_pphh_noalloc",
    "ccdgpu_trace_arm", "ccdgpu_trace_read", "ccdgpu_solve_batch", "ccdgpu_set_schedule",
    "ccdgpu_get_schedule", "ccdgpu_autotune", "ccdgpu_ladder_profile", "ccdgpu_kernel_profile",
    "ccdgpu_mbpt2", "ccdgpu_reference_energy", "ccdgpu_release_cached_memory",
    "ccdgpu_build_channels", "ccdgpu_inject_wait_timeout", "ccdgpu_trace_read_end",
]


def gpu_lib():
    """Load libccdgpu.so.  Raises if the CUDA library was not built: there is no fallback."""
    global _gpu
    if _gpu is None:
        path = os.path.join(_HERE, "libccdgpu.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing; run coupled_cluster_doubles_b200.build.build_all()")
        lib = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        lib.ccdgpu_default_options.argtypes = [P(Options)]
        lib.ccdgpu_default_options.restype = None
        lib.ccdgpu_create.argtypes = [P(Problem), P(Options), P(vp)]
        lib.ccdgpu_destroy.argtypes = [vp]
        lib.ccdgpu_destroy.restype = None
        lib.ccdgpu_strerror.argtypes = [ctypes.c_int]
        lib.ccdgpu_strerror.restype = ctypes.c_char_p
        lib.ccdgpu_reset.argtypes = [vp]
        lib.ccdgpu_set_t2.argtypes = [vp, P(c_dbl), c_u64]
        lib.ccdgpu_get_t2.argtypes = [vp, P(c_dbl), c_u64]
        lib.ccdgpu_t2_size.argtypes = [vp]
        lib.ccdgpu_t2_size.restype = c_u64
        lib.ccdgpu_step.argtypes = [vp, c_dbl, P(c_dbl)]
        lib.ccdgpu_solve.argtypes = [vp, c_dbl, c_i64, c_dbl, P(Result)]
        for f in ("ccdgpu_calc_t2diff_p2_p1hh", "ccdgpu_calc_t2diff_h2pp_h1",
                  "ccdgpu_calc_t2diff_phhp", "ccdgpu_calc_t2diff_pphh",
                  "ccdgpu_map_from_distributed", "ccdgpu_map_to_distributed"):
            getattr(lib, f).argtypes = [vp]
        lib.ccdgpu_calc_t2_pphh.argtypes = [vp, c_dbl, P(c_dbl)]
        lib.ccdgpu_read_chain.argtypes = [vp, c_i32, P(c_dbl), c_u64, P(c_u64)]
        lib.ccdgpu_get_profile.argtypes = [vp, P(Profile)]
        lib.ccdgpu_enable_profiling.argtypes = [vp, c_i32]
        lib.ccdgpu_work_per_iteration.argtypes = [vp, P(c_dbl), P(c_dbl), P(c_dbl)]
        lib.ccdgpu_energy_history.argtypes = [vp, P(c_dbl), c_i64, P(c_i64)]
        lib.ccdgpu_stream.argtypes = [vp]
        lib.ccdgpu_stream.restype = vp
        lib.ccdgpu_calc_channel_t2diff_pphh_noalloc.argtypes = [vp, vp, vp, vp, vp, c_i64, c_i64, vp]
        lib.ccdgpu_calc_channel_t2diff_pphh_noalloc.restype = ctypes.c_int
        lib.ccdgpu_trace_arm.argtypes = [vp, c_i64]
        lib.ccdgpu_solve_batch.argtypes = [P(vp), c_i32, c_dbl, c_i64, c_dbl, P(Result)]
        lib.ccdgpu_set_schedule.argtypes = [vp, P(Schedule)]
        lib.ccdgpu_get_schedule.argtypes = [vp, P(Schedule)]
        lib.ccdgpu_autotune.argtypes = [vp, c_i32, P(Schedule), P(c_dbl), P(c_dbl)]
        lib.ccdgpu_ladder_profile.argtypes = [vp, c_i32, P(c_dbl), P(c_dbl), P(c_dbl)]
        lib.ccdgpu_kernel_profile.argtypes = [vp, c_i32, P(c_dbl), P(c_dbl), P(c_dbl)]
        lib.ccdgpu_mbpt2.argtypes = [vp, c_i32, P(c_dbl)]
        lib.ccdgpu_reference_energy.argtypes = [vp, P(c_dbl), P(c_dbl), P(c_dbl)]
        lib.ccdgpu_release_cached_memory.argtypes = []
        lib.ccdgpu_release_cached_memory.restype = None
        lib.ccdgpu_trace_read.argtypes = [vp, P(c_u64), P(c_u64), c_i32]
        lib.ccdgpu_inject_wait_timeout.argtypes = [vp]
        lib.ccdgpu_trace_read_end.argtypes = [vp, P(c_u64), c_i32]
        _gpu = lib
    return _gpu
