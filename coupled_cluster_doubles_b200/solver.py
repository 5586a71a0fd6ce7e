"""Python front end of the B200 CCD solver (libccdgpu.so through its C ABI).

Mirrors the reference's loop (main.cpp:491-682) and stage functions (calc.hpp):

    solver = CCDSolver(System.electron_gas(r_s=1.0, n_shells=19, n_particle_shells=2))
    res = solver.solve(tol=1e-12)          # stop rule and 101-iteration cap of main.cpp
    t2 = solver.t2()                       # t2_pphh data order

    solver.calc_t2diff_pphh()              # calcT2Diff_pphh  (calc.cpp:205)
    solver.calc_t2diff_phhp()              # calcT2Diff_phhp  (calc.cpp:315)
    ...

Errors come back as CCDGPUError carrying the library's status code; there is no CPU fallback.
"""
import ctypes

import numpy as np

from . import _native

PREC = {"fp64": 0, "mixed": 1, "mixed_bf16": 1, "mixed_bf16x3": 2}
PATH = {"fused": 0, "tables": 1}
VMODE = {"stored": 0, "on_the_fly": 1, "in_ladder": 2}

CHAIN_T2 = 0
CHAIN_T2_OLD = 1
CHAIN_DIFF_PPHH = 2
CHAIN_DIFF_PHHP = 3
CHAIN_OLD_PHHP = 4
CHAIN_DIFF_H2PP_H1 = 5
CHAIN_DIFF_P2_P1HH = 6
CHAIN_GATHERED0 = 8

MAP_NAMES = ["iab_j", "jab_i", "a_bij", "b_aij", "ai_jb", "aj_ib", "bi_ja", "bj_ia"]


class CCDGPUError(RuntimeError):
    def __init__(self, status, where=""):
        lib = _native.gpu_lib()
        msg = lib.ccdgpu_strerror(status).decode()
        super().__init__(f"{where}: {msg} (status {status})")
        self.status = status


def _check(rc, where):
    if rc != 0:
        raise CCDGPUError(rc, where)


class Result:
    def __init__(self, r):
        self.e_corr = r.e_corr
        self.e_diff = r.e_diff
        self.iterations = int(r.iterations)
        self.converged = bool(r.converged)
        self.polish_iterations = int(r.polish_iterations)
        self.seconds = r.seconds

    def __repr__(self):
        return (f"Result(e_corr={self.e_corr!r}, iterations={self.iterations}, "
                f"converged={self.converged}, seconds={self.seconds:.6f})")


def solve_batch(solvers, tol=1e-8, max_iters=100, mixing=0.5, check=True):
    """Solve several independent systems together (ccdgpu_solve_batch): every solver's device
    loop is in flight at once.  Returns one Result per solver; with check=False a failed solve
    (for example a diverging iteration, e_corr non-finite) does not raise."""
    n = len(solvers)
    hs = (ctypes.c_void_p * n)(*[s._h for s in solvers])
    rs = (_native.Result * n)()
    rc = _native.gpu_lib().ccdgpu_solve_batch(hs, n, tol, max_iters, mixing, rs)
    if check:
        _check(rc, "ccdgpu_solve_batch")
    return [Result(r) for r in rs]


class CCDSolver:
    def __init__(self, system, precision="fp64", path="fused", v_mode="stored", device=0,
                 use_graph=True, polish_threshold=1e-6, device_loop=True):
        lib = _native.gpu_lib()
        self.system = system  # keeps the host problem alive during create
        opt = _native.Options()
        lib.ccdgpu_default_options(ctypes.byref(opt))
        opt.device = device
        opt.precision = PREC[precision]
        opt.path = PATH[path]
        opt.v_mode = VMODE[v_mode]
        opt.use_graph = int(bool(use_graph))
        opt.device_loop = int(bool(device_loop))
        opt.polish_threshold = polish_threshold
        self._h = ctypes.c_void_p()
        _check(lib.ccdgpu_create(system.problem, ctypes.byref(opt), ctypes.byref(self._h)),
               "ccdgpu_create")
        self.n_t2 = int(lib.ccdgpu_t2_size(self._h))
        self.path = path
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None):
            _native.gpu_lib().ccdgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def reset(self):
        _check(_native.gpu_lib().ccdgpu_reset(self._h), "ccdgpu_reset")

    def step(self, mixing=0.5):
        e = ctypes.c_double()
        _check(_native.gpu_lib().ccdgpu_step(self._h, mixing, ctypes.byref(e)), "ccdgpu_step")
        return e.value

    def solve(self, tol=1e-8, max_iters=100, mixing=0.5):
        r = _native.Result()
        _check(_native.gpu_lib().ccdgpu_solve(self._h, tol, max_iters, mixing, ctypes.byref(r)),
               "ccdgpu_solve")
        return Result(r)

    def t2(self, out=None):
        if out is None:
            out = np.empty(self.n_t2)
        _check(_native.gpu_lib().ccdgpu_get_t2(
            self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self.n_t2),
            "ccdgpu_get_t2")
        return out

    def set_t2(self, t2):
        t2 = np.ascontiguousarray(t2, dtype=np.float64)
        _check(_native.gpu_lib().ccdgpu_set_t2(
            self._h, t2.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), t2.size),
            "ccdgpu_set_t2")

    def chain(self, chain_id):
        lib = _native.gpu_lib()
        n = ctypes.c_uint64()
        _check(lib.ccdgpu_read_chain(self._h, chain_id, None, 0, ctypes.byref(n)), "read_chain")
        out = np.empty(n.value)
        _check(lib.ccdgpu_read_chain(self._h, chain_id,
                                     out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     n.value, None), "read_chain")
        return out

    def energy_history(self):
        n = ctypes.c_int64()
        out = np.zeros(128)
        _check(_native.gpu_lib().ccdgpu_energy_history(
            self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 128, ctypes.byref(n)),
            "ccdgpu_energy_history")
        return out[:n.value].copy()

    def enable_profiling(self, on=True):
        _check(_native.gpu_lib().ccdgpu_enable_profiling(self._h, int(bool(on))), "profiling")

    def profile(self):
        p = _native.Profile()
        _check(_native.gpu_lib().ccdgpu_get_profile(self._h, ctypes.byref(p)), "profile")
        return {k: (list(getattr(p, k)) if k == "ms_create" else getattr(p, k))
                for k, _ in p._fields_}

    def schedule(self):
        sch = _native.Schedule()
        _check(_native.gpu_lib().ccdgpu_get_schedule(self._h, ctypes.byref(sch)), "schedule")
        return {"thin_split_mul": sch.thin_split_mul, "wide_split_mul": sch.wide_split_mul,
                "tc_split_mul": sch.tc_split_mul, "mid_split_mul": sch.mid_split_mul}

    def set_schedule(self, thin_split_mul=1, wide_split_mul=3, tc_split_mul=2, mid_split_mul=0):
        sch = _native.Schedule(thin_split_mul, wide_split_mul, tc_split_mul, mid_split_mul)
        _check(_native.gpu_lib().ccdgpu_set_schedule(self._h, ctypes.byref(sch)), "set_schedule")

    def autotune(self, reps=5):
        """Pick the pp-ladder schedule by timing the candidates on this GPU (ccdgpu_autotune).
        Returns (schedule dict, ms per FP64 ladder, ms per tensor-core ladder)."""
        sch = _native.Schedule()
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(_native.gpu_lib().ccdgpu_autotune(self._h, reps, ctypes.byref(sch), ctypes.byref(a),
                                                 ctypes.byref(b)), "ccdgpu_autotune")
        return self.schedule(), a.value, b.value

    def ladder_profile(self, reps=5):
        """Each pp-ladder class alone (ccdgpu_ladder_profile): {class: (ms, flops, bytes)}."""
        ms, fl, by = (ctypes.c_double * 4)(), (ctypes.c_double * 4)(), (ctypes.c_double * 4)()
        _check(_native.gpu_lib().ccdgpu_ladder_profile(self._h, reps, ms, fl, by),
               "ccdgpu_ladder_profile")
        names = ["fp64_thin", "fp64_mid", "fp64_wide", "tensor_core"]
        return {n: (ms[k], fl[k], by[k]) for k, n in enumerate(names) if ms[k] > 0}

    def mbpt2(self, init_t2=False):
        """E_MBPT2 computed on the device (ccdgpu_mbpt2); init_t2=True also starts T2 from the
        first-order amplitudes instead of zero."""
        e = ctypes.c_double()
        _check(_native.gpu_lib().ccdgpu_mbpt2(self._h, int(bool(init_t2)), ctypes.byref(e)),
               "ccdgpu_mbpt2")
        return e.value

    def reference_energy(self, sp_energy_bare):
        """E_ref and the normal-ordered single-particle energies computed on the device from
        the bare ones and the system's model (ccdgpu_reference_energy): (e_ref, energies)."""
        bare = np.ascontiguousarray(sp_energy_bare, dtype=np.float64)
        out = np.zeros_like(bare)
        e = ctypes.c_double()
        dp = ctypes.POINTER(ctypes.c_double)
        _check(_native.gpu_lib().ccdgpu_reference_energy(
            self._h, bare.ctypes.data_as(dp), ctypes.byref(e), out.ctypes.data_as(dp)),
            "ccdgpu_reference_energy")
        return e.value, out

    def kernel_profile(self, reps=5):
        """Ring, hh-ladder and one-body kernel classes alone (ccdgpu_kernel_profile):
        {class: (ms, flops, bytes)}; classes without work are left out."""
        ms, fl, by = (ctypes.c_double * 7)(), (ctypes.c_double * 7)(), (ctypes.c_double * 7)()
        _check(_native.gpu_lib().ccdgpu_kernel_profile(self._h, reps, ms, fl, by),
               "ccdgpu_kernel_profile")
        names = ["ring_small", "ring_mid", "ring_large", "hh_small", "hh_large", "onebody",
                 "hh_reduce"]
        return {n: (ms[k], fl[k], by[k]) for k, n in enumerate(names) if by[k] > 0}

    TRACE_KERNELS = ["ring_small", "ring_mid", "ring_large", "hh_small", "hh_large", "onebody",
                     "ladder_thin", "ladder_mid", "ladder_wide", "ladder_tc", "assemble",
                     "loop_ctl", "energy", "retile", "ladder_reduce", "hh_reduce", "phhp_gather"]

    def trace_arm(self, iteration):
        """Record kernel start times of iteration `iteration` of the next solve (-1 disarms)."""
        _check(_native.gpu_lib().ccdgpu_trace_arm(self._h, int(iteration)), "ccdgpu_trace_arm")

    def trace_read(self, with_end=False):
        """{kernel: (first CTA start, last CTA start)} in ns, relative to the earliest start;
        with_end=True adds the time the last CTA finished (None where a kernel does not record
        it).  Kernels that did not run in the traced iteration are left out."""
        n = len(self.TRACE_KERNELS)
        first = (ctypes.c_uint64 * n)()
        last = (ctypes.c_uint64 * n)()
        end = (ctypes.c_uint64 * n)()
        lib = _native.gpu_lib()
        _check(lib.ccdgpu_trace_read(self._h, first, last, n), "ccdgpu_trace_read")
        _check(lib.ccdgpu_trace_read_end(self._h, end, n), "ccdgpu_trace_read_end")
        ran = [k for k in range(n) if first[k] != 2**64 - 1]
        if not ran:
            return {}
        t0 = min(first[k] for k in ran)
        if with_end:
            return {self.TRACE_KERNELS[k]: (first[k] - t0, last[k] - t0,
                                            end[k] - t0 if end[k] else None) for k in ran}
        return {self.TRACE_KERNELS[k]: (first[k] - t0, last[k] - t0) for k in ran}

    def inject_wait_timeout(self):
        """Failure-path test hook (ccdgpu_inject_wait_timeout): the next step() makes a bounded
        device wait of the FP64 pp ladder run out and raises CCDGPUError(CCDGPU_ERR_TIMEOUT)."""
        _check(_native.gpu_lib().ccdgpu_inject_wait_timeout(self._h), "inject_wait_timeout")

    def stream_ptr(self):
        """The handle's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return _native.gpu_lib().ccdgpu_stream(self._h)

    def work_per_iteration(self):
        f, b, lf = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(_native.gpu_lib().ccdgpu_work_per_iteration(
            self._h, ctypes.byref(f), ctypes.byref(b), ctypes.byref(lf)), "work")
        return {"flops": f.value, "ladder_bytes": b.value, "ladder_flops": lf.value}

    # Stage entry points with the reference's names (calc.hpp, Chain.hpp, main.cpp:591-665).
    def calc_t2diff_p2_p1hh(self):
        _check(_native.gpu_lib().ccdgpu_calc_t2diff_p2_p1hh(self._h), "calcT2Diff_p2_p1hh")

    def calc_t2diff_h2pp_h1(self):
        _check(_native.gpu_lib().ccdgpu_calc_t2diff_h2pp_h1(self._h), "calcT2Diff_h2pp_h1")

    def calc_t2diff_phhp(self):
        _check(_native.gpu_lib().ccdgpu_calc_t2diff_phhp(self._h), "calcT2Diff_phhp")

    def calc_t2diff_pphh(self):
        _check(_native.gpu_lib().ccdgpu_calc_t2diff_pphh(self._h), "calcT2Diff_pphh")

    def map_from_distributed(self):
        _check(_native.gpu_lib().ccdgpu_map_from_distributed(self._h), "mapFromDistributed")

    def calc_t2_pphh(self, mixing=0.5):
        e = ctypes.c_double()
        _check(_native.gpu_lib().ccdgpu_calc_t2_pphh(self._h, mixing, ctypes.byref(e)),
               "calcT2_pphh")
        return e.value

    def map_to_distributed(self):
        _check(_native.gpu_lib().ccdgpu_map_to_distributed(self._h), "mapToDistributed")
