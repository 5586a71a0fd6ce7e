"""Host-side CCD systems (the reference's basis + channel + V + remap-table setup).

`System` wraps one ccdhost_system built by libccdhost.so.  Its `.problem` pointer is the
`ccdgpu_problem` that the solver consumes; `.array(name)` exposes the builder's flat arrays
(channel dims, maps, remap tables, V slabs) for tests.  Constructors mirror the reference CLI
(parse.cpp:131-244); `tables=False` leaves the eight remap tables to the
device (ccdgpu_create derives them):

    System.pairing(xi=1.0, g=0.5, n_pair_states=4, n_particles=4)      # --pairing -x -g -l -n
    System.inf_matter(density=0.08, tz_max=1, n_shells=4, n_particle_shells=2)  # --infMatter
    System.electron_gas(r_s=0.5, n_shells=4, n_particle_shells=2)      # --electronGas
"""
import ctypes

import numpy as np

from . import _native

_DT = {1: np.float64, 2: np.uint64, 4: np.int32}


class BuildError(RuntimeError):
    pass


LOAD_V_PPPP, NO_TABLES, NO_V, DEVICE_CHANNELS = 1, 2, 4, 8  # ccdhost_flags


def _flags(load_v_pppp, tables, v_blocks=True, device_channels=False):
    """Builder flags: V_pppp built on the host or not; remap tables built on the host, or left
    to ccdgpu_create, which then derives them on the device; with v_blocks=False no V block at
    all (ccdgpu_create generates them on the device; the solver needs v_mode="on_the_fly");
    device_channels=True builds the channel dimensions and maps on the current CUDA device."""
    return ((LOAD_V_PPPP if load_v_pppp else 0) | (0 if tables else NO_TABLES) |
            (0 if v_blocks else NO_V) | (DEVICE_CHANNELS if device_channels else 0))


class System:
    def __init__(self, handle, kind, params):
        self._h = handle
        self.kind = kind
        self.params = params
        lib = _native.host_lib()
        self.problem = lib.ccdhost_problem(self._h)
        p = self.problem.contents
        self.n_sp = int(p.n_sp)
        self.n_particles = int(p.n_particles)
        self.n_channels = int(p.n_channels)
        self.reference_energy = float(lib.ccdhost_reference_energy(self._h))
        self.mbpt2 = float(lib.ccdhost_mbpt2(self._h))

    @staticmethod
    def _build(fn, *args, kind, params):
        lib = _native.host_lib()
        h = ctypes.c_void_p()
        rc = getattr(lib, fn)(*args, ctypes.byref(h))
        if rc != 0:
            raise BuildError(f"{fn} failed with status {rc}")
        return System(h, kind, params)

    @classmethod
    def pairing(cls, xi=1.0, g=0.5, n_pair_states=4, n_particles=4, load_v_pppp=True,
                tables=True, v_blocks=True, device_channels=False):
        return cls._build("ccdhost_build_pairing", float(xi), float(g), int(n_pair_states),
                          int(n_particles),
                          _flags(load_v_pppp, tables, v_blocks, device_channels),
                          kind="pairing",
                          params=dict(xi=xi, g=g, n_pair_states=n_pair_states,
                                      n_particles=n_particles))

    @classmethod
    def inf_matter(cls, density=0.08, tz_max=1, n_shells=4, n_particle_shells=2,
                   load_v_pppp=True, tables=True, v_blocks=True, device_channels=False):
        return cls._build("ccdhost_build_inf_matter", float(density), int(tz_max),
                          int(n_shells), int(n_particle_shells),
                          _flags(load_v_pppp, tables, v_blocks, device_channels),
                          kind="inf_matter",
                          params=dict(density=density, tz_max=tz_max, n_shells=n_shells,
                                      n_particle_shells=n_particle_shells))

    @classmethod
    def electron_gas(cls, r_s=0.5, n_shells=4, n_particle_shells=2, load_v_pppp=True,
                     tables=True, v_blocks=True, device_channels=False):
        return cls._build("ccdhost_build_electron_gas", float(r_s), int(n_shells),
                          int(n_particle_shells),
                          _flags(load_v_pppp, tables, v_blocks, device_channels),
                          kind="electron_gas",
                          params=dict(r_s=r_s, n_shells=n_shells,
                                      n_particle_shells=n_particle_shells))

    def array(self, name):
        lib = _native.host_lib()
        data = ctypes.c_void_p()
        count = ctypes.c_uint64()
        dtype = ctypes.c_int32()
        rc = lib.ccdhost_array(self._h, name.encode(), ctypes.byref(data), ctypes.byref(count),
                               ctypes.byref(dtype))
        if rc != 0:
            raise KeyError(name)
        dt = np.dtype(_DT[dtype.value])
        n = count.value
        if n == 0:
            return np.zeros(0, dtype=dt)
        buf = (ctypes.c_char * (n * dt.itemsize)).from_address(data.value)
        return np.frombuffer(buf, dtype=dt, count=n).copy()

    def chan_dims(self):
        return self.array("chan_dims").reshape(-1, 4)

    def t2_size(self):
        d = self.chan_dims()
        return int((d[:, 0] * d[:, 1]).sum())

    def close(self):
        if self._h:
            _native.host_lib().ccdhost_free(self._h)
            self._h = None
            self.problem = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
