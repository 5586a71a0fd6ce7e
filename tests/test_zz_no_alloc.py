"""The allocation-free channel entry point against the solver's own stage entry point.

ccdgpu_calc_channel_t2diff_pphh_noalloc serves callers that cannot allocate device memory (a
host that owns all device memory through its own pool or budget): every buffer is supplied by
the caller and its intermediate lives in a fixed scratch array inside the library.  This test
computes the ladder term of every amplitude-carrying channel of a small system with it, twice
in a row, and compares with ccdgpu_calc_t2diff_pphh (the stage entry point, which works on the
solver's own device chains) at the stage tolerance of the parity tests.  The test allocates its
device buffers with torch; the entry point itself allocates nothing.
"""
import numpy as np
import pytest

from coupled_cluster_doubles_b200 import CCDSolver, _native, solver as solver_mod
from helpers import golden, system_for

pytestmark = pytest.mark.gpu

STATUS_UNSUPPORTED = -7


def _host(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


def test_noalloc_channel_ladder_matches_stage_entry_point():
    import torch

    lib = _native.gpu_lib()
    g = golden("pnm14_s4")
    dev = torch.device("cuda:0")
    with system_for(g) as s, CCDSolver(s, path="tables") as sol:
        for _ in range(3):
            sol.step(0.5)
        sol.calc_t2diff_pphh()
        d_ref = sol.chain(solver_mod.CHAIN_DIFF_PPHH)
        t2 = sol.chain(solver_mod.CHAIN_T2_OLD)
        assert np.any(t2)
        p = s.problem.contents
        dims = s.chan_dims()
        stream = torch.cuda.current_stream(dev)
        off = checked = 0
        for c in range(s.n_channels):
            pp, hh = int(dims[c, 0]), int(dims[c, 1])
            if not (pp and hh):
                continue
            vp = torch.from_numpy(_host(p.v_pppp[c], pp * pp)).to(dev)
            vx = torch.from_numpy(_host(p.v_hhpp[c], hh * pp)).to(dev)
            vh = torch.from_numpy(_host(p.v_hhhh[c], hh * hh)).to(dev)
            tb = torch.from_numpy(t2[off:off + pp * hh].copy()).to(dev)
            ref = d_ref[off:off + pp * hh]
            scale = max(float(np.max(np.abs(ref))), 1e-300)
            for _ in range(2):  # two calls in a row share the scratch array
                out = torch.full((pp * hh,), float("nan"), dtype=torch.float64, device=dev)
                rc = lib.ccdgpu_calc_channel_t2diff_pphh_noalloc(
                    vp.data_ptr(), vx.data_ptr(), vh.data_ptr(), tb.data_ptr(), out.data_ptr(),
                    pp, hh, stream.cuda_stream)
                assert rc == 0
                torch.cuda.synchronize(dev)
                got = out.cpu().numpy()
                assert np.max(np.abs(got - ref)) <= 1e-12 * scale
            off += pp * hh
            checked += 1
        assert checked > 0


def test_noalloc_rejects_sizes_beyond_scratch():
    import torch

    lib = _native.gpu_lib()
    dev = torch.device("cuda:0")
    buf = torch.zeros(8, dtype=torch.float64, device=dev)
    ptr = buf.data_ptr()
    stream = torch.cuda.current_stream(dev).cuda_stream
    assert lib.ccdgpu_calc_channel_t2diff_pphh_noalloc(ptr, ptr, ptr, ptr, ptr, 100000, 72,
                                                       stream) == STATUS_UNSUPPORTED
    assert lib.ccdgpu_calc_channel_t2diff_pphh_noalloc(ptr, ptr, ptr, ptr, ptr, 10, 73,
                                                       stream) == STATUS_UNSUPPORTED
