"""The allocation-free channel entry point against the CPU oracle and the stage entry point.

ccdgpu_calc_channel_t2diff_pphh_noalloc serves callers that cannot allocate device memory (a
host that owns all device memory through its own pool or budget): every buffer is supplied by
the caller and its intermediate lives in a fixed scratch array inside the library.

- Every amplitude-carrying channel of the electron gas N=54, |n|^2 <= 20 (pp up to 724, so up
  to 12 split-K slices of 64 rows; hh up to 54, so the X kernel takes more than 48 KB of
  dynamic shared memory) is computed twice in a row, from two different amplitude sets, and
  compared with the oracle (oracle/ccd_oracle.c, calc.cpp:132-203) and with
  ccdgpu_calc_t2diff_pphh (the stage entry point on the solver's own device chains).  The
  second call uses other amplitudes, so a stale X or a ticket counter that was not reset
  would show.
- A synthetic channel at the capacity limit (hh = 72, pp = 3136: 49 slices) against numpy.

Tolerance: 1e-12 of the channel's largest |D| (the stage tolerance of the parity tests).  The
test allocates its device buffers with torch; the entry point itself allocates nothing.
"""
import numpy as np
import pytest

from coupled_cluster_doubles_b200 import CCDSolver, _native, solver as solver_mod
from helpers import golden, system_for
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

STATUS_UNSUPPORTED = -7
RTOL = 1e-12


def _host(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


def _call(lib, dev, stream, vp, vx, vh, t, pp, hh):
    import torch
    out = torch.full((pp * hh,), float("nan"), dtype=torch.float64, device=dev)
    rc = lib.ccdgpu_calc_channel_t2diff_pphh_noalloc(vp.data_ptr(), vx.data_ptr(), vh.data_ptr(),
                                                    t.data_ptr(), out.data_ptr(), pp, hh,
                                                    stream.cuda_stream)
    assert rc == 0
    torch.cuda.synchronize(dev)
    return out.cpu().numpy()


def _close(got, ref):
    scale = max(float(np.max(np.abs(ref))), 1e-300)
    return float(np.max(np.abs(got - ref))) <= RTOL * scale


def test_noalloc_channel_ladder_matches_oracle_and_stage_entry_point():
    import torch

    lib = _native.gpu_lib()
    g = golden("eg54_s19")
    dev = torch.device("cuda:0")
    with system_for(g) as s, CCDSolver(s, path="tables") as sol:
        # Two amplitude sets: after two and after three iterations (t2Old = T2 after a step).
        refs = []
        sol.step(0.5)
        for _ in range(2):
            sol.step(0.5)
            sol.calc_t2diff_pphh()
            t2 = sol.chain(solver_mod.CHAIN_T2_OLD)
            d_stage = sol.chain(solver_mod.CHAIN_DIFF_PPHH)
            oracle = Oracle(s)
            oracle.set_t2(t2)
            oracle.calc_t2diff_pphh()
            d_oracle = oracle.chain(solver_mod.CHAIN_DIFF_PPHH)
            oracle.close()
            refs.append((t2, d_stage, d_oracle))
        t2_a, t2_b = refs[0][0], refs[1][0]
        assert np.any(t2_a) and np.max(np.abs(t2_a - t2_b)) > 0
        p = s.problem.contents
        dims = s.chan_dims()
        stream = torch.cuda.current_stream(dev)
        off = checked = multi_slice = wide = 0
        for c in range(s.n_channels):
            pp, hh = int(dims[c, 0]), int(dims[c, 1])
            if not (pp and hh):
                continue
            vp = torch.from_numpy(_host(p.v_pppp[c], pp * pp)).to(dev)
            vx = torch.from_numpy(_host(p.v_hhpp[c], hh * pp)).to(dev)
            vh = torch.from_numpy(_host(p.v_hhhh[c], hh * hh)).to(dev)
            sl = slice(off, off + pp * hh)
            # Two calls in a row share the scratch array; the second from other amplitudes.
            for t2, d_stage, d_oracle in refs:
                tb = torch.from_numpy(t2[sl].copy()).to(dev)
                got = _call(lib, dev, stream, vp, vx, vh, tb, pp, hh)
                assert _close(got, d_oracle[sl]), (c, pp, hh)
                assert _close(got, d_stage[sl]), (c, pp, hh)
            off += pp * hh
            checked += 1
            multi_slice += pp > 64
            wide += hh > 48
        assert checked > 0 and multi_slice > 0 and wide > 0


def test_noalloc_at_capacity_limit_matches_numpy():
    import torch

    lib = _native.gpu_lib()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    pp, hh = 3136, 72  # 32 + (49 + 1) * 72^2 = 259232 <= 262144 doubles of scratch
    rng = np.random.default_rng(7)
    for call in range(2):  # two calls in a row, different inputs
        v_pppp = rng.standard_normal((pp, pp)) / pp
        v_hhpp = rng.standard_normal((hh, pp)) / pp
        v_hhhh = rng.standard_normal((hh, hh))
        t2 = rng.standard_normal((pp, hh)) * (0.1 + call)
        x = v_hhhh + 0.5 * (v_hhpp @ t2)
        d_ref = 0.5 * (t2 @ x) + 0.5 * (v_pppp @ t2)
        args = [torch.from_numpy(np.ascontiguousarray(a).ravel()).to(dev)
                for a in (v_pppp, v_hhpp, v_hhhh, t2)]
        got = _call(lib, dev, stream, *args, pp, hh)
        assert _close(got, d_ref.ravel()), call


def test_noalloc_rejects_sizes_beyond_scratch():
    import torch

    lib = _native.gpu_lib()
    dev = torch.device("cuda:0")
    buf = torch.zeros(8, dtype=torch.float64, device=dev)
    ptr = buf.data_ptr()
    stream = torch.cuda.current_stream(dev).cuda_stream
    call = lib.ccdgpu_calc_channel_t2diff_pphh_noalloc
    assert call(ptr, ptr, ptr, ptr, ptr, 100000, 72, stream) == STATUS_UNSUPPORTED
    assert call(ptr, ptr, ptr, ptr, ptr, 10, 73, stream) == STATUS_UNSUPPORTED
    # One row past the capacity at hh = 72: 50 slices need 32 + 51 * 72^2 > 262144 doubles.
    assert call(ptr, ptr, ptr, ptr, ptr, 3137, 72, stream) == STATUS_UNSUPPORTED
