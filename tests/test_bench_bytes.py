"""bench.py's count of the bytes ccdgpu_create moves host -> device (the e2e line's
h2d_bytes_per_step), for every problem form the bench builds: with host tables or not, with
host V or not.  The V_pppp term counts the rows a <= b only, as create uploads them."""
import os
import sys

import numpy as np
import pytest

from helpers import golden, system_for

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
import bench  # noqa: E402


@pytest.mark.parametrize("name", ["eg14_s19", "pnm14_s4", "pairing_gp0.5"])
def test_problem_bytes_per_form(name):
    g = golden(name)
    with system_for(g) as s:
        d = s.chan_dims().astype(np.int64)
        act = (d[:, 0] > 0) & (d[:, 1] > 0)
        pm = s.array("pp_map").reshape(-1, 2)
        # rows a <= b per active channel, independently of the bench's reduceat
        rows, o = [], 0
        for c in range(len(d)):
            n = int(d[c, 0])
            if act[c]:
                rows.append(int((pm[o:o + n, 0] <= pm[o:o + n, 1]).sum()))
            o += n
        pppp = 8 * int((np.array(rows) * d[act, 0]).sum())
        full = bench._problem_bytes(s, with_v_pppp=True, with_tables=True)
        no_pppp = bench._problem_bytes(s, with_v_pppp=False, with_tables=True)
        assert full - no_pppp == pppp
        n_t = int((d[act, 0] * d[act, 1]).sum())
        npart = s.n_sp - s.n_particles
        assert (bench._problem_bytes(s, with_v_pppp=False, with_tables=True)
                - bench._problem_bytes(s, with_v_pppp=False, with_tables=False)
                == 24 * 8 * n_t - 16 * npart * s.n_particles)
        no_v = bench._problem_bytes(s, with_v_pppp=False, with_tables=False, with_v=False)
        assert 0 < no_v < bench._problem_bytes(s, with_v_pppp=False, with_tables=False)
