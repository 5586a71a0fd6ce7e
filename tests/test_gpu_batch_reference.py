"""The batched electron-gas sweep (bench.py --config batch24: 24 systems, N in {14, 38, 54} x
r_s from 0.5 to 8, solved together by ccdgpu_solve_batch) against the reference's own outcome
for every member (tests/golden/batch24.npz, made by tests/golden/make_batch_golden.py with the
unmodified reference at the sweep's stop threshold).

The reference loop (main.cpp:508-519) stops when |dE| <= tol, at 101 iterations, or at the first
non-finite energy (|dE| > tol is then false).  A member converges, reaches the cap or diverges
in FP64 exactly as in the reference, with the same iteration count (+-1) and energy; in mixed
precision the members the reference converges converge, to 1e-7 per particle plus the stop
threshold, and the others do not converge.
"""
import math
import os

import numpy as np
import pytest

from coupled_cluster_doubles_b200 import CCDSolver, System, solve_batch
from helpers import GOLDEN

pytestmark = pytest.mark.gpu


def _outcome(r):
    if not math.isfinite(r.e_corr):
        return "diverged"
    return "converged" if r.converged else "capped"


def _solve(g, precision):
    systems = [System.electron_gas(r_s=float(rs), n_shells=int(ns), n_particle_shells=int(p),
                                   load_v_pppp=False)
               for rs, ns, p in zip(g["r_s"], g["n_shells"], g["n_particle_shells"])]
    sols = [CCDSolver(s, precision=precision, v_mode="on_the_fly") for s in systems]
    try:
        return solve_batch(sols, tol=float(g["tol"][0]), max_iters=100, check=False)
    finally:
        for s in sols:
            s.close()
        for s in systems:
            s.close()


def _golden():
    return dict(np.load(os.path.join(GOLDEN, "batch24.npz")))


def test_batch_fp64_outcomes_match_reference():
    g = _golden()
    tol = float(g["tol"][0])
    res = _solve(g, "fp64")
    for k, r in enumerate(res):
        want = str(g["status"][k])
        assert _outcome(r) == want, (k, _outcome(r), want)
        if want == "converged":
            e_ref = float(g["e_final"][k])
            assert abs(r.iterations - int(g["iterations"][k])) <= 1, k
            assert abs(r.e_corr - e_ref) <= 2 * tol + 1e-10 * abs(e_ref), (k, r.e_corr, e_ref)
        elif want == "capped":
            assert r.iterations == int(g["iterations"][k]) == 101, k


def test_batch_mixed_converges_where_reference_does():
    g = _golden()
    tol = float(g["tol"][0])
    res = _solve(g, "mixed_bf16")
    for k, r in enumerate(res):
        want = str(g["status"][k])
        n = int(g["n"][k])
        if want == "converged":
            e_ref = float(g["e_final"][k])
            assert _outcome(r) == "converged", (k, _outcome(r))
            assert abs(r.e_corr - e_ref) <= 2 * tol + 1e-7 * n, (k, r.e_corr, e_ref)
        else:
            assert _outcome(r) != "converged", (k, _outcome(r), want)
