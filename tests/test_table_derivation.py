"""The remap-table derivation the device runs when a problem carries no loadMaps tables
(pair_sizes_kernel, row_scan_kernel, derive_tables_kernel), restated in numpy and checked
against the reference's own tables on the CPU.

loadMaps (load.cpp:389-532) builds the eight tables from the channel maps alone.  The device
derivation uses only the pair lists, the block offsets inside the three-body chains (exclusive
sums of block sizes over the partner index) and the modified-channel position of every
(particle, hole) pair.  This test states that arithmetic once more and requires the result to
equal the tables the reference wrote, entry for entry (the builder's copies of them are
bit-identical to the reference's dumps, checked by test_builder_golden).
"""
import numpy as np
import pytest

from helpers import EXTRA, MAPS, SMALL, golden, system_for


def derive_tables(s):
    nh, nsp = s.n_particles, s.n_sp
    npart = nsp - nh
    d = s.chan_dims().astype(np.int64)                        # pp, hh, hp, ph
    md = s.array("chan_mod_dims").reshape(-1, 4).astype(np.int64)
    pp = s.array("pp_map").reshape(-1, 2).astype(np.int64)
    hh = s.array("hh_map").reshape(-1, 2).astype(np.int64)
    phm = s.array("ph_mod_map").reshape(-1, 2).astype(np.int64)   # (a, i)
    hpm = s.array("hp_mod_map").reshape(-1, 2).astype(np.int64)   # (j, b)
    nch = len(d)
    off = lambda n: np.concatenate([[0], np.cumsum(n)])
    pp_off, hh_off = off(d[:, 0]), off(d[:, 1])
    ph_off, hp_off = off(md[:, 3]), off(md[:, 2])
    # Block sizes, then exclusive sums over the partner index (pair_sizes + row_scan).
    hsz = np.zeros((nh, nh), np.int64)
    psz = np.zeros((npart, npart), np.int64)
    ch_of_hh = np.repeat(np.arange(nch), d[:, 1])
    ch_of_pp = np.repeat(np.arange(nch), d[:, 0])
    hsz[hh[:, 0], hh[:, 1]] = d[ch_of_hh, 0]
    psz[pp[:, 0] - nh, pp[:, 1] - nh] = d[ch_of_pp, 1]
    hblk = np.cumsum(hsz, axis=1) - hsz
    pblk = np.cumsum(psz, axis=1) - psz
    # Modified channel, row (ph') and column (hp') of every (particle, hole) pair.
    mch = np.full((npart, nh), -1, np.int64)
    mrow = np.full((npart, nh), -1, np.int64)
    mcol = np.full((npart, nh), -1, np.int64)
    ch_of_ph = np.repeat(np.arange(nch), md[:, 3])
    ch_of_hp = np.repeat(np.arange(nch), md[:, 2])
    mch[phm[:, 0] - nh, phm[:, 1]] = ch_of_ph
    mrow[phm[:, 0] - nh, phm[:, 1]] = np.arange(len(phm)) - ph_off[ch_of_ph]
    mcol[hpm[:, 1] - nh, hpm[:, 0]] = np.arange(len(hpm)) - hp_off[ch_of_hp]
    tabs = [[] for _ in range(8)]
    for c in np.nonzero((d[:, 0] > 0) & (d[:, 1] > 0))[0]:
        P = pp[pp_off[c]:pp_off[c + 1]]
        H = hh[hh_off[c]:hh_off[c + 1]]
        AB, IJ = np.meshgrid(np.arange(len(P)), np.arange(len(H)), indexing="ij")
        AB, IJ = AB.ravel(), IJ.ravel()
        a, b = P[AB, 0], P[AB, 1]
        i, j = H[IJ, 0], H[IJ, 1]
        zero = np.zeros_like(a)
        tabs[0].append(np.stack([j, hblk[j, i] + AB, zero], 1))
        tabs[1].append(np.stack([i, hblk[i, j] + AB, zero], 1))
        tabs[2].append(np.stack([a - nh, zero, pblk[a - nh, b - nh] + IJ], 1))
        tabs[3].append(np.stack([b - nh, zero, pblk[b - nh, a - nh] + IJ], 1))
        for k, (x, y, u, v) in enumerate([(a, i, j, b), (a, j, i, b), (b, i, j, a), (b, j, i, a)]):
            tabs[4 + k].append(np.stack([mch[x - nh, y], mrow[x - nh, y], mcol[v - nh, u]], 1))
    return [np.concatenate(t).astype(np.uint64).ravel() for t in tabs]


@pytest.mark.parametrize("name", SMALL + ["eg54_s19"] + EXTRA)
def test_table_derivation_reproduces_reference_tables(name):
    g = golden(name)
    with system_for(g) as s:
        derived = derive_tables(s)
        for k, n in enumerate(MAPS):
            np.testing.assert_array_equal(derived[k], s.array(n), err_msg=n)
