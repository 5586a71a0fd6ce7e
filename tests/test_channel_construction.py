"""The channel construction the device runs for ccdgpu_build_channels (pair_channel_kernel,
the one-rank ffdBalance order, place_pairs_kernel + sort_segments_kernel), restated in numpy
and checked against the reference's own channel dimensions and maps on the CPU.

Channel of an ordered pair (ElectronGasSPBasis.cpp:572-624, InfMatterSPBasis.cpp:458-510,
PairingSPBasis.cpp:168-181): total (regular) or difference (modified) momentum, spin and
isospin, numbered in one box of (4 nmax + 1)^3 x 3 x t slots.  Channels are ordered by cost
descending, index ascending (balance.cpp:91-144 with one rank); each channel's lists hold its
pairs by kind (pp, hh, hp, ph) in (p, q) order.
"""
import numpy as np
import pytest

from helpers import EXTRA, SMALL, golden, system_for


def channel_rule(g, qn):
    if g["kind"] == "pairing":
        return None
    tz_max = g["params"].get("tz_max", 1)
    chan_tz, mod_tz = (-2, 0) if tz_max == 1 else (2, 2)
    return int(np.abs(qn[:, :3]).max()), chan_tz, mod_tz


def pair_channels(g, qn, nch):
    a, b = qn[:, None, :].astype(np.int64), qn[None, :, :].astype(np.int64)
    rule = channel_rule(g, qn)
    if rule is None:  # pairing: spin sum / difference
        return (a[..., 1] + b[..., 1] + 2) // 2, (a[..., 1] - b[..., 1] + 2) // 2
    nmax, chan_tz, mod_tz = rule
    n, s = 4 * nmax + 1, 3
    t, tm = 2 + chan_tz // 2 if chan_tz >= 0 else 1, 1 + mod_tz
    c = ((a[..., 0] + b[..., 0] + n // 2) * n * n * s * t + (a[..., 1] + b[..., 1] + n // 2) * n * s * t
         + (a[..., 2] + b[..., 2] + n // 2) * s * t + (a[..., 3] + b[..., 3] + 2) // 2 * t
         + (a[..., 4] + b[..., 4] + 2) // 2)
    m = ((a[..., 0] - b[..., 0] + n // 2) * n * n * s * tm + (a[..., 1] - b[..., 1] + n // 2) * n * s * tm
         + (a[..., 2] - b[..., 2] + n // 2) * s * tm + (a[..., 3] - b[..., 3] + 2) // 2 * tm
         + (a[..., 4] - b[..., 4] + mod_tz) // 2)
    assert c.max() < nch and m.max() < nch
    return c, m


def build_channels(g, s):
    nsp, nh, nch = s.n_sp, s.n_particles, s.n_channels
    qn = s.array("qn").reshape(nsp, -1)
    c0, m0 = pair_channels(g, qn, nch)
    p, q = np.meshgrid(np.arange(nsp), np.arange(nsp), indexing="ij")
    kind = np.where(p < nh, np.where(q < nh, 1, 2), np.where(q < nh, 3, 0))  # pp hh hp ph
    d0 = np.zeros((nch, 4), np.int64)
    m0d = np.zeros((nch, 4), np.int64)
    np.add.at(d0, (c0.ravel(), kind.ravel()), 1)
    np.add.at(m0d, (m0.ravel(), kind.ravel()), 1)
    pp_, hh_, hp_, ph_ = (d0[:, k].astype(np.float64) for k in range(4))
    cost = (hh_ * hh_ + hh_ * hp_ + hh_ * pp_ + hp_ * ph_ + hp_ * pp_ + pp_ * pp_ + hp_ * ph_
            + hp_ * hp_)
    order = np.lexsort((np.arange(nch), -cost))   # cost descending, index ascending
    inv = np.empty(nch, np.int64)
    inv[order] = np.arange(nch)
    dims, mdims = d0[order], m0d[order]
    # Lists: stable sort of the (p, q)-ordered pairs by (kind, permuted channel).
    flat_pq = np.stack([p.ravel(), q.ravel()], 1)
    lists = {}
    for name, ch in (("", inv[c0.ravel()]), ("mod", inv[m0.ravel()])):
        key = kind.ravel() * nch + ch
        srt = np.argsort(key, kind="stable")
        lists[name] = {k: flat_pq[srt][kind.ravel()[srt] == k] for k in range(4)}
    return dims, mdims, lists


@pytest.mark.parametrize("name", SMALL + ["eg54_s19"] + EXTRA)
def test_channel_construction_reproduces_reference(name):
    g = golden(name)
    with system_for(g) as s:
        dims, mdims, lists = build_channels(g, s)
        np.testing.assert_array_equal(dims, s.chan_dims().astype(np.int64))
        np.testing.assert_array_equal(mdims, s.array("chan_mod_dims").reshape(-1, 4))
        np.testing.assert_array_equal(lists[""][0].ravel(), s.array("pp_map"))
        np.testing.assert_array_equal(lists[""][1].ravel(), s.array("hh_map"))
        np.testing.assert_array_equal(lists["mod"][3].ravel(), s.array("ph_mod_map"))
        np.testing.assert_array_equal(lists["mod"][2].ravel(), s.array("hp_mod_map"))
