"""The index mappings of the device V generators (gen_v_hhhh_kernel, gen_v_pphh_kernel,
gen_v_mod_kernel, gen_v3_kernel): which pair of which channel map goes into which argument of
the antisymmetrised matrix element, and where the element lands.  Restated here in numpy for
the pairing model and the electron gas, and checked against the reference's own V blocks
(load.cpp:112-318; the builder's copies are bit-identical to the reference's dumps)."""
import numpy as np
import pytest

from helpers import golden, system_for


def tbme_fn(s, kind):
    qn = s.array("qn").reshape(s.n_sp, -1).astype(np.int64)
    m = s.problem.contents.model.contents
    if kind == "pairing":
        g = m.params[0]

        def v(p, q, r, t):  # PairingSPBasis.cpp:127-141
            a, b, c, d = qn[p], qn[q], qn[r], qn[t]
            ok = (a[:, 0] == b[:, 0]) & (c[:, 0] == d[:, 0]) & (a[:, 1] == -b[:, 1]) & (-c[:, 1] == d[:, 1])
            out = np.where(ok, -0.5 * g, 0.0)
            return np.where(ok & (a[:, 1] == -c[:, 1]), -out, out)
        return v
    L, e_sq = m.params[0], m.params[1]

    def direct(p, q, r, t):  # ElectronGasSPBasis.cpp:424-448
        qi, qj, qk, ql = qn[p], qn[q], qn[r], qn[t]
        ok = (qi[:, 3] == qk[:, 3]) & (qj[:, 3] == ql[:, 3])
        ok &= np.all(qi[:, :3] + qj[:, :3] == qk[:, :3] + ql[:, :3], axis=1)
        prefactor = e_sq / (L * L * L)
        rel = np.zeros(len(p))
        for i in range(3):
            term = 2 * np.pi * (qi[:, i] - qk[:, i]) / L
            rel = rel + term * term
        with np.errstate(divide="ignore"):
            val = prefactor * 4 * np.pi / (rel + 0.0 * 0.0)
        return np.where(ok & (rel >= 1e-5), val, 0.0)

    return lambda p, q, r, t: direct(p, q, r, t) - direct(p, q, t, r)


@pytest.mark.parametrize("name", ["pairing_gp0.5", "eg14_s19"])
def test_generator_mappings_reproduce_reference_v(name):
    g = golden(name)
    with system_for(g) as s:
        v = tbme_fn(s, g["kind"])
        nh = s.n_particles
        d = s.chan_dims().astype(np.int64)
        md = s.array("chan_mod_dims").reshape(-1, 4).astype(np.int64)
        pp = s.array("pp_map").reshape(-1, 2).astype(np.int64)
        hh = s.array("hh_map").reshape(-1, 2).astype(np.int64)
        ph = s.array("ph_mod_map").reshape(-1, 2).astype(np.int64)   # (b, j)
        hp = s.array("hp_mod_map").reshape(-1, 2).astype(np.int64)   # (i, a)
        off = lambda n: np.concatenate([[0], np.cumsum(n)])
        po, ho, pho, hpo = off(d[:, 0]), off(d[:, 1]), off(md[:, 3]), off(md[:, 2])
        act = np.nonzero((d[:, 0] > 0) & (d[:, 1] > 0))[0]
        hhhh, hhpp = [], []
        for c in act:
            P, H = pp[po[c]:po[c + 1]], hh[ho[c]:ho[c + 1]]
            x, y = np.meshgrid(np.arange(len(H)), np.arange(len(H)), indexing="ij")
            x, y = x.ravel(), y.ravel()
            hhhh.append(v(H[x, 0], H[x, 1], H[y, 0], H[y, 1]))          # gen_v_hhhh_kernel
            ab, ij = np.meshgrid(np.arange(len(P)), np.arange(len(H)), indexing="ij")
            ab, ij = ab.ravel(), ij.ravel()
            vt = v(H[ij, 0], H[ij, 1], P[ab, 0], P[ab, 1])              # gen_v_pphh_kernel:
            hhpp.append(vt.reshape(len(P), len(H)).T.ravel())           # V_pphh = V_hhpp^T
        np.testing.assert_allclose(np.concatenate(hhhh), s.array("v_hhhh"), rtol=1e-14, atol=0)
        np.testing.assert_allclose(np.concatenate(hhpp), s.array("v_hhpp"), rtol=1e-14, atol=0)
        hpph, hphp = [], []
        for c in np.nonzero((md[:, 3] > 0) & (md[:, 2] > 0))[0]:
            BJ, IA = ph[pho[c]:pho[c + 1]], hp[hpo[c]:hpo[c + 1]]
            k, x = np.meshgrid(np.arange(len(BJ)), np.arange(len(IA)), indexing="ij")
            k, x = k.ravel(), x.ravel()
            vt = v(IA[x, 0], BJ[k, 1], IA[x, 1], BJ[k, 0])              # gen_v_mod_kernel,
            hpph.append(vt.reshape(len(BJ), len(IA)).T.ravel())         # stored ph' x hp'
            x, y = np.meshgrid(np.arange(len(IA)), np.arange(len(IA)), indexing="ij")
            x, y = x.ravel(), y.ravel()
            hphp.append(v(IA[x, 0], IA[y, 1], IA[x, 1], IA[y, 0]))
        np.testing.assert_allclose(np.concatenate(hpph), s.array("v_hpph_mod"), rtol=1e-14, atol=0)
        np.testing.assert_allclose(np.concatenate(hphp), s.array("v_hphp_mod"), rtol=1e-14, atol=0)
        # Three-body V (gen_v3_kernel): blocks of hpp(k) by j, of phh(a) by b.
        npart = s.n_sp - nh
        hsz = np.zeros((nh, nh), np.int64)
        psz = np.zeros((npart, npart), np.int64)
        hsz[hh[:, 0], hh[:, 1]] = d[np.repeat(np.arange(len(d)), d[:, 1]), 0]
        psz[pp[:, 0] - nh, pp[:, 1] - nh] = d[np.repeat(np.arange(len(d)), d[:, 0]), 1]
        hblk, pblk = np.cumsum(hsz, 1) - hsz, np.cumsum(psz, 1) - psz
        tb = s.array("three_body_dims").reshape(-1, 2).astype(np.int64)   # phh, hpp
        o_h, o_p = off(tb[:nh, 1]), off(tb[nh:, 0])
        v3h, v3p = np.zeros(o_h[-1]), np.zeros(o_p[-1])
        for c in act:
            P, H = pp[po[c]:po[c + 1]], hh[ho[c]:ho[c + 1]]
            x, ab = np.meshgrid(np.arange(len(H)), np.arange(len(P)), indexing="ij")
            x, ab = x.ravel(), ab.ravel()
            k, j = H[x, 0], H[x, 1]
            v3h[o_h[k] + hblk[k, j] + ab] = v(k, j, P[ab, 0], P[ab, 1])
            y, ij = np.meshgrid(np.arange(len(P)), np.arange(len(H)), indexing="ij")
            y, ij = y.ravel(), ij.ravel()
            a, b = P[y, 0] - nh, P[y, 1] - nh
            v3p[o_p[a] + pblk[a, b] + ij] = v(H[ij, 0], H[ij, 1], P[y, 0], P[y, 1])
        np.testing.assert_allclose(v3h, s.array("v_h_hpp"), rtol=1e-14, atol=0)
        np.testing.assert_allclose(v3p, s.array("v_phh_p"), rtol=1e-14, atol=0)


@pytest.mark.parametrize("name", ["pairing_gp0.5", "eg14_s19"])
def test_normal_order_formula_reproduces_reference(name):
    """normal_order_kernel (SPBasis.cpp:7-40): e'_p = e_p + sum_{j<A} <pj|v|pj> and
    E_ref = sum_{i,j<A} 1/2 <ij|v|ij> + sum_{i<A} e_i, from the bare energies."""
    g = golden(name)
    with system_for(g) as s:
        v = tbme_fn(s, g["kind"])
        nh, nsp = s.n_particles, s.n_sp
        bare = s.array("sp_energy_bare")
        p, j = np.meshgrid(np.arange(nsp), np.arange(nh), indexing="ij")
        corr = v(p.ravel(), j.ravel(), p.ravel(), j.ravel()).reshape(nsp, nh)
        np.testing.assert_allclose(bare + corr.sum(axis=1), s.array("sp_energy"), rtol=1e-13,
                                   atol=1e-14)
        i, jj = np.meshgrid(np.arange(nh), np.arange(nh), indexing="ij")
        e_ref = 0.5 * v(i.ravel(), jj.ravel(), i.ravel(), jj.ravel()).sum() + bare[:nh].sum()
        assert e_ref == pytest.approx(float(g["scalars"][0]), rel=1e-13)


def _vgen_codes(qn, orb):
    """An orbital's code in the ladder's generator: momentum bytes biased by 64, 21 in byte 3
    for spin up."""
    q = qn[orb]
    return ((q[..., 0] + 64) | ((q[..., 1] + 64) << 8) | ((q[..., 2] + 64) << 16) |
            (np.where(q[..., 3] > 0, 21, 0) << 24)).astype(np.int64)


def _q2_index(x, y):
    """(x - y + 0x80808080) ^ 0x80808080 as four signed bytes, dotted with itself (dp4a)."""
    d = ((x - y + 0x80808080) & 0xFFFFFFFF) ^ 0x80808080
    out = np.zeros(np.broadcast(x, y).shape, dtype=np.int64)
    for sh in (0, 8, 16, 24):
        b = (d >> sh) & 0xFF
        b = np.where(b >= 128, b - 256, b)
        out += b * b
    return out


@pytest.mark.parametrize("name", ["eg14_s19", "eg14_r2"])
def test_ladder_v_generator_codes_reproduce_reference_v(name):
    """The electron-gas V generator inside the tensor-core ladder (pp_ladder_tc_kernel with
    GEN): V[ab,cd] = w(idx(n_a, n_c)) - w(idx(n_b, n_c)), where the index is q^2 for equal spins
    and q^2 + 441 (a zero entry) otherwise, from codes with the spin in byte 3 and a table w by
    index.  Restated in numpy over every packed row a <= b and K column c < d of every channel,
    against the reference's V_pppp blocks (FP32 table, as the 2-term split uses)."""
    g = golden(name)
    with system_for(g) as s:
        qn = s.array("qn").reshape(s.n_sp, -1).astype(np.int64)
        m = s.problem.contents.model.contents
        L, e_sq = m.params[0], m.params[1]
        assert np.abs(qn[:, :3]).max() <= 6
        q2 = np.arange(3 * 144 + 441 + 1, dtype=np.float64)
        with np.errstate(divide="ignore"):
            tab = np.where((q2 > 0) & (q2 <= 432),
                           e_sq / L ** 3 * 4 * np.pi / ((2 * np.pi / L) ** 2 * q2), 0.0)
        tab = tab.astype(np.float32)
        d = s.chan_dims().astype(np.int64)
        pp = s.array("pp_map").reshape(-1, 2).astype(np.int64)
        vp = s.array("v_pppp")
        po = np.concatenate([[0], np.cumsum(d[:, 0])])
        voff = 0
        checked = 0
        for c in np.nonzero((d[:, 0] > 0) & (d[:, 1] > 0))[0]:
            P = pp[po[c]:po[c + 1]]
            n = len(P)
            ref = vp[voff:voff + n * n].reshape(n, n)
            voff += n * n
            rows = np.nonzero(P[:, 0] <= P[:, 1])[0]
            cols = np.nonzero(P[:, 0] < P[:, 1])[0]
            if not len(rows) or not len(cols):
                continue
            na = _vgen_codes(qn, P[rows, 0][:, None])
            nb = _vgen_codes(qn, P[rows, 1][:, None])
            nc = _vgen_codes(qn, P[cols, 0][None, :])
            i1, i2 = _q2_index(na, nc), _q2_index(nb, nc)
            assert i1.max() < len(tab) and i2.max() < len(tab)
            v = (tab[i1] - tab[i2]).astype(np.float64)
            want = ref[np.ix_(rows, cols)]
            scale = max(float(np.abs(want).max()), 1e-300)
            assert np.max(np.abs(v - want)) <= 2e-7 * scale, c
            checked += 1
        assert checked > 10


@pytest.mark.parametrize("name", ["eg14_s19", "eg54c36_r2", "eg54c36_r05"])
def test_folded_momentum_table_is_exact(name):
    """The device keeps the electron gas's direct term by momentum transfer d = n_a - n_c stored
    by component magnitude (|dx|, |dy|, |dz|).  The reference's expression
    (ElectronGasSPBasis.cpp:424-448) sees each component through (2 pi d_i / L)^2, and a
    negated component gives the same bits, so every entry of the full range [-R, R]^3 equals
    its folded one exactly."""
    g = golden(name)
    with system_for(g, load_v_pppp=False) as s:
        qn = s.array("qn").reshape(s.n_sp, -1).astype(np.int64)
        m = s.problem.contents.model.contents
        L, e_sq = m.params[0], m.params[1]
    R = 2 * int(np.abs(qn[:, :3]).max())
    d = np.stack(np.meshgrid(*[np.arange(-R, R + 1)] * 3, indexing="ij"), -1).reshape(-1, 3)

    def direct(dd):
        prefactor = e_sq / (L * L * L)
        rel = np.zeros(len(dd))
        for i in range(3):
            term = 2 * np.pi * dd[:, i] / L
            rel = rel + term * term
        with np.errstate(divide="ignore"):
            val = prefactor * 4 * np.pi / (rel + 0.0 * 0.0)
        return np.where(rel >= 1e-5, val, 0.0)

    full, folded = direct(d), direct(np.abs(d))
    assert np.array_equal(full.view(np.uint64), folded.view(np.uint64))
