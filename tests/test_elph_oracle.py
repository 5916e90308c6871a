"""CPU checks of the electron-phonon oracle (no GPU).

The reference ships no numeric fixture for this path (its el-ph test has no
assertion and its coupling file is not distributed), so the C++ oracle is
pinned here by properties of the physics and by an independent numpy
restatement of ElScatteringMatrix::builder (el_scattering.cpp:38-405) on a
tiny case.
"""
import numpy as np
import pytest

import oracle
from phoebe_b200 import constants as C
from phoebe_b200 import lattice, synth


@pytest.fixture(scope="module")
def model():
    return synth.elph_model(nw=8, ncell_h=1, ncell_e=1, ncell_p=1)


def test_wannier_hamiltonian_diagonalisation(model):
    wan = oracle.ElectronH0Wannier(model.Re, model.degE, model.H)
    rng = np.random.default_rng(1)
    k = rng.normal(size=(5, 3)) * 0.3
    E, U = wan.diagonalize(k)
    for i in range(len(k)):
        ph = np.exp(1j * model.Re @ k[i])
        Hk = np.einsum("r,rmn->mn", ph, model.H)
        assert np.allclose(Hk, Hk.conj().T, atol=1e-14)
        np.testing.assert_allclose(U[i] @ np.diag(E[i]) @ U[i].conj().T, Hk, atol=1e-13)
        assert np.all(np.diff(E[i]) >= 0)


def test_wannier_velocities_match_energy_differences(model):
    wan = oracle.ElectronH0Wannier(model.Re, model.degE, model.H)
    k = np.array([[0.21, -0.13, 0.07], [0.4, 0.1, -0.3]])
    E, U, v = wan.diagonalize(k, velocities=True)
    h = 1e-5
    for i in range(len(k)):
        for c in range(3):
            kp, km = k[i].copy(), k[i].copy()
            kp[c] += h
            km[c] -= h
            d = (wan.diagonalize(kp)[0][0] - wan.diagonalize(km)[0][0]) / (2 * h)
            nondeg = np.ones(8, bool)
            gaps = np.diff(E[i])
            nondeg[:-1] &= gaps > 1e-4
            nondeg[1:] &= gaps > 1e-4
            np.testing.assert_allclose(v[i, nondeg, c], d[nondeg], rtol=1e-5, atol=1e-9)
    _, _, v0 = wan.diagonalize(np.zeros((1, 3)), velocities=True)
    assert np.all(v0 == 0.0)


def test_coupling_is_gauge_invariant(model):
    wan = oracle.ElectronH0Wannier(model.Re, model.degE, model.H)
    elph = oracle.InteractionElPhWan(model.Re, model.degE, model.Rp, model.degP, model.g)
    k1 = np.array([0.1, 0.2, -0.05])
    k2 = np.array([[0.3, -0.1, 0.2], [-0.2, 0.05, 0.1]])
    _, U1 = wan.diagonalize(k1)
    _, U2 = wan.diagonalize(k2)
    ev3 = np.stack([np.linalg.qr(np.random.default_rng(i).normal(size=(6, 6)) + 0j)[0] for i in range(2)])
    q3 = k2 - k1
    elph.cache_elph(U1[0][:, 2:6], k1)
    a = elph.calc_coupling_squared(U2[:, :, 1:7], np.array([6, 6]), ev3, q3)
    rng = np.random.default_rng(7)
    elph.cache_elph(U1[0][:, 2:6] * np.exp(1j * rng.uniform(0, 6, 4)), k1)
    U2g = U2[:, :, 1:7] * np.exp(1j * rng.uniform(0, 6, (2, 1, 6)))
    b = elph.calc_coupling_squared(U2g, np.array([6, 6]), ev3, q3)
    np.testing.assert_allclose(a, b, rtol=1e-11, atol=1e-14 * a.max())
    assert a.max() > 0


def _numpy_el_builder(model, kmesh, qmesh, Ek, Uk, vk, lo, hi, Eq, evq, kcart, recip, k1list, temps, mu,
                      smearing, sigma, norm):
    """Direct numpy restatement of the el-ph linewidth builder (independent of the C++ oracle)."""
    nw, nph = model.H.shape[1], Eq.shape[1]
    out = np.zeros((len(temps), len(k1list), nw))
    qT = recip / np.asarray(kmesh)[:, None]
    f = [kmesh[i] // qmesh[i] for i in range(3)]
    cut = 5.0 / C.ryToCmm1

    def delta(e, v):
        if smearing == "gaussian":
            x = e / sigma
            return 0.0 if x > 6 else np.exp(-x * x) / sigma / np.sqrt(np.pi)
        if np.linalg.norm(v) == 0 and e == 0:
            return 1.0
        s = np.sqrt(np.sum((qT @ v) ** 2) / 6)
        if s == 0:
            return 0.0
        s = max(s, C.adaptiveBroadeningCutoff)
        if abs(e) > 2 * s:
            return 0.0
        x = e / s
        return np.exp(-x * x) / np.sqrt(np.pi) / s / C.erf2

    def sym(c, e1, e2, e3):
        for axis, e in ((0, e1), (1, e2), (2, e3)):
            c = np.moveaxis(c, axis, 0)
            i = 0
            while i < len(e):
                d = 1
                while i + d < len(e) and abs(e[i] - e[i + d]) < 1e-6:
                    d += 1
                c[i:i + d] = c[i:i + d].sum(0) / float(d)
                i += d
            c = np.moveaxis(c, 0, axis)
        return c

    for i1, ik1 in enumerate(k1list):
        l1, h1 = lo[ik1], hi[ik1]
        if h1 <= l1:
            continue
        U1 = Uk[ik1][:, l1:h1]
        ph = np.exp(1j * model.Re @ kcart[ik1]) / model.degE
        g1 = np.einsum("r,rpnab->pnab", ph, model.g.astype(np.complex128))
        cached = np.einsum("pnab,ac->pncb", g1, U1)
        x1, y1, z1 = np.unravel_index(ik1, kmesh[::-1])[::-1]
        for iq in range(int(np.prod(qmesh))):
            qx, qy, qz = np.unravel_index(iq, qmesh[::-1])[::-1]
            ik2 = ((x1 + f[0] * qx) % kmesh[0]) + kmesh[0] * (((y1 + f[1] * qy) % kmesh[1]) +
                                                            kmesh[1] * ((z1 + f[2] * qz) % kmesh[2]))
            l2, h2 = lo[ik2], hi[ik2]
            if h2 <= l2:
                continue
            q3 = kcart[ik2] - kcart[ik1]
            php = np.exp(1j * model.Rp @ q3) / model.degP
            g3 = np.einsum("p,pncb->ncb", php, cached)
            g4 = np.einsum("ncb,nm->mcb", g3, evq[iq])
            gf = np.einsum("bd,mcb->cdm", np.conj(Uk[ik2][:, l2:h2]), g4)
            c = sym(np.abs(gf) ** 2, Ek[ik1, l1:h1], Ek[ik2, l2:h2], Eq[iq])
            for b2 in range(h2 - l2):
                for b1 in range(h1 - l1):
                    for nu in range(nph):
                        en3 = Eq[iq, nu]
                        if en3 < cut:
                            continue
                        v = vk[ik1, l1 + b1] - vk[ik2, l2 + b2]
                        en1, en2 = Ek[ik1, l1 + b1], Ek[ik2, l2 + b2]
                        d1, d2 = delta(en1 - en2 + en3, v), delta(en1 - en2 - en3, v)
                        if d1 <= 0 and d2 <= 0:
                            continue
                        for it, T in enumerate(temps):
                            f2 = 1.0 / (np.exp((en2 - mu) / T) + 1.0)
                            n3 = 1.0 / (np.exp(en3 / T) - 1.0)
                            out[it, i1, l1 + b1] += c[b1, b2, nu] * ((f2 + n3) * d1 + (1 - f2 + n3) * d2) * norm / en3 * np.pi
        e = Ek[ik1, l1:h1]
        row = out[0, i1, l1:h1].copy()
        for b in range(h1 - l1):
            m = np.abs(e - e[b]) < 1e-6
            out[0, i1, l1 + b] = row[m].sum() / float(m.sum())
    return out


@pytest.mark.parametrize("smearing", ["adaptive", "gaussian"])
def test_oracle_el_builder_matches_numpy_restatement(model, smearing):
    cr = model.crystal
    kmesh, qmesh = (4, 4, 4), (2, 2, 2)
    wan = oracle.ElectronH0Wannier(model.Re, model.degE, model.H)
    kc = lattice.Mesh(cr, kmesh).cartesian_coords()
    Ek, Uk, vk = wan.diagonalize(kc, velocities=True)
    ph = oracle.PhononH0(cr, synth.diamond_fc2(cr))
    qc = lattice.Mesh(cr, qmesh).cartesian_coords()
    Eq, evq = ph.diagonalize(qc)
    mu = float(np.median(Ek))
    lo, hi = synth.active_window(Ek, mu, 0.05)
    assert (hi > lo).sum() > 10
    elph = oracle.InteractionElPhWan(model.Re, model.degE, model.Rp, model.degP, model.g)
    temps = np.array([C.kelvin_to_ry(300.0), C.kelvin_to_ry(900.0)])
    k1 = np.arange(0, 64, 3)
    sigma = 0.01
    A = oracle.el_linewidths(elph, kmesh, qmesh, Ek, Uk, vk, lo, hi, Eq, evq, kc, cr.reciprocal_cell, k1, temps, mu,
                             smearing, sigma, 1.0 / 8)
    B = _numpy_el_builder(model, kmesh, qmesh, Ek, Uk, vk, lo, hi, Eq, evq, kc, cr.reciprocal_cell, k1, temps, mu,
                          smearing, sigma, 1.0 / 8)
    assert np.abs(B).max() > 0
    np.testing.assert_allclose(A, B, rtol=1e-10, atol=1e-14 * np.abs(B).max())
