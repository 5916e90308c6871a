"""Electron-phonon Wannier path on the GPU against the CPU FP64 oracle.

ElectronH0Wannier (FT + eigensolve + Hellmann-Feynman velocities),
InteractionElPhWan (cacheElPh, calcCouplingSquared) and the linewidth builder
of ElScatteringMatrix: FP64 GPU results agree with the oracle to 1e-10
relative (couplings, linewidths) on the same inputs.
"""
import numpy as np
import pytest

import oracle
from phoebe_b200 import constants as C
from phoebe_b200 import lattice, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def model():
    return synth.elph_model(nw=8, ncell_h=1, ncell_e=1, ncell_p=1)


def test_wannier_bands_match_oracle(ctx, model):
    from phoebe_b200.core import ElectronH0Wannier
    cr = model.crystal
    wan = ElectronH0Wannier(ctx, cr, model.Re, model.degE, model.H)
    ref = oracle.ElectronH0Wannier(model.Re, model.degE, model.H)
    k = lattice.Mesh(cr, (5, 5, 5)).cartesian_coords()
    E, U, v = wan.diagonalizeWithVelocities(k)
    Eo, Uo, vo = ref.diagonalize(k, velocities=True)
    scale = np.abs(Eo).max()
    np.testing.assert_allclose(E, Eo, rtol=0, atol=1e-12 * scale)
    # eigenvectors up to a phase per band (non-degenerate bands): |<u_gpu|u_orc>| = 1
    ov = np.abs(np.einsum("kwb,kwb->kb", np.conj(U), Uo))
    gaps = np.minimum(np.abs(np.diff(Eo, axis=1, prepend=-1e9)), np.abs(np.diff(Eo, axis=1, append=1e9)))
    nd = gaps > 1e-6
    np.testing.assert_allclose(ov[nd], 1.0, atol=1e-9)
    vs = np.abs(vo).max()
    np.testing.assert_allclose(v, vo, rtol=0, atol=1e-6 * vs)
    bands = wan.populate((5, 5, 5))
    Eb, _, vb = bands.get()
    np.testing.assert_allclose(Eb, E, rtol=0, atol=1e-13 * scale)
    # the mesh path forms k on the host in C++: an ulp of k moves the finite
    # difference (step 1e-8) of H by ~1e-8 of the velocity scale
    np.testing.assert_allclose(vb, v, rtol=0, atol=1e-6 * vs)
    bands.close()
    wan.close()


def test_couplings_match_oracle(ctx, model):
    from phoebe_b200.core import InteractionElPhWan
    ref_wan = oracle.ElectronH0Wannier(model.Re, model.degE, model.H)
    k1 = np.array([0.11, -0.23, 0.05])
    k2 = np.random.default_rng(3).normal(size=(9, 3)) * 0.4
    _, U1 = ref_wan.diagonalize(k1)
    _, U2 = ref_wan.diagonalize(k2)
    ev3 = np.stack([np.linalg.qr(np.random.default_rng(10 + i).normal(size=(6, 6)) +
                                 1j * np.random.default_rng(20 + i).normal(size=(6, 6)))[0] for i in range(9)])
    q3 = k2 - k1
    nb2s = np.array([6, 5, 6, 3, 6, 1, 6, 4, 6], dtype=np.int32)
    U2p = np.zeros((9, 8, 6), dtype=np.complex128)
    for i in range(9):
        U2p[i, :, :nb2s[i]] = U2[i][:, 1:1 + nb2s[i]]
    ref = oracle.InteractionElPhWan(model.Re, model.degE, model.Rp, model.degP, model.g)
    ref.cache_elph(U1[0][:, 2:7], k1)
    co = ref.calc_coupling_squared(U2p, nb2s, ev3, q3)
    gpu = InteractionElPhWan(ctx, model.Re, model.degE, model.Rp, model.degP, model.g)
    gpu.cacheElPh(U1[0][:, 2:7], k1)
    out = gpu.calcCouplingSquared([U2p[i][:, :nb2s[i]] for i in range(9)], ev3, q3)
    for i in range(9):
        a, b = out[i], co[i, :, :nb2s[i], :]
        assert a.shape == b.shape
        np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-14 * np.abs(co).max())
    assert np.abs(co).max() > 0
    gpu.close()


@pytest.mark.parametrize("smearing,kmesh,qmesh", [("adaptive", (6, 6, 6), (3, 3, 3)),
                                                  ("gaussian", (4, 4, 4), (2, 2, 2))])
def test_el_linewidths_match_oracle(ctx, model, smearing, kmesh, qmesh):
    from phoebe_b200.core import (ElectronH0Wannier, ElScatteringMatrix, InteractionElPhWan, PhononH0)
    cr = model.crystal
    wan = ElectronH0Wannier(ctx, cr, model.Re, model.degE, model.H)
    el = wan.populate(kmesh, withVelocities=True)
    h0 = PhononH0(ctx, cr, synth.diamond_fc2(cr))
    ph = h0.populate(qmesh, withVelocities=False)
    gpu = InteractionElPhWan(ctx, model.Re, model.degE, model.Rp, model.degP, model.g)
    Ek, Uk, vk = el.get()
    Eq, evq, _ = ph.get(velocities=False)
    mu = float(np.median(Ek))
    window = 0.05
    temps = np.array([C.kelvin_to_ry(300.0), C.kelvin_to_ry(900.0)])
    nk = int(np.prod(kmesh))
    k1 = np.arange(0, nk, 2 if nk > 100 else 1, dtype=np.int32)
    sigma = 0.01
    sm = ElScatteringMatrix(gpu, el, ph, temps, mu, window, smearing, sigma)
    A = sm.setup(k1)
    lo, hi = synth.active_window(Ek, mu, window)
    kc = lattice.Mesh(cr, kmesh).cartesian_coords()
    ref = oracle.InteractionElPhWan(model.Re, model.degE, model.Rp, model.degP, model.g)
    B = oracle.el_linewidths(ref, kmesh, qmesh, Ek, Uk, vk, lo, hi, Eq, evq, kc, cr.reciprocal_cell, k1, temps, mu,
                             smearing, sigma, 1.0 / np.prod(qmesh))
    assert np.abs(B).max() > 0
    big = np.abs(B) > 1e-9 * np.abs(B).max()
    rel = np.abs(A - B)[big] / np.abs(B)[big]
    assert rel.max() < 1e-10, rel.max()
    assert np.abs(A - B)[~big].max(initial=0.0) < 1e-15 * np.abs(B).max()
    # inactive states carry no linewidth
    for i, ik in enumerate(k1):
        mask = np.ones(8, bool)
        mask[lo[ik]:hi[ik]] = False
        assert np.all(A[:, i, mask] == 0.0)
    gpu.close()
    ph.close()
    h0.close()
    el.close()
    wan.close()


def test_el_linewidths_split_precision(ctx, model):
    """Tensor-core (BF16 x3) Rp transform: linewidths within 1e-5 of the FP64 path."""
    from phoebe_b200.core import (ElectronH0Wannier, ElScatteringMatrix, InteractionElPhWan, PhononH0)
    cr = model.crystal
    kmesh, qmesh = (8, 8, 8), (4, 4, 4)
    wan = ElectronH0Wannier(ctx, cr, model.Re, model.degE, model.H)
    el = wan.populate(kmesh, withVelocities=True)
    h0 = PhononH0(ctx, cr, synth.diamond_fc2(cr))
    ph = h0.populate(qmesh, withVelocities=False)
    gpu = InteractionElPhWan(ctx, model.Re, model.degE, model.Rp, model.degP, model.g)
    Ek = el.get(velocities=False)[0]
    mu = float(np.median(Ek))
    temps = np.array([C.kelvin_to_ry(300.0)])
    k1 = np.arange(0, 512, 3, dtype=np.int32)
    sm = ElScatteringMatrix(gpu, el, ph, temps, mu, 0.05, "adaptive")
    A64 = sm.setup(k1)
    gpu.setPrecision("split_bf16")
    A16 = sm.setup(k1)
    assert np.abs(A64).max() > 0
    big = np.abs(A64) > 1e-6 * np.abs(A64).max()
    rel = np.abs(A16 - A64)[big] / np.abs(A64)[big]
    print("split vs fp64, small el-ph model: max rel %.3e" % rel.max())
    assert rel.max() < 1e-5, rel.max()
    gpu.setPrecision("fp64")
    # back on the FP64 path (atomic accumulation order varies between runs)
    np.testing.assert_allclose(sm.setup(k1), A64, rtol=1e-13, atol=0)
    gpu.close()
    ph.close()
    h0.close()
    el.close()
    wan.close()


def test_el_linewidths_split_precision_full_model(ctx):
    """The el-ph benchmark model (343 electron and 343 phonon vectors, 40^3 k,
    20^3 q): split-precision linewidths of a sample of active k1 within 1e-5 of
    the FP64 path (the FP64 path itself is pinned to the oracle on the small
    model above)."""
    from phoebe_b200.core import (ElectronH0Wannier, ElScatteringMatrix, InteractionElPhWan, PhononH0)
    model = synth.elph_model(nw=8, ncell_h=3, ncell_e=3, ncell_p=3)
    cr = model.crystal
    wan = ElectronH0Wannier(ctx, cr, model.Re, model.degE, model.H)
    el = wan.populate((40, 40, 40), withVelocities=True)
    h0 = PhononH0(ctx, cr, synth.diamond_fc2(cr))
    ph = h0.populate((20, 20, 20), withVelocities=False)
    gpu = InteractionElPhWan(ctx, model.Re, model.degE, model.Rp, model.degP, model.g)
    Ek = el.get(velocities=False)[0]
    mu = float(np.median(Ek))
    window = 0.3 / C.energyRyToEv
    lo, hi = synth.active_window(Ek, mu, window)
    active = np.nonzero(hi > lo)[0]
    k1 = np.sort(np.random.default_rng(5).choice(active, 12, replace=False)).astype(np.int32)
    temps = np.array([C.kelvin_to_ry(300.0)])
    sm = ElScatteringMatrix(gpu, el, ph, temps, mu, window, "adaptive")
    A64 = sm.setup(k1)
    gpu.setPrecision("split_bf16")
    A16 = sm.setup(k1)
    big = np.abs(A64) > 1e-6 * np.abs(A64).max()
    rel = np.abs(A16 - A64)[big] / np.abs(A64)[big]
    print("split vs fp64, full el-ph model: max rel %.3e, median %.3e over %d linewidths"
          % (rel.max(), np.median(rel), big.sum()))
    assert big.sum() >= 8
    assert rel.max() < 1e-5, rel.max()
    gpu.close()
    ph.close()
    h0.close()
    el.close()
    wan.close()
