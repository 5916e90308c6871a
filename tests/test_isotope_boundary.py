"""Isotope (ph_scattering.cpp:616-793) and boundary (:819-860) scattering.

CPU: the oracle's isotope and boundary terms equal an independent numpy
restatement of the reference formulas (including the adaptive isotope delta
that takes its width from v1 and is halved), and the host finalize step with
a boundary length equals the oracle's.  GPU: the builder with isotope and
boundary scattering matches the oracle to 1e-10 on the fused nb = 6 path
(adaptive and Gaussian) and on the shared-memory path (15 branches, with a
q2 window); the split path with isotope scattering stays within 1e-5 of FP64."""
import numpy as np
import pytest

import oracle
from phoebe_b200 import constants as C
from phoebe_b200 import lattice, synth

G_DIAMOND = np.array([2.0e-4, 5.0e-4])   # per-atom isotope mass variances (distinct to test indexing)


def _oracle_inputs(cr, fc2, mesh):
    h0 = oracle.PhononH0(cr, fc2)
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    E, U = h0.diagonalize(q)
    return E, U, h0.velocities(q), q


def _numpy_isotope(E, U, vg, mesh, recip, T, smearing, sigma, g):
    """ph_scattering.cpp:616-793, linewidth mode, restated with numpy."""
    nq, nb = E.shape
    nat = nb // 3
    norm = 1.0 / nq
    qT = np.asarray(recip) / np.asarray(mesh)[:, None]
    ecut = 0.001 / C.ryToCmm1
    ok = (E >= C.phExcludeCutoff) & (E >= ecut)
    out = np.zeros((len(T), nq * nb))
    bose = [np.where(E > 0, 1.0 / np.expm1(np.maximum(E, 1e-300) / t), 0.0) for t in T]
    Ua = U.reshape(nq, nat, 3, nb)
    # Z[q1, q2, at, b1, b2] = sum_k conj(U1) U2
    Z = np.einsum("pakb,qakc->pqabc", Ua.conj(), Ua)
    term = np.einsum("pqabc,a->pqbc", np.abs(Z) ** 2, g)
    e1 = E[:, None, :, None]
    e2 = E[None, :, None, :]
    de = e1 - e2
    if smearing == "gaussian":
        x = de / sigma
        dl = np.where(x > 6, 0.0, np.exp(-x * x) / sigma / np.sqrt(np.pi))
    else:
        v1 = vg[:, None, :, None, :]
        s = np.sqrt(((v1 @ qT.T) ** 2).sum(-1) / 6)
        s = np.where((s != 0) & (s < C.adaptiveBroadeningCutoff), C.adaptiveBroadeningCutoff, s)
        vz = np.all(v1 == 0, axis=-1)
        sd = np.where(s > 0, s, 1.0)
        x = de / sd
        d = np.where(np.abs(de) > 2 * s, 0.0, np.exp(-x * x) / np.sqrt(np.pi) / sd / C.erf2)
        d = np.where(s == 0, 0.0, d)
        dl = 0.5 * np.where(vz & (de == 0), 1.0, d)
    rate = np.pi * 0.5 * norm * e1 * e2 * dl * term
    rate = np.where(ok[:, None, :, None] & ok[None, :, None, :], rate, 0.0)
    for c, b in enumerate(bose):
        n1 = b[:, None, :, None]
        n2 = b[None, :, None, :]
        out[c] = (rate * (n1 * n2 + 0.5 * (n1 + n2))).sum(axis=(1, 3)).ravel()
    return out


@pytest.mark.parametrize("smearing", ["gaussian", "adaptive"])
def test_oracle_isotope_term_vs_numpy(diamond, smearing):
    cr, mesh = diamond["crystal"], (3, 3, 3)
    E, U, vg, q = _oracle_inputs(cr, diamond["fc2"], mesh)
    T = np.array([C.kelvin_to_ry(300.0), C.kelvin_to_ry(700.0)])
    sigma = 0.3 / C.ryToTHz
    from phoebe_b200.core import isotope_coupling
    g = isotope_coupling(cr, G_DIAMOND)
    v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    a = v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, smearing, sigma, finalize=False)
    b = v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, smearing, sigma, finalize=False,
                      isotope_coupling=g)
    ref = _numpy_isotope(E, U, vg, mesh, cr.reciprocal_cell, T, smearing, sigma, g)
    assert np.abs(ref).max() > 0
    np.testing.assert_allclose(b - a, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())


def test_oracle_boundary_term_and_host_finalize(diamond):
    from phoebe_b200.core import finalize_linewidths
    cr, mesh = diamond["crystal"], (3, 3, 3)
    E, U, vg, q = _oracle_inputs(cr, diamond["fc2"], mesh)
    T = np.array([C.kelvin_to_ry(300.0), C.kelvin_to_ry(700.0)])
    L = 1.0e6   # Bohr
    v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    a = v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, "adaptive", 0.0)
    b = v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, "adaptive", 0.0, boundary_length=L)
    ok = E >= C.phExcludeCutoff
    for c, t in enumerate(T):
        with np.errstate(divide="ignore", over="ignore"):
            x = np.sinh(E / 2 / t)
            bd = np.where(ok, np.linalg.norm(vg, axis=-1) / L * 0.25 / x / x, 0.0)
        np.testing.assert_allclose((b - a)[c], bd.ravel(), rtol=1e-10, atol=1e-14 * np.abs(bd).max())
    # the host finalize of partial sums equals the oracle's own finalize
    part = v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, "adaptive", 0.0, finalize=False)
    fin = finalize_linewidths(part, E, vg, T, L)
    np.testing.assert_allclose(fin, b, rtol=1e-12, atol=1e-14 * np.abs(b).max())


def _compare(A_gpu, A_ref, rtol):
    scale = np.abs(A_ref).max()
    assert scale > 0
    big = np.abs(A_ref) > 1e-6 * scale
    rel = np.abs(A_gpu - A_ref)[big] / np.abs(A_ref)[big]
    assert rel.max() < rtol, rel.max()
    assert np.abs(A_gpu - A_ref)[~big].max(initial=0.0) < rtol * 1e-6 * scale


def _gpu_oracle(ctx, cr, fc2, fc3, mesh, smearing, g, L, window=False, precision="fp64"):
    from phoebe_b200.core import Interaction3Ph, PhononH0, PhScatteringMatrix
    T = np.array([C.kelvin_to_ry(300.0), C.kelvin_to_ry(600.0)])
    sigma = 0.3 / C.ryToTHz
    h0 = PhononH0(ctx, cr, fc2)
    bands = h0.populate(mesh, withVelocities=True)
    E, U, vg = bands.get()
    win = synth.q2_window(E, mesh) if window else None
    v3 = Interaction3Ph(ctx, cr, fc3, precision=precision)
    A_gpu = PhScatteringMatrix(v3, bands, T, smearing, sigma, window=win, isotope_coupling=g,
                               boundary_length=L).setup()
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    A_ref = oracle.Interaction3Ph(cr, fc3).linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, smearing, sigma,
                                                       window=win, isotope_coupling=g, boundary_length=L)
    for o in (v3, bands, h0):
        o.close()
    return A_gpu, A_ref


@pytest.mark.gpu
@pytest.mark.parametrize("smearing,mesh", [("adaptive", (6, 6, 6)), ("gaussian", (4, 4, 4))])
def test_fused_path_isotope_boundary_vs_oracle(ctx, diamond, smearing, mesh):
    from phoebe_b200.core import isotope_coupling
    cr = diamond["crystal"]
    A_gpu, A_ref = _gpu_oracle(ctx, cr, diamond["fc2"], diamond["fc3"], mesh, smearing,
                               isotope_coupling(cr, G_DIAMOND), 2.0e5)
    _compare(A_gpu, A_ref, 1e-10)


@pytest.mark.gpu
def test_generic_path_isotope_boundary_window_vs_oracle(ctx):
    from phoebe_b200.core import isotope_coupling
    w = synth.perovskite_workload(mesh=(3, 3, 3), num_pairs=150, fc_grid=(4, 4, 4))
    g = isotope_coupling(w.crystal, [1.2e-4, 3.0e-4, 4.0e-5, 4.0e-5, 4.0e-5])
    A_gpu, A_ref = _gpu_oracle(ctx, w.crystal, w.fc2, w.fc3, (3, 3, 3), "adaptive", g, 5.0e5, window=True)
    _compare(A_gpu, A_ref, 1e-10)


@pytest.mark.gpu
def test_split_path_with_isotopes(ctx, diamond):
    from phoebe_b200.core import isotope_coupling
    cr = diamond["crystal"]
    g = isotope_coupling(cr, G_DIAMOND)
    A16, _ = _gpu_oracle(ctx, cr, diamond["fc2"], diamond["fc3"], (6, 6, 6), "adaptive", g, 0.0,
                         precision="split_bf16")
    A64, _ = _gpu_oracle(ctx, cr, diamond["fc2"], diamond["fc3"], (6, 6, 6), "adaptive", g, 0.0)
    _compare(A16, A64, 1e-5)
