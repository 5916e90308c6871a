"""Batched uneven instances: the 5-atom perovskite-like cell (15 branches)
with a per-q1 energy window on q2 (the workload has no counterpart in the
reference; the oracle applies the identical filter).

CPU: the window's properties, and the oracle builder with a window that
keeps everything equals the oracle without one.  GPU: the shared-memory FP64
builder (any nb <= 16, windows) matches the oracle to 1e-10 on the 15-branch
cell with and without windows, and on the 6-branch diamond cell a window
that keeps every pair reproduces the fused nb = 6 kernel; the batched
15x15 eigensolve matches the oracle's."""
import numpy as np
import pytest

import oracle
from phoebe_b200 import constants as C
from phoebe_b200 import lattice, synth


@pytest.fixture(scope="module")
def perovskite():
    # the 15-branch cell of the batched workload with a reduced FC3 (150 pairs)
    # and FC2 grid so that the oracle finishes in seconds
    return synth.perovskite_workload(mesh=(4, 4, 4), num_pairs=150, fc_grid=(4, 4, 4))


def _oracle_bands(w, mesh):
    h0 = oracle.PhononH0(w.crystal, w.fc2)
    q = lattice.Mesh(w.crystal, mesh).cartesian_coords()
    E, U = h0.diagonalize(q)
    return E, U, h0.velocities(q), q


def test_window_properties(perovskite):
    mesh = (4, 4, 4)
    E, *_ = _oracle_bands(perovskite, mesh)
    energy, cut = synth.q2_window(E, mesh)
    nq = E.shape[0]
    keep = energy[None, :] <= cut[:, None]          # (q1, q2)
    frac = keep.mean(axis=1)
    assert frac.min() >= 0.2 - 1e-12 and frac.max() <= 1.0
    assert frac.min() < 0.6 and frac.std() > 0.05  # uneven
    m = np.arange(nq)
    ix, iy, iz = m % 4, (m // 4) % 4, m // 16
    neg = ((4 - iz) % 4) * 16 + ((4 - iy) % 4) * 4 + (4 - ix) % 4
    np.testing.assert_array_equal(keep, keep[:, neg])   # q2 and -q2 together
    e2, c2 = synth.q2_window(E, mesh)
    np.testing.assert_array_equal(cut, c2)


def test_oracle_window_keeping_everything_is_no_window(diamond):
    mesh = (4, 4, 4)
    cr = diamond["crystal"]
    h0 = oracle.PhononH0(cr, diamond["fc2"])
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    E, U = h0.diagonalize(q)
    vg = h0.velocities(q)
    v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    T = np.array([C.kelvin_to_ry(300.0)])
    a = v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, "adaptive", 0.0)
    nq = E.shape[0]
    b = v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, "adaptive", 0.0,
                      window=(np.zeros(nq), np.zeros(nq)))
    np.testing.assert_array_equal(a, b)
    c = v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, "adaptive", 0.0,
                      window=(np.ones(nq), np.zeros(nq)), finalize=False)
    assert np.all(c == 0.0)


def _compare(A_gpu, A_ref, rtol):
    scale = np.abs(A_ref).max()
    assert scale > 0
    big = np.abs(A_ref) > 1e-6 * scale
    rel = np.abs(A_gpu - A_ref)[big] / np.abs(A_ref)[big]
    assert rel.max() < rtol, rel.max()
    assert np.abs(A_gpu - A_ref)[~big].max(initial=0.0) < rtol * 1e-6 * scale


def _gpu_vs_oracle(ctx, w, mesh, smearing, temps_k, window):
    from phoebe_b200.core import Interaction3Ph, PhononH0, PhScatteringMatrix
    cr = w.crystal
    T = np.array([C.kelvin_to_ry(t) for t in temps_k])
    sigma = 0.3 / C.ryToTHz
    h0 = PhononH0(ctx, cr, w.fc2)
    bands = h0.populate(mesh, withVelocities=True)
    E, U, vg = bands.get()
    win = synth.q2_window(E, mesh) if window else None
    v3 = Interaction3Ph(ctx, cr, w.fc3)
    A_gpu = PhScatteringMatrix(v3, bands, T, smearing, sigma, window=win).setup()
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    A_ref = oracle.Interaction3Ph(cr, w.fc3).linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, smearing,
                                                         sigma, window=win)
    for o in (v3, bands, h0):
        o.close()
    return A_gpu, A_ref


@pytest.mark.gpu
@pytest.mark.parametrize("smearing,window", [("adaptive", False), ("adaptive", True), ("gaussian", True)])
def test_fifteen_branches_vs_oracle(ctx, perovskite, smearing, window):
    A_gpu, A_ref = _gpu_vs_oracle(ctx, perovskite, (4, 4, 4), smearing, (300.0, 600.0), window)
    _compare(A_gpu, A_ref, 1e-10)


@pytest.mark.gpu
def test_fifteen_branches_odd_mesh_window(ctx, perovskite):
    A_gpu, A_ref = _gpu_vs_oracle(ctx, perovskite, (3, 3, 3), "adaptive", (300.0,), True)
    _compare(A_gpu, A_ref, 1e-10)


@pytest.mark.gpu
def test_window_on_diamond_vs_oracle(ctx, diamond):
    w = synth.Workload("diamond", diamond["crystal"], diamond["fc2"], diamond["fc3"], (6, 6, 6), (300.0,),
                       "adaptive", 0.0)
    A_gpu, A_ref = _gpu_vs_oracle(ctx, w, (6, 6, 6), "adaptive", (300.0,), True)
    _compare(A_gpu, A_ref, 1e-10)


@pytest.mark.gpu
def test_generic_kernel_equals_fused_kernel(ctx, diamond):
    """nb = 6 with a window that keeps every pair runs the shared-memory kernel;
    it must give the fused register-tiled kernel's result."""
    from phoebe_b200.core import Interaction3Ph, PhononH0, PhScatteringMatrix
    cr = diamond["crystal"]
    T = np.array([C.kelvin_to_ry(100.0), C.kelvin_to_ry(300.0)])
    h0 = PhononH0(ctx, cr, diamond["fc2"])
    bands = h0.populate((6, 6, 6), withVelocities=True)
    v3 = Interaction3Ph(ctx, cr, diamond["fc3"])
    A_fused = PhScatteringMatrix(v3, bands, T, "adaptive").setup()
    everything = (np.zeros(bands.nq), np.zeros(bands.nq))
    A_generic = PhScatteringMatrix(v3, bands, T, "adaptive", window=everything).setup()
    _compare(A_generic, A_fused, 1e-12)


@pytest.mark.gpu
def test_fifteen_band_eigensolve_vs_oracle(ctx):
    """Dynamical-matrix interpolation over the 7x7x7 FC2 grid and the batched
    15x15 Hermitian eigensolve of the 24^3 mesh in one launch (populate);
    a sample of points against the oracle."""
    from phoebe_b200.core import PhononH0
    cr = synth.perovskite_crystal()
    fc2 = synth.perovskite_fc2(cr, (7, 7, 7))
    h0 = PhononH0(ctx, cr, fc2)
    mesh = (24, 24, 24)
    bands = h0.populate(mesh, withVelocities=False)
    E, U, _ = bands.get(velocities=False)
    assert E.shape == (13824, 15)
    idx = np.random.default_rng(4).choice(13824, 64, replace=False)
    q = lattice.Mesh(cr, mesh).cartesian_coords()[idx]
    Eo, Uo = oracle.PhononH0(cr, fc2).diagonalize(q)
    scale = np.abs(Eo).max()
    np.testing.assert_allclose(E[idx], Eo, rtol=0, atol=1e-12 * scale)
    # mass-scaled eigenvectors: U^dag M U = 1, and the oracle's dynamical
    # matrix is reproduced from them (phases of degenerate bands are free)
    m = np.repeat(cr.atomic_masses, 3)
    for k in range(8):
        G = U[idx[k]].conj().T @ (m[:, None] * U[idx[k]])
        np.testing.assert_allclose(G, np.eye(15), atol=1e-10)
        Po = Uo[k] @ np.diag(Eo[k]) @ (m[:, None] * Uo[k]).conj().T
        Pg = U[idx[k]] @ np.diag(E[idx[k]]) @ (m[:, None] * U[idx[k]]).conj().T
        np.testing.assert_allclose(Pg, Po, atol=1e-10 * np.abs(Po).max())
    bands.close()
    h0.close()
