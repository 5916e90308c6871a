"""GPU linewidth builder (PhScatteringMatrix::builder, linewidth mode) vs the
oracle's restatement of the reference builder.

Parity is checked on identical band structures (the GPU's energies,
eigenvectors and velocities fed to both), where the FP64 path must agree to
1e-10 relative; end to end (each side computes its own band structure) the
agreement is limited by the 1e-8 finite-difference velocities of adaptive
smearing and is checked at 1e-6 (Gaussian) / 1e-4 (adaptive)."""
import numpy as np
import pytest

import oracle
from phoebe_b200 import constants as C
from phoebe_b200 import lattice

pytestmark = pytest.mark.gpu


def _compare(A_gpu, A_ref, rtol):
    scale = np.abs(A_ref).max()
    big = np.abs(A_ref) > 1e-6 * scale
    rel = np.abs(A_gpu - A_ref)[big] / np.abs(A_ref)[big]
    assert rel.max() < rtol, rel.max()
    assert np.abs(A_gpu - A_ref)[~big].max(initial=0.0) < rtol * 1e-6 * scale


def _run(ctx, diamond, mesh, smearing, temps_k, same_bands=True):
    from phoebe_b200.core import Interaction3Ph, PhononH0, PhScatteringMatrix
    cr = diamond["crystal"]
    T = np.array([C.kelvin_to_ry(t) for t in temps_k])
    sigma = 0.3 / C.ryToTHz
    h0 = PhononH0(ctx, cr, diamond["fc2"])
    bands = h0.populate(mesh, withVelocities=True)
    v3 = Interaction3Ph(ctx, cr, diamond["fc3"])
    sm = PhScatteringMatrix(v3, bands, T, smearing, sigma)
    A_gpu = sm.setup()
    E, U, vg = bands.get()
    m = lattice.Mesh(cr, mesh)
    if not same_bands:
        ref_h0 = oracle.PhononH0(cr, diamond["fc2"])
        q = m.cartesian_coords()
        E, U = ref_h0.diagonalize(q)
        vg = ref_h0.velocities(q)
    ref_v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    A_ref = ref_v3.linewidths(mesh, E, U, vg, m.cartesian_coords(), cr.reciprocal_cell, T,
                              smearing, sigma)
    return A_gpu, A_ref, sm, E, vg, T


def test_gaussian_8x8x8_same_bands(ctx, diamond):
    A_gpu, A_ref, sm, E, vg, T = _run(ctx, diamond, (8, 8, 8), "gaussian", (300.0,))
    assert np.abs(A_ref).max() > 0
    _compare(A_gpu, A_ref, 1e-10)
    # thermal conductivity from the same A_out
    k_gpu = sm.thermalConductivity(diamond["crystal"].volume) / C.thConductivityAuToSi
    k_ref = oracle.rta_kappa(E, vg, A_ref, T, 512, diamond["crystal"].volume)
    np.testing.assert_allclose(k_gpu, k_ref, rtol=1e-9, atol=1e-12 * np.abs(k_ref).max())


def test_adaptive_6x6x6_three_temperatures(ctx, diamond):
    A_gpu, A_ref, *_ = _run(ctx, diamond, (6, 6, 6), "adaptive", (100.0, 300.0, 600.0))
    _compare(A_gpu, A_ref, 1e-10)


def test_odd_mesh_adaptive(ctx, diamond):
    A_gpu, A_ref, *_ = _run(ctx, diamond, (5, 5, 5), "adaptive", (300.0,))
    _compare(A_gpu, A_ref, 1e-10)


def test_end_to_end_independent_band_structures(ctx, diamond):
    A_gpu, A_ref, *_ = _run(ctx, diamond, (6, 6, 6), "gaussian", (300.0,), same_bands=False)
    _compare(A_gpu, A_ref, 1e-6)


def test_excluded_gamma_modes_are_zero(ctx, diamond):
    A_gpu, A_ref, sm, E, vg, T = _run(ctx, diamond, (4, 4, 4), "gaussian", (300.0,))
    assert np.all(A_gpu[:, :3] == 0.0)   # acoustic modes at Gamma (iq = 0)
    assert np.all(A_gpu[:, 3:6] > 0.0)
