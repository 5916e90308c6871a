"""GPU harmonic path vs the oracle (mirrors test/kokkosHamiltonians.cpp:356-451
and test/velocityTest.cpp:5-67: energies 1e-12 rel, reconstructed dynamical
matrix 1e-12 of its norm, velocities 1e-5 rel / 1e-7 abs, zero at Gamma)."""
import numpy as np
import pytest

import oracle
from phoebe_b200 import lattice

pytestmark = pytest.mark.gpu


def _cases(diamond, si_golden):
    return [(diamond["crystal"], diamond["fc2"]), (si_golden["crystal"], si_golden["fc2"])]


def _random_q(cr, n, seed):
    rng = np.random.default_rng(seed)
    crys = rng.uniform(-0.5, 1.0, size=(n, 3))
    crys[0] = 0.0
    crys[1] = [0.5, 0.0, 0.0]
    crys[2] = [0.5, 0.5, 0.0]
    return crys @ cr.reciprocal_cell.T


def test_energies_and_eigenvectors(ctx, diamond, si_golden):
    from phoebe_b200.core import PhononH0
    for cr, fc in _cases(diamond, si_golden):
        q = _random_q(cr, 200, 5)
        ref = oracle.PhononH0(cr, fc)
        gpu = PhononH0(ctx, cr, fc)
        E0, U0 = ref.diagonalize(q, mass_scaling=False)
        E1, U1 = gpu.diagonalizeFromCoordinates(q, withMassScaling=False)
        # eigenvalues w2 carry an absolute error ~eps*|D|; omega = sqrt|w2| of the
        # acoustic Gamma modes is noise, so near-zero modes are compared in w2
        w2_0 = np.sign(E0) * E0 ** 2
        w2_1 = np.sign(E1) * E1 ** 2
        np.testing.assert_allclose(w2_1, w2_0, rtol=0, atol=1e-13 * np.abs(w2_0).max())
        big = np.abs(w2_0) > 1e-8 * np.abs(w2_0).max()
        np.testing.assert_allclose(E1[big], E0[big], rtol=1e-12)
        D0 = np.einsum("qab,qb,qcb->qac", U0, w2_0, U0.conj())
        D1 = np.einsum("qab,qb,qcb->qac", U1, w2_1, U1.conj())
        norm = np.abs(D0).max()
        np.testing.assert_allclose(D1, D0, atol=1e-12 * norm)
        I = np.einsum("qab,qac->qbc", U1.conj(), U1)
        np.testing.assert_allclose(I, np.broadcast_to(np.eye(cr.num_bands), I.shape), atol=1e-12)
        # mass scaling divides rows by sqrt(m)
        _, U2 = gpu.diagonalizeFromCoordinates(q[:5])
        m = np.repeat(cr.atomic_masses, 3)
        np.testing.assert_allclose(np.abs(U2), np.abs(U1[:5]) / np.sqrt(m)[None, :, None], rtol=1e-13)


def test_group_velocities(ctx, diamond, si_golden):
    from phoebe_b200.core import PhononH0
    for cr, fc in _cases(diamond, si_golden):
        q = _random_q(cr, 100, 7)
        ref = oracle.PhononH0(cr, fc)
        gpu = PhononH0(ctx, cr, fc)
        v0 = ref.velocities(q)
        E1, U1, v1 = gpu.diagonalizeWithVelocities(q)
        np.testing.assert_allclose(v1, v0, rtol=1e-5, atol=1e-7)
        assert np.all(v1[0] == 0.0)  # Gamma


def test_mesh_band_structure(ctx, diamond):
    from phoebe_b200.core import PhononH0
    cr, fc = diamond["crystal"], diamond["fc2"]
    gpu = PhononH0(ctx, cr, fc)
    bands = gpu.populate((4, 4, 4))
    E, U, vg = bands.get()
    m = lattice.Mesh(cr, (4, 4, 4))
    q = m.cartesian_coords()
    E2, U2, v2 = gpu.diagonalizeWithVelocities(q)
    # same kernel on (up to rounding of the Cartesian mesh points) the same q
    np.testing.assert_allclose(E, E2, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(vg, v2, rtol=1e-6, atol=1e-9)
    ref = oracle.PhononH0(cr, fc)
    E0, _ = ref.diagonalize(q)
    w2, w2_0 = np.sign(E) * E ** 2, np.sign(E0) * E0 ** 2
    np.testing.assert_allclose(w2, w2_0, rtol=0, atol=1e-13 * np.abs(w2_0).max())


def test_errors_are_reported(ctx, diamond):
    from phoebe_b200 import _abi
    from phoebe_b200.core import PhononH0
    gpu = PhononH0(ctx, diamond["crystal"], diamond["fc2"])
    L = _abi.load()
    rc = L.phx_ph_diag(gpu.h, -1, None, 1, None, None)
    assert rc == _abi.PHX_ERR_ARG
    assert "bad arguments" in _abi.last_error(ctx.h)
