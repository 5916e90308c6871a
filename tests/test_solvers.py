"""Exact BTE solvers (Omini-Sparavigna iterations and conjugate gradients,
src/apps/phonon_transport_app.cpp:197-383) on the scattering matrix.

The synthetic diamond's matrix has near-zero modes (energy conservation
under a finite smearing), for which the Omini-Sparavigna iterations diverge
on these coarse meshes, as the reference's would (its "max BTE iterations"
error).  The tests add boundary scattering (grains of 3e3 to 3e4 Bohr), which
makes the iterations converge; conjugate gradients need a symmetric matrix,
i.e. Gaussian smearing, or the reference's symmetrisation (A + A^T) / 2.

CPU: with the oracle's stored matrix (diamond 4x4x4 and 5x5x5), the solvers
converge to the conductivity of the direct solve of A f = b; their first
iterate is the RTA conductivity of the oracle; the reference's convergence
measure (the smallest relative change of the tensor) is reproduced.  GPU: the
solvers fed by the stored matrix in device memory give, iteration by
iteration, the conductivities of the same solvers fed by the oracle's
products (8x8x8); the symmetrised stored matrix equals the oracle's
symmetrised, and the matrix-free product equals the stored one."""
import numpy as np
import pytest

import oracle
from phoebe_b200 import constants as C
from phoebe_b200 import lattice, solvers


def _oracle_matrix(diamond, mesh, smearing, T, L):
    cr = diamond["crystal"]
    h0 = oracle.PhononH0(cr, diamond["fc2"])
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    E, U = h0.diagonalize(q)
    vg = h0.velocities(q)
    M, lw = oracle.Interaction3Ph(cr, diamond["fc3"]).scattering_matrix(
        mesh, E, U, vg, q, cr.reciprocal_cell, T, smearing, 0.3 / C.ryToTHz, boundary_length=L)
    return E, vg, M, lw


def _problem(diamond, E, vg, T, mesh):
    cr = diamond["crystal"]
    return solvers.BteProblem(E, vg, [T], int(np.prod(mesh)), lattice.calc_volume(cr.direct_cell))


@pytest.mark.parametrize("mesh,smearing,L", [((4, 4, 4), "gaussian", 3.0e3), ((5, 5, 5), "adaptive", 3.0e4)])
def test_solvers_reach_direct_solution(diamond, mesh, smearing, L):
    T = C.kelvin_to_ry(300.0)
    E, vg, M, lw = _oracle_matrix(diamond, mesh, smearing, T, L)
    P = _problem(diamond, E, vg, T, mesh)
    diag = lw[None, :]

    def dot(x):
        return oracle.smatrix_dot(M, E, x)

    def offdot(x):
        return oracle.smatrix_dot(M, E, x, off_diagonal=True)

    k_exact = solvers.exact(P, M)
    d = np.diagonal(k_exact, axis1=1, axis2=2)
    assert d.min() > 0
    k_it, h_it = solvers.iterative(P, diag, offdot, threshold=1e-12, max_iter=300)
    np.testing.assert_allclose(np.diagonal(k_it, axis1=1, axis2=2), d, rtol=1e-9)
    if smearing == "gaussian":
        k_cg, _ = solvers.variational(P, diag, dot, threshold=1e-12, max_iter=400)
        np.testing.assert_allclose(np.diagonal(k_cg, axis1=1, axis2=2), d, rtol=1e-9)
    else:
        # the reference's remedy for a non-symmetric matrix before conjugate gradients
        S = 0.5 * (M + M.T)
        k_cg, _ = solvers.variational(P, diag, lambda x: oracle.smatrix_dot(S, E, x), threshold=1e-12,
                                      max_iter=400)
        np.testing.assert_allclose(np.diagonal(k_cg, axis1=1, axis2=2),
                                   np.diagonal(solvers.exact(P, S), axis1=1, axis2=2), rtol=1e-9)
    # the RTA conductivity the solvers start from, as phx_ph_rta_kappa's oracle computes it
    rta = oracle.rta_kappa(E, vg, diag, [T], int(np.prod(mesh)), lattice.calc_volume(diamond["crystal"].direct_cell))
    np.testing.assert_allclose(h_it[0], rta, rtol=1e-12, atol=1e-15 * np.abs(rta).max())
    # the full solution differs from the RTA (the matrix is not diagonal)
    assert np.abs(d - np.diagonal(rta, axis1=1, axis2=2)).max() > 1e-4 * d.max()


def test_reference_convergence_measure():
    old = np.array([[[1.0, 0.0, 0.0], [0.0, 2.0, 0.0], [0.0, 0.0, 4.0]]])
    new = np.array([[[1.1, 0.0, 0.0], [0.0, 2.0 + 1e-3, 0.0], [0.0, 0.0, 4.4]]])
    assert solvers.relative_change(new, old) == pytest.approx(5e-4)
    with pytest.raises(solvers.BteNotConverged):
        P = solvers.BteProblem(np.array([1e-3, 2e-3]), np.ones((2, 3)), [1e-3], 1, 1.0)

        def grow(x):
            return 10.0 * x
        solvers.iterative(P, np.ones((1, 2)), grow, threshold=1e-12, max_iter=5)


@pytest.mark.gpu
def test_gpu_solvers_match_oracle_fed_solvers(ctx, diamond):
    from phoebe_b200.core import Interaction3Ph, PhononH0, PhScatteringMatrix
    cr, mesh = diamond["crystal"], (8, 8, 8)
    T = C.kelvin_to_ry(300.0)
    h0 = PhononH0(ctx, cr, diamond["fc2"])
    bands = h0.populate(mesh, withVelocities=True)
    E, U, vg = bands.get()
    v3 = Interaction3Ph(ctx, cr, diamond["fc3"])
    L = 3.0e4
    stored = PhScatteringMatrix(v3, bands, [T], "adaptive", boundary_length=L, in_memory=True)
    diag = stored.setup()
    free = PhScatteringMatrix(v3, bands, [T], "adaptive", boundary_length=L)
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    M, lw = oracle.Interaction3Ph(cr, diamond["fc3"]).scattering_matrix(mesh, E, U, vg, q, cr.reciprocal_cell, T,
                                                                        "adaptive", 0.0, boundary_length=L)
    P = _problem(diamond, E, vg, T, mesh)
    kw = dict(threshold=1e-10, max_iter=100)
    k_gpu, h_gpu = solvers.iterative(P, diag, stored.offDiagonalDot, **kw)
    k_ref, h_ref = solvers.iterative(P, lw[None, :], lambda x: oracle.smatrix_dot(M, E, x, off_diagonal=True), **kw)
    assert len(h_gpu) == len(h_ref) > 5
    for a, b in zip(h_gpu, h_ref):
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-12 * np.abs(b).max())
    # the matrix-free product (one builder pass) on the solvers' right-hand side
    x = P.drift
    np.testing.assert_allclose(free.dot(x), stored.dot(x), rtol=1e-10, atol=1e-13 * np.abs(stored.dot(x)).max())
    # symmetrised in device memory, then conjugate gradients
    stored.symmetrize()
    S = 0.5 * (M + M.T)
    ns = E.size
    np.testing.assert_allclose(stored.getMatrixRows(0, ns), S, rtol=0, atol=1e-10 * np.abs(S).max())
    # the first 12 conjugate-gradient steps, step by step (the solve needs ~210);
    # the steps amplify the last-bit differences of the products' summation
    # order (FP64 atomics), from ~1e-15 to ~1e-9 of the tensor by step 25
    hist = []
    for dot in (stored.dot, lambda x: oracle.smatrix_dot(S, E, x)):
        with pytest.raises(solvers.BteNotConverged) as e:
            solvers.variational(P, diag if dot is stored.dot else lw[None, :], dot, threshold=0.0, max_iter=12)
        hist.append(e.value.history)
    for a, b in zip(*hist):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-9 * np.abs(b).max())
    stored.close()
    for o in (v3, bands, h0):
        o.close()
