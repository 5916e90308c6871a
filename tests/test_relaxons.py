"""Relaxon solver (src/apps/phonon_transport_app.cpp:386-420): a2Omega,
the eigendecomposition of the stored matrix's upper triangle, and the
conductivity of calcFromRelaxons without symmetries.

CPU: the oracle's relaxon conductivity equals the direct solve of A f = b
with A the symmetric matrix of A's upper triangle (for Gaussian smearing, A
itself), to 1e-12; the host solver fed by the same eigenvectors gives the
oracle's conductivity; the JSON file has the reference's keys and units.
GPU (8x8x8 diamond, adaptive smearing, boundary scattering): a2Omega in
device memory equals the oracle's; the eigenvalues equal LAPACK's on the
oracle's Omega; the eigenvectors satisfy S theta = theta lambda, S the
symmetric matrix of Omega's upper triangle; the
relaxon conductivity equals the oracle's, with all eigenvalues (k = 0 and
k = ns) and with the smallest half; a relaxon solve before the eigensolve,
products and a second eigensolve afterwards are refused."""
import json

import numpy as np
import pytest

import oracle
from phoebe_b200 import constants as C
from phoebe_b200 import lattice, output, solvers


def _matrix(diamond, mesh, smearing, T, L, E=None, U=None, vg=None):
    cr = diamond["crystal"]
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    if E is None:
        h0 = oracle.PhononH0(cr, diamond["fc2"])
        E, U = h0.diagonalize(q)
        vg = h0.velocities(q)
    sigma = 0.3 / C.ryToTHz if smearing == "gaussian" else 0.0
    M, lw = oracle.Interaction3Ph(cr, diamond["fc3"]).scattering_matrix(
        mesh, E, U, vg, q, cr.reciprocal_cell, T, smearing, sigma, boundary_length=L)
    return E, vg, M, lw


def _problem(diamond, E, vg, T, mesh):
    return solvers.BteProblem(E, vg, [T], int(np.prod(mesh)), lattice.calc_volume(diamond["crystal"].direct_cell))


def _numpy_solve(lam, theta):
    g = np.where(lam > 0.0, 1.0 / np.where(lam > 0.0, lam, 1.0), 0.0)
    return lambda x: (theta @ (g[:, None] * (theta.T @ x.T))).T


@pytest.mark.parametrize("mesh,smearing,L", [((4, 4, 4), "gaussian", 3.0e3), ((5, 5, 5), "adaptive", 3.0e4)])
def test_relaxons_equal_direct_solve(diamond, mesh, smearing, L):
    T = C.kelvin_to_ry(300.0)
    E, vg, M, lw = _matrix(diamond, mesh, smearing, T, L)
    P = _problem(diamond, E, vg, T, mesh)
    Om, diag = oracle.a2omega(M, lw, E, T)
    np.testing.assert_allclose(np.diagonal(Om), diag, rtol=1e-13)
    vol = lattice.calc_volume(diamond["crystal"].direct_cell)
    lam, theta, kappa = oracle.relaxons(Om, E, vg, T, int(np.prod(mesh)), vol)
    # the excluded states (Gamma acoustic) are the zero eigenvalues; the rest are positive
    assert (lam == 0.0).sum() == (P.excluded).sum() == 3 and lam.min() == 0.0
    # the eigensolver reads the upper triangle: the matrix it diagonalizes is triu(A) + triu(A, 1)^T
    S = np.triu(M) + np.triu(M, 1).T
    k_exact = solvers.exact(P, S)[0]
    np.testing.assert_allclose(kappa, k_exact, rtol=0, atol=1e-12 * np.abs(k_exact).max())
    if smearing == "gaussian":
        np.testing.assert_allclose(kappa, solvers.exact(P, M)[0], rtol=0, atol=1e-12 * np.abs(k_exact).max())
    # the host solver with the same eigenvectors
    k_host = solvers.relaxons(P, _numpy_solve(lam, theta))
    np.testing.assert_allclose(k_host[0], kappa, rtol=0, atol=1e-13 * np.abs(kappa).max())
    # the relaxon conductivity is not the RTA one
    rta = oracle.rta_kappa(E, vg, lw[None, :], [T], int(np.prod(mesh)), vol)[0]
    assert np.abs(np.diagonal(kappa) - np.diagonal(rta)).max() > 1e-3 * np.abs(kappa).max()


def test_relaxons_json(tmp_path):
    lam = np.array([0.0, 2.0e-7, 5.0e-6])
    T = C.kelvin_to_ry(300.0)
    out = output.relaxons_relaxation_times_json(tmp_path / "relaxons_relaxation_times.json", lam, [T])
    d = json.loads((tmp_path / "relaxons_relaxation_times.json").read_text())
    assert d == out
    assert sorted(d) == ["chemicalPotentials", "particleType", "relaxationTimeUnit", "relaxationTimes",
                         "temperatureUnit", "temperatures"]
    assert d["relaxationTimeUnit"] == "fs" and d["particleType"] == "phonon"
    assert d["temperatures"] == pytest.approx([300.0], rel=1e-12)
    t = d["relaxationTimes"][0]
    assert t[0] is None
    assert t[1] == pytest.approx(C.energyRyToFs / 2.0e-7, rel=1e-15)
    assert t[2] == pytest.approx(C.energyRyToFs / 5.0e-6, rel=1e-15)


@pytest.mark.gpu
def test_gpu_relaxons_match_oracle(ctx, diamond):
    from phoebe_b200._abi import PhxError
    from phoebe_b200.core import Interaction3Ph, PhononH0, PhScatteringMatrix
    cr, mesh = diamond["crystal"], (8, 8, 8)
    T = C.kelvin_to_ry(300.0)
    L = 3.0e4
    h0 = PhononH0(ctx, cr, diamond["fc2"])
    bands = h0.populate(mesh, withVelocities=True)
    E, U, vg = bands.get()
    v3 = Interaction3Ph(ctx, cr, diamond["fc3"])
    _, _, M, lw = _matrix(diamond, mesh, "adaptive", T, L, E, U, vg)
    Om, diag = oracle.a2omega(M, lw, E, T)
    P = _problem(diamond, E, vg, T, mesh)
    vol = lattice.calc_volume(cr.direct_cell)
    ns = E.size
    scale = np.abs(Om).max()
    for k in (0, ns // 2, ns):
        A = PhScatteringMatrix(v3, bands, [T], "adaptive", boundary_length=L, in_memory=True)
        A.setup()
        A.a2Omega()
        A.a2Omega()   # a second call does nothing (isMatrixOmega)
        np.testing.assert_allclose(A.internalDiagonal[0], diag, rtol=1e-10, atol=0)
        np.testing.assert_allclose(A.getMatrixRows(0, ns), Om, rtol=0, atol=1e-10 * scale)
        with pytest.raises(PhxError):
            A.dot(P.drift)
        with pytest.raises(PhxError):
            A.diagonalize(ns + 1)
        with pytest.raises(PhxError):
            A.relaxonSolve(P.drift[0])   # before the eigensolve
        lam = A.diagonalize(k)
        lam_ref, theta_ref, k_ref = oracle.relaxons(Om, E, vg, T, int(np.prod(mesh)), vol, num_eigenvalues=k)
        assert lam.size == lam_ref.size == (k or ns)   # k = ns: all of them, as the reference
        np.testing.assert_allclose(lam, lam_ref, rtol=0, atol=1e-9 * np.abs(lam_ref).max())
        theta = A.getMatrixRows(0, ns)[:, :lam.size]
        # eigenpairs of the symmetric matrix of Omega's upper triangle
        res = (np.triu(Om) + np.triu(Om, 1).T) @ theta - theta * lam[None, :]
        assert np.abs(res).max() < 1e-9 * np.abs(lam_ref).max()
        kappa = solvers.relaxons(P, A.relaxonSolve)[0]
        np.testing.assert_allclose(kappa, k_ref, rtol=0, atol=1e-8 * np.abs(k_ref).max())
        if k in (0, ns):
            k_exact = solvers.exact(P, np.triu(M) + np.triu(M, 1).T)[0]
            np.testing.assert_allclose(kappa, k_exact, rtol=0, atol=1e-8 * np.abs(k_exact).max())
        with pytest.raises(PhxError):
            A.diagonalize(k)
        with pytest.raises(PhxError):
            A.symmetrize()
        A.close()
    for o in (v3, bands, h0):
        o.close()


_MG_CHECK = r"""
import numpy as np
import oracle
from phoebe_b200 import constants as C, lattice, solvers, synth
from phoebe_b200.core import Context, Interaction3Ph, PhononH0, PhScatteringMatrix
cr = synth.diamond_crystal()
fc2, fc3 = synth.diamond_fc2(cr), synth.random_fc3(cr, 400, synth.SEED_BASE)
mesh, T, L = (8, 8, 8), C.kelvin_to_ry(300.0), 3.0e4
ctx = Context(0)
h0 = PhononH0(ctx, cr, fc2)
bands = h0.populate(mesh, withVelocities=True)
E, U, vg = bands.get()
v3 = Interaction3Ph(ctx, cr, fc3)
q = lattice.Mesh(cr, mesh).cartesian_coords()
M, lw = oracle.Interaction3Ph(cr, fc3).scattering_matrix(mesh, E, U, vg, q, cr.reciprocal_cell, T, "adaptive",
                                                         0.0, boundary_length=L)
Om, _ = oracle.a2omega(M, lw, E, T)
vol = lattice.calc_volume(cr.direct_cell)
P = solvers.BteProblem(E, vg, [T], int(np.prod(mesh)), vol)
ns = E.size
for k in (0, ns // 2):
    A = PhScatteringMatrix(v3, bands, [T], "adaptive", boundary_length=L, in_memory=True)
    A.setup()
    A.a2Omega()
    lam = A.diagonalize(k)
    lam_ref, _, k_ref = oracle.relaxons(Om, E, vg, T, int(np.prod(mesh)), vol, num_eigenvalues=k)
    assert lam.size == lam_ref.size == (k or ns)
    np.testing.assert_allclose(lam, lam_ref, rtol=0, atol=1e-9 * np.abs(lam_ref).max())
    theta = A.getMatrixRows(0, ns)[:, :lam.size]
    res = (np.triu(Om) + np.triu(Om, 1).T) @ theta - theta * lam[None, :]
    assert np.abs(res).max() < 1e-9 * np.abs(lam_ref).max()
    kappa = solvers.relaxons(P, A.relaxonSolve)[0]
    np.testing.assert_allclose(kappa, k_ref, rtol=0, atol=1e-8 * np.abs(k_ref).max())
    A.close()
print("multi-GPU eigensolver path ok")
"""


@pytest.mark.gpu
def test_gpu_relaxons_through_the_multi_gpu_solver():
    """The eigensolve of matrices that the single-GPU solvers refuse (20^3,
    48 000 states) runs on cuSOLVER's multi-GPU solver over this one device,
    after the upper triangle is mirrored onto the lower one; PHX_EIG_MG=1
    forces that path on the 8x8x8 matrix, checked against the same oracle.
    The library opens that solver when first needed, and it needs the
    toolkit's cuBLAS, so the check runs in a process that has not loaded
    PyTorch (whose wheel brings an older cuBLAS)."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _MG_CHECK], cwd=root, capture_output=True, text=True, timeout=900,
                       env={**os.environ, "PHX_EIG_MG": "1"})
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "multi-GPU eigensolver path ok" in r.stdout
