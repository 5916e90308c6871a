"""Scattering-matrix modes of the builder: switchCase 0 (matrix in memory) and
switchCase 1 (matrix-vector product), src/bte/ph_scattering.cpp:382-431,
520-572, 714-759, 846-933; ScatteringMatrix::dot / offDiagonalDot of a stored
matrix, src/bte/scattering.cpp:180-330.

CPU: the oracle's matrix equals an independent numpy restatement built from
the oracle's couplings (Gaussian smearing, 3x3x3 mesh); its diagonal is the
un-averaged linewidth of the linewidth mode; its matrix-vector mode equals
the stored matrix times x (isotope and boundary scattering included, two
temperatures); the stored-matrix dot skips excluded states and the
off-diagonal dot the diagonal; with Gaussian smearing the matrix is
symmetric.  GPU: the stored matrix, its dot products, the matrix-free
product, and q2 slices match the oracle to 1e-10; at the 20x20x20 mesh the
stored matrix (18.4 GB) is symmetric under Gaussian smearing, its diagonal is
the linewidth mode's, and the matrix-free product equals the stored one."""
import numpy as np
import pytest

import oracle
from phoebe_b200 import constants as C
from phoebe_b200 import lattice


def _bands(cr, fc2, mesh):
    h0 = oracle.PhononH0(cr, fc2)
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    E, U = h0.diagonalize(q)
    return E, U, h0.velocities(q), q


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _numpy_matrix(cr, fc3, mesh, E, U, T, sigma):
    """switchCase 0, Gaussian smearing, restated from the couplings: for each
    (q1 b1, q2 b2), + sum_b3 W+ - sum_b3 (W-1 + W-2) off the diagonal, the
    un-averaged linewidth on it, rows and columns of excluded states zero."""
    nq, nb = E.shape
    ns = nq * nb
    n0, n1, n2 = mesh
    idx = np.arange(nq)
    ix, iy, iz = idx % n0, (idx // n0) % n1, idx // (n0 * n1)

    def add(a, b, s):
        return (((iz[a] + s * iz[b]) % n2) * n0 * n1 + ((iy[a] + s * iy[b]) % n1) * n0 + (ix[a] + s * ix[b]) % n0)

    q = lattice.Mesh(cr, mesh).cartesian_coords()
    v3 = oracle.Interaction3Ph(cr, fc3)
    bose = np.where(E > 0, 1.0 / np.expm1(np.maximum(E, 1e-300) / T), 0.0)
    excl = E < C.phExcludeCutoff
    ecut = 0.001 / C.ryToCmm1
    ok = ~excl & (E >= ecut)
    norm = 1.0 / nq

    def gauss(x):
        y = x / sigma
        return np.where(y > 6, 0.0, np.exp(-y * y) / sigma / np.sqrt(np.pi))

    M = np.zeros((ns, ns))
    lw = np.zeros(ns)
    for iq2 in range(nq):
        v3.cache_d3(q[iq2])
        i3p = np.array([add(i, iq2, 1) for i in range(nq)])
        i3m = np.array([add(i, iq2, -1) for i in range(nq)])
        cp, cm = v3.couplings_squared(q, U, U[iq2], U[i3p], U[i3m])
        for iq1 in range(nq):
            Vp = oracle.symmetrize_coupling(cp[iq1], E[iq1], E[iq2], E[i3p[iq1]])
            Vm = oracle.symmetrize_coupling(cm[iq1], E[iq1], E[iq2], E[i3m[iq1]])
            e1, e2 = E[iq1][:, None, None], E[iq2][None, :, None]
            o12 = (ok[iq1][:, None, None] & ok[iq2][None, :, None])
            for V, q3, sgn in ((Vp, i3p[iq1], 1.0), (Vm, i3m[iq1], -1.0)):
                e3 = E[q3][None, None, :]
                o = o12 & ok[q3][None, None, :]
                f1, f2, f3 = bose[iq1][:, None, None], bose[iq2][None, :, None], bose[q3][None, None, :]
                pref = np.pi * 0.25 * V * norm / np.where(o, e1 * e2 * e3, 1.0)
                if sgn > 0:
                    r = pref * f1 * f2 * (f3 + 1) * gauss(e1 + e2 - e3)
                else:
                    r = pref * (f3 * f1 * (f2 + 1) * gauss(e1 + e3 - e2) + f2 * f3 * (f1 + 1) * gauss(e2 + e3 - e1))
                r = np.where(o, r, 0.0).sum(axis=2)
                rows = iq1 * nb + np.arange(nb)
                cols = iq2 * nb + np.arange(nb)
                M[np.ix_(rows, cols)] += sgn * r
                lw[rows] += 0.5 * r.sum(axis=1)
    ex = excl.ravel()
    lw[ex] = 0.0
    M[np.ix_(ex, ex)] = 0.0
    M[np.diag_indices(ns)] = lw
    return M, lw


def test_oracle_matrix_vs_numpy(diamond):
    cr, mesh = diamond["crystal"], (3, 3, 3)
    E, U, vg, q = _bands(cr, diamond["fc2"], mesh)
    T = C.kelvin_to_ry(300.0)
    sigma = 0.3 / C.ryToTHz
    v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    M, lw = v3.scattering_matrix(mesh, E, U, vg, q, cr.reciprocal_cell, T, "gaussian", sigma)
    Mn, lwn = _numpy_matrix(cr, diamond["fc3"], mesh, E, U, T, sigma)
    assert np.abs(Mn - np.diag(np.diag(Mn))).max() > 0
    assert _rel(M, Mn) < 1e-12
    np.testing.assert_allclose(lw, lwn, rtol=1e-12, atol=1e-14 * np.abs(lwn).max())


@pytest.mark.parametrize("smearing", ["gaussian", "adaptive"])
def test_oracle_diagonal_is_unaveraged_linewidth(diamond, smearing):
    cr, mesh = diamond["crystal"], (4, 4, 4)
    E, U, vg, q = _bands(cr, diamond["fc2"], mesh)
    T = C.kelvin_to_ry(300.0)
    sigma = 0.3 / C.ryToTHz
    v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    M, lw = v3.scattering_matrix(mesh, E, U, vg, q, cr.reciprocal_cell, T, smearing, sigma)
    raw = v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, [T], smearing, sigma, finalize=False)[0]
    raw[E.ravel() < C.phExcludeCutoff] = 0.0
    np.testing.assert_allclose(lw, raw, rtol=1e-12, atol=1e-14 * np.abs(raw).max())
    np.testing.assert_array_equal(np.diag(M), lw)
    ex = E.ravel() < C.phExcludeCutoff
    assert ex.any() and np.all(M[ex] == 0.0) and np.all(M[:, ex] == 0.0)


def test_oracle_matrix_free_product_equals_stored(diamond):
    from phoebe_b200.core import isotope_coupling
    cr, mesh = diamond["crystal"], (4, 4, 4)
    E, U, vg, q = _bands(cr, diamond["fc2"], mesh)
    temps = np.array([C.kelvin_to_ry(200.0), C.kelvin_to_ry(500.0)])
    g = isotope_coupling(cr, [2.0e-4, 5.0e-4])
    L = 3.0e5
    v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    ns = E.size
    x = np.random.default_rng(3).normal(size=(2, 2, 3, ns))
    y = v3.scattering_dot(mesh, E, U, vg, q, cr.reciprocal_cell, temps, "adaptive", 0.0, x, isotope_coupling=g,
                          boundary_length=L)
    for c, T in enumerate(temps):
        M, lw = v3.scattering_matrix(mesh, E, U, vg, q, cr.reciprocal_cell, T, "adaptive", 0.0,
                                     isotope_coupling=g, boundary_length=L)
        ref = np.einsum("rs,vis->vir", M, x[:, c])
        assert _rel(y[:, c], ref) < 1e-12
        # the stored-matrix dot equals the plain product (excluded rows and columns are zero)
        np.testing.assert_allclose(oracle.smatrix_dot(M, E, x[:, c]), ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())
        off = oracle.smatrix_dot(M, E, x[:, c], off_diagonal=True)
        np.testing.assert_allclose(off, ref - lw[None, None, :] * x[:, c], rtol=1e-10,
                                   atol=1e-13 * np.abs(ref).max())


def test_oracle_stored_dot_skips_excluded(diamond):
    rng = np.random.default_rng(5)
    ns = 30
    M = rng.normal(size=(ns, ns))
    E = np.abs(rng.normal(size=ns)) * 1e-3
    E[[2, 7]] = 0.0
    x = rng.normal(size=(2, 3, ns))
    keep = E >= C.phExcludeCutoff
    Mk = M * keep[:, None] * keep[None, :]
    np.testing.assert_allclose(oracle.smatrix_dot(M, E, x), np.einsum("rs,vis->vir", Mk, x), rtol=1e-13, atol=1e-13)
    Mo = M - np.diag(np.diag(M))
    np.testing.assert_allclose(oracle.smatrix_dot(M, E, x, off_diagonal=True), np.einsum("rs,vis->vir", Mo, x),
                               rtol=1e-13, atol=1e-13)


def test_oracle_gaussian_matrix_is_symmetric(diamond):
    cr, mesh = diamond["crystal"], (4, 4, 4)
    E, U, vg, q = _bands(cr, diamond["fc2"], mesh)
    v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    M, _ = v3.scattering_matrix(mesh, E, U, vg, q, cr.reciprocal_cell, C.kelvin_to_ry(300.0), "gaussian",
                                0.3 / C.ryToTHz)
    assert np.abs(M - np.diag(np.diag(M))).max() > 0
    assert _rel(M, M.T) < 1e-9


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def _gpu_setup(ctx, diamond, mesh):
    from phoebe_b200.core import Interaction3Ph, PhononH0
    cr = diamond["crystal"]
    h0 = PhononH0(ctx, cr, diamond["fc2"])
    bands = h0.populate(mesh, withVelocities=True)
    v3 = Interaction3Ph(ctx, cr, diamond["fc3"])
    return h0, bands, v3


def _close(*objs):
    for o in objs:
        o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("smearing,mesh", [("gaussian", (4, 4, 4)), ("adaptive", (6, 6, 6))])
def test_gpu_stored_matrix_vs_oracle(ctx, diamond, smearing, mesh):
    from phoebe_b200.core import PhScatteringMatrix, isotope_coupling
    cr = diamond["crystal"]
    h0, bands, v3 = _gpu_setup(ctx, diamond, mesh)
    E, U, vg = bands.get()
    T = C.kelvin_to_ry(300.0)
    sigma = 0.3 / C.ryToTHz
    g = isotope_coupling(cr, [2.0e-4, 5.0e-4])
    sm = PhScatteringMatrix(v3, bands, [T], smearing, sigma, isotope_coupling=g, boundary_length=2.0e5,
                            in_memory=True)
    diag = sm.setup()[0]
    ns = E.size
    A = sm.getMatrixRows(0, ns)
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    M, lw = oracle.Interaction3Ph(cr, diamond["fc3"]).scattering_matrix(
        mesh, E, U, vg, q, cr.reciprocal_cell, T, smearing, sigma, isotope_coupling=g, boundary_length=2.0e5)
    assert _rel(A, M) < 1e-10
    np.testing.assert_allclose(diag, lw, rtol=1e-10, atol=1e-14 * np.abs(lw).max())
    # rows in two pieces equal the whole
    np.testing.assert_array_equal(np.vstack([sm.getMatrixRows(0, 7), sm.getMatrixRows(7, ns - 7)]), A)
    x = np.random.default_rng(8).normal(size=(3, 1, 3, ns))
    for off in (False, True):
        y = sm.offDiagonalDot(x) if off else sm.dot(x)
        ref = oracle.smatrix_dot(M, E, x[:, 0], off_diagonal=off)
        assert _rel(y[:, 0], ref) < 1e-10
    sm.close()
    _close(v3, bands, h0)


@pytest.mark.gpu
def test_gpu_matrix_free_product_vs_oracle(ctx, diamond):
    from phoebe_b200.core import PhScatteringMatrix, isotope_coupling
    cr, mesh = diamond["crystal"], (6, 6, 6)
    h0, bands, v3 = _gpu_setup(ctx, diamond, mesh)
    E, U, vg = bands.get()
    temps = np.array([C.kelvin_to_ry(150.0), C.kelvin_to_ry(450.0)])
    g = isotope_coupling(cr, [2.0e-4, 5.0e-4])
    ns = E.size
    x = np.random.default_rng(9).normal(size=(5, 2, 3, ns))   # 5 vectors: two passes of 4
    sm = PhScatteringMatrix(v3, bands, temps, "adaptive", isotope_coupling=g, boundary_length=4.0e5)
    y = sm.dot(x)
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    ref = oracle.Interaction3Ph(cr, diamond["fc3"]).scattering_dot(
        mesh, E, U, vg, q, cr.reciprocal_cell, temps, "adaptive", 0.0, x, isotope_coupling=g, boundary_length=4.0e5)
    assert _rel(y, ref) < 1e-10
    assert sm.stats.pairs == bands.nq ** 2
    # one vector without the batch axis; the reference's offDiagonalDot without a stored matrix
    np.testing.assert_allclose(sm.dot(x[0]), y[0], rtol=1e-12, atol=1e-13 * np.abs(y).max())
    sm.setup()
    off = sm.offDiagonalDot(x[0])
    np.testing.assert_allclose(off, y[0] - sm.internalDiagonal[:, None, :] * x[0], rtol=1e-12,
                               atol=1e-13 * np.abs(y).max())
    _close(v3, bands, h0)


@pytest.mark.gpu
def test_gpu_matrix_q2_slices_sum_to_whole(ctx, diamond):
    from phoebe_b200.core import PhScatteringMatrix
    mesh = (4, 4, 4)
    h0, bands, v3 = _gpu_setup(ctx, diamond, mesh)
    T = [C.kelvin_to_ry(300.0)]
    ns = bands.nq * bands.nb
    parts = []
    for a, b in ((0, 21), (21, 50), (50, 64)):
        sm = PhScatteringMatrix(v3, bands, T, "adaptive", in_memory=True)
        sm.setup(a, b, finalize=False)
        parts.append(sm.getMatrixRows(0, ns))
        sm.close()
    whole = PhScatteringMatrix(v3, bands, T, "adaptive", in_memory=True)
    whole.setup(finalize=False)
    W = whole.getMatrixRows(0, ns)
    assert _rel(sum(parts), W) < 1e-12
    # the matrix-free product over the same slices
    x = np.random.default_rng(2).normal(size=(1, 3, ns))
    free = PhScatteringMatrix(v3, bands, T, "adaptive")
    ys = sum(free.dot(x, a, b, finalize=False) for a, b in ((0, 21), (21, 50), (50, 64)))
    yw = free.dot(x, finalize=False)
    assert _rel(ys, yw) < 1e-12
    whole.close()
    _close(v3, bands, h0)


@pytest.mark.gpu
def test_gpu_matrix_modes_reject_bad_arguments(ctx, diamond):
    from phoebe_b200.core import PhScatteringMatrix
    from phoebe_b200._abi import PhxError
    h0, bands, v3 = _gpu_setup(ctx, diamond, (4, 4, 4))
    with pytest.raises(ValueError):
        PhScatteringMatrix(v3, bands, [1e-3, 2e-3], "adaptive", in_memory=True).setup()
    nq = bands.nq
    sm = PhScatteringMatrix(v3, bands, [1e-3], "adaptive", window=(np.zeros(nq), np.zeros(nq)), in_memory=True)
    with pytest.raises(PhxError):
        sm.setup()
    _close(v3, bands, h0)


@pytest.mark.gpu
def test_gpu_full_mesh_matrix_properties(ctx, diamond):
    """20x20x20 (48 000 states, an 18.4 GB matrix in device memory)."""
    from phoebe_b200.core import PhScatteringMatrix
    h0, bands, v3 = _gpu_setup(ctx, diamond, (20, 20, 20))
    T = [C.kelvin_to_ry(300.0)]
    sigma = 0.3 / C.ryToTHz
    ns = bands.nq * bands.nb
    sm = PhScatteringMatrix(v3, bands, T, "gaussian", sigma, in_memory=True)
    diag = sm.setup()[0]
    raw = PhScatteringMatrix(v3, bands, T, "gaussian", sigma).setup(finalize=False)[0]
    E = bands.get(velocities=False)[0].ravel()
    raw[E < C.phExcludeCutoff] = 0.0
    np.testing.assert_allclose(diag, raw, rtol=1e-11, atol=1e-14 * np.abs(raw).max())
    # symmetric under Gaussian smearing: compare row blocks with column blocks
    rng = np.random.default_rng(1)
    for r0 in rng.choice(ns - 64, 3, replace=False):
        rows = sm.getMatrixRows(int(r0), 64)                    # A[r0:r0+64, :]
        assert np.abs(rows).max() > 0
        # A[c, r0:r0+64] == A[r0:r0+64, c]
        cidx = rng.choice(ns, 32, replace=False)
        colsT = np.stack([sm.getMatrixRows(int(c), 1)[0, r0:r0 + 64] for c in cidx])
        assert np.abs(colsT - rows[:, cidx].T).max() <= 1e-9 * np.abs(rows).max()
    x = rng.normal(size=(2, 1, 3, ns))
    y_stored = sm.dot(x)
    free = PhScatteringMatrix(v3, bands, T, "gaussian", sigma)
    y_free = free.dot(x)
    assert _rel(y_free, y_stored) < 1e-11
    sm.close()
    _close(v3, bands, h0)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["split_fp16", "split_bf16"])
def test_gpu_split_matrix_modes_vs_fp64(ctx, diamond, precision):
    """The tensor-core path in both matrix modes against the FP64 path: stored
    matrix (8x8x8), its diagonal, and the matrix-free product (two
    temperatures, isotope and boundary scattering); errors relative to the
    largest element at the linewidths' 1e-5 bar (measured: FP16 operands
    9.4e-7, diagonal 1.8e-6, product 6.5e-7; BF16 1.2e-6 and 2.4e-6)."""
    from phoebe_b200.core import PhScatteringMatrix, isotope_coupling
    cr, mesh = diamond["crystal"], (8, 8, 8)
    h0, bands, v3 = _gpu_setup(ctx, diamond, mesh)
    ns = bands.nq * bands.nb
    T = [C.kelvin_to_ry(300.0)]
    ref = PhScatteringMatrix(v3, bands, T, "adaptive", in_memory=True)
    d64 = ref.setup()[0]
    A64 = ref.getMatrixRows(0, ns)
    ref.close()
    v3.setPrecision(precision)
    sm = PhScatteringMatrix(v3, bands, T, "adaptive", in_memory=True)
    d16 = sm.setup()[0]
    A16 = sm.getMatrixRows(0, ns)
    sm.close()
    scale = np.abs(A64).max()
    err = np.abs(A16 - A64).max() / scale
    off = A64 - np.diag(np.diag(A64))
    big = np.abs(off) > 1e-2 * np.abs(off).max()
    rel_big = (np.abs(A16 - A64)[big] / np.abs(A64)[big]).max()
    dbig = np.abs(d64) > 1e-6 * np.abs(d64).max()
    derr = (np.abs(d16 - d64)[dbig] / np.abs(d64)[dbig]).max()
    print("\n%s stored matrix: max |dA|/max|A| %.2e, largest off-diagonal elements %.2e, diagonal %.2e"
          % (precision, err, rel_big, derr))
    # a single element is a sum of a few triplets: relative to itself its error is larger
    # (measured 4.7e-5 with FP16 operands, 1.6e-4 with BF16) than that of the sums
    assert err < 1e-5 and derr < 1e-5 and rel_big < 1e-3
    # matrix-free, two temperatures, isotope and boundary scattering
    g = isotope_coupling(cr, [2.0e-4, 5.0e-4])
    temps = np.array([C.kelvin_to_ry(150.0), C.kelvin_to_ry(450.0)])
    x = np.random.default_rng(12).normal(size=(2, 2, 3, ns))
    y16 = PhScatteringMatrix(v3, bands, temps, "adaptive", isotope_coupling=g, boundary_length=4.0e5).dot(x)
    v3.setPrecision("fp64")
    y64 = PhScatteringMatrix(v3, bands, temps, "adaptive", isotope_coupling=g, boundary_length=4.0e5).dot(x)
    yerr = np.abs(y16 - y64).max() / np.abs(y64).max()
    print("%s matrix-free product: max |dy|/max|y| %.2e" % (precision, yerr))
    assert yerr < 1e-5
    _close(v3, bands, h0)
