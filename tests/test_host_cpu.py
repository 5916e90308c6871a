"""CPU-only checks: oracle self-consistency, host logic of the product, ABI exports."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from phoebe_b200 import constants as C
from phoebe_b200 import lattice, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_oracle_eigensolver_matches_lapack():
    """Householder + QL solver of the oracle against LAPACK (numpy.linalg)."""
    rng = np.random.default_rng(0)
    # direct check through a real symmetric dynamical matrix
    for n in (3, 6, 15, 36):
        A = rng.normal(size=(n, n))
        S = A + A.T
        masses = np.ones(n)
        R = np.zeros((1, 3))
        w = np.ones(1)
        M = S.reshape(1, n, n).copy()
        E = np.zeros((1, n))
        U = np.zeros((1, n, n, 2))
        q = np.zeros((1, 3))
        L = oracle.lib()
        p = oracle._p
        rc = L.orc_ph_diag(n, 1, p(R), p(w), p(M), p(masses), 1, p(q), 0, p(E), p(U))
        assert rc == 0
        w2 = np.sign(E[0]) * E[0] ** 2
        np.testing.assert_allclose(w2, np.linalg.eigvalsh(S), rtol=1e-11, atol=1e-11)
        Uc = U[0, ..., 0] + 1j * U[0, ..., 1]
        np.testing.assert_allclose(Uc.conj().T @ Uc, np.eye(n), atol=1e-12)
        np.testing.assert_allclose((Uc * w2) @ Uc.conj().T, S, atol=1e-11)


def test_ws_reorder_product_matches_oracle(diamond, si_golden):
    from phoebe_b200.core import ws_reorder
    for cr, fc in ((diamond["crystal"], diamond["fc2"]), (si_golden["crystal"], si_golden["fc2"])):
        R1, w1, M1 = ws_reorder(cr, fc)
        R2, w2, M2 = oracle.ws_reorder(cr, fc)
        assert R1.shape == R2.shape
        np.testing.assert_array_equal(w1, w2)
        # R may differ in the last bit (FMA contraction in one of the builds)
        np.testing.assert_allclose(R1, R2, rtol=1e-15, atol=1e-14)
        np.testing.assert_array_equal(M1, M2)
        # sum of weights per atom pair equals the coarse-grid size
        assert abs(w1.sum() - np.prod(fc.shape[2:5]) * cr.num_atoms ** 2) < 1e-8


def test_abi_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "phx_abi.h")).read()
    names = sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(phx_\w+)\s*\(", hdr, re.M)))
    assert len(names) >= 20
    lib = ctypes.CDLL(os.path.join(ROOT, "phoebe_b200", "libphx.so"))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    from phoebe_b200 import _abi
    assert set(names) <= set(_abi.SIGNATURES), set(names) - set(_abi.SIGNATURES)


def test_abi_reports_no_device_on_cpu():
    from phoebe_b200 import _abi
    L = _abi.load()
    h = ctypes.c_void_p()
    rc = L.phx_ctx_create(0, ctypes.byref(h))
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        assert rc == _abi.PHX_ERR_NODEV
        assert "device" in _abi.last_error().lower()
    elif rc == 0:
        L.phx_ctx_destroy(h)


def test_mesh_integer_q3_matches_reference_rounding(diamond):
    """q3 = q1 +/- q2 by integer mesh arithmetic equals the reference's
    Cartesian round trip + round() lookup (points.cpp:404-423)."""
    cr = diamond["crystal"]
    rng = np.random.default_rng(1)
    for mesh in ((8, 8, 8), (20, 20, 20), (6, 5, 4)):
        m = lattice.Mesh(cr, mesh)
        n = m.num_points
        i1 = rng.integers(0, n, 4000)
        i2 = rng.integers(0, n, 4000)
        q1, q2 = m.cartesian_coords(i1), m.cartesian_coords(i2)
        for sgn in (+1, -1):
            ref = m.index_of(m.cartesian_to_crystal(q1 + sgn * q2))
            a = np.stack([i1 % mesh[0], (i1 // mesh[0]) % mesh[1], i1 // (mesh[0] * mesh[1])], 1)
            b = np.stack([i2 % mesh[0], (i2 // mesh[0]) % mesh[1], i2 // (mesh[0] * mesh[1])], 1)
            c = np.mod(a + sgn * b, mesh)
            mine = c[:, 2] * mesh[0] * mesh[1] + c[:, 1] * mesh[0] + c[:, 0]
            np.testing.assert_array_equal(ref, mine)


def test_synthetic_fc3_symmetric_and_asr(diamond):
    fc3 = diamond["fc3"]
    assert fc3.num_pairs == 400
    assert fc3.residual < 1e-12
    D3 = fc3.D3
    nat = 2
    # ASR: sum over R3 and atom c of Phi(0a, R2 b, R3 c) vanishes
    s = D3.reshape(6, 6, nat, 3, D3.shape[3], D3.shape[4]).sum(axis=(2, 4))
    assert np.abs(s).max() < 1e-11 * np.abs(D3).max()
    assert D3.shape[3] == D3.shape[4]  # nr2 == nr3 by permutation closure


def test_synthetic_fc2_sum_rule(diamond):
    fc = diamond["fc2"]
    s = fc.sum(axis=(2, 3, 4, 6))
    assert np.abs(s).max() < 1e-12


def test_counter_rng_reproducible():
    a = synth.CounterRNG(123).normal(5, 1000)
    b = synth.CounterRNG(123).normal(5, 1000)
    np.testing.assert_array_equal(a, b)
    assert abs(a.mean()) < 0.15 and abs(a.std() - 1) < 0.1


def test_time_reversal_identity_of_the_vertex(diamond):
    """Design check behind the fused builder: symmetrised |V-(q1,-q2)|^2 equals
    symmetrised |V+(q1,q2)|^2 (same q3), computed by the oracle."""
    cr = diamond["crystal"]
    h0 = oracle.PhononH0(cr, diamond["fc2"])
    v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    m = lattice.Mesh(cr, (6, 6, 6))
    n = m.num_points
    rng = np.random.default_rng(3)
    for _ in range(4):
        i1, i2 = rng.integers(0, n, 2)
        i2m = m.index_of(-m.crystal_coords(i2))[0]
        i3 = m.index_of(m.cartesian_to_crystal(m.cartesian_coords(i1) + m.cartesian_coords(i2)))[0]
        q = m.cartesian_coords([i1, i2, i2m, i3])
        E, U = h0.diagonalize(q)
        v3.cache_d3(q[1])
        P, _ = v3.couplings_squared(q[0][None], U[0][None], U[1], U[3][None], U[3][None])
        v3.cache_d3(q[2])
        _, Mm = v3.couplings_squared(q[0][None], U[0][None], U[2], U[3][None], U[3][None])
        Ps = oracle.symmetrize_coupling(P[0], E[0], E[1], E[3])
        Ms = oracle.symmetrize_coupling(Mm[0], E[0], E[2], E[3])
        np.testing.assert_allclose(Ms, Ps, rtol=1e-9, atol=1e-12 * np.abs(Ps).max())
