"""GPU Interaction3Ph (cacheD3 + getCouplingsSquared through the C ABI).

Mirrors test/interaction3phTest.cpp: Coupling3Ph000 and Coupling3Ph210 on
the reference's own fixtures, then element-wise parity with the oracle on
random pairs of the synthetic diamond workload (same eigenvectors on both
sides, so |V|^2 is compared without symmetrisation)."""
import numpy as np
import pytest

import oracle
from phoebe_b200 import lattice

pytestmark = pytest.mark.gpu


def test_coupling_000_gpu(ctx, si_golden):
    from phoebe_b200.core import Interaction3Ph, PhononH0
    cr, z = si_golden["crystal"], si_golden["z"]
    h0 = PhononH0(ctx, cr, si_golden["fc2"])
    v3 = Interaction3Ph(ctx, cr, si_golden["fc3"])
    q = np.zeros(3)
    E, U = h0.diagonalizeFromCoordinates(q)
    v3.cacheD3(q)
    cp, cm = v3.getCouplingsSquared(q[None], q, [U[0]], U[0], [U[0]], [U[0]])
    assert np.array_equal(cp[0], cm[0])
    x1 = z["golden000_plus"][3:, 3:, 3:].sum()
    x2 = cp[0][3:, 3:, 3:].sum()
    assert abs((x1 - x2) / x1) < 1e-7


def test_coupling_210_gpu(ctx, si_golden):
    from phoebe_b200.core import Interaction3Ph, PhononH0
    cr, z = si_golden["crystal"], si_golden["z"]
    h0 = PhononH0(ctx, cr, si_golden["fc2"])
    v3 = Interaction3Ph(ctx, cr, si_golden["fc3"])
    mesh = lattice.Mesh(cr, z["mesh210"])
    qs = mesh.cartesian_coords(z["iq210"])
    E, U = h0.diagonalizeFromCoordinates(qs)
    v3.cacheD3(qs[1])
    cp, cm = v3.getCouplingsSquared(qs[0][None], qs[1], [U[0]], U[1], [U[2]], [U[2]])
    Ps = oracle.symmetrize_coupling(cp[0], E[0], E[1], E[2])
    Ms = oracle.symmetrize_coupling(cm[0], E[0], E[1], E[2])
    for mine, gold in ((Ps, z["golden210_plus"]), (Ms, z["golden210_mins"])):
        x1, x3 = mine[:2].sum(), gold[:2].sum()
        assert abs((x1 - x3) / x1) < 1e-7


def test_couplings_match_oracle(ctx, diamond):
    from phoebe_b200.core import Interaction3Ph
    cr = diamond["crystal"]
    ref_h0 = oracle.PhononH0(cr, diamond["fc2"])
    ref_v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    v3 = Interaction3Ph(ctx, cr, diamond["fc3"])
    m = lattice.Mesh(cr, (10, 10, 10))
    rng = np.random.default_rng(11)
    n = m.num_points
    for _ in range(3):
        iq2 = int(rng.integers(n))
        iq1 = rng.integers(0, n, 17)
        q1 = m.cartesian_coords(iq1)
        q2 = m.cartesian_coords(iq2)
        E1, U1 = ref_h0.diagonalize(q1)
        _, U2 = ref_h0.diagonalize(q2)
        _, U3p = ref_h0.diagonalize(q1 + q2)
        _, U3m = ref_h0.diagonalize(q1 - q2)
        ref_v3.cache_d3(q2)
        P0, M0 = ref_v3.couplings_squared(q1, U1, U2[0], U3p, U3m)
        v3.cacheD3(q2)
        cp, cm = v3.getCouplingsSquared(q1, q2, list(U1), U2[0], list(U3p), list(U3m))
        P1, M1 = np.stack(cp), np.stack(cm)
        scale = max(np.abs(P0).max(), np.abs(M0).max())
        np.testing.assert_allclose(P1, P0, rtol=1e-11, atol=1e-13 * scale)
        np.testing.assert_allclose(M1, M0, rtol=1e-11, atol=1e-13 * scale)


def test_ragged_band_counts(ctx, diamond):
    """Windows give fewer bands per point; outputs are ragged (nb1, nb2, nb3)."""
    from phoebe_b200.core import Interaction3Ph
    cr = diamond["crystal"]
    ref_h0 = oracle.PhononH0(cr, diamond["fc2"])
    ref_v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    v3 = Interaction3Ph(ctx, cr, diamond["fc3"])
    m = lattice.Mesh(cr, (8, 8, 8))
    q1 = m.cartesian_coords([3, 77, 200])
    q2 = m.cartesian_coords(45)
    E1, U1 = ref_h0.diagonalize(q1)
    _, U2 = ref_h0.diagonalize(q2)
    _, U3p = ref_h0.diagonalize(q1 + q2)
    _, U3m = ref_h0.diagonalize(q1 - q2)
    ref_v3.cache_d3(q2)
    P0, M0 = ref_v3.couplings_squared(q1, U1, U2[0], U3p, U3m)
    nb1 = [6, 4, 2]
    nb3p = [5, 6, 3]
    nb3m = [2, 6, 6]
    nb2 = 4
    v3.cacheD3(q2)
    cp, cm = v3.getCouplingsSquared(q1, q2, [U1[i][:, :nb1[i]] for i in range(3)], U2[0][:, :nb2],
                                    [U3p[i][:, :nb3p[i]] for i in range(3)],
                                    [U3m[i][:, :nb3m[i]] for i in range(3)])
    for i in range(3):
        np.testing.assert_allclose(cp[i], P0[i][:nb1[i], :nb2, :nb3p[i]], rtol=1e-11, atol=1e-25)
        np.testing.assert_allclose(cm[i], M0[i][:nb1[i], :nb2, :nb3m[i]], rtol=1e-11, atol=1e-25)


def test_couplings_before_cache_is_an_error(ctx, diamond):
    from phoebe_b200 import _abi
    from phoebe_b200.core import Interaction3Ph
    v3 = Interaction3Ph(ctx, diamond["crystal"], diamond["fc3"])
    U = np.eye(6, dtype=complex)
    with pytest.raises(_abi.PhxError) as ei:
        v3.getCouplingsSquared(np.zeros((1, 3)), np.zeros(3), [U], U, [U], [U])
    assert ei.value.status == _abi.PHX_ERR_STATE


# Split precisions of the drop-in call: the R3 transform of the q1 batch as one
# tensor-core GEMM with hi/lo operands and FP32 accumulation, the eigenvector
# contractions in FP64.  Stated bounds, relative to the largest |V|^2 of the
# batch: FP16 hi/lo (11 + 11 bits) 2e-6, BF16 hi/lo (8 + 8 bits) 2e-5; the
# large couplings (above 1e-2 of the largest) also element-wise within 1e-4
# (FP16) and 1e-3 (BF16) relative.
SPLIT_BOUNDS = {"split_fp16": (2e-6, 1e-4), "split_bf16": (2e-5, 1e-3)}


@pytest.mark.parametrize("precision", ["split_fp16", "split_bf16"])
def test_split_couplings_match_oracle(ctx, diamond, precision):
    from phoebe_b200.core import Interaction3Ph
    cr = diamond["crystal"]
    ref_h0 = oracle.PhononH0(cr, diamond["fc2"])
    ref_v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    v3 = Interaction3Ph(ctx, cr, diamond["fc3"], precision=precision)
    m = lattice.Mesh(cr, (10, 10, 10))
    rng = np.random.default_rng(11)
    n = m.num_points
    glob, elem = SPLIT_BOUNDS[precision]
    for _ in range(3):
        iq2 = int(rng.integers(n))
        iq1 = rng.integers(0, n, 130)              # more than one 128-row GEMM tile
        q1 = m.cartesian_coords(iq1)
        q2 = m.cartesian_coords(iq2)
        _, U1 = ref_h0.diagonalize(q1)
        _, U2 = ref_h0.diagonalize(q2)
        _, U3p = ref_h0.diagonalize(q1 + q2)
        _, U3m = ref_h0.diagonalize(q1 - q2)
        ref_v3.cache_d3(q2)
        P0, M0 = ref_v3.couplings_squared(q1, U1, U2[0], U3p, U3m)
        v3.cacheD3(q2)
        cp, cm = v3.getCouplingsSquared(q1, q2, list(U1), U2[0], list(U3p), list(U3m))
        P1, M1 = np.stack(cp), np.stack(cm)
        scale = max(np.abs(P0).max(), np.abs(M0).max())
        for a, b in ((P1, P0), (M1, M0)):
            assert np.abs(a - b).max() < glob * scale, (precision, np.abs(a - b).max() / scale)
            big = np.abs(b) > 1e-2 * scale
            assert (np.abs(a - b)[big] / np.abs(b)[big]).max() < elem


@pytest.mark.parametrize("precision", ["split_fp16", "split_bf16"])
def test_split_couplings_reference_goldens(ctx, si_golden, precision):
    """Coupling3Ph210 of the reference's own test (rel 1e-3 there) on the split path."""
    from phoebe_b200.core import Interaction3Ph, PhononH0
    cr, z = si_golden["crystal"], si_golden["z"]
    h0 = PhononH0(ctx, cr, si_golden["fc2"])
    v3 = Interaction3Ph(ctx, cr, si_golden["fc3"], precision=precision)
    mesh = lattice.Mesh(cr, z["mesh210"])
    qs = mesh.cartesian_coords(z["iq210"])
    E, U = h0.diagonalizeFromCoordinates(qs)
    v3.cacheD3(qs[1])
    cp, cm = v3.getCouplingsSquared(qs[0][None], qs[1], [U[0]], U[1], [U[2]], [U[2]])
    Ps = oracle.symmetrize_coupling(cp[0], E[0], E[1], E[2])
    Ms = oracle.symmetrize_coupling(cm[0], E[0], E[1], E[2])
    for mine, gold in ((Ps, z["golden210_plus"]), (Ms, z["golden210_mins"])):
        x1, x3 = mine[:2].sum(), gold[:2].sum()
        assert abs((x1 - x3) / x1) < 1e-5
