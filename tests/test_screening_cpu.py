"""CPU checks of the learned-screening path: the network oracle's gradient
against central finite differences, and the per-triplet contributions of the
screening module against the oracle builder (their sum over q2 is the
unaveraged linewidth)."""
import numpy as np
import pytest

import oracle
from oracle import mlp
from phoebe_b200 import constants as C
from phoebe_b200 import lattice, screening, synth


@pytest.mark.parametrize("rounded", [False, True])
def test_oracle_gradient_matches_finite_differences(rounded):
    dims = mlp.layer_dims(12, 24, 3)
    p = mlp.init_params(12, 24, 3, seed=3).astype(np.float64)
    rng = np.random.default_rng(4)
    X = rng.normal(size=(50, 12))
    t = rng.normal(size=50)
    if rounded:
        # rounded weights: perturb the already-rounded values by exactly representable steps
        p = mlp.bf16(p).astype(np.float64)
    _, g = mlp.loss_and_grad(p, X, t, dims, rounded=False)
    h = 1e-6
    idx = rng.choice(len(p), 40, replace=False)
    fd = []
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd.append((mlp.loss_and_grad(pp, X, t, dims, rounded=False)[0] -
                   mlp.loss_and_grad(pm, X, t, dims, rounded=False)[0]) / (2 * h))
    np.testing.assert_allclose(np.array(fd), g[idx], rtol=1e-6, atol=1e-9 * np.abs(g).max())


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-3], dtype=np.float32)
    r = mlp.bf16(x)
    # exactly representable values are unchanged; halfway values go to even
    assert mlp.bf16(np.float32(1.0 + 2 ** -7)) == np.float32(1.0 + 2 ** -7)
    assert mlp.bf16(np.float32(1.0 + 2 ** -8)) == np.float32(1.0)
    assert mlp.bf16(np.float32(1.0 + 3 * 2 ** -8)) == np.float32(1.0 + 2 ** -6)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)


class _OracleVertex:
    """The oracle vertex behind the GPU mirror's cacheD3 / getCouplingsSquared names."""

    def __init__(self, cr, fc3):
        self.v = oracle.Interaction3Ph(cr, fc3)

    def cacheD3(self, q2):
        self.v.cache_d3(q2)

    def getCouplingsSquared(self, q1s, q2, ev1s, ev2, ev3p, ev3m):
        cp, cm = self.v.couplings_squared(q1s, np.stack(ev1s), ev2, np.stack(ev3p), np.stack(ev3m))
        return list(cp), list(cm)


@pytest.mark.parametrize("smearing", ["adaptive", "gaussian"])
def test_contributions_sum_to_oracle_linewidths(smearing):
    cr = synth.diamond_crystal()
    fc2 = synth.diamond_fc2(cr)
    fc3 = synth.random_fc3(cr, 400, synth.SEED_BASE)
    mesh = (4, 4, 4)
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    h0 = oracle.PhononH0(cr, fc2)
    E, U = h0.diagonalize(q)
    vg = h0.velocities(q)
    T = C.kelvin_to_ry(300.0)
    sigma = 0.3 / C.ryToTHz
    c = screening.triplet_contributions(_OracleVertex(cr, fc3), mesh, q, E, U, vg, cr.reciprocal_cell, T,
                                        list(range(len(q))), smearing, sigma)
    A = oracle.Interaction3Ph(cr, fc3).linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, [T], smearing, sigma,
                                                  finalize=False)[0].reshape(len(q), 6)
    S = c.sum(axis=(0, 3, 4))
    assert A.max() > 0
    np.testing.assert_allclose(S, A, rtol=1e-10, atol=1e-13 * A.max())


def test_pair_level_screening_bound(diamond):
    """Upper bound of any screen at the granularity of (q1, q2) pairs, for
    the 1e-3 linewidth error budget: for every q1, skip its q2 pairs in
    increasing order of their largest relative contribution to the q1 modes
    while the skipped total stays below 1e-3.  Even this perfect screen
    skips about 1% of the pairs (1.2% at 8x8x8, 1.7% at 12x12x12 measured the
    same way), so screening cannot give the builder a large factor on this
    workload."""
    cr, mesh = diamond["crystal"], (6, 6, 6)
    h0 = oracle.PhononH0(cr, diamond["fc2"])
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    E, U = h0.diagonalize(q)
    vg = h0.velocities(q)
    v3 = oracle.Interaction3Ph(cr, diamond["fc3"])
    T = [C.kelvin_to_ry(300.0)]
    nq = len(q)
    contrib = np.stack([v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, "adaptive", 0.0, q2_list=[i],
                                      finalize=False)[0].reshape(nq, 6) for i in range(nq)])   # (q2, q1, b1)
    G = contrib.sum(axis=0)
    np.testing.assert_allclose(G.ravel(), v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, "adaptive", 0.0,
                                                        finalize=False)[0], rtol=1e-12, atol=1e-30)
    ok = (E >= C.phExcludeCutoff) & (G > 0)
    rel = np.where(ok[None], contrib / np.where(G > 0, G, 1.0)[None], 0.0).max(axis=2)    # (q2, q1)
    skippable = np.mean([(np.cumsum(np.sort(rel[:, i])) < 1e-3).sum() / nq for i in range(nq)])
    assert 0.0 < skippable < 0.05
