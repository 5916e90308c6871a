"""The oracle against the reference's ShengBTE golden couplings.

Mirrors test/interaction3phTest.cpp: Coupling3Ph000 (:9-127) and
Coupling3Ph210 (:129-350), with the same invariants and tolerances (and a
tighter check, since the oracle reproduces the goldens to their 8 digits).
"""
import numpy as np

import oracle
from phoebe_b200 import lattice


def test_coupling_000(si_golden):
    cr, z = si_golden["crystal"], si_golden["z"]
    h0 = oracle.PhononH0(cr, si_golden["fc2"])
    v3 = oracle.Interaction3Ph(cr, si_golden["fc3"])
    q = np.zeros(3)
    E, U = h0.diagonalize(q)
    v3.cache_d3(q)
    P, M = v3.couplings_squared(q[None], U, U[0], U, U)
    assert np.array_equal(P, M)  # ASSERT_EQ(couplingPlus, couplingMins) at Gamma
    x1 = z["golden000_plus"][3:, 3:, 3:].sum()
    x2 = P[0][3:, 3:, 3:].sum()
    rel = abs((x1 - x2) / x1)
    assert rel < 1e-4          # reference tolerance
    assert rel < 1e-7          # the goldens carry 8 significant digits


def test_coupling_210(si_golden):
    cr, z = si_golden["crystal"], si_golden["z"]
    h0 = oracle.PhononH0(cr, si_golden["fc2"])
    v3 = oracle.Interaction3Ph(cr, si_golden["fc3"])
    mesh = lattice.Mesh(cr, z["mesh210"])
    qs = mesh.cartesian_coords(z["iq210"])
    # q3 = q1 + q2 and q1 - q2 fall on iq = 200 (interaction3phTest.cpp:299-309)
    assert mesh.index_of(mesh.cartesian_to_crystal(qs[0] + qs[1]))[0] == 200
    assert mesh.index_of(mesh.cartesian_to_crystal(qs[0] - qs[1]))[0] == 200
    E, U = h0.diagonalize(qs)
    v3.cache_d3(qs[1])
    P, M = v3.couplings_squared(qs[0][None], U[0][None], U[1], U[2][None], U[2][None])
    Ps = oracle.symmetrize_coupling(P[0], E[0], E[1], E[2])
    Ms = oracle.symmetrize_coupling(M[0], E[0], E[1], E[2])
    gp, gm = z["golden210_plus"], z["golden210_mins"]
    for mine, gold in ((Ps, gp), (Ms, gp), (Ms, gm)):
        x1, x3 = mine[:2].sum(), gold[:2].sum()
        assert abs((x1 - x3) / x1) < 1e-3   # reference tolerance
        assert abs((x1 - x3) / x1) < 1e-7


def test_nr2_equals_nr3(si_golden):
    D3 = si_golden["fc3"].D3
    assert D3.shape[3] == D3.shape[4]
