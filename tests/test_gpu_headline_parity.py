"""Parity on the benchmark's own workload: the 20x20x20 diamond mesh (8000
points), 400 FC3 pairs, adaptive smearing, 100/300/600 K.

* The plain FP64 builder against the oracle on q2 slices of the full mesh
  (every q1), at the FP64 bar of 1e-10 relative.  The builder evaluates the
  "+" vertex of (q1, q2) once and uses it for the "+" process of (q1, q2) and
  the "-" process of (q1, -q2); the oracle, like the reference, takes both
  processes of each q2.  The slices are therefore mesh rows (x varies, y and
  z fixed) whose union is closed under q -> -q: the row through Gamma, and a
  generic row with its mirror image.
* The split path against the FP64 path over the whole mesh: linewidths within
  1e-5 relative and the RTA conductivity within 1e-4
  (bar 1e-3)."""
import numpy as np
import pytest

import oracle
from phoebe_b200 import constants as C
from phoebe_b200 import lattice

pytestmark = pytest.mark.gpu

MESH = (20, 20, 20)
TEMPS = (100.0, 300.0, 600.0)


@pytest.fixture(scope="module")
def headline(ctx, diamond):
    from phoebe_b200.core import PhononH0
    h0 = PhononH0(ctx, diamond["crystal"], diamond["fc2"])
    bands = h0.populate(MESH, withVelocities=True)
    T = np.array([C.kelvin_to_ry(t) for t in TEMPS])
    yield bands, T
    bands.close()
    h0.close()


def _row(y, z):
    n0, n1 = MESH[0], MESH[1]
    b = n0 * (y + n1 * z)
    return b, b + n0


def test_fp64_q2_slices_match_oracle_at_20(ctx, diamond, headline):
    from phoebe_b200.core import Interaction3Ph, PhScatteringMatrix
    bands, T = headline
    cr = diamond["crystal"]
    v3 = Interaction3Ph(ctx, cr, diamond["fc3"], precision="fp64")
    sm = PhScatteringMatrix(v3, bands, T, "adaptive")
    rows = [_row(0, 0), _row(3, 7), _row(MESH[1] - 3, MESH[2] - 7)]
    A_gpu = sum(sm.setup(b, e, finalize=False) for b, e in rows)
    q2_list = np.concatenate([np.arange(b, e) for b, e in rows])
    # the union is closed under negation
    m = lattice.Mesh(cr, MESH)
    neg = set()
    for iq in q2_list:
        ix, iy, iz = iq % 20, (iq // 20) % 20, iq // 400
        neg.add((-ix % 20) + 20 * ((-iy % 20) + 20 * (-iz % 20)))
    assert neg == set(q2_list.tolist())
    E, U, vg = bands.get()
    A_ref = oracle.Interaction3Ph(cr, diamond["fc3"]).linewidths(
        MESH, E, U, vg, m.cartesian_coords(), cr.reciprocal_cell, T, "adaptive", 0.0,
        q2_list=q2_list, finalize=False)
    scale = np.abs(A_ref).max()
    assert scale > 0
    big = np.abs(A_ref) > 1e-6 * scale
    rel = np.abs(A_gpu - A_ref)[big] / np.abs(A_ref)[big]
    assert rel.max() < 1e-10, rel.max()
    assert np.abs(A_gpu - A_ref)[~big].max(initial=0.0) < 1e-16 * scale
    v3.close()


def test_split_matches_fp64_on_the_whole_20_mesh(ctx, diamond, headline):
    from phoebe_b200.core import Interaction3Ph, PhScatteringMatrix
    bands, T = headline
    cr = diamond["crystal"]
    out = {}
    for prec in ("fp64", "split_fp16"):
        v3 = Interaction3Ph(ctx, cr, diamond["fc3"], precision=prec)
        sm = PhScatteringMatrix(v3, bands, T, "adaptive")
        A = sm.setup()
        out[prec] = (A, sm.thermalConductivity(cr.volume), sm.stats)
        v3.close()
    A64, k64, _ = out["fp64"]
    A16, k16, st = out["split_fp16"]
    E = bands.get(velocities=False)[0].reshape(-1)
    ok = E >= C.phExcludeCutoff
    big = ok[None, :] & (np.abs(A64) > 1e-8 * np.abs(A64).max())
    rel = np.abs(A16 - A64)[big] / np.abs(A64)[big]
    assert rel.max() < 1e-5, rel.max()
    # diagonal conductivity components, every temperature
    for t in range(len(T)):
        d64, d16 = np.diagonal(k64[t]), np.diagonal(k16[t])
        assert np.abs(d16 - d64).max() < 1e-4 * np.abs(d64).max(), (t, d16, d64)
    # the near-cut-off event list held every event of every launch
    assert 0 < st.edge_events_peak <= st.edge_events_cap
