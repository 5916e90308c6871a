"""The builder for cells with many branches (csrc/wide.cu): any nb up to 48,
FP64 and split precision (tcgen05 R3 transform), optional per-q1 q2 window,
one persistent kernel per chunk of q2 fed by a work queue.

* nb = 36, the 12-atom cell of the learned-screening workload, with a reduced
  FC3 (150 pairs) on 3^3 and 4^3 meshes: FP64 against the oracle at 1e-10,
  the split precisions against FP64 at 1e-5.
* nb = 15, the perovskite cell, with and without the q2 window: the split
  path against the shared-memory FP64 builder at 1e-5; the FP64 path of this
  builder (PHX_WIDE=1) against it at 1e-10.
* nb = 6, the diamond cell, forced onto this builder (PHX_WIDE=1): both
  precisions against the fused nb = 6 FP64 kernel."""
import os

import numpy as np
import pytest

import oracle
from phoebe_b200 import constants as C
from phoebe_b200 import lattice, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def twelve():
    cr = synth.twelve_atom_crystal(synth.SEED_BASE + 4)
    return {"crystal": cr, "fc2": synth.twelve_atom_fc2(cr), "fc3": synth.random_fc3(cr, 150, synth.SEED_BASE + 4)}


@pytest.fixture(scope="module")
def perovskite():
    return synth.perovskite_workload(mesh=(4, 4, 4), num_pairs=150, fc_grid=(4, 4, 4))


class _Wide:
    """PHX_WIDE=1 for the duration of a block."""

    def __enter__(self):
        os.environ["PHX_WIDE"] = "1"

    def __exit__(self, *a):
        os.environ.pop("PHX_WIDE", None)


def _rel(A, B, lo=1e-6):
    """max relative difference of A against B on entries above lo of B's largest"""
    scale = np.abs(B).max()
    assert scale > 0
    big = np.abs(B) > lo * scale
    return float((np.abs(A - B)[big] / np.abs(B)[big]).max()), float(np.abs(A - B)[~big].max(initial=0.0) / scale)


def _setup(ctx, cr, fc2, fc3, mesh):
    from phoebe_b200.core import PhononH0
    h0 = PhononH0(ctx, cr, fc2)
    return h0, h0.populate(mesh, withVelocities=True)


def _lw(ctx, cr, fc3, bands, T, smearing, precision, window=None, sigma=0.3 / C.ryToTHz):
    from phoebe_b200.core import Interaction3Ph, PhScatteringMatrix
    v3 = Interaction3Ph(ctx, cr, fc3, precision=precision)
    sm = PhScatteringMatrix(v3, bands, T, smearing, sigma, window=window)
    A = sm.setup()
    st = sm.stats
    v3.close()
    return A, st


@pytest.mark.parametrize("mesh,smearing,temps", [((4, 4, 4), "adaptive", (150.0, 300.0)),
                                                 ((3, 3, 3), "gaussian", (300.0,))])
def test_36_branches_fp64_matches_oracle_split_matches_fp64(ctx, twelve, mesh, smearing, temps):
    cr, fc3 = twelve["crystal"], twelve["fc3"]
    assert cr.num_bands == 36
    h0, bands = _setup(ctx, cr, twelve["fc2"], fc3, mesh)
    T = np.array([C.kelvin_to_ry(t) for t in temps])
    A64, st = _lw(ctx, cr, fc3, bands, T, smearing, "fp64")
    assert st.pair_launches >= 1
    E, U, vg = bands.get()
    m = lattice.Mesh(cr, mesh)
    ref = oracle.Interaction3Ph(cr, fc3).linewidths(mesh, E, U, vg, m.cartesian_coords(), cr.reciprocal_cell, T,
                                                    smearing, 0.3 / C.ryToTHz)
    rel, small = _rel(A64, ref)
    assert rel < 1e-10 and small < 1e-16, (rel, small)
    ok = (E.reshape(-1) >= C.phExcludeCutoff)[None, :]
    for prec in ("split_fp16", "split_bf16"):
        As, _ = _lw(ctx, cr, fc3, bands, T, smearing, prec)
        big = ok & (np.abs(A64) > 1e-8 * np.abs(A64).max())
        r = (np.abs(As - A64)[big] / np.abs(A64)[big]).max()
        assert r < 1e-5, (prec, r)
    bands.close()
    h0.close()


@pytest.mark.parametrize("windowed", [False, True])
def test_15_branches_split_and_wide_fp64_match_shared_memory_builder(ctx, perovskite, windowed):
    w = perovskite
    mesh = (4, 4, 4)
    h0, bands = _setup(ctx, w.crystal, w.fc2, w.fc3, mesh)
    T = np.array([C.kelvin_to_ry(t) for t in (300.0, 600.0)])
    window = None
    if windowed:
        window = synth.q2_window(bands.get(velocities=False)[0], mesh)
    A64, _ = _lw(ctx, w.crystal, w.fc3, bands, T, "adaptive", "fp64", window)   # shared-memory builder
    with _Wide():
        Aw, _ = _lw(ctx, w.crystal, w.fc3, bands, T, "adaptive", "fp64", window)
    rel, small = _rel(Aw, A64)
    assert rel < 1e-10 and small < 1e-16, (rel, small)
    E = bands.get(velocities=False)[0]
    ok = (E.reshape(-1) >= C.phExcludeCutoff)[None, :]
    big = ok & (np.abs(A64) > 1e-8 * np.abs(A64).max())
    for prec in ("split_fp16", "split_bf16"):
        As, st = _lw(ctx, w.crystal, w.fc3, bands, T, "adaptive", prec, window)
        r = (np.abs(As - A64)[big] / np.abs(A64)[big]).max()
        assert r < 1e-5, (prec, r)
        assert st.pair_launches >= 1
    bands.close()
    h0.close()


def test_6_branches_on_the_wide_builder_match_fused_kernel(ctx, diamond):
    cr = diamond["crystal"]
    mesh = (6, 6, 6)
    h0, bands = _setup(ctx, cr, diamond["fc2"], diamond["fc3"], mesh)
    T = np.array([C.kelvin_to_ry(t) for t in (100.0, 300.0, 600.0)])
    A64, _ = _lw(ctx, cr, diamond["fc3"], bands, T, "adaptive", "fp64")       # fused nb = 6 kernel
    with _Wide():
        Aw, _ = _lw(ctx, cr, diamond["fc3"], bands, T, "adaptive", "fp64")
        As, _ = _lw(ctx, cr, diamond["fc3"], bands, T, "adaptive", "split_fp16")
    rel, small = _rel(Aw, A64)
    assert rel < 1e-10 and small < 1e-16, (rel, small)
    E = bands.get(velocities=False)[0]
    ok = (E.reshape(-1) >= C.phExcludeCutoff)[None, :]
    big = ok & (np.abs(A64) > 1e-8 * np.abs(A64).max())
    r = (np.abs(As - A64)[big] / np.abs(A64)[big]).max()
    assert r < 1e-5, r
    bands.close()
    h0.close()
