"""CUDA graphs and the launch-plan autotuner of the linewidth builder.

The first call of a builder configuration runs eagerly, the second captures
its device work into a CUDA graph, later identical calls replay it
(stats.graph 0, 1, then 2); the
results equal those of eager launches (PHX_GRAPHS=0) -- bit for bit on the
FP64 path, to 1e-6 on the split path, whose FP32 shared-memory accumulation
order varies from run to run -- and values copied in outside the graph (the
temperatures) take effect on replay.  The autotuner
picks one of its candidate plans, and the tuned plan gives the default
plan's linewidths."""
import os

import numpy as np
import pytest

from phoebe_b200 import constants as C

pytestmark = pytest.mark.gpu


def _setup(ctx, diamond, mesh, precision):
    from phoebe_b200.core import Interaction3Ph, PhononH0
    cr = diamond["crystal"]
    h0 = PhononH0(ctx, cr, diamond["fc2"])
    bands = h0.populate(mesh, withVelocities=True)
    v3 = Interaction3Ph(ctx, cr, diamond["fc3"], precision=precision)
    return h0, bands, v3


class _env:
    def __init__(self, **kv):
        self.kv = kv

    def __enter__(self):
        self.old = {k: os.environ.get(k) for k in self.kv}
        os.environ.update(self.kv)

    def __exit__(self, *a):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


@pytest.mark.parametrize("precision", ["fp64", "split_bf16"])
def test_graph_capture_and_replay(ctx, diamond, precision):
    from phoebe_b200.core import PhScatteringMatrix
    h0, bands, v3 = _setup(ctx, diamond, (8, 8, 8), precision)
    T1 = np.array([C.kelvin_to_ry(t) for t in (100.0, 300.0)])
    T2 = np.array([C.kelvin_to_ry(t) for t in (200.0, 600.0)])
    if precision == "fp64":
        same = np.testing.assert_array_equal
    else:
        def same(x, y):
            np.testing.assert_allclose(x, y, rtol=1e-6, atol=1e-12 * np.abs(y).max())
    sm = PhScatteringMatrix(v3, bands, T1, "adaptive")
    a0 = sm.setup().copy()
    assert sm.stats.graph == 0
    a1 = sm.setup().copy()
    assert sm.stats.graph == 1
    a2 = sm.setup().copy()
    assert sm.stats.graph == 2
    same(a0, a1)
    same(a1, a2)
    assert sm.stats.pair_launches >= 1 and sm.stats.ms_pair > 0.0
    with _env(PHX_GRAPHS="0"):
        e1 = sm.setup().copy()
        assert sm.stats.graph == 0
    same(a1, e1)
    # new temperature values, same shapes: the graph replays with them
    sm2 = PhScatteringMatrix(v3, bands, T2, "adaptive")
    b = sm2.setup().copy()
    assert sm2.stats.graph == 2
    with _env(PHX_GRAPHS="0"):
        eb = sm2.setup().copy()
    same(b, eb)
    assert np.abs(b - a1).max() > 0
    for o in (v3, bands, h0):
        o.close()


def test_generic_path_graph(ctx, diamond):
    from phoebe_b200.core import PhScatteringMatrix
    h0, bands, v3 = _setup(ctx, diamond, (4, 4, 4), "fp64")
    T = np.array([C.kelvin_to_ry(300.0)])
    everything = (np.zeros(bands.nq), np.zeros(bands.nq))
    sm = PhScatteringMatrix(v3, bands, T, "adaptive", window=everything)
    sm.setup()
    a = sm.setup().copy()
    assert sm.stats.graph == 1
    b = sm.setup().copy()
    assert sm.stats.graph == 2
    # shared-memory atomics: the order of the last bits may differ
    np.testing.assert_allclose(a, b, rtol=1e-13, atol=0)
    for o in (v3, bands, h0):
        o.close()


@pytest.mark.parametrize("precision,cands", [("fp64", {(512, 8), (512, 4), (512, 16), (1024, 16)}),
                                             ("split_bf16", {(448, 7), (448, 14), (896, 14), (896, 28),
                                                             (1792, 14), (1792, 28)})])
def test_autotuned_plan(ctx, diamond, precision, cands):
    from phoebe_b200.core import PhScatteringMatrix
    h0, bands, v3 = _setup(ctx, diamond, (12, 12, 12), precision)
    T = np.array([C.kelvin_to_ry(300.0)])
    sm = PhScatteringMatrix(v3, bands, T, "adaptive")
    tuned = sm.setup().copy()
    # a chunk longer than the q2 range is clipped to it
    assert (sm.stats.plan_chunk, sm.stats.plan_slots) in {(min(c, bands.nq), sl) for c, sl in cands}
    with _env(PHX_TUNE="0", PHX_GRAPHS="0"):
        default = sm.setup().copy()
    tol = 1e-12 if precision == "fp64" else 1e-6
    big = np.abs(default) > 1e-6 * np.abs(default).max()
    assert (np.abs(tuned - default)[big] / np.abs(default)[big]).max() < tol
    for o in (v3, bands, h0):
        o.close()
