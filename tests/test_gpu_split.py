"""Split-precision (BF16 x3 on tcgen05) path: the tensor-core GEMM building
block against numpy, then whole-builder linewidths against the FP64 path.

North-star bar for the split path: linewidth max relative error <= 1e-5 and
thermal conductivity within 0.1% of the FP64 result (checked at 1e-4 here)."""
import ctypes

import numpy as np
import pytest

from phoebe_b200 import constants as C

pytestmark = pytest.mark.gpu


def test_tc_gemm_selftest(ctx):
    from phoebe_b200 import _abi
    rng = np.random.default_rng(0)
    for N, Kp in ((144, 96), (64, 16), (256, 48)):
        A = rng.normal(size=(128, Kp)).astype(np.float32)
        B = rng.normal(size=(N, Kp)).astype(np.float32)
        Cm = np.zeros((128, N), dtype=np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        _abi.check(_abi.load().phx_diag_tc_gemm(ctx.h, N, Kp, A.ctypes.data_as(fp),
                                                B.ctypes.data_as(fp), Cm.ctypes.data_as(fp)), ctx.h)
        ref = A.astype(np.float64) @ B.astype(np.float64).T
        # BF16 hi+lo keeps ~16 bits per operand: each product is exact to
        # ~2^-17 relative, so the error is ~1e-5 of sum_k |A||B|
        scale = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64).T
        err = (np.abs(Cm - ref) / scale).max()
        assert err < 3e-5, (N, Kp, err)


def _builder(ctx, diamond, mesh, smearing, temps_k, precision):
    from phoebe_b200.core import Interaction3Ph, PhononH0, PhScatteringMatrix
    cr = diamond["crystal"]
    T = np.array([C.kelvin_to_ry(t) for t in temps_k])
    h0 = PhononH0(ctx, cr, diamond["fc2"])
    bands = h0.populate(mesh, withVelocities=True)
    v3 = Interaction3Ph(ctx, cr, diamond["fc3"], precision=precision)
    sm = PhScatteringMatrix(v3, bands, T, smearing, 0.3 / C.ryToTHz)
    A = sm.setup()
    k = sm.thermalConductivity(cr.volume)
    E, _, _ = bands.get(velocities=False)
    return A, k, E, sm


CASES = [((8, 8, 8), "gaussian", (300.0,)),
         ((10, 10, 10), "adaptive", (100.0, 300.0, 600.0)),
         # coarse meshes: pairs whose FP64 velocity difference is non-zero but
         # lost in FP32 (width floored), and small linewidths built from
         # triplets with strong cancellation in V (FP16 hi/lo needed for 1e-5)
         ((6, 6, 6), "adaptive", (300.0, 600.0)),
         ((8, 8, 8), "adaptive", (300.0,)),
         ((5, 5, 5), "adaptive", (100.0, 200.0, 300.0, 600.0))]


@pytest.mark.parametrize("mesh,smearing,temps,precision",
                         [c + ("split_fp16",) for c in CASES] + [c + ("split_bf16",) for c in CASES[:3]])
def test_split_linewidths_match_fp64(ctx, diamond, mesh, smearing, temps, precision):
    A64, k64, E, _ = _builder(ctx, diamond, mesh, smearing, temps, "fp64")
    A16, k16, _, sm = _builder(ctx, diamond, mesh, smearing, temps, precision)
    # linewidths Gamma = A / n(n+1) on non-excluded states
    ok = E.reshape(-1) >= C.phExcludeCutoff
    big = ok[None, :] & (np.abs(A64) > 1e-8 * np.abs(A64).max())
    rel = np.abs(A16 - A64)[big] / np.abs(A64)[big]
    assert rel.max() < 1e-5, rel.max()
    np.testing.assert_allclose(k16, k64, rtol=1e-4)
    assert sm.stats.kernel_launches > 0


def test_near_cutoff_events_beyond_the_list_capacity(ctx, diamond):
    """The split path records triplets whose adaptive-delta cut-off test is
    too close for FP32 and re-decides them in FP64 after each pair launch.
    With the event list capped below what a chunk produces, the chunk applies
    none of its events and is re-run in smaller q2 pieces with the rates off;
    the linewidths must not change (beyond rounding)."""
    from phoebe_b200 import _abi
    L = _abi.load()
    mesh, temps = (8, 8, 8), (300.0,)
    A0, k0, E, sm0 = _builder(ctx, diamond, mesh, "adaptive", temps, "split_fp16")
    assert sm0.stats.edge_events_cap == 2 ** 18
    assert sm0.stats.edge_overflow_chunks == 0
    peak = sm0.stats.edge_events_peak
    assert peak > 4      # this mesh has near-cut-off events
    try:
        _abi.check(L.phx_debug_set_split_edge_cap(peak // 3), ctx.h)
        A1, k1, _, sm1 = _builder(ctx, diamond, mesh, "adaptive", temps, "split_fp16")
        assert sm1.stats.edge_events_cap == peak // 3
        assert sm1.stats.edge_overflow_chunks >= 1
    finally:
        _abi.check(L.phx_debug_set_split_edge_cap(0), ctx.h)
    ok = E.reshape(-1) >= C.phExcludeCutoff
    big = ok[None, :] & (np.abs(A0) > 1e-8 * np.abs(A0).max())
    rel = np.abs(A1 - A0)[big] / np.abs(A0)[big]
    assert rel.max() < 1e-6, rel.max()
    # and the capped run still matches the FP64 path at the split bar
    A64, _, _, _ = _builder(ctx, diamond, mesh, "adaptive", temps, "fp64")
    rel64 = np.abs(A1 - A64)[big] / np.abs(A64)[big]
    assert rel64.max() < 1e-5, rel64.max()
