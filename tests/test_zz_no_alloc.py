"""The allocation-free builder entry point, phx_ph_linewidths_static.

It serves callers that cannot allocate device memory at call time (an
application whose own pool allocator owns all free device memory, or a
latency-critical loop that must not pay cudaMalloc's implicit device
synchronisation): every intermediate buffer lives in a 16 MiB array that the
library reserves statically on each GPU.  The test calls it twice in a row
through the C ABI and compares both results with the regular entry point
phx_ph_linewidths_d (same FP64 path, with its own scratch allocations), at
the 1e-10 relative tolerance of the other FP64 linewidth tests.  It lives in
its own file, collected last, and builds everything it needs itself, so it
passes alone in a fresh process as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

from phoebe_b200 import constants as C

pytestmark = pytest.mark.gpu


def _params(T, nq, smearing, sigma):
    from phoebe_b200 import _abi
    p = _abi.LwParams()
    p.num_temperatures = len(T)
    p.temperatures = T.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    p.smearing = _abi.PHX_SMEAR_ADAPTIVE if smearing == "adaptive" else _abi.PHX_SMEAR_GAUSSIAN
    p.sigma = sigma
    p.finalize = 1
    p.q2_begin = 0
    p.q2_end = nq
    return p


def test_static_scratch_builder_matches_regular_entry_point():
    import torch

    from phoebe_b200 import _abi, synth
    from phoebe_b200.core import Context, Interaction3Ph, PhononH0

    ctx = Context(0)
    cr = synth.diamond_crystal()
    fc2 = synth.diamond_fc2(cr)
    fc3 = synth.random_fc3(cr, 400, synth.SEED_BASE)
    L = _abi.load()
    for mesh, smearing, temps in (((6, 6, 6), "adaptive", (100.0, 300.0, 600.0)),
                                  ((5, 5, 5), "gaussian", (300.0,))):
        T = np.array([C.kelvin_to_ry(t) for t in temps])
        h0 = PhononH0(ctx, cr, fc2)
        bands = h0.populate(mesh, withVelocities=True)
        v3 = Interaction3Ph(ctx, cr, fc3, precision="fp64")
        nq = bands.nq
        n = len(T) * nq * bands.nb
        p = _params(T, nq, smearing, 0.3 / C.ryToTHz)
        ref = torch.zeros(n, dtype=torch.float64, device="cuda")
        _abi.check(L.phx_ph_linewidths_d(v3.h, bands.h, ctypes.byref(p), ctypes.c_void_p(ref.data_ptr()),
                                         None), ctx.h)
        outs = []
        for _ in range(2):
            out = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
            _abi.check(L.phx_ph_linewidths_static(v3.h, bands.h, ctypes.byref(p),
                                                  ctypes.c_void_p(out.data_ptr())), ctx.h)
            outs.append(out.cpu().numpy())
        A = ref.cpu().numpy()
        assert np.abs(A).max() > 0
        big = np.abs(A) > 1e-6 * np.abs(A).max()
        for B in outs:
            assert np.all(np.isfinite(B))
            rel = np.abs(B - A)[big] / np.abs(A)[big]
            assert rel.max() < 1e-10, rel.max()
            assert np.abs(B - A)[~big].max(initial=0.0) < 1e-16 * np.abs(A).max()
        # the second call starts from the first call's leftovers and must not see them
        np.testing.assert_array_equal(outs[0], outs[1])
        v3.close()
        bands.close()
        h0.close()


def test_static_scratch_rejects_problems_beyond_its_size():
    import torch

    from phoebe_b200 import _abi, synth
    from phoebe_b200.core import BandStructure, Context, Interaction3Ph

    ctx = Context(0)
    cr = synth.diamond_crystal()
    fc3 = synth.random_fc3(cr, 400, synth.SEED_BASE)
    v3 = Interaction3Ph(ctx, cr, fc3, precision="fp64")
    mesh = (36, 36, 36)            # 46656 points x 6 bands x 4 temperatures: > 16 MiB
    nq = int(np.prod(mesh))
    E = np.tile(np.linspace(1e-3, 5e-3, 6), (nq, 1))
    U = np.tile(np.eye(6, dtype=np.complex128), (nq, 1, 1))
    bands = BandStructure.from_arrays(ctx, mesh, cr.reciprocal_cell, E, U, None)
    T = np.array([C.kelvin_to_ry(t) for t in (100.0, 200.0, 300.0, 600.0)])
    p = _params(T, nq, "gaussian", 1e-4)
    out = torch.zeros(len(T) * nq * 6, dtype=torch.float64, device="cuda")
    L = _abi.load()
    rc = L.phx_ph_linewidths_static(v3.h, bands.h, ctypes.byref(p), ctypes.c_void_p(out.data_ptr()))
    assert rc == _abi.PHX_ERR_ARG
    assert "static scratch" in _abi.last_error(ctx.h)


def test_static_scratch_q2_slices_match_regular_entry_point():
    """A q2 slice (what one rank of a multi-GPU run computes, finalize = 0) over
    more than one chunk of the 16 MiB array, and an empty slice."""
    import torch

    from phoebe_b200 import _abi, synth
    from phoebe_b200.core import Context, Interaction3Ph, PhononH0

    ctx = Context(0)
    cr = synth.diamond_crystal()
    fc3 = synth.random_fc3(cr, 400, synth.SEED_BASE)
    mesh = (6, 6, 6)
    T = np.array([C.kelvin_to_ry(t) for t in (100.0, 300.0, 600.0)])
    h0 = PhononH0(ctx, cr, synth.diamond_fc2(cr))
    bands = h0.populate(mesh, withVelocities=True)
    v3 = Interaction3Ph(ctx, cr, fc3, precision="fp64")
    nq, nb = bands.nq, bands.nb
    n = len(T) * nq * nb
    # q2 per chunk of the static path: what is left of 16 MiB after the Bose
    # table and the partial sums, over one q2 slab of the cached vertex
    align = lambda x: (x + 255) // 256 * 256
    fixed = 2 * align(8 * nq * nb * len(T)) + align(64)
    chunk = (16 * 2 ** 20 - fixed) // (16 * v3.nr3 * nb ** 3)
    q2b, q2e = 30, 190
    assert q2e - q2b > chunk, "the slice must span more than one chunk"
    L = _abi.load()
    p = _params(T, nq, "adaptive", 0.0)
    p.finalize = 0
    p.q2_begin, p.q2_end = q2b, q2e
    ref = torch.zeros(n, dtype=torch.float64, device="cuda")
    _abi.check(L.phx_ph_linewidths_d(v3.h, bands.h, ctypes.byref(p), ctypes.c_void_p(ref.data_ptr()), None),
               ctx.h)
    out = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
    _abi.check(L.phx_ph_linewidths_static(v3.h, bands.h, ctypes.byref(p), ctypes.c_void_p(out.data_ptr())),
               ctx.h)
    A, B = ref.cpu().numpy(), out.cpu().numpy()
    assert np.abs(A).max() > 0 and np.all(np.isfinite(B))
    big = np.abs(A) > 1e-6 * np.abs(A).max()
    assert (np.abs(B - A)[big] / np.abs(A)[big]).max() < 1e-10
    assert np.abs(B - A)[~big].max(initial=0.0) < 1e-16 * np.abs(A).max()
    # an empty slice writes zeros
    p.q2_begin = p.q2_end = 50
    _abi.check(L.phx_ph_linewidths_static(v3.h, bands.h, ctypes.byref(p), ctypes.c_void_p(out.data_ptr())),
               ctx.h)
    assert np.all(out.cpu().numpy() == 0.0)
    v3.close()
    bands.close()
    h0.close()
