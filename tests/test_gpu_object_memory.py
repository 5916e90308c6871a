"""Device memory of the library's objects: stream-ordered allocations from the
device's memory pool (band structures, couplings, phonon Hamiltonians).

GPU: objects created and destroyed repeatedly reuse the pool's memory (free
device memory stays flat after the first round, and the results are
unchanged); objects that outlive their context can still be destroyed; a new
context works after an old one was destroyed."""
import numpy as np
import pytest

from phoebe_b200 import constants as C

pytestmark = pytest.mark.gpu


def _build(ctx, diamond, mesh):
    from phoebe_b200.core import Interaction3Ph, PhononH0, PhScatteringMatrix
    h0 = PhononH0(ctx, diamond["crystal"], diamond["fc2"])
    bands = h0.populate(mesh, withVelocities=True)
    v3 = Interaction3Ph(ctx, diamond["crystal"], diamond["fc3"])
    A = PhScatteringMatrix(v3, bands, [C.kelvin_to_ry(300.0)], "adaptive").setup()
    return h0, bands, v3, A


def test_objects_reuse_pool_memory(diamond):
    import torch
    from phoebe_b200.core import Context
    ctx = Context(0)
    ref = None
    free = []
    for i in range(12):
        h0, bands, v3, A = _build(ctx, diamond, (6, 6, 6))
        if ref is None:
            ref = A
        np.testing.assert_allclose(A, ref, rtol=1e-12, atol=0)
        for o in (v3, bands, h0):
            o.close()
        ctx.synchronize()
        free.append(torch.cuda.mem_get_info(0)[0])
    # after the first round the pool holds what a round needs; later rounds take nothing more
    assert max(free[1:]) - min(free[1:]) < 64 << 20
    ctx.close()


def test_objects_outliving_their_context(diamond):
    from phoebe_b200.core import Context
    ctx = Context(0)
    h0, bands, v3, A = _build(ctx, diamond, (4, 4, 4))
    ctx.close()
    for o in (v3, bands, h0):
        o.close()
    ctx2 = Context(0)
    h0, bands, v3, A2 = _build(ctx2, diamond, (4, 4, 4))
    np.testing.assert_allclose(A2, A, rtol=1e-12, atol=0)
    for o in (v3, bands, h0):
        o.close()
    ctx2.close()
