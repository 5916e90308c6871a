"""The multi-rank form of the product builder on one GPU.

Two processes (gloo process group, world size 2) each call libphx's FP64 and
split linewidth builders on their contiguous q2 slice with finalize = 0; the
partial vectors are summed with an all-reduce and finalized once
(finalize_linewidths).  That must equal one process's whole builder, as in
bench.py --gpus N (the reference's q2 split and allReduceSum,
src/bte/ph_scattering.cpp:800).  The two processes launch independent kernels
on the same GPU; nothing on the device waits for the other process.  Also
here: the linewidth-mode counterpart of the matrix modes' slice test, q2
slices of one process summing to the whole call."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from phoebe_b200 import constants as C

pytestmark = pytest.mark.gpu

MESH = (6, 6, 6)
TEMPS = (100.0, 300.0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _objects(ctx, precision):
    from phoebe_b200 import synth
    from phoebe_b200.core import Interaction3Ph, PhononH0, PhScatteringMatrix
    cr = synth.diamond_crystal()
    h0 = PhononH0(ctx, cr, synth.diamond_fc2(cr))
    bands = h0.populate(MESH, withVelocities=True)
    v3 = Interaction3Ph(ctx, cr, synth.random_fc3(cr, 400, synth.SEED_BASE), precision=precision)
    T = np.array([C.kelvin_to_ry(t) for t in TEMPS])
    return h0, bands, v3, PhScatteringMatrix(v3, bands, T, "adaptive")


def _rank_main(rank, world, port, out_path, precision):
    import torch
    import torch.distributed as dist
    from phoebe_b200.core import Context, finalize_linewidths, q2_slice
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ctx = Context(0)
        h0, bands, v3, sm = _objects(ctx, precision)
        b, e = q2_slice(rank, world, bands.nq)
        part = sm.setup(b, e, finalize=False)
        t = torch.from_numpy(part.copy())
        dist.all_reduce(t)
        A = finalize_linewidths(t.numpy(), bands.get(velocities=False)[0])
        if rank == 0:
            np.save(out_path, A)
        for o in (v3, bands, h0):
            o.close()
        ctx.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-12), ("split_fp16", 1e-6)])
def test_two_ranks_equal_one_process(ctx, tmp_path, precision, rtol):
    out = str(tmp_path / "a2.npy")
    sp = mp.get_context("spawn")
    port = _free_port()
    procs = [sp.Process(target=_rank_main, args=(r, 2, port, out, precision)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    A2 = np.load(out)
    h0, bands, v3, sm = _objects(ctx, precision)
    A1 = sm.setup()
    assert np.abs(A1).max() > 0
    # the split path sums its FP32 per-q2 accumulators in FP64 per slot, so a
    # different q2 split changes the last bits of the FP32 partial sums
    np.testing.assert_allclose(A2, A1, rtol=rtol, atol=rtol * 1e-3 * np.abs(A1).max())
    for o in (v3, bands, h0):
        o.close()


@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-12), ("split_fp16", 1e-6)])
def test_linewidth_q2_slices_sum_to_whole(ctx, precision, rtol):
    from phoebe_b200.core import finalize_linewidths
    h0, bands, v3, sm = _objects(ctx, precision)
    nq = bands.nq
    cuts = (0, 37, 101, 150, nq)
    parts = sum(sm.setup(a, b, finalize=False) for a, b in zip(cuts[:-1], cuts[1:]))
    whole = sm.setup(finalize=False)
    scale = np.abs(whole).max()
    assert scale > 0
    assert np.abs(parts - whole).max() < rtol * scale
    A = sm.setup()
    E = bands.get(velocities=False)[0]
    assert np.abs(finalize_linewidths(parts, E) - A).max() < rtol * scale
    for o in (v3, bands, h0):
        o.close()
