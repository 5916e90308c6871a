"""The multi-rank form of the builder on CPU ranks (gloo, world size 2).

Each rank takes its contiguous q2 slice (the reference splits the q2 loop
over MPI ranks), builds unfinalised partial linewidths with the oracle,
the partials are summed with an all-reduce, and the finalize step
(degeneracy averaging, exclusions) runs once on the sum.  The result must
equal the single-process builder.  bench.py --gpus N uses the same slicing
and reduction with NCCL.
"""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _setup():
    import oracle
    from phoebe_b200 import constants as C
    from phoebe_b200 import lattice, synth
    cr = synth.diamond_crystal()
    fc2 = synth.diamond_fc2(cr)
    fc3 = synth.random_fc3(cr, 400, synth.SEED_BASE)
    mesh = (4, 4, 4)
    q = lattice.Mesh(cr, mesh).cartesian_coords()
    h0 = oracle.PhononH0(cr, fc2)
    E, U = h0.diagonalize(q)
    vg = h0.velocities(q)
    T = np.array([C.kelvin_to_ry(t) for t in (100.0, 300.0)])
    return oracle.Interaction3Ph(cr, fc3), mesh, q, E, U, vg, cr.reciprocal_cell, T


def _rank_main(rank, world, port, out_path):
    import torch
    import torch.distributed as dist
    from phoebe_b200.core import finalize_linewidths, q2_slice
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        v3, mesh, q, E, U, vg, recip, T = _setup()
        b, e = q2_slice(rank, world, len(q))
        part = v3.linewidths(mesh, E, U, vg, q, recip, T, "adaptive", 0.0, q2_list=np.arange(b, e),
                             finalize=False)
        t = torch.from_numpy(part.copy())
        dist.all_reduce(t)
        A = finalize_linewidths(t.numpy(), E)
        if rank == 0:
            np.save(out_path, A)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_equal_one_process(tmp_path):
    out = str(tmp_path / "a2.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    A2 = np.load(out)
    v3, mesh, q, E, U, vg, recip, T = _setup()
    A1 = v3.linewidths(mesh, E, U, vg, q, recip, T, "adaptive", 0.0, finalize=True)
    assert np.abs(A1).max() > 0
    np.testing.assert_allclose(A2, A1, rtol=1e-12, atol=1e-15 * np.abs(A1).max())


def test_q2_slices_partition_the_mesh():
    from phoebe_b200.core import q2_slice
    for nq in (1, 7, 512, 8000):
        for world in (1, 2, 3, 4, 8):
            s = [q2_slice(r, world, nq) for r in range(world)]
            assert s[0][0] == 0 and s[-1][1] == nq
            assert all(s[i][1] == s[i + 1][0] for i in range(world - 1))
            assert max(e - b for b, e in s) - min(e - b for b, e in s) <= 1
