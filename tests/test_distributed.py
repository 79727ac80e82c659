"""One solve over several ranks: the communicator over torch.distributed, the strided
trajectory shares and the gathered results (gloo ranks on the CPU)."""

from __future__ import annotations

import os

import numpy as np

from beamtracer_b200.distributed import merge_planes, share


def test_shares_cover_every_trajectory_once():
    for n in (0, 1, 7, 100):
        for size in (1, 2, 3, 8):
            got = sorted(i for r in range(size) for i in range(n)[share(n, r, size)])
            assert got == list(range(n))


def _rank(rank, world, port, out):
    try:
        out.put(_rank_body(rank, world, port))
    except Exception as error:  # report it to the parent instead of hanging it
        import traceback

        out.put((rank, "error", traceback.format_exc(), error.__class__.__name__, 0))


def _rank_body(rank, world, port):
    import torch
    import torch.distributed as dist

    from beamtracer_b200.distributed import TorchComm
    from beamtracer_b200.model import BeamOptics
    from tests.vlasov_cases import diode

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    comm = TorchComm()
    charge = torch.full((1, 5), float(rank + 1), dtype=torch.float64)
    comm.allreduce_tensor(charge)
    model = BeamOptics(diode(current_density=10.0), comm=comm)
    particles, _ = model._particles()
    ys = comm.allgather(particles.position[1].tolist())
    planes = [(np.full((3, rank + 1), rank, float), np.zeros((3, rank + 1)),
               np.full(rank + 1, 1e-9), np.zeros(rank + 1, np.int32), np.ones(rank + 1, np.int8))]
    parts = comm.allgather(planes)
    merged = merge_planes(parts, [9.9e-3])
    size = comm.Get_size()
    dist.destroy_process_group()
    return (rank, charge.tolist(), ys, merged[0].point.tolist(), size)


def test_two_ranks_share_reduce_and_gather():
    import multiprocessing as mp
    import socket

    from beamtracer_b200.model import BeamOptics
    from tests.vlasov_cases import diode

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict((r[0], r[1:]) for r in (out.get(timeout=180) for _ in procs))
    for p in procs:
        p.join(timeout=60)
    for rank, r in results.items():
        assert r[0] != "error", r[1]
    whole = BeamOptics(diode(current_density=10.0))._particles()[0].position[1]
    for rank in (0, 1):
        charge, ys, points, size = results[rank]
        assert size == 2
        assert charge == [[3.0] * 5]
        assert sorted(ys[0] + ys[1]) == sorted(whole.tolist())
        assert ys[rank] == whole[rank::2].tolist()
        assert np.asarray(points).shape == (3, 3)  # rank 0's crossing, then rank 1's two
        assert np.asarray(points)[0].tolist() == [0.0, 1.0, 1.0]
