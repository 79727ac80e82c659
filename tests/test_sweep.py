"""The batched design sweep's candidates and their partition across ranks."""

from __future__ import annotations

import os

import pytest

from beamtracer_b200.einzel import design_cost, share_of_designs, sweep_designs


def test_sweep_designs_are_seeded_and_in_range():
    a, b = sweep_designs(64), sweep_designs(64)
    assert a == b
    assert len({d.shape for d in a}) == 3
    for d in a:
        assert 3e3 <= d.voltages[1] <= 12e3 and 3e-3 <= d.aperture <= 7e-3
        assert 2000 <= d.trajectories <= 20000
        assert 10e-3 <= d.centres[2] - d.centres[1] <= 25e-3


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_every_candidate_is_solved_once_and_the_load_is_balanced(world):
    designs = sweep_designs(256)
    shares = [share_of_designs(designs, r, world) for r in range(world)]
    flat = sorted(k for s in shares for k in s)
    assert flat == list(range(256))
    loads = [sum(design_cost(designs[k]) for k in s) for s in shares]
    biggest = max(design_cost(d) for d in designs)
    assert max(loads) - min(loads) <= biggest


def _rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    designs = sweep_designs(40)
    mine = share_of_designs(designs, rank, world)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    dist.destroy_process_group()
    out.put((rank, gathered))


def test_ranks_agree_on_the_partition_without_talking():
    import multiprocessing as mp
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    for rank in (0, 1):
        gathered = results[rank]
        assert sorted(gathered[0] + gathered[1]) == list(range(40))
        assert gathered[rank] == share_of_designs(sweep_designs(40), rank, 2)
