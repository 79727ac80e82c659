"""One solve split over two ranks (gloo between two processes on one GPU: the charges are
summed on the host, so no kernel waits on another rank) against the same solve on one
rank: the strided trajectory shares, the summed node charges and the gathered crossings
give the same converged potential and beam moments."""

from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _config():
    from tests.vlasov_cases import extraction

    return extraction(1.0, iterations=6, tolerance=0.0)


def _rank(rank, world, port, out):
    try:
        import torch
        import torch.distributed as dist

        from beamtracer_b200.distributed import TorchComm
        from beamtracer_b200.model import BeamOptics

        torch.cuda.set_device(0)
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=world)
        model = BeamOptics(_config(), comm=TorchComm()).run()
        m = model.beam_moments(7.5e-3)
        result = (rank, model.potential.copy(), m.current, m.rms_size, m.emittance,
                  int(model.state.trace.status.size))  # fmt: skip
        dist.destroy_process_group()
        out.put(result)
    except Exception:
        import traceback

        out.put((rank, "error", traceback.format_exc(), 0, 0, 0))


def test_two_ranks_equal_one():
    import multiprocessing as mp
    import socket

    from beamtracer_b200.model import BeamOptics

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = {r[0]: r[1:] for r in (out.get(timeout=600) for _ in procs)}
    for p in procs:
        p.join(timeout=60)
    for r in results.values():
        assert not (isinstance(r[0], str) and r[0] == "error"), r[1]
    single = BeamOptics(_config()).run()
    m = single.beam_moments(7.5e-3)
    for rank in (0, 1):
        phi, current, size, emittance, launched = results[rank]
        np.testing.assert_allclose(phi, single.potential, rtol=0, atol=1e-9 * 2000.0)
        assert current == pytest.approx(m.current, rel=1e-9)
        assert size == pytest.approx(m.rms_size, rel=1e-7)
        assert emittance == pytest.approx(m.emittance, rel=1e-6)
        assert launched == single.state.trace.status.size
