"""One solve over several GPUs: the reference's MPI communicator calls over
``torch.distributed`` (one process per GPU, NCCL between GPUs).

``BeamOptics(config, comm=TorchComm())`` traces every ``size``-th trajectory on each rank
(``model.py:445-447``), sums the node charges of every iteration over the ranks before the
density is formed (``tracer.py:1341-1342``: the reference's ``Allreduce``), solves the same
field on every rank (the same density gives the same potential, so every rank stops at the
same iteration), and gathers the plane crossings, statuses and kept trajectories at the end
(``model.py:461-495``).  A device tensor is reduced in place with the process group's
backend (NCCL for CUDA tensors; a CPU backend such as gloo reduces a host copy).
"""

from __future__ import annotations

from typing import Any

import numpy as np


class TorchComm:
    """``Get_rank``, ``Get_size``, ``allgather`` and a summing ``allreduce`` of a device
    tensor, over a ``torch.distributed`` process group (the default one if None)."""

    def __init__(self, group: Any = None) -> None:
        import torch.distributed as dist

        if not dist.is_initialized():
            raise RuntimeError("TorchComm needs an initialised torch.distributed process group")
        self.dist = dist
        self.group = group

    def Get_rank(self) -> int:  # noqa: N802 - the reference's communicator interface
        return self.dist.get_rank(self.group)

    def Get_size(self) -> int:  # noqa: N802
        return self.dist.get_world_size(self.group)

    def allgather(self, obj: Any) -> list:
        out = [None] * self.Get_size()
        self.dist.all_gather_object(out, obj, group=self.group)
        return out

    def allreduce_tensor(self, tensor) -> Any:
        """Sum ``tensor`` over the ranks in place (on the host when the backend cannot take
        device tensors); return it."""
        backend = self.dist.get_backend(self.group)
        if tensor.is_cuda and backend != "nccl":
            host = tensor.cpu()
            self.dist.all_reduce(host, group=self.group)
            tensor.copy_(host)
        else:
            self.dist.all_reduce(tensor, group=self.group)
        return tensor


def share(n: int, rank: int, size: int) -> slice:
    """The trajectories of a rank: every ``size``-th from ``rank`` (``model.py:445-447``)."""
    return slice(rank, n, size) if size > 1 else slice(None)


def merge_planes(parts: list[list[tuple]], positions: list[float]):
    """The plane crossings of every rank, rank after rank (``model.py:461-477``): ``parts``
    holds, per rank, per plane, ``(point, velocity, current, species, direction)``."""
    from beamtracer_b200.tracer import PlaneHits

    merged = []
    for k, x in enumerate(positions):
        hits = PlaneHits(x)
        for part in parts:
            hits.append(*part[k])
        merged.append(hits)
    return merged


def gather_trace(comm: TorchComm, trace) -> None:
    """Give every rank the crossings, statuses, electrodes and kept trajectories of all
    (``model.py:461-495``), in rank order."""
    planes = [(h.point, h.velocity, h.current, h.species, h.direction) for h in trace.planes]
    parts = comm.allgather(planes)
    trace.planes = merge_planes(parts, [h.position_x for h in trace.planes])
    trace.status = np.concatenate(comm.allgather(np.asarray(trace.status)))
    trace.electrode = np.concatenate(comm.allgather(np.asarray(trace.electrode)))
    trace.trajectories = [t for part in comm.allgather(list(trace.trajectories)) for t in part]
    trace.trajectory_species = np.concatenate(
        comm.allgather(np.asarray(trace.trajectory_species)))  # fmt: skip
