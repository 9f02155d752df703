"""A batch of meshes split across GPUs: one process per GPU, no collective.

Meshes are independent units of work, so the multi-GPU form of the batched
call is a static partition: every rank refines its own share of the meshes on
its own GPU, and nothing crosses between GPUs on the data path.  The split is
by predicted output (refined quads, nnz * 4^(levels-1) for a mesh of nnz
corners): largest mesh first, each to the rank with the least work so far
(ties to the lowest rank), so the ranks finish together to within one mesh.
Each rank keeps its meshes in batch order.

The reference has no multi-GPU path; its caller loops over meshes on one GPU
(source/main.cpp:84-113).  ``partition`` / ``shard_indices`` are pure host
logic (tested with gloo ranks on the CPU); ``ShardedBatch`` runs a rank's
share through ``slak_batch_*`` on the rank's device.
"""
from __future__ import annotations

import os
from typing import Callable, List, Optional, Sequence, Union

from .mesh import Mesh


def predicted_quads(nnz: int, levels: int) -> int:
    """Refined quads after `levels` levels of a mesh with `nnz` corners (the
    first level makes one quad per corner, each later level four per quad)."""
    if levels < 1:
        return 0
    return int(nnz) * 4 ** (int(levels) - 1)


def partition(work: Sequence[int], world_size: int) -> List[int]:
    """Owner rank of every item: largest first, each to the least-loaded rank."""
    if world_size < 1:
        raise ValueError(f"partition: world_size must be at least 1, got {world_size}")
    if any(w < 0 for w in work):
        raise ValueError("partition: work must be non-negative")
    load = [0] * world_size
    owner = [0] * len(work)
    for k in sorted(range(len(work)), key=lambda k: (-work[k], k)):
        r = min(range(world_size), key=lambda r: (load[r], r))
        owner[k] = r
        load[r] += work[k]
    return owner


def shard_indices(work: Sequence[int], rank: int, world_size: int) -> List[int]:
    """Indices of rank `rank`'s items, in batch order."""
    if not 0 <= rank < world_size:
        raise ValueError(f"shard_indices: rank {rank} outside 0..{world_size - 1}")
    owner = partition(work, world_size)
    return [k for k, o in enumerate(owner) if o == rank]


def rank_and_world(rank: Optional[int] = None, world_size: Optional[int] = None):
    """(rank, world size): the arguments, else torch.distributed's process
    group when one is initialised, else RANK / WORLD_SIZE from the environment
    (torchrun), else (0, 1)."""
    if rank is not None and world_size is not None:
        return int(rank), int(world_size)
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist.get_rank(), dist.get_world_size()
    except ImportError:
        pass
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


MeshSource = Union[Mesh, Callable[[], Mesh]]


class ShardedBatch:
    """This rank's share of a batch, refined on this rank's GPU.

    ``meshes``: host meshes, or callables that make them (only this rank's are
    called, so a rank never builds another rank's geometry; then ``work`` must
    be given).  ``work``: predicted output per mesh (default
    ``predicted_quads(nnz, levels)``).  The device is LOCAL_RANK's unless
    ``device`` is given.  ``output(i)`` takes the mesh's index in the whole
    batch and returns None for a mesh another rank owns."""

    def __init__(self, meshes: Sequence[MeshSource], levels: Sequence[int], scheme: int, flags: int = 0,
                 work: Optional[Sequence[int]] = None, rank: Optional[int] = None,
                 world_size: Optional[int] = None, device: Optional[int] = None, stream=None):
        from . import api
        if len(levels) != len(meshes):
            raise ValueError(f"ShardedBatch: {len(meshes)} meshes but {len(levels)} level counts")
        if work is None:
            if any(callable(m) for m in meshes):
                raise ValueError("ShardedBatch: pass `work` when meshes are made on demand")
            work = [predicted_quads(m.nnz, l) for m, l in zip(meshes, levels)]
        elif len(work) != len(meshes):
            raise ValueError(f"ShardedBatch: {len(meshes)} meshes but {len(work)} work figures")
        self.rank, self.world_size = rank_and_world(rank, world_size)
        self.indices = shard_indices(work, self.rank, self.world_size)
        torch = api._torch()
        if device is None:
            device = int(os.environ.get("LOCAL_RANK", "0")) % torch.cuda.device_count()
        torch.cuda.set_device(device)
        self.device = device
        host = [meshes[k]() if callable(meshes[k]) else meshes[k] for k in self.indices]
        self._dms = [api.DeviceMesh.from_host(m) for m in host]
        self._slot = {k: j for j, k in enumerate(self.indices)}
        self.levels = [int(levels[k]) for k in self.indices]
        self._batch = api.Batch(self._dms, self.levels, scheme, flags, stream=stream) if self.indices else None

    def execute(self, stream=None) -> None:
        if self._batch is not None:
            self._batch.execute(stream)

    def check(self, stream=None) -> None:
        if self._batch is not None:
            self._batch.check(stream)

    def output(self, i: int):
        j = self._slot.get(int(i))
        return None if j is None else self._batch.output(j)

    @property
    def launches(self) -> int:
        return self._batch.launches if self._batch is not None else 0

    @property
    def waves(self) -> int:
        return self._batch.waves if self._batch is not None else 0

    def close(self) -> None:
        if self._batch is not None:
            self._batch.close()
            self._batch = None
