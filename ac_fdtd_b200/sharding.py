"""Independent rooms spread over GPUs, one process per GPU.

Rooms never exchange data, so a batch shards with no collective on the data path: each rank
runs a ``RoomBatch`` of its share of the rooms, and only the receiver recordings travel, once,
to the rank that asks for them (``torch.distributed`` object gather over whatever backend the
process group uses -- NCCL between GPUs, gloo for the CPU tests).

Shares are balanced by cell count with the longest-processing-time rule: rooms in decreasing
size, each to the rank with the fewest cells so far. The largest share is at most 4/3 of the
optimum.
"""

from __future__ import annotations

import numpy as np

__all__ = ["partition_rooms", "ShardedRooms"]


def partition_rooms(cell_counts, world_size: int) -> list[list[int]]:
    """Room indices per rank, balanced by cells (greedy, deterministic)."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(cell_counts)), key=lambda r: (-int(cell_counts[r]), r))
    loads = [0] * world_size
    shares: list[list[int]] = [[] for _ in range(world_size)]
    for r in order:
        rank = min(range(world_size), key=lambda q: (loads[q], q))
        shares[rank].append(r)
        loads[rank] += int(cell_counts[r])
    return [sorted(share) for share in shares]


class ShardedRooms:
    """This rank's part of a room list, run as one batch, with a gather of the recordings.

    ``make_batch(specs)`` builds the local batch (in production a ``RoomBatch`` on this rank's
    GPU, e.g. ``functools.partial(RoomBatch, device=local_rank)``; tests pass a stand-in);
    ``rank``/``world_size`` default to the current process group.
    """

    def __init__(self, specs, make_batch, rank: int | None = None, world_size: int | None = None):
        import torch.distributed as dist

        if rank is None:
            rank = dist.get_rank() if dist.is_initialized() else 0
        if world_size is None:
            world_size = dist.get_world_size() if dist.is_initialized() else 1
        self.rank, self.world_size = rank, world_size
        counts = [int(np.prod(spec["grid"].shape if hasattr(spec["grid"], "shape")
                              else (spec["grid"].nx, spec["grid"].ny, spec["grid"].nz)))
                  for spec in specs]
        self.shares = partition_rooms(counts, world_size)
        self.local_rooms = self.shares[rank]
        self.local_index = {room: i for i, room in enumerate(self.local_rooms)}
        self.batch = make_batch([specs[r] for r in self.local_rooms]) if self.local_rooms else None
        self.local_cells = sum(counts[r] for r in self.local_rooms)

    def owns(self, room: int) -> bool:
        return room in self.local_index

    def add_volume_source(self, room: int, point, signal) -> None:
        if self.owns(room):
            self.batch.add_volume_source(self.local_index[room], point, signal)

    def add_pressure_receiver(self, room: int, point) -> None:
        if self.owns(room):
            self.batch.add_pressure_receiver(self.local_index[room], point)

    def run(self, n_steps: int) -> None:
        if self.batch is not None:
            self.batch.run(n_steps)

    def gather_recordings(self, dst: int = 0):
        """Every room's recordings, in room order, on rank ``dst`` (None elsewhere)."""
        import torch.distributed as dist

        local = {room: self.batch.recorded_pressure(self.local_index[room])
                 for room in self.local_rooms}
        if self.world_size == 1 or not dist.is_initialized():
            return [local[r] for r in sorted(local)]
        gathered = [None] * self.world_size if self.rank == dst else None
        dist.gather_object(local, gathered, dst=dst)
        if self.rank != dst:
            return None
        merged = {}
        for part in gathered:
            merged.update(part)
        return [merged[r] for r in sorted(merged)]
