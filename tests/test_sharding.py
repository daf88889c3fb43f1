"""Sharding independent rooms over ranks: the balance rule, and the gather across two gloo
processes on the CPU (a stand-in batch replaces the GPU one; the data path has no collective)."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ac_fdtd_b200 import Grid
from ac_fdtd_b200.sharding import ShardedRooms, partition_rooms


def test_partition_is_balanced_complete_and_deterministic():
    rng = np.random.default_rng(0)
    counts = rng.integers(60, 200, 64) ** 3
    for world in (1, 2, 3, 4, 8):
        shares = partition_rooms(counts, world)
        assert sorted(r for share in shares for r in share) == list(range(64))
        loads = [sum(counts[r] for r in share) for share in shares]
        # LPT: the largest share is within 4/3 of the ideal, and here much closer.
        assert max(loads) <= 4 / 3 * max(counts.sum() / world, counts.max())
        assert shares == partition_rooms(counts, world)
    assert partition_rooms([5, 1, 1], 4)[3] == []


class FakeBatch:
    """Stands in for RoomBatch: recordings are a function of the room and step count."""

    def __init__(self, specs):
        self.specs = specs
        self.steps = 0
        self.receivers = [[] for _ in specs]

    def add_volume_source(self, room, point, signal):
        pass

    def add_pressure_receiver(self, room, point):
        self.receivers[room].append(point)

    def run(self, n):
        self.steps += n

    def recorded_pressure(self, room):
        tag = self.specs[room]["tag"]
        return np.full((len(self.receivers[room]), self.steps), float(tag))


def _worker(rank, world, port, specs, queue):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sharded = ShardedRooms(specs, FakeBatch)
        for room in range(len(specs)):
            sharded.add_pressure_receiver(room, (0.1, 0.1, 0.1))
        sharded.run(5)
        result = sharded.gather_recordings(dst=0)
        queue.put((rank, sharded.local_rooms, None if result is None else [r.tolist() for r in result]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_gather_every_room_in_order():
    specs = [dict(grid=Grid(dx=0.05, nx=n, ny=n, nz=n), tag=t)
             for t, n in enumerate((9, 4, 7, 5, 8, 3))]
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(rank, 2, port, specs, queue)) for rank in range(2)]
    for p in procs:
        p.start()
    results = {}
    for _ in procs:
        rank, rooms, gathered = queue.get(timeout=120)
        results[rank] = (rooms, gathered)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(results[0][0] + results[1][0]) == list(range(6))
    assert results[1][1] is None
    gathered = results[0][1]
    assert len(gathered) == 6
    for room, rec in enumerate(gathered):
        assert np.array(rec).shape == (1, 5)
        assert np.all(np.array(rec) == room)
