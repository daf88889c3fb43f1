"""The x-slab decomposition of one room, on the CPU: slab ranges, the coefficient blocks the
parts are built from (checked cell by cell against the whole room), and the ghost exchange
schedule over gloo ranks (a stencil run in slabs equals the whole-array run bit for bit)."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ac_fdtd_b200 import AIR, AbsorbingLayer, AirAbsorption, Grid, WallAdmittances
from ac_fdtd_b200.boundaries import FACES
from ac_fdtd_b200.coefficients import room_coefficients
from ac_fdtd_b200.slabs import slab_coefficients, slab_ranges


def test_slab_ranges_cover_the_room_evenly():
    for nx, parts in ((10, 1), (10, 3), (7, 7), (384, 8), (385, 8)):
        ranges = slab_ranges(nx, parts)
        assert ranges[0][0] == 0 and ranges[-1][1] == nx
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
        sizes = [x1 - x0 for x0, x1 in ranges]
        assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    for nx, parts in ((3, 4), (5, 0)):
        with pytest.raises(ValueError):
            slab_ranges(nx, parts)


def _pair_used(shells, shape, cell):
    """The wall pair the pressure sweep applies at ``cell``: the entry of the first face, in
    FACES order, that the cell lies on (as the kernel's shell lookup does), or None."""
    n = shape
    for face, (axis, side) in enumerate(FACES):
        if cell[axis] != (0 if side == 0 else n[axis] - 1):
            continue
        b, c = [a for a in range(3) if a != axis]
        pairs = shells[face].reshape(n[b], n[c], 2)
        return tuple(pairs[cell[b], cell[c]])
    return None


@pytest.mark.parametrize("parts", [2, 3, 9])
def test_every_owned_cell_gets_the_rooms_wall_pair_and_layer_profiles(parts):
    grid = Grid(dx=0.05, nx=9, ny=5, nz=6)
    block = room_coefficients(grid, AIR, 1.0, np.float64,
                              WallAdmittances(0.3, 0.1, 0.7, 0.0, 0.2, 0.5),
                              AbsorbingLayer(thickness=3, faces=((0, 0), (0, 1), (2, 1))),
                              AirAbsorption())
    shape = block.shape
    for x0, x1 in slab_ranges(shape[0], parts):
        local, gx0 = slab_coefficients(block, x0, x1)
        ghosts = (x0 > 0) + (x1 < shape[0])
        assert local.shape == (x1 - x0 + ghosts, shape[1], shape[2])
        assert gx0 == (x0 - 1 if x0 > 0 else 0)
        gx1 = gx0 + local.shape[0]
        np.testing.assert_array_equal(local.layer_cell[0], block.layer_cell[0][gx0:gx1])
        np.testing.assert_array_equal(local.layer_face[0], block.layer_face[0][gx0:gx1 + 1])
        for a in (1, 2):
            np.testing.assert_array_equal(local.layer_cell[a], block.layer_cell[a])
            np.testing.assert_array_equal(local.layer_face[a], block.layer_face[a])
        for i in range(x0, x1):
            for j in range(shape[1]):
                for k in range(shape[2]):
                    want = _pair_used(block.wall_shell, shape, (i, j, k))
                    got = _pair_used(local.wall_shell, local.shape, (i - gx0, j, k))
                    assert got == want, (x0, x1, i, j, k)
        # scalars travel unchanged
        assert (local.vel_coef, local.pres_coef, local.src_coef, local.relax_scale, local.dt) == \
            (block.vel_coef, block.pres_coef, block.src_coef, block.relax_scale, block.dt)


def test_walls_given_per_patch_cut_cell_by_cell_too():
    from ac_fdtd_b200.boundaries import WallPatches

    grid = Grid(dx=0.05, nx=8, ny=6, nz=7)
    patches = WallPatches(np.random.default_rng(3).uniform(0.0, 0.8, (6, 3, 3)))
    block = room_coefficients(grid, AIR, 1.0, np.float32, patches)
    for x0, x1 in slab_ranges(grid.nx, 3):
        local, gx0 = slab_coefficients(block, x0, x1)
        for i in range(x0, x1):
            for j in range(grid.ny):
                for k in range(grid.nz):
                    assert _pair_used(local.wall_shell, local.shape, (i - gx0, j, k)) == \
                        _pair_used(block.wall_shell, block.shape, (i, j, k))


def test_rigid_rooms_and_rooms_without_layer_cut_too():
    block = room_coefficients(Grid(dx=0.05, nx=6, ny=3, nz=4), AIR, 1.0, np.float32)
    local, gx0 = slab_coefficients(block, 2, 4)
    assert local.wall_shell is None and local.layer_cell is None
    assert local.shape == (4, 3, 4) and gx0 == 1
    with pytest.raises(ValueError):
        slab_coefficients(block, 4, 7)


# ---------------------------------------------------------------- the exchange over gloo

def _stencil(u, steps):
    """A whole-array explicit 1-D diffusion along x with fixed zero ends (float64)."""
    u = u.copy()
    for _ in range(steps):
        padded = np.concatenate([np.zeros((1,) + u.shape[1:]), u, np.zeros((1,) + u.shape[1:])])
        u = padded[1:-1] + 0.25 * ((padded[:-2] - padded[1:-1]) + (padded[2:] - padded[1:-1]))
    return u


def _exchange_worker(rank, world, port, u0, steps, queue):
    import torch
    import torch.distributed as dist

    from ac_fdtd_b200.slabs import exchange_ghosts

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        x0, x1 = slab_ranges(u0.shape[0], world)[rank]
        # local array: [left ghost] owned planes [right ghost]; ghosts at the room's ends stay 0
        left, right = x0 > 0, x1 < u0.shape[0]
        local = torch.zeros((x1 - x0 + 2,) + u0.shape[1:], dtype=torch.float64)
        local[1:-1] = torch.from_numpy(u0[x0:x1])

        def exchange():
            exchange_ghosts(local[1], local[-2], local[0] if left else None,
                            local[-1] if right else None, rank, world)

        exchange()
        for _ in range(steps):
            inner = local[1:-1] + 0.25 * ((local[:-2] - local[1:-1]) + (local[2:] - local[1:-1]))
            local[1:-1] = inner
            exchange()
        queue.put((rank, x0, local[1:-1].numpy().copy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_exchanging_ghost_planes_reproduce_the_whole_array(world):
    u0 = np.random.default_rng(world).standard_normal((11, 4, 3))
    steps = 7
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_exchange_worker, args=(rank, world, port, u0, steps, queue))
             for rank in range(world)]
    for p in procs:
        p.start()
    parts = sorted(queue.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assembled = np.concatenate([part for _, _, part in parts])
    np.testing.assert_array_equal(assembled, _stencil(u0, steps))


# ---------------------------------------------------------------- point routing (stub ABI)

@pytest.fixture
def stub(monkeypatch):
    from ac_fdtd_b200 import _native
    from tests.test_host_logic import StubLibrary

    lib = StubLibrary()
    monkeypatch.setattr(_native, "_lib", lib)
    monkeypatch.setattr(_native, "library", lambda: lib)
    return lib


def test_points_go_to_the_part_owning_their_cell(stub):
    from ac_fdtd_b200.slabs import SlabGroup

    grid = Grid(dx=0.05, nx=10, ny=4, nz=5)
    group = SlabGroup(grid, dtype=np.float32, parts=3, walls=WallAdmittances.uniform(0.2))
    assert [(s.x0, s.x1, s.gx0) for s in group.slabs] == [(0, 4, 0), (4, 7, 3), (7, 10, 6)]
    assert [s.solver.coefficients.shape[0] for s in group.slabs] == [5, 5, 4]
    for x, part in ((0.0, 0), (0.199, 0), (0.2, 1), (0.349, 1), (0.35, 2), (0.5, 2), (9.0, 2)):
        owners = [s.owned_cell((x, 0.1, 0.1)) for s in group.slabs]
        assert [q for q, c in enumerate(owners) if c is not None] == [part], x
        i = grid.cell_index((x, 0.1, 0.1))[0]
        assert owners[part] == (i - group.slabs[part].gx0, 2, 2)
    receivers = [group.add_pressure_receiver((x, 0.1, 0.1)) for x in (0.46, 0.01, 0.3)]
    assert receivers == [0, 1, 2]
    assert group._receivers == [(2, 0), (0, 0), (1, 0)]
    group.add_volume_source((0.26, 0.1, 0.1), np.ones(3))
    assert [len(s.solver._sources) for s in group.slabs] == [0, 1, 0]
    flat, _ = group.slabs[1].solver._sources[0]
    assert np.unravel_index(flat, group.slabs[1].solver._shape) == (2, 2, 2)
