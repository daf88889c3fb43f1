"""One room cut into x slabs over several GPUs, with a ghost-plane exchange every step.

A room larger than one GPU's memory, or one wanted faster than one GPU runs it, is cut along x
into contiguous slabs of planes, one per part. Each part's solver holds its own planes plus one
ghost plane on each side that has a neighbour. Its coefficients are the whole room's, cut to
those planes: wall pairs on the room's own x faces only (neutral pairs (1, 0) on a cut), layer
profiles at their positions in the whole room. Every owned cell and face therefore performs
the single-room arithmetic, and the owned planes equal a one-GPU run of the room bit for bit.

After every step each part sends its first owned p plane to the left neighbour's right ghost
and its last owned p plane to the right neighbour's left ghost. The next velocity sweep then
computes every owned face, including the two faces shared with ghosts, from current pressures,
so only pressure planes travel: (ny + 1) x pz elements each way per cut and step (604 KB at
384^2 fp32 in the padded layout). Nothing owned reads a ghost cell except that pressure, in
the velocity sweep; where the sweeps also update ghost cells (the copy path), the exchange
overwrites them before the next step.

Two ways to run the parts:

* ``SlabGroup`` -- every part in this process (one GPU or several). With the two-sweep and the
  fused schemes the exchange is part of the step: each part's pressure update stores its first
  and last own planes straight into the neighbours' ghost planes (peer stores across GPUs,
  ``acf_run_slabs``), and the steps are ordered so that no kernel waits on another; the staged
  scheme copies the ghost planes after each step (``acf_copy_plane``);
* ``DistributedSlabRoom`` -- this rank's part, one process per GPU, planes exchanged by
  ``exchange_ghosts`` over ``torch.distributed`` (NCCL between GPUs; gloo in the CPU tests).

The reference runs one room in one shared-memory process; the slab decomposition is this
backend's addition. Energy sums each part's owned cells and faces on its GPU
(``acf_energy_terms_planes``) and adds the seven sums over the parts.
"""

from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _native
from .boundaries import FACES
from .coefficients import room_coefficients
from .grid import Grid, cell_index
from .medium import AIR
from .solver import CudaAcousticFDTD, energy_from_terms

__all__ = ["slab_ranges", "slab_coefficients", "SlabRoom", "SlabGroup", "DistributedSlabRoom",
           "exchange_ghosts"]

_P_FIELD = 0


def slab_ranges(nx: int, parts: int) -> list[tuple[int, int]]:
    """Contiguous x-plane ranges [x0, x1) of ``parts`` slabs, sizes differing by at most one."""
    nx, parts = int(nx), int(parts)
    if parts < 1 or parts > nx:
        raise ValueError(f"cannot cut {nx} x planes into {parts} slabs")
    base, extra = divmod(nx, parts)
    ranges, x0 = [], 0
    for part in range(parts):
        x1 = x0 + base + (1 if part < extra else 0)
        ranges.append((x0, x1))
        x0 = x1
    return ranges


def slab_coefficients(block, x0: int, x1: int):
    """The coefficient block of the planes [x0, x1) of a room, with its ghost planes.

    Returns ``(local_block, gx0)``: the local grid covers the room's planes [gx0, gx1), one more
    on each side that has a neighbour. Wall pairs of the y and z faces and the x layer profiles
    are the room's entries for those planes; an x face keeps the room's pairs only where it is
    the room's own wall, and is neutral (1, 0) on a cut.
    """
    nx, ny, nz = block.shape
    if not 0 <= x0 < x1 <= nx:
        raise ValueError(f"slab [{x0}, {x1}) outside the room's {nx} x planes")
    gx0 = x0 - 1 if x0 > 0 else 0
    gx1 = x1 + 1 if x1 < nx else nx
    local = dataclasses.replace(block, shape=(gx1 - gx0, ny, nz))
    if block.wall_shell is not None:
        shells = []
        for face, (axis, side) in enumerate(FACES):
            pairs = block.wall_shell[face]
            if axis == 0:
                on_wall = (side == 0 and gx0 == 0) or (side == 1 and gx1 == nx)
                if on_wall:
                    shells.append(pairs.copy())
                else:
                    neutral = np.zeros((ny, nz, 2))
                    neutral[..., 0] = 1.0
                    shells.append(neutral.reshape(-1))
            else:
                across = nz if axis == 1 else ny       # the face's other axis besides x
                cut = pairs.reshape(nx, across, 2)[gx0:gx1]
                shells.append(np.ascontiguousarray(cut).reshape(-1))
        local.wall_shell = shells
    if block.layer_cell is not None:
        local.layer_cell = [np.ascontiguousarray(block.layer_cell[0][gx0:gx1])] + \
            [a.copy() for a in block.layer_cell[1:]]
        local.layer_face = [np.ascontiguousarray(block.layer_face[0][gx0:gx1 + 1])] + \
            [a.copy() for a in block.layer_face[1:]]
    return local, gx0


class SlabRoom:
    """The planes [x0, x1) of a room (part ``part`` of ``parts``), with their ghost planes.

    The room is described by the arguments of ``CudaAcousticFDTD``; points are given in the
    room's coordinates and belong to the part whose planes hold their cell.
    """

    def __init__(self, grid, medium=AIR, courant: float = 1.0, dtype=np.float64, walls=None,
                 absorbing_layer=None, air_absorption=None, *, part: int, parts: int,
                 device: int | None = None, scheme: str = "two_sweeps") -> None:
        block = room_coefficients(grid, medium, courant, dtype, walls, absorbing_layer,
                                  air_absorption)
        self.room_shape = block.shape
        self.dx = float(grid.dx)
        self.part, self.parts = int(part), int(parts)
        self.x0, self.x1 = slab_ranges(block.shape[0], parts)[part]
        local, self.gx0 = slab_coefficients(block, self.x0, self.x1)
        self.has_left = self.x0 > 0
        self.has_right = self.x1 < block.shape[0]
        nx, ny, nz = local.shape
        self.solver = CudaAcousticFDTD(Grid(dx=self.dx, nx=nx, ny=ny, nz=nz), medium, courant,
                                       dtype, walls, absorbing_layer, air_absorption,
                                       device=device, scheme=scheme, coefficients=local)
        self.dt = self.solver.dt
        self.dtype = self.solver.dtype

    # local x planes (every field has nx + 1 of them; p uses the first nx)
    @property
    def first_owned(self) -> int:
        return self.x0 - self.gx0

    @property
    def last_owned(self) -> int:
        return self.x1 - 1 - self.gx0

    @property
    def left_ghost(self) -> int:
        return 0

    @property
    def right_ghost(self) -> int:
        return self.x1 - self.gx0

    def owned_cell(self, point):
        """Local (i, j, k) of the cell holding ``point``, or None when another part owns it."""
        i, j, k = cell_index(self.dx, self.room_shape, point)
        if not self.x0 <= i < self.x1:
            return None
        return (i - self.gx0, j, k)

    def add_volume_source(self, point, signal) -> bool:
        """Add the source here if this part owns its cell; returns whether it did."""
        cell = self.owned_cell(point)
        if cell is not None:
            self.solver.add_volume_source_at(cell, signal)
        return cell is not None

    def add_pressure_receiver(self, point) -> int | None:
        """Local receiver index if this part owns the point's cell, else None."""
        cell = self.owned_cell(point)
        return None if cell is None else self.solver.add_pressure_receiver_at(cell)

    def energy_terms(self) -> np.ndarray:
        """The seven energy sums over this part's owned cells and faces (the room's far x face
        on the last part); the parts' sums add up to the whole room's."""
        return self.solver.energy_terms(planes=(self.first_owned, self.last_owned + 1),
                                        far_face=not self.has_right)

    def plane_view(self, plane: int):
        """A torch tensor over local p plane ``plane`` in device memory (no copy)."""
        import torch

        pointer, strides = self.solver.field_pointer(_P_FIELD)
        count = int(strides[0])
        address = pointer + plane * count * self.dtype.itemsize
        return torch.as_tensor(_DeviceArray(address, count, self.dtype),
                               device=f"cuda:{self.solver.device}")

    def owned(self, array: np.ndarray, faces: bool = False) -> np.ndarray:
        """The owned x range of a local field snapshot (``faces``: x faces, with the room's far
        face on the last part)."""
        hi = self.x1 - self.gx0 + (1 if faces and not self.has_right else 0)
        return array[self.x0 - self.gx0: hi]

    def close(self) -> None:
        self.solver.close()


class _DeviceArray:
    """A one-dimensional device buffer described by the CUDA array interface."""

    def __init__(self, address: int, count: int, dtype: np.dtype):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": np.dtype(dtype).str,
                                         "data": (int(address), False), "version": 3,
                                         "strides": None}


class _SlabSet:
    """Fields assembled over a list of parts (every part, or this rank's)."""

    slabs: list[SlabRoom]

    def _assemble(self, getter, faces: bool = False) -> np.ndarray:
        return np.concatenate([s.owned(getter(s), faces) for s in self.slabs], axis=0)


class SlabGroup(_SlabSet):
    """Every part of one room in this process, stepped in lockstep.

    With the two-sweep scheme the ghost exchange is part of each pressure sweep (peer stores,
    ``acf_run_slabs``); with the others the ghost planes are copied after each step.
    ``devices`` (optional) lists the GPU of each part (cycled); by default all parts share the
    library's current device. Results equal ``CudaAcousticFDTD`` on the whole room bit for bit.
    """

    def __init__(self, grid, medium=AIR, courant: float = 1.0, dtype=np.float64, walls=None,
                 absorbing_layer=None, air_absorption=None, *, parts: int, devices=None,
                 scheme: str = "two_sweeps") -> None:
        self.slabs = [SlabRoom(grid, medium, courant, dtype, walls, absorbing_layer,
                               air_absorption, part=q, parts=parts,
                               device=None if not devices else devices[q % len(devices)],
                               scheme=scheme)
                      for q in range(parts)]
        self.dt = self.slabs[0].dt
        self._lib = _native.library()
        self._receivers: list[tuple[int, int]] = []   # (part, local receiver)
        self._several_devices = len({s.solver.device for s in self.slabs}) > 1

    @property
    def step_index(self) -> int:
        return self.slabs[0].solver.step_index

    def add_volume_source(self, point, signal) -> None:
        owners = [s.add_volume_source(point, signal) for s in self.slabs]
        if sum(owners) != 1:
            raise RuntimeError(f"point {point} is owned by {sum(owners)} parts, not one")

    def add_pressure_receiver(self, point) -> int:
        for q, s in enumerate(self.slabs):
            local = s.add_pressure_receiver(point)
            if local is not None:
                self._receivers.append((q, local))
                return len(self._receivers) - 1
        raise RuntimeError(f"point {point} is owned by no part")

    def _copy(self, dst: SlabRoom, dst_plane: int, src: SlabRoom, src_plane: int) -> None:
        _native.check(self._lib.acf_copy_plane(dst.solver._handle, dst_plane, src.solver._handle,
                                               src_plane, _P_FIELD, None), "acf_copy_plane")

    def exchange(self) -> None:
        """Refresh every ghost p plane from its owner."""
        if self._several_devices:
            for s in self.slabs:
                s.solver.synchronize()
        for left, right in zip(self.slabs, self.slabs[1:]):
            self._copy(right, right.left_ghost, left, left.last_owned)
            self._copy(left, left.right_ghost, right, right.first_owned)
        if self._several_devices:
            for s in self.slabs:
                s.solver.synchronize()

    def run(self, n_steps: int) -> None:
        """Advance every part. With the two-sweep or the fused scheme each step's pressure update
        also stores the boundary planes into the neighbours' ghost planes (``acf_run_slabs``: no
        exchange step; the fused steps replay from a CUDA graph on one GPU); the staged scheme
        steps part by part and copies the ghost planes after each step."""
        n_steps = int(n_steps)
        if n_steps <= 0:
            return
        for s in self.slabs:
            s.solver.flush()      # state written on the host reaches the device first
        self.exchange()           # ghost planes from the current state
        if all(s.solver.scheme in ("two_sweeps", "fused") for s in self.slabs) and \
                len({s.solver.scheme for s in self.slabs}) == 1:
            n = len(self.slabs)
            for s in self.slabs:
                s.solver.prepare_points()
            handles = (ctypes.c_void_p * n)(*[s.solver._handle.value for s in self.slabs])
            own_lo = (ctypes.c_int32 * n)(*[s.first_owned for s in self.slabs])
            own_hi = (ctypes.c_int32 * n)(*[s.last_owned + 1 for s in self.slabs])
            _native.check(self._lib.acf_run_slabs(handles, n, own_lo, own_hi, n_steps,
                                                  self.step_index, None), "acf_run_slabs")
            for s in self.slabs:
                s.solver.advanced(n_steps)
            return
        for _ in range(n_steps):
            for s in self.slabs:
                s.solver.run(1)
            self.exchange()

    def synchronize(self) -> None:
        for s in self.slabs:
            s.solver.synchronize()

    def energy(self) -> float:
        """The whole room's acoustic energy (``CudaAcousticFDTD.energy``), from every part's sums."""
        solver = self.slabs[0].solver
        if self._several_devices:
            # The last pressure sweep of a part stores into its neighbours' ghost planes from
            # the neighbour's GPU; each part's sums read its ghost p plane on its own stream,
            # which nothing orders after those peer stores. Finish every GPU's work first.
            self.synchronize()
        terms = np.sum([s.energy_terms() for s in self.slabs], axis=0)
        return energy_from_terms(terms, solver.medium, float(solver.grid.dx), self.dt)

    @property
    def p(self) -> np.ndarray:
        return self._assemble(lambda s: s.solver.p)

    @property
    def velocity(self) -> list[np.ndarray]:
        return [self._assemble(lambda s: s.solver.velocity[0], faces=True),
                self._assemble(lambda s: s.solver.velocity[1]),
                self._assemble(lambda s: s.solver.velocity[2])]

    def recording(self, receiver: int) -> np.ndarray:
        part, local = self._receivers[receiver]
        return self.slabs[part].solver.recording(local)

    @property
    def recorded_pressure(self) -> np.ndarray:
        return np.stack([self.recording(r) for r in range(len(self._receivers))]) \
            if self._receivers else np.zeros((0, self.step_index), dtype=self.slabs[0].dtype)

    def close(self) -> None:
        for s in self.slabs:
            s.close()


def exchange_ghosts(first_owned, last_owned, left_ghost, right_ghost, rank: int, world: int,
                    group=None) -> None:
    """One ghost exchange of the x-slab decomposition over ``torch.distributed``.

    Rank r sends ``first_owned`` to r - 1 and ``last_owned`` to r + 1, and receives r - 1's last
    plane into ``left_ghost`` and r + 1's first into ``right_ghost``. The four operations of a
    rank go out as one batch, so neighbours never wait on each other in a cycle (with NCCL a
    single group launch); it returns when they are complete. Tensors absent at the room's ends
    may be None.
    """
    import torch.distributed as dist

    ops = []
    if rank > 0:
        ops.append(dist.P2POp(dist.isend, first_owned, rank - 1, group))
        ops.append(dist.P2POp(dist.irecv, left_ghost, rank - 1, group))
    if rank < world - 1:
        ops.append(dist.P2POp(dist.isend, last_owned, rank + 1, group))
        ops.append(dist.P2POp(dist.irecv, right_ghost, rank + 1, group))
    if ops:
        for request in dist.batch_isend_irecv(ops):
            request.wait()


class DistributedSlabRoom(_SlabSet):
    """This rank's part of a room cut into one slab per rank (one process per GPU).

    The process group must be initialised; ``device`` is this rank's GPU (default: the
    library's current device -- pass the local rank unless CUDA_VISIBLE_DEVICES already narrows
    the process to one GPU). Recordings stay with the rank that owns each receiver;
    ``gather_recordings`` brings them to one rank.
    """

    def __init__(self, grid, medium=AIR, courant: float = 1.0, dtype=np.float64, walls=None,
                 absorbing_layer=None, air_absorption=None, *, device: int | None = None,
                 group=None, scheme: str = "two_sweeps") -> None:
        import torch
        import torch.distributed as dist

        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.slab = SlabRoom(grid, medium, courant, dtype, walls, absorbing_layer, air_absorption,
                             part=self.rank, parts=self.world, device=device, scheme=scheme)
        # NCCL's point-to-point calls run on torch's current device: make it this part's GPU.
        torch.cuda.set_device(self.slab.solver.device)
        self.slabs = [self.slab]
        self.dt = self.slab.dt
        self._receivers: list[int | None] = []

    @property
    def step_index(self) -> int:
        return self.slab.solver.step_index

    def add_volume_source(self, point, signal) -> bool:
        return self.slab.add_volume_source(point, signal)

    def add_pressure_receiver(self, point) -> int:
        """Global receiver index (the same on every rank); this rank records it if it owns it."""
        self._receivers.append(self.slab.add_pressure_receiver(point))
        return len(self._receivers) - 1

    def exchange(self) -> None:
        """Refresh both ghost planes from the neighbours. With NCCL nothing waits on the host:
        the solver and NCCL's calls are ordered on the device (the solver runs on the legacy
        default stream, torch's current stream, which NCCL's stream waits for before the
        transfer and which waits for the transfer before the next step). Other backends move
        host-visible data, so the device is synchronised around them."""
        import torch
        import torch.distributed as dist

        if self.world == 1:
            return
        s = self.slab
        on_device = dist.get_backend(self.group) == "nccl" and s.solver._stream.value in (None, 0)
        if not on_device:
            s.solver.synchronize()
        # Views over the current copy of p (the fused schemes alternate between two copies).
        planes = (s.plane_view(s.first_owned), s.plane_view(s.last_owned),
                  s.plane_view(s.left_ghost) if s.has_left else None,
                  s.plane_view(s.right_ghost) if s.has_right else None)
        exchange_ghosts(*planes, self.rank, self.world, self.group)
        if not on_device:
            torch.cuda.synchronize(s.solver.device)

    def run(self, n_steps: int) -> None:
        n_steps = int(n_steps)
        if n_steps <= 0:
            return
        self.slab.solver.flush()
        if self.world == 1:              # no cut: the whole room, in CUDA graphs
            self.slab.solver.run(n_steps)
            return
        self.exchange()
        for _ in range(n_steps):
            self.slab.solver.run(1)
            self.exchange()

    @property
    def p(self) -> np.ndarray:
        """This rank's owned planes of p."""
        return self._assemble(lambda s: s.solver.p)

    def energy(self) -> float:
        """The whole room's acoustic energy: every rank's sums, all-reduced (collective)."""
        import torch
        import torch.distributed as dist

        terms = torch.tensor(self.slab.energy_terms(), dtype=torch.float64)
        if dist.get_backend(self.group) == "nccl":
            terms = terms.cuda(self.slab.solver.device)
        dist.all_reduce(terms, group=self.group)
        solver = self.slab.solver
        return energy_from_terms(terms.cpu().numpy(), solver.medium, float(solver.grid.dx),
                                 self.dt)

    def gather_recordings(self, dst: int = 0) -> np.ndarray | None:
        """Every receiver's recording on rank ``dst`` (None elsewhere)."""
        import torch.distributed as dist

        mine = {r: self.slab.solver.recording(local)
                for r, local in enumerate(self._receivers) if local is not None}
        gathered = [None] * self.world if self.rank == dst else None
        dist.gather_object(mine, gathered, dst=dst, group=self.group)
        if self.rank != dst:
            return None
        merged = {}
        for part in gathered:
            merged.update(part)
        return np.stack([merged[r] for r in range(len(self._receivers))]) if merged else None

    def close(self) -> None:
        self.slab.close()

