"""``RoomBatch``: many rooms of different sizes advanced together on one GPU.

Each room is described by the arguments of ``CudaAcousticFDTD`` (grid, medium, courant, walls,
absorbing_layer, air_absorption); all rooms share the precision and the number of ISO
relaxation processes and step in lockstep. Each sweep is a single launch over a flat tile
table that covers every room (one CTA per tile, or a persistent grid striding over the table):
two launches a step with ``scheme="two_sweeps"``, one with ``scheme="fused"`` (the velocity and
pressure updates of a step in one sweep, ping-ponging the fields as ``CudaAcousticFDTD`` does
with the same scheme). Long runs replay CUDA graphs of those launches. Per room, the arithmetic
is exactly that of the single-room solver, so every room's fields and recordings equal a
``CudaAcousticFDTD`` run of that room alone, bit for bit, under either scheme.

The reference solves one room per solver object (``src/ac_fdtd/scheme.py:82``); batching is
this backend's addition for workloads of many rooms or many source positions.
"""

from __future__ import annotations

import ctypes
import weakref

import numpy as np

from . import _native
from .coefficients import room_coefficients
from .grid import cell_index
from .medium import AIR
from .solver import DEFAULT_STEPS_PER_GRAPH, _as_double_pointer, raise_for_status

__all__ = ["RoomBatch"]


def _free_batch(handle):
    if handle:
        _native.library().acf_batch_destroy(handle)


class RoomBatch:
    """A batch of rooms; ``rooms`` is a list of dicts of ``CudaAcousticFDTD`` arguments."""

    def __init__(self, rooms, dtype=np.float32, *, stream: int = 0,
                 steps_per_graph: int = DEFAULT_STEPS_PER_GRAPH,
                 differentiable_walls: bool = False, scheme: str = "two_sweeps",
                 device: int | None = None) -> None:
        if not rooms:
            raise ValueError("a batch needs at least one room")
        self.dtype = np.dtype(dtype)
        self._lib = _native.library()
        count = ctypes.c_int(0)
        _native.check(self._lib.acf_device_count(ctypes.byref(count)), "acf_device_count")
        if count.value < 1:
            raise RuntimeError("no CUDA device is visible; the cuda backend has no CPU path")
        if device is not None:      # else the library's current device (0 unless set)
            _native.check(self._lib.acf_set_device(int(device)), "acf_set_device")
        self.specs = [dict(room) for room in rooms]
        self.blocks = []
        self._force_walls = differentiable_walls
        configs = (_native.AcfConfig * len(rooms))()
        keep = []
        for r, spec in enumerate(self.specs):
            block = room_coefficients(spec["grid"], spec.get("medium", AIR),
                                      spec.get("courant", 1.0), self.dtype, spec.get("walls"),
                                      spec.get("absorbing_layer"), spec.get("air_absorption"),
                                      force_walls=differentiable_walls)
            self.blocks.append(block)
            config = configs[r]
            config.nx, config.ny, config.nz = block.shape
            config.precision = self.dtype.itemsize
            config.n_relax = block.n_relax
            config.vel_coef = block.vel_coef
            config.pres_coef = block.pres_coef
            config.src_coef = block.src_coef
            config.relax_scale = block.relax_scale
            for q in range(block.n_relax):
                config.relax_decay[q] = block.relax_decay[q]
                config.relax_mean[q] = block.relax_mean[q]
                config.relax_gain[q] = block.relax_gain[q]
            if block.wall_shell is not None:
                for f, shell in enumerate(block.wall_shell):
                    keep.append(shell)
                    config.wall_shell[f] = _as_double_pointer(shell)
            if block.layer_cell is not None:
                for a in range(3):
                    keep += [block.layer_cell[a], block.layer_face[a]]
                    config.cell[a] = _as_double_pointer(block.layer_cell[a])
                    config.face[a] = _as_double_pointer(block.layer_face[a])
        handle = ctypes.c_void_p()
        _native.check(self._lib.acf_batch_create(len(rooms), configs, ctypes.byref(handle)),
                      "acf_batch_create")
        self._handle = handle
        self._finalizer = weakref.finalize(self, _free_batch, handle.value)
        self._stream = ctypes.c_void_p(int(stream))
        _native.check(self._lib.acf_batch_set_graph(handle, int(steps_per_graph)),
                      "acf_batch_set_graph")
        self.step_index = 0
        self._sources = [[] for _ in rooms]
        self._receivers = [[] for _ in rooms]
        self._dirty_sources: set[int] = set()
        self._dirty_receivers: set[int] = set()
        self.scheme = "two_sweeps"
        self.set_scheme(scheme)

    # ------------------------------------------------------------------ geometry
    def __len__(self) -> int:
        return len(self.specs)

    @property
    def shapes(self):
        return [block.shape for block in self.blocks]

    @property
    def n_cells(self) -> int:
        return int(sum(np.prod(s) for s in self.shapes))

    def dt(self, room: int) -> float:
        return self.blocks[room].dt

    def _flat(self, room: int, point) -> int:
        block = self.blocks[room]
        return int(np.ravel_multi_index(cell_index(block.dx, block.shape, point), block.shape))

    # ------------------------------------------------------------------ points
    def add_volume_source(self, room: int, point, signal) -> None:
        self._sources[room].append((self._flat(room, point),
                                    np.asarray(signal, dtype=self.dtype).reshape(-1)))
        self._dirty_sources.add(room)

    def add_pressure_receiver(self, room: int, point) -> int:
        self._receivers[room].append((self._flat(room, point), self.step_index))
        self._dirty_receivers.add(room)
        return len(self._receivers[room]) - 1

    def _push_points(self) -> None:
        for room in sorted(self._dirty_sources):
            sources = self._sources[room]
            stride = max((s.size for _, s in sources), default=0)
            cells = np.array([c for c, _ in sources], dtype=np.int64)
            lengths = np.array([s.size for _, s in sources], dtype=np.int64)
            signals = np.zeros((len(sources), max(stride, 1)))
            for q, (_, s) in enumerate(sources):
                signals[q, : s.size] = s
            _native.check(self._lib.acf_batch_set_sources(
                self._handle, room, len(sources), cells.ctypes.data_as(_native._I64P),
                lengths.ctypes.data_as(_native._I64P), _as_double_pointer(signals), stride),
                "acf_batch_set_sources")
        self._dirty_sources.clear()
        for room in sorted(self._dirty_receivers):
            receivers = self._receivers[room]
            cells = np.array([c for c, _ in receivers], dtype=np.int64)
            starts = np.array([s for _, s in receivers], dtype=np.int64)
            _native.check(self._lib.acf_batch_set_receivers(
                self._handle, room, len(receivers), cells.ctypes.data_as(_native._I64P),
                starts.ctypes.data_as(_native._I64P)), "acf_batch_set_receivers")
        self._dirty_receivers.clear()

    def recording(self, room: int, receiver: int) -> np.ndarray:
        self._push_points()
        _, start = self._receivers[room][receiver]
        n = self.step_index - start
        row = np.empty(n, dtype=self.dtype)
        if n > 0:
            _native.check(self._lib.acf_batch_read_recording(
                self._handle, room, receiver, start, n, row.ctypes.data, self._stream),
                "acf_batch_read_recording")
        return row

    def recorded_pressure(self, room: int) -> np.ndarray:
        rows = [self.recording(room, r) for r in range(len(self._receivers[room]))]
        if not rows:
            return np.zeros((0, 0))
        if len({row.size for row in rows}) > 1:
            raise ValueError("receivers of this room were added at different steps")
        return np.stack(rows)

    # ------------------------------------------------------------------ state
    def _shape(self, room: int, field: int):
        shape = list(self.blocks[room].shape)
        if 1 <= field <= 3:
            shape[field - 1] += 1
        return tuple(shape)

    def get_field(self, room: int, field: int) -> np.ndarray:
        out = np.empty(self._shape(room, field), dtype=self.dtype)
        _native.check(self._lib.acf_batch_download(self._handle, room, field, out.ctypes.data,
                                                   self._stream), "acf_batch_download")
        self.synchronize()
        return out

    def set_field(self, room: int, field: int, values) -> None:
        array = np.ascontiguousarray(values, dtype=self.dtype)
        if array.shape != self._shape(room, field):
            raise ValueError(f"shape {array.shape}, expected {self._shape(room, field)}")
        _native.check(self._lib.acf_batch_upload(self._handle, room, field, array.ctypes.data,
                                                 self._stream), "acf_batch_upload")
        self.synchronize()

    def p(self, room: int) -> np.ndarray:
        return self.get_field(room, _native.FIELD_P)

    def velocity(self, room: int) -> list[np.ndarray]:
        return [self.get_field(room, _native.FIELD_VX + a) for a in range(3)]

    # ------------------------------------------------------------------ stepping
    def run(self, n_steps: int) -> None:
        n_steps = int(n_steps)
        if n_steps <= 0:
            return
        self._push_points()
        _native.check(self._lib.acf_batch_run(self._handle, n_steps, self.step_index,
                                              self._stream), "acf_batch_run")
        self.step_index += n_steps

    def set_coefficients(self, room: int, walls=None, absorbing_layer=None,
                         air_absorption=None) -> None:
        """Replace one room's walls, layer and air (same grid, relaxation count and features)."""
        from .solver import config_from_block

        spec = self.specs[room]
        block = room_coefficients(spec["grid"], spec.get("medium", AIR), spec.get("courant", 1.0),
                                  self.dtype, walls, absorbing_layer, air_absorption,
                                  force_walls=self._force_walls)
        config, keep = config_from_block(block)
        _native.check(self._lib.acf_batch_set_coefficients(self._handle, room, ctypes.byref(config)),
                      "acf_batch_set_coefficients")
        del keep
        spec.update(walls=walls, absorbing_layer=absorbing_layer, air_absorption=air_absorption)
        self.blocks[room] = block

    SCHEMES = {"two_sweeps": _native.SCHEME_TWO_SWEEPS, "fused": _native.SCHEME_FUSED}

    def set_scheme(self, scheme: str) -> None:
        """``"two_sweeps"`` (a velocity launch and a pressure launch per step, in place) or
        ``"fused"`` (one launch per step into a second copy of every room's p and v, (8 + 2R)
        instead of (12 + 2R) elements moved per cell). Results are bit-identical."""
        if scheme not in self.SCHEMES:
            raise ValueError(f"scheme must be one of {sorted(self.SCHEMES)}, got {scheme!r}")
        _native.check(self._lib.acf_batch_set_scheme(self._handle, self.SCHEMES[scheme]),
                      "acf_batch_set_scheme")
        self.scheme = scheme

    def set_prefetch(self, enabled: bool | None = None) -> None:
        """L2 prefetch of each next x plane: ``None`` (default) turns it on when every room's
        fields together exceed the GPU's L2, ``True``/``False`` force it. Results never depend
        on it."""
        mode = -1 if enabled is None else int(bool(enabled))
        _native.check(self._lib.acf_batch_set_prefetch(self._handle, mode),
                      "acf_batch_set_prefetch")

    def reset_state(self) -> None:
        """Every room at rest (all fields zero), on the device."""
        _native.check(self._lib.acf_batch_reset_state(self._handle, self._stream),
                      "acf_batch_reset_state")

    def synchronize(self) -> None:
        """Wait for the device, then raise if a sweep of any room produced a non-finite
        pressure (``ACF_ERR_NUMERIC``); the batch's state is then not valid."""
        _native.check(self._lib.acf_synchronize(self._stream), "acf_synchronize")
        status = ctypes.c_int32(0)
        _native.check(self._lib.acf_batch_device_status(self._handle, ctypes.byref(status)),
                      "acf_batch_device_status")
        raise_for_status(status.value)

    def set_launch(self, block_threads: int = 128, planes: int = 8, ctas_per_sm: int = 0) -> None:
        _native.check(self._lib.acf_batch_set_launch(self._handle, int(block_threads), int(planes),
                                                     int(ctas_per_sm)), "acf_batch_set_launch")

    def energy(self, room: int) -> float:
        terms = np.zeros(7)
        block = self.blocks[room]
        _native.check(self._lib.acf_batch_energy_terms(self._handle, room, block.dx,
                                                       _as_double_pointer(terms), self._stream),
                      "acf_batch_energy_terms")
        medium = self.specs[room].get("medium", AIR)
        rho, c = float(medium.density), float(medium.sound_speed)
        potential = terms[0] / (2.0 * rho * c**2)
        kinetic = sum(0.5 * rho * terms[1 + a] for a in range(3))
        coupling = sum(terms[4 + a] for a in range(3))
        return block.dx**3 * (potential + kinetic - 0.5 * block.dt * coupling)

    def profile(self, enable: bool) -> None:
        _native.check(self._lib.acf_batch_profile_enable(self._handle, int(bool(enable))),
                      "acf_batch_profile_enable")

    def profile_read(self) -> tuple[float, float, int]:
        a, b, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        _native.check(self._lib.acf_batch_profile_read(self._handle, ctypes.byref(a),
                                                       ctypes.byref(b), ctypes.byref(n)),
                      "acf_batch_profile_read")
        return a.value, b.value, n.value

    def launch_count(self) -> int:
        return int(self._lib.acf_batch_launch_count(self._handle))

    def close(self) -> None:
        self._finalizer()
