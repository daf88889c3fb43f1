"""``CudaAcousticFDTD``: the reference solver surface over the sm_100a kernels.

Same constructor, methods and properties as ac-fdtd's ``AcousticFDTD`` (``src/ac_fdtd/
scheme.py:82-389``) and ``CAcousticFDTD`` (``src/ac_fdtd/c_backend.py:160-382``): a caller swaps
the class and nothing else. The state lives on the GPU; ``p``, ``velocity`` and
``relaxation_states`` are host snapshots in pinned memory, refreshed from the device on every
access, and whatever is written into them is uploaded before the next ``run``. Arrays obtained
before a ``run`` are not updated by it: read the property again afterwards.

There is no CPU path. If the CUDA library cannot be loaded or no GPU is present, the
constructor raises.
"""

from __future__ import annotations

import ctypes
import weakref

import numpy as np

from . import _native
from .coefficients import room_coefficients
from .grid import cell_index
from .medium import AIR

__all__ = ["CudaAcousticFDTD", "DEFAULT_STEPS_PER_GRAPH", "pinned_array"]

#: Steps captured per CUDA graph for long runs; shorter runs launch step by step.
DEFAULT_STEPS_PER_GRAPH = 64


def _as_double_pointer(array: np.ndarray):
    return array.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def config_from_block(block):
    """Fill an ``acf_config`` from a coefficient block; returns it with the arrays it points to."""
    config = _native.AcfConfig()
    config.nx, config.ny, config.nz = block.shape
    config.precision = block.dtype.itemsize
    config.n_relax = block.n_relax
    config.vel_coef = block.vel_coef
    config.pres_coef = block.pres_coef
    config.src_coef = block.src_coef
    config.relax_scale = block.relax_scale
    for r in range(block.n_relax):
        config.relax_decay[r] = block.relax_decay[r]
        config.relax_mean[r] = block.relax_mean[r]
        config.relax_gain[r] = block.relax_gain[r]
    keep = []
    if block.wall_shell is not None:
        for f, shell in enumerate(block.wall_shell):
            keep.append(shell)
            config.wall_shell[f] = _as_double_pointer(shell)
    if block.layer_cell is not None:
        for a in range(3):
            keep += [block.layer_cell[a], block.layer_face[a]]
            config.cell[a] = _as_double_pointer(block.layer_cell[a])
            config.face[a] = _as_double_pointer(block.layer_face[a])
    return config, keep


def energy_from_terms(terms, medium, dx: float, dt: float) -> float:
    """The reference's energy (``scheme.py:365-389``) from the seven sums of ``acf_energy_terms``:
    dx^3 (sum p^2 / (2 rho c^2) + sum rho v^2 / 2 - dt/2 sum v . grad p)."""
    rho = float(medium.density)
    c = float(medium.sound_speed)
    potential = terms[0] / (2.0 * rho * c**2)
    kinetic = 0.0
    coupling = 0.0
    for axis in range(3):
        kinetic += 0.5 * rho * terms[1 + axis]
        coupling += terms[4 + axis]
    return dx**3 * (potential + kinetic - 0.5 * dt * coupling)


def _free_native(handle):
    if handle:
        _native.library().acf_destroy(handle)


class _PinnedBlock:
    """Pinned host memory owned by the numpy arrays that view it; freed with the last view."""

    def __init__(self, lib, shape, dtype: np.dtype):
        self._lib = lib
        self.pointer = ctypes.c_void_p()
        nbytes = int(np.prod(shape)) * dtype.itemsize
        _native.check(lib.acf_host_alloc(nbytes, ctypes.byref(self.pointer)), "acf_host_alloc")
        self.__array_interface__ = {
            "shape": tuple(shape), "typestr": dtype.str, "version": 3,
            "data": (self.pointer.value or 0, False),
        }

    def __del__(self):
        if self.pointer.value:
            self._lib.acf_host_free(self.pointer)
            self.pointer = ctypes.c_void_p()


def raise_for_status(word: int) -> None:
    """Turn a device status word (``acf_device_status``) into the error it reports."""
    if word & _native.STATUS_NON_FINITE:
        raise _native.NativeError(_native.ERR_NUMERIC, "acf_device_status",
                                  "a sweep produced a non-finite pressure (NaN or infinity); "
                                  "the state is not valid")
    if word & _native.STATUS_WAIT_TIMEOUT:
        raise _native.NativeError(_native.ERR_STATE, "acf_device_status",
                                  "a sweep timed out waiting (a staged sweep for its bulk "
                                  "copies, a two-step sweep for its neighbours); the solver "
                                  "state is not valid")


def pinned_array(shape, dtype=np.float32) -> np.ndarray:
    """A zeroed numpy array in page-locked host memory (full-speed host<->device copies)."""
    array = np.asarray(_PinnedBlock(_native.library(), tuple(shape), np.dtype(dtype)))
    array[...] = 0
    return array


class CudaAcousticFDTD:
    """The staggered pressure-velocity leapfrog on one B200, two fused sweeps per step.

    Args mirror ``AcousticFDTD.__init__`` (``scheme.py:107-116``); ``stream`` is an optional
    ``cudaStream_t`` handle (an int) to run on, and ``steps_per_graph`` the CUDA-graph chunk.
    """

    def __init__(self, grid, medium=AIR, courant: float = 1.0, dtype=np.float64, walls=None,
                 absorbing_layer=None, air_absorption=None, *, stream: int = 0,
                 steps_per_graph: int = DEFAULT_STEPS_PER_GRAPH,
                 differentiable_walls: bool = False, scheme: str = "two_sweeps",
                 device: int | None = None, coefficients=None) -> None:
        # ``coefficients``: a prepared block for ``grid`` (a slab of a larger room cuts its own
        # from the whole room's); otherwise built from the arguments as the reference does.
        if coefficients is None:
            block = room_coefficients(grid, medium, courant, dtype, walls, absorbing_layer,
                                      air_absorption, force_walls=differentiable_walls)
        else:
            block = coefficients
            if tuple(block.shape) != (int(grid.nx), int(grid.ny), int(grid.nz)):
                raise ValueError(f"coefficient block of shape {block.shape} for a grid of "
                                 f"{(grid.nx, grid.ny, grid.nz)}")
        self._force_walls = differentiable_walls
        self.grid = grid
        self.medium = medium
        self.courant = courant
        self.dtype = block.dtype
        self.walls = walls
        self.absorbing_layer = absorbing_layer
        self.air_absorption = air_absorption
        self.dt = block.dt
        self.step_index = 0
        self.coefficients = block
        self._shape = block.shape
        self._stream = ctypes.c_void_p(int(stream))

        self._lib = _native.library()
        count = ctypes.c_int(0)
        _native.check(self._lib.acf_device_count(ctypes.byref(count)), "acf_device_count")
        if count.value < 1:
            raise RuntimeError("no CUDA device is visible; the cuda backend has no CPU path")
        if device is not None:      # else the library's current device (0 unless set)
            _native.check(self._lib.acf_set_device(int(device)), "acf_set_device")

        config, keep = config_from_block(block)
        handle = ctypes.c_void_p()
        _native.check(self._lib.acf_create(ctypes.byref(config), ctypes.byref(handle)), "acf_create")
        self._handle = handle
        self._finalizer = weakref.finalize(self, _free_native, handle.value)
        _native.check(self._lib.acf_set_graph(handle, int(steps_per_graph)), "acf_set_graph")

        # Host snapshots: name -> ndarray, plus which are current and which were handed out.
        self._mirror: dict[int, np.ndarray] = {}
        self._mirror_current: set[int] = set()
        self._mirror_exposed: set[int] = set()

        self._sources: list[tuple[int, np.ndarray]] = []
        self._receivers: list[tuple[int, int]] = []  # (flat cell, start step)
        self._sources_dirty = False
        self._receivers_dirty = False
        self.set_scheme(scheme)

    # ------------------------------------------------------------------ geometry / time
    @property
    def time(self) -> float:
        return self.step_index * self.dt

    @property
    def sample_rate(self) -> float:
        return 1.0 / self.dt

    @property
    def n_relax(self) -> int:
        return self.coefficients.n_relax

    def _flat(self, point) -> int:
        index = cell_index(float(self.grid.dx), self._shape, point)
        return int(np.ravel_multi_index(index, self._shape))

    # ------------------------------------------------------------------ state mirrors
    def _field_shape(self, field: int) -> tuple[int, int, int]:
        shape = list(self._shape)
        if 1 <= field <= 3:
            shape[field - 1] += 1
        return tuple(shape)

    def _mirror_array(self, field: int) -> np.ndarray:
        if field not in self._mirror:
            block = _PinnedBlock(self._lib, self._field_shape(field), self.dtype)
            self._mirror[field] = np.asarray(block)
        return self._mirror[field]

    def _pull(self, fields) -> None:
        pending = [f for f in fields if f not in self._mirror_current]
        for f in pending:
            array = self._mirror_array(f)
            _native.check(self._lib.acf_download(self._handle, f, array.ctypes.data, self._stream),
                          "acf_download")
        if pending:
            self.synchronize()
            self._mirror_current.update(pending)

    def _flush(self) -> None:
        """Upload every snapshot the caller may have written since it was handed out."""
        if not self._mirror_exposed:
            return
        for f in sorted(self._mirror_exposed):
            array = self._mirror[f]
            _native.check(self._lib.acf_upload(self._handle, f, array.ctypes.data, self._stream),
                          "acf_upload")
        # The copies read pinned memory asynchronously; finish them before the caller can
        # write into the snapshots again.
        self.synchronize()
        self._mirror_exposed.clear()

    def _expose(self, fields) -> list[np.ndarray]:
        self._pull(fields)
        self._mirror_exposed.update(fields)
        return [self._mirror[f] for f in fields]

    @property
    def p(self) -> np.ndarray:
        """Pressure p^n, shape (nx, ny, nz); a writable host snapshot."""
        return self._expose([_native.FIELD_P])[0]

    @p.setter
    def p(self, value) -> None:
        self.p[...] = value

    @property
    def velocity(self) -> list[np.ndarray]:
        """[vx, vy, vz] at n - 1/2, shapes from ``Grid.velocity_shape``; writable snapshots."""
        return self._expose([_native.FIELD_VX, _native.FIELD_VY, _native.FIELD_VZ])

    @property
    def vx(self) -> np.ndarray:
        return self._expose([_native.FIELD_VX])[0]

    @property
    def vy(self) -> np.ndarray:
        return self._expose([_native.FIELD_VY])[0]

    @property
    def vz(self) -> np.ndarray:
        return self._expose([_native.FIELD_VZ])[0]

    def set_state(self, p=None, velocity=None, relaxation=None) -> int:
        """Upload state straight from caller arrays (reference layout, solver dtype).

        Arrays in pinned memory (see :func:`pinned_array`) move at full link speed. Returns the
        number of bytes copied host to device.
        """
        self._flush()
        items = []
        if p is not None:
            items.append((_native.FIELD_P, p))
        if velocity is not None:
            items += [(_native.FIELD_VX + a, v) for a, v in enumerate(velocity)]
        if relaxation is not None:
            if len(relaxation) != self.n_relax:
                raise ValueError(f"expected {self.n_relax} relaxation states, got {len(relaxation)}")
            items += [(_native.FIELD_PSI0 + r, s) for r, s in enumerate(relaxation)]
        total = 0
        keep = []
        for field, array in items:
            array = np.ascontiguousarray(array, dtype=self.dtype)
            if array.shape != self._field_shape(field):
                raise ValueError(f"field {field}: shape {array.shape}, expected {self._field_shape(field)}")
            keep.append(array)
            _native.check(self._lib.acf_upload(self._handle, field, array.ctypes.data, self._stream),
                          "acf_upload")
            self._mirror_current.discard(field)
            total += array.nbytes
        self.synchronize()
        return total

    def reset_state(self) -> None:
        """Put the room at rest: p, v and the relaxation states to zero, on the device."""
        self._pressure_only_started = False
        self._mirror_exposed -= {_native.FIELD_VX, _native.FIELD_VY, _native.FIELD_VZ}
        self._flush()
        _native.check(self._lib.acf_reset_state(self._handle, self._stream), "acf_reset_state")
        self._mirror_current.clear()

    def get_state(self, p=None, velocity=None) -> int:
        """Download p and/or the velocities into caller arrays; returns bytes copied."""
        self._flush()
        items = []
        if p is not None:
            items.append((_native.FIELD_P, p))
        if velocity is not None:
            items += [(_native.FIELD_VX + a, v) for a, v in enumerate(velocity)]
        total = 0
        for field, array in items:
            if (array.shape != self._field_shape(field) or array.dtype != self.dtype
                    or not array.flags.c_contiguous):
                raise ValueError(f"field {field}: need a C-contiguous {self.dtype} array of shape "
                                 f"{self._field_shape(field)}")
            _native.check(self._lib.acf_download(self._handle, field, array.ctypes.data, self._stream),
                          "acf_download")
            total += array.nbytes
        self.synchronize()
        return total

    @property
    def relaxation_states(self) -> list[np.ndarray]:
        """The ISO relaxation states psi_r, one (nx, ny, nz) snapshot per process."""
        return self._expose([_native.FIELD_PSI0 + r for r in range(self.n_relax)])

    # ------------------------------------------------------------------ sources / receivers
    def add_volume_source(self, point, signal) -> None:
        """Soft volume source at the cell containing ``point`` (``scheme.py:231-244``)."""
        values = np.asarray(signal, dtype=self.dtype).reshape(-1)
        self._sources.append((self._flat(point), values))
        self._sources_dirty = True

    def clear_sources(self) -> None:
        """Remove every volume source (receivers and state are kept)."""
        self._sources = []
        self._sources_dirty = True

    def add_pressure_receiver(self, point) -> int:
        """Record p at ``point`` after every step from now on (``scheme.py:246-255``)."""
        self._receivers.append((self._flat(point), self.step_index))
        self._receivers_dirty = True
        return len(self._receivers) - 1

    def add_volume_source_at(self, cell, signal) -> None:
        """``add_volume_source`` for the cell with index ``(i, j, k)``."""
        values = np.asarray(signal, dtype=self.dtype).reshape(-1)
        self._sources.append((int(np.ravel_multi_index(tuple(int(c) for c in cell), self._shape)),
                              values))
        self._sources_dirty = True

    def add_pressure_receiver_at(self, cell) -> int:
        """``add_pressure_receiver`` for the cell with index ``(i, j, k)``."""
        flat = int(np.ravel_multi_index(tuple(int(c) for c in cell), self._shape))
        self._receivers.append((flat, self.step_index))
        self._receivers_dirty = True
        return len(self._receivers) - 1

    def _push_points(self) -> None:
        if self._sources_dirty:
            n = len(self._sources)
            stride = max((s.size for _, s in self._sources), default=0)
            cells = np.array([c for c, _ in self._sources], dtype=np.int64)
            lengths = np.array([s.size for _, s in self._sources], dtype=np.int64)
            signals = np.zeros((n, max(stride, 1)), dtype=np.float64)
            for q, (_, s) in enumerate(self._sources):
                signals[q, : s.size] = s
            _native.check(self._lib.acf_set_sources(
                self._handle, n, cells.ctypes.data_as(_native._I64P),
                lengths.ctypes.data_as(_native._I64P), _as_double_pointer(signals), stride),
                "acf_set_sources")
            self._sources_dirty = False
        if self._receivers_dirty:
            cells = np.array([c for c, _ in self._receivers], dtype=np.int64)
            starts = np.array([s for _, s in self._receivers], dtype=np.int64)
            _native.check(self._lib.acf_set_receivers(
                self._handle, len(self._receivers), cells.ctypes.data_as(_native._I64P),
                starts.ctypes.data_as(_native._I64P)), "acf_set_receivers")
            self._receivers_dirty = False

    @property
    def recorded_pressure(self) -> np.ndarray:
        """Every receiver's samples as ``(channel, sample)`` (``scheme.py:257-262``).

        Like the reference, receivers added part-way through have fewer samples, and asking
        for a ragged set raises instead of padding.
        """
        if not self._receivers:
            return np.zeros((0, 0))
        self._push_points()
        rows = []
        for r, (_, start) in enumerate(self._receivers):
            n = self.step_index - start
            row = np.empty(n, dtype=self.dtype)
            if n > 0:
                _native.check(self._lib.acf_read_recording(
                    self._handle, r, start, n, row.ctypes.data, self._stream), "acf_read_recording")
            rows.append(row)
        if len({row.size for row in rows}) > 1:
            raise ValueError(
                "receivers were added at different steps, so their recordings have different "
                f"lengths {[row.size for row in rows]}; read them one by one with recording(r)"
            )
        return np.stack(rows)

    def recorded_pressure_device(self):
        """``recorded_pressure`` as a CUDA tensor ``(channel, sample)`` in the solver's dtype,
        copied device to device (for post-processing on the GPU; ``postprocess``)."""
        import torch

        self._push_points()
        starts = {start for _, start in self._receivers}
        if len(starts) > 1:
            raise ValueError("receivers were added at different steps; their recordings are ragged")
        n = self.step_index - (starts.pop() if starts else 0)
        dtype = torch.float64 if self.dtype == np.float64 else torch.float32
        out = torch.empty((len(self._receivers), max(n, 0)), dtype=dtype,
                          device=f"cuda:{self.device}")
        for r, (_, start) in enumerate(self._receivers):
            if n > 0:
                _native.check(self._lib.acf_read_recording(
                    self._handle, r, start, n, out[r].data_ptr(), self._stream), "acf_read_recording")
        return out

    def recording(self, receiver: int) -> np.ndarray:
        """Samples of one receiver since it was added."""
        self._push_points()
        _, start = self._receivers[receiver]
        n = self.step_index - start
        row = np.empty(n, dtype=self.dtype)
        if n > 0:
            _native.check(self._lib.acf_read_recording(
                self._handle, receiver, start, n, row.ctypes.data, self._stream),
                "acf_read_recording")
        return row

    def probe_pressure(self, point) -> float:
        return float(self.p[cell_index(float(self.grid.dx), self._shape, point)])

    def probe_velocity(self, point, axis: int) -> float:
        return float(self.velocity[axis][cell_index(float(self.grid.dx), self._shape, point)])

    # ------------------------------------------------------------------ stepping
    def run(self, n_steps: int) -> None:
        """Advance ``n_steps`` on the GPU; asynchronous with respect to the host."""
        n_steps = int(n_steps)
        if n_steps <= 0:
            return
        self._flush()
        self._push_points()
        _native.check(self._lib.acf_run(self._handle, n_steps, self.step_index, self._stream),
                      "acf_run")
        self.step_index += n_steps
        self._mirror_current.clear()
        if self.scheme == "pressure_only":      # no velocities are kept from here on
            self._mirror_exposed -= {_native.FIELD_VX, _native.FIELD_VY, _native.FIELD_VZ}
            self._pressure_only_started = True

    def step(self) -> None:
        self.run(1)

    def flush(self) -> None:
        """Upload what was written into the host snapshots now (``run`` does it by itself)."""
        self._flush()

    def prepare_points(self) -> None:
        """Push added sources and receivers to the device now (``run`` does it by itself); for
        callers that advance the solver through another entry point (``acf_run_slabs``)."""
        self._push_points()

    def advanced(self, n_steps: int) -> None:
        """Record that another entry point advanced this solver by ``n_steps``."""
        self.step_index += int(n_steps)
        self._mirror_current.clear()

    @property
    def device(self) -> int:
        """The GPU this solver's state lives on."""
        return int(self._lib.acf_solver_device(self._handle))

    def field_pointer(self, field: int) -> tuple[int, tuple[int, int, int]]:
        """Device address of a field in the padded layout and its (x, y, z) element strides;
        valid until the next ``run`` (the fused schemes alternate between two copies)."""
        pointer = ctypes.c_void_p()
        strides = (ctypes.c_int64 * 3)()
        _native.check(self._lib.acf_field_pointer(self._handle, int(field), ctypes.byref(pointer),
                                                  strides), "acf_field_pointer")
        return int(pointer.value or 0), (int(strides[0]), int(strides[1]), int(strides[2]))

    def synchronize(self) -> None:
        """Wait for the device, then raise if a sweep reported a non-finite pressure or a
        staged sweep gave up waiting (``check_device``)."""
        _native.check(self._lib.acf_synchronize(self._stream), "acf_synchronize")
        self.check_device()

    def check_device(self) -> None:
        """Raise :class:`~ac_fdtd_b200._native.NativeError` if a sweep produced a non-finite
        pressure (status ``ACF_ERR_NUMERIC``) or a staged sweep gave up waiting for its copies
        (``ACF_ERR_STATE``); the state is then not valid. Clears the device's report."""
        status = ctypes.c_int32(0)
        _native.check(self._lib.acf_device_status(self._handle, ctypes.byref(status)),
                      "acf_device_status")
        raise_for_status(status.value)

    # ------------------------------------------------------------------ diagnostics
    def energy_terms(self, planes: tuple[int, int] | None = None,
                     far_face: bool = True) -> np.ndarray:
        """The seven FP64 device sums behind :meth:`energy` (see ``acf_energy_terms``);
        ``planes=(x_begin, x_end)`` restricts them to those x planes (``far_face``: with the
        face nx when x_end = nx), as a slab of a larger room needs."""
        self._flush()
        terms = np.zeros(7)
        if planes is None:
            _native.check(self._lib.acf_energy_terms(self._handle, float(self.grid.dx),
                                                     _as_double_pointer(terms), self._stream),
                          "acf_energy_terms")
        else:
            _native.check(self._lib.acf_energy_terms_planes(
                self._handle, float(self.grid.dx), int(planes[0]), int(planes[1]),
                int(bool(far_face)), _as_double_pointer(terms), self._stream),
                "acf_energy_terms_planes")
        return terms

    def energy(self) -> float:
        """Acoustic energy of the stored (p^n, v^{n-1/2}) pair in joules (``scheme.py:365-389``).

        The sums are accumulated in FP64 on the device in either precision.
        """
        if self.scheme == "pressure_only" and getattr(self, "_pressure_only_started", False):
            return self.pressure_only_energy()
        return energy_from_terms(self.energy_terms(), self.medium, float(self.grid.dx), self.dt)

    def pressure_only_energy(self) -> float:
        """The pressure-only scheme's conserved energy after its latest step, in joules:
        dx^3 / (2 rho c^2) (sum (p^{n+1} - p^n)^2 / lam2 - sum p^{n+1} L p^n), lam2 = c_p c_v
        and L the rigid-face Laplacian (``acf_pressure_only_energy_terms``). Constant with rigid
        walls, non-increasing with impedance walls and no sources."""
        self._flush()
        terms = np.zeros(2)
        _native.check(self._lib.acf_pressure_only_energy_terms(
            self._handle, _as_double_pointer(terms), self._stream), "acf_pressure_only_energy_terms")
        block = self.coefficients
        lam2 = float(np.dtype(self.dtype).type(block.vel_coef * block.pres_coef))
        rho, c = float(self.medium.density), float(self.medium.sound_speed)
        return float(self.grid.dx) ** 3 / (2.0 * rho * c**2) * (terms[0] / lam2 - terms[1])

    def set_coefficients(self, walls=None, absorbing_layer=None, air_absorption=None) -> None:
        """Replace the wall, layer and air coefficients, keeping the grid and the state.

        The new set must have the same relaxation count and the same presence of walls and
        layer as the one the solver was built with.
        """
        block = room_coefficients(self.grid, self.medium, self.courant, self.dtype, walls,
                                  absorbing_layer, air_absorption, force_walls=self._force_walls)
        config, keep = config_from_block(block)
        _native.check(self._lib.acf_set_coefficients(self._handle, ctypes.byref(config)),
                      "acf_set_coefficients")
        del keep
        self.walls, self.absorbing_layer, self.air_absorption = walls, absorbing_layer, air_absorption
        self.coefficients = block

    SCHEMES = {"two_sweeps": _native.SCHEME_TWO_SWEEPS, "fused": _native.SCHEME_FUSED,
               "staged": _native.SCHEME_FUSED_STAGED,
               "pressure_only": _native.SCHEME_PRESSURE_ONLY}

    def set_scheme(self, scheme: str) -> None:
        """``"two_sweeps"`` (velocity sweep, then pressure sweep, in place), ``"fused"`` (one
        sweep into a second copy of p and v) or ``"staged"`` (the fused sweep with its inputs
        streamed into shared memory by bulk copies). Results are bit-identical; the fused steps
        move (8 + 2R) elements per cell instead of (12 + 2R) and need four more fields of
        memory. ``"pressure_only"``: the second-order wave equation on p alone (rigid or
        impedance walls, no absorbing layer or air absorption), 3 elements per cell and step;
        its first step is the p-v step from the state as it stands, so pressures and recordings
        equal the other schemes' to rounding, and from then on no velocities are kept
        (``velocity`` raises; ``energy`` is the scheme's own conserved quadratic form)."""
        if scheme not in self.SCHEMES:
            raise ValueError(f"scheme must be one of {sorted(self.SCHEMES)}, got {scheme!r}")
        if scheme == "pressure_only" and (self.coefficients.layer_cell is not None
                                          or self.n_relax > 0):
            raise ValueError("the pressure-only scheme has no absorbing layer or air absorption: "
                             "the second-order pressure equation keeps no velocity or relaxation "
                             "state for them")
        self._flush()
        _native.check(self._lib.acf_set_scheme(self._handle, self.SCHEMES[scheme]), "acf_set_scheme")
        if scheme == "pressure_only" and getattr(self, "scheme", None) != "pressure_only":
            self._pressure_only_started = False
        self.scheme = scheme
        self._mirror_current.clear()

    def set_prefetch(self, enabled: bool | None = None) -> None:
        """L2 prefetch of each next x plane in the marching kernels: ``None`` (default) turns
        it on when the fields a step streams exceed the GPU's L2, ``True``/``False`` force it.
        Results never depend on it."""
        mode = -1 if enabled is None else int(bool(enabled))
        _native.check(self._lib.acf_set_prefetch(self._handle, mode), "acf_set_prefetch")

    @property
    def prefetch(self) -> bool:
        """Whether the L2 prefetch is in effect for this room."""
        return self._lib.acf_get_prefetch(self._handle) == 1

    def set_time_blocking(self, steps_per_launch: int = 2) -> None:
        """Steps per launch of the fused single-precision sweep: 2 takes every x plane through
        two steps in one sweep (temporal blocking: the state is read and written once per two
        steps), 1 goes back to one step per launch. Results are identical either way. Needs
        float32 and nz a multiple of 4 (``NativeError`` otherwise); takes effect while the
        scheme is ``"fused"``."""
        _native.check(self._lib.acf_set_time_blocking(self._handle, int(steps_per_launch)),
                      "acf_set_time_blocking")

    @property
    def time_blocking(self) -> int:
        """Steps per launch of the fused sweep (1 or 2)."""
        return self._lib.acf_get_time_blocking(self._handle)

    def set_launch(self, block_threads: int = 256, planes: int = 4) -> None:
        """Launch geometry of the sweeps (threads per block, x planes per block)."""
        _native.check(self._lib.acf_set_launch(self._handle, int(block_threads), int(planes)),
                      "acf_set_launch")

    def set_staging(self, rows: int = 2, stages: int = 0, planes: int | None = None,
                    vector: int = 4) -> None:
        """Geometry of the staged scheme: y rows per CTA, ring buffers (0: automatic), z
        elements per thread (2 or 4) and, if given, x planes per CTA (which also sets 128
        threads per block for the other schemes)."""
        _native.check(self._lib.acf_set_staging(self._handle, int(rows), int(stages), int(vector)),
                      "acf_set_staging")
        if planes is not None:
            _native.check(self._lib.acf_set_launch(self._handle, 128, int(planes)),
                          "acf_set_launch")

    def launch_count(self) -> int:
        return int(self._lib.acf_launch_count(self._handle))

    def profile(self, enable: bool) -> None:
        """Time each sweep with CUDA events during subsequent runs (step-by-step launches)."""
        _native.check(self._lib.acf_profile_enable(self._handle, int(bool(enable))),
                      "acf_profile_enable")

    def profile_read(self) -> tuple[float, float, int]:
        """(velocity-sweep ms, pressure-sweep ms, steps timed) since profiling was enabled."""
        a, b, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        _native.check(self._lib.acf_profile_read(self._handle, ctypes.byref(a), ctypes.byref(b),
                                                 ctypes.byref(n)), "acf_profile_read")
        return a.value, b.value, n.value

    def close(self) -> None:
        """Release the device state now instead of at garbage collection."""
        self._finalizer()
        self._mirror.clear()
