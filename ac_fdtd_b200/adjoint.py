"""Gradients of receiver-signal losses by the hand-written adjoint kernels.

``DifferentiableRoom`` wraps one ``CudaAcousticFDTD``: ``forward`` runs the leapfrog while
recording what the parameter gradients need, ``backward`` takes dL/d(recordings) and runs the
transposed leapfrog backward in time on the GPU (``acf_adjoint_run``), returning gradients with
respect to

* the source signals (every sample),
* the wall admittances -- six per-wall values, or per patch for ``WallPatches`` walls,
* the ISO relaxation strengths Delta_r and times tau_r of the air,
* the initial pressure and velocity fields.

Walls and sources need only the pressure history on the boundary cells, kept for every step of
the forward run. The air needs the divergence and relaxation states of every cell at every
step. When that history fits in device memory the recorded run keeps it for every step;
otherwise it is recomputed segment by segment from full-state checkpoints taken every
``checkpoint_every`` steps (default ceil(sqrt(T))), because the lossy scheme cannot be run
backward stably. ``room_response`` exposes the same computation as a
``torch.autograd.Function``. The reference's solvers are not differentiable.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native
from .boundaries import FACES, WallAdmittances, patch_index
from .medium import AIR
from .solver import CudaAcousticFDTD, _as_double_pointer

__all__ = ["DifferentiableRoom", "DifferentiableBatch", "RoomGradients", "FixedProcesses",
           "room_response", "shell_face_gradients", "wall_gradients"]


class FixedProcesses:
    """Air given directly as relaxation processes (strength, relaxation time) per process."""

    def __init__(self, strengths, relaxation_times):
        from .air import RelaxationProcess

        self._processes = tuple(RelaxationProcess(float(s), float(t))
                                for s, t in zip(strengths, relaxation_times, strict=True))

    def processes(self, sound_speed, dt):
        return self._processes


@dataclass
class RoomGradients:
    signal: np.ndarray                       # (n_sources, n_steps)
    walls: np.ndarray | None = None          # (6,) for WallAdmittances, (6, P, P) for patches
    wall_cells: list | None = None           # dL/dxi at every cell of each face, six 2D maps
    strength: np.ndarray | None = None       # dL/dDelta_r
    relaxation_time: np.ndarray | None = None
    air_coefficients: dict = field(default_factory=dict)
    initial_p: np.ndarray | None = None


def _first_face_slots(shape):
    """For each face, the shell slot (face_off of first face + index) of every cell on it."""
    n = shape
    sizes = [n[1] * n[2], n[1] * n[2], n[0] * n[2], n[0] * n[2], n[0] * n[1], n[0] * n[1]]
    face_off = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    slots = []
    for axis, side in FACES:
        b, c = [a for a in range(3) if a != axis]
        coords = [None, None, None]
        coords[axis] = np.full((n[b], n[c]), 0 if side == 0 else n[axis] - 1)
        coords[b], coords[c] = np.meshgrid(np.arange(n[b]), np.arange(n[c]), indexing="ij")
        i, j, k = coords
        slot = np.full((n[b], n[c]), -1, dtype=np.int64)
        # first face in FACES order, as the kernels' shell_face does
        rules = [(i == 0, 0, j * n[2] + k), (i == n[0] - 1, 1, j * n[2] + k),
                 (j == 0, 2, i * n[2] + k), (j == n[1] - 1, 3, i * n[2] + k),
                 (k == 0, 4, i * n[1] + j), (k == n[2] - 1, 5, i * n[1] + j)]
        for mask, f, idx in rules:
            take = mask & (slot < 0)
            slot[take] = face_off[f] + idx[take]
        slots.append(slot)
    return slots


def shell_face_gradients(shape, grad_a, scale):
    """dL/dxi at every cell of each face from dL/da per shell slot (a = scale * sum xi)."""
    return [scale * grad_a[slot] for slot in _first_face_slots(shape)]


def wall_gradients(walls, shape, grad_a, sound_speed, dt, dx):
    """dL/dxi per wall (six values) or per patch ((6, P, P) for ``WallPatches``), and the
    per-cell maps, from dL/da per shell slot."""
    cells = shell_face_gradients(shape, grad_a, sound_speed * dt / (2.0 * dx))
    if hasattr(walls, "patch_values"):
        P = walls.patches
        g = np.zeros((6, P, P))
        for f, (axis, _) in enumerate(FACES):
            b, c = [a for a in range(3) if a != axis]
            ib = patch_index(shape[b], P)
            ic = patch_index(shape[c], P)
            np.add.at(g[f], (ib[:, None], ic[None, :]), cells[f])
        return g, cells
    return np.array([m.sum() for m in cells]), cells


def _air_chain(processes, c, rho, dx, dt, dgain, dmean, ddecay, dscale):
    """dL/dDelta_r and dL/dtau_r from the gradients of the scheme's relaxation coefficients.

    decay = exp(-dt/tau), mean = dt (tau/dt)(1 - decay), gain = rho c_r^2 Delta / dx with
    c_r^2 = c^2 / (1 + sum Delta), relax_scale = dt sum gain (scheme.py:166-191).
    """
    strength = np.array([p.strength for p in processes])
    tau = np.array([p.relaxation_time for p in processes])
    total = 1.0 + strength.sum()
    relaxed = c**2 / total
    d_relaxed = -c**2 / total**2                      # d relaxed / d Delta_k (any k)
    # d gain_r / d Delta_k = rho/dx (relaxed [r == k] + Delta_r d_relaxed)
    jac = rho / dx * (relaxed * np.eye(strength.size) + np.outer(strength, np.full(strength.size, d_relaxed)))
    dgain_total = dgain + dt * dscale                 # relax_scale = dt * sum(gain)
    d_strength = jac.T @ dgain_total
    decay = np.exp(-dt / tau)
    ddecay_dtau = decay * dt / tau**2
    dmean_dtau = (1.0 - decay) - tau * ddecay_dtau
    d_tau = ddecay * ddecay_dtau + dmean * dmean_dtau
    return d_strength, d_tau


class DifferentiableRoom:
    """One room whose receiver signals can be differentiated with the adjoint kernels."""

    def __init__(self, grid, medium=AIR, courant: float = 1.0, dtype=np.float32, walls=None,
                 absorbing_layer=None, air_absorption=None, *, max_steps: int,
                 wrt=("signal", "walls"), checkpoint_every: int | None = None) -> None:
        self.wrt = set(wrt)
        self.solver = CudaAcousticFDTD(grid, medium, courant, dtype, walls or WallAdmittances(),
                                       absorbing_layer, air_absorption,
                                       differentiable_walls="walls" in self.wrt,
                                       steps_per_graph=0)
        self.max_steps = int(max_steps)
        flags = 0
        if "walls" in self.wrt:
            flags |= _native.GRAD_WALLS
        if "air" in self.wrt:
            if self.solver.n_relax == 0:
                raise ValueError("air gradients need air absorption")
            flags |= _native.GRAD_AIR
        lib = self.solver._lib
        # None: the library keeps the whole D/psi history when it fits in device memory (no
        # recompute), else checkpoints every ceil(sqrt(max_steps)) steps.
        _native.check(lib.acf_adjoint_prepare(self.solver._handle, flags, self.max_steps,
                                              int(checkpoint_every or 0)), "acf_adjoint_prepare")
        self.checkpoint_every = int(lib.acf_adjoint_checkpoint_interval(self.solver._handle))
        self._shell_size = int(lib.acf_adjoint_shell_size(self.solver._handle))
        self.n_steps = 0

    @property
    def dt(self) -> float:
        return self.solver.dt

    def set_parameters(self, walls=None, air_absorption=None, absorbing_layer=None) -> None:
        self.solver.set_coefficients(walls if walls is not None else self.solver.walls,
                                     absorbing_layer if absorbing_layer is not None else self.solver.absorbing_layer,
                                     air_absorption if air_absorption is not None else self.solver.air_absorption)

    def forward(self, n_steps: int, p0=None) -> np.ndarray:
        """Run n_steps from rest (or from p0), recording the history; return the recordings."""
        if not 0 < n_steps <= self.max_steps:
            raise ValueError(f"n_steps must be in 1..{self.max_steps}")
        s = self.solver
        s.reset_state()
        if p0 is not None:
            s.set_state(p=p0)
        s.step_index = 0
        s._flush()
        s._push_points()
        _native.check(s._lib.acf_forward_record(s._handle, int(n_steps), 0, s._stream),
                      "acf_forward_record")
        s.step_index = int(n_steps)
        s._mirror_current.clear()
        self.n_steps = int(n_steps)
        return s.recorded_pressure

    def backward(self, grad_recordings) -> RoomGradients:
        s = self.solver
        n = self.n_steps
        grad = np.ascontiguousarray(grad_recordings, dtype=np.float64).reshape(len(s._receivers), n)
        n_src = len(s._sources)
        grad_src = np.zeros((n_src, n))
        grad_shell = np.zeros(self._shell_size) if "walls" in self.wrt else None
        n_air = 3 * s.n_relax + 1
        grad_air = np.zeros(n_air) if "air" in self.wrt else None

        def ptr(a):
            return None if a is None else _as_double_pointer(a)

        _native.check(s._lib.acf_adjoint_run(s._handle, ptr(grad), ptr(grad_src), ptr(grad_shell),
                                             ptr(grad_air), s._stream), "acf_adjoint_run")
        out = RoomGradients(signal=grad_src)
        block = s.coefficients
        c, rho = float(s.medium.sound_speed), float(s.medium.density)
        if grad_shell is not None:
            out.walls, out.wall_cells = wall_gradients(s.walls, block.shape, grad_shell, c,
                                                       block.dt, block.dx)
        if grad_air is not None:
            R = s.n_relax
            dgain, dmean, ddecay, dscale = grad_air[:R], grad_air[R:2 * R], grad_air[2 * R:3 * R], grad_air[3 * R]
            out.air_coefficients = dict(gain=dgain, mean=dmean, decay=ddecay, relax_scale=dscale)
            processes = s.air_absorption.processes(c, block.dt)
            out.strength, out.relaxation_time = _air_chain(processes, c, rho, block.dx, block.dt,
                                                           dgain, dmean, ddecay, dscale)
        p0 = np.empty(block.shape, dtype=s.dtype)
        _native.check(s._lib.acf_adjoint_download(s._handle, _native.FIELD_P, p0.ctypes.data,
                                                  s._stream), "acf_adjoint_download")
        out.initial_p = p0
        return out


class DifferentiableBatch:
    """Many rooms differentiated together: one batched forward and one batched adjoint per
    gradient, with every room's walls (per wall or per patch) and sources as parameters."""

    def __init__(self, rooms, dtype=np.float32, *, max_steps: int) -> None:
        from .batch import RoomBatch

        self.batch = RoomBatch(rooms, dtype=dtype, steps_per_graph=0, differentiable_walls=True)
        self.max_steps = int(max_steps)
        lib = self.batch._lib
        _native.check(lib.acf_batch_adjoint_prepare(self.batch._handle, self.max_steps),
                      "acf_batch_adjoint_prepare")
        self._shell_sizes = [int(lib.acf_batch_adjoint_shell_size(self.batch._handle, r))
                             for r in range(len(self.batch))]
        self.n_steps = 0

    def set_walls(self, room: int, walls) -> None:
        spec = self.batch.specs[room]
        self.batch.set_coefficients(room, walls, spec.get("absorbing_layer"),
                                    spec.get("air_absorption"))

    def forward(self, n_steps: int):
        """Run every room from rest for n_steps; return each room's recordings."""
        if not 0 < n_steps <= self.max_steps:
            raise ValueError(f"n_steps must be in 1..{self.max_steps}")
        b = self.batch
        b.reset_state()
        b.step_index = 0
        b._push_points()
        _native.check(b._lib.acf_batch_forward_record(b._handle, int(n_steps), 0, b._stream),
                      "acf_batch_forward_record")
        b.step_index = int(n_steps)
        self.n_steps = int(n_steps)
        return [b.recorded_pressure(r) for r in range(len(b))]

    def backward(self, grad_recordings) -> list[RoomGradients]:
        """Given dL/d(recordings) per room, the gradients of every room."""
        b = self.batch
        n = self.n_steps
        grad = np.ascontiguousarray(np.concatenate(
            [np.asarray(g, dtype=np.float64).reshape(len(b._receivers[r]), n)
             for r, g in enumerate(grad_recordings)], axis=0))
        n_src = sum(len(s) for s in b._sources)
        grad_src = np.zeros((max(n_src, 1), n))
        grad_shell = np.zeros(sum(self._shell_sizes))
        _native.check(b._lib.acf_batch_adjoint_run(b._handle, _as_double_pointer(grad),
                                                   _as_double_pointer(grad_src),
                                                   _as_double_pointer(grad_shell), b._stream),
                      "acf_batch_adjoint_run")
        out = []
        src_row = shell_at = 0
        for r in range(len(b)):
            block, spec = b.blocks[r], b.specs[r]
            medium = spec.get("medium", AIR)
            k = len(b._sources[r])
            g = RoomGradients(signal=grad_src[src_row:src_row + k])
            src_row += k
            shell = grad_shell[shell_at:shell_at + self._shell_sizes[r]]
            shell_at += self._shell_sizes[r]
            g.walls, g.wall_cells = wall_gradients(spec.get("walls") or WallAdmittances(),
                                                   block.shape, shell,
                                                   float(medium.sound_speed), block.dt, block.dx)
            out.append(g)
        return out


def room_response(room: DifferentiableRoom, source_point, xi, signal, n_steps: int):
    """Receiver recordings as a differentiable function of the six wall admittances ``xi`` and
    one source ``signal`` (torch tensors); gradients come from the adjoint kernels."""
    import torch

    class _Response(torch.autograd.Function):
        @staticmethod
        def forward(ctx, xi_t, signal_t):
            room.set_parameters(walls=WallAdmittances(*[float(v) for v in xi_t.detach().cpu()]))
            room.solver.clear_sources()
            room.solver.add_volume_source(source_point, signal_t.detach().cpu().numpy())
            return torch.as_tensor(room.forward(n_steps).astype(np.float64))

        @staticmethod
        def backward(ctx, grad_out):
            g = room.backward(grad_out.detach().cpu().numpy())
            return torch.as_tensor(g.walls), torch.as_tensor(g.signal[0])

    return _Response.apply(xi, signal)
