"""ORACLE -- test infrastructure only: drives the reference's compiled C backend.

``oracle/Makefile`` compiles ac-fdtd's ``src/ac_fdtd/c/acfdtd.c`` unmodified into
``oracle/_ref/acfdtd_{f32,f64}.so``. This module is a ctypes driver of that library, with the
setup of the reference's own driver ``src/ac_fdtd/c_backend.py:170-356`` (coefficients rounded
from FP64, relaxation scale from the FP64 gain sum, all-ones profiles without a layer). It is
the CPU baseline and the reference arm of ``bench.py``; it never runs in the product path.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

from .leapfrog import oracle_cell_index, oracle_layer_factors, oracle_processes, oracle_wall_list

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
MAX_RELAX = 4
_libs: dict[str, ctypes.CDLL] = {}


def library_path(dtype) -> Path:
    return REF_DIR / f"acfdtd_{'f64' if np.dtype(dtype) == np.float64 else 'f32'}.so"


def available() -> bool:
    return library_path(np.float64).exists() and library_path(np.float32).exists()


def build(reference: str | None = None) -> bool:
    """Compile the reference C backend from the ac-fdtd checkout at ``reference`` (default: the
    ``AC_FDTD_REFERENCE`` environment variable) if its sources are there; True if the libraries
    exist afterwards. Without a checkout, only libraries built earlier count."""
    reference = reference or os.environ.get("AC_FDTD_REFERENCE")
    if reference and Path(reference, "src/ac_fdtd/c/acfdtd.c").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), f"REFERENCE={reference}"], check=True,
                       capture_output=True)
    return available()


def _struct(dtype):
    real = ctypes.c_double if np.dtype(dtype) == np.float64 else ctypes.c_float
    rp = ctypes.POINTER(real)
    ip = ctypes.POINTER(ctypes.c_int64)

    class State(ctypes.Structure):  # field order of acfdtd.c:56-97
        _fields_ = [
            ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
            ("n_relax", ctypes.c_int32), ("n_wall", ctypes.c_int64), ("n_sources", ctypes.c_int64),
            ("n_receivers", ctypes.c_int64), ("n_steps", ctypes.c_int64),
            ("source_length", ctypes.c_int64),
            ("vel_coef", real), ("pres_coef", real), ("src_coef", real), ("relax_scale", real),
            ("p", rp), ("vx", rp), ("vy", rp), ("vz", rp), ("psi", rp),
            ("relax_decay", real * MAX_RELAX), ("relax_mean", real * MAX_RELAX),
            ("relax_gain", real * MAX_RELAX),
            ("cell", rp * 3), ("face", rp * 3), ("has_layer", ctypes.c_int32),
            ("wall_index", ip), ("wall_from_updated", rp), ("wall_from_previous", rp),
            ("wall_scratch", rp), ("source_index", ip), ("source_signal", rp),
            ("receiver_index", ip), ("recording", rp),
        ]

    return State, real


def _library(dtype) -> ctypes.CDLL:
    key = str(np.dtype(dtype))
    if key not in _libs:
        lib = ctypes.CDLL(str(library_path(dtype)))
        lib.acfdtd_struct_size.restype = ctypes.c_size_t
        lib.acfdtd_set_threads.restype = ctypes.c_int
        lib.acfdtd_set_threads.argtypes = [ctypes.c_int]
        lib.acfdtd_thread_count.restype = ctypes.c_int
        lib.acfdtd_run.restype = None
        lib.acfdtd_run.argtypes = [ctypes.c_void_p, ctypes.c_int64]
        State, _ = _struct(dtype)
        if lib.acfdtd_struct_size() != ctypes.sizeof(State):
            raise RuntimeError("ctypes mirror of the reference acfdtd struct does not match")
        _libs[key] = lib
    return _libs[key]


class RefCSolver:
    """The reference C time loop on host arrays (same API subset as the solvers)."""

    def __init__(self, grid, medium, courant=1.0, dtype=np.float64, walls=None,
                 absorbing_layer=None, air_absorption=None, threads: int = 0):
        self.dtype = dt_ = np.dtype(dtype)
        self.lib = _library(dt_)
        self.threads = self.lib.acfdtd_set_threads(int(threads))
        self.shape = shape = (int(grid.nx), int(grid.ny), int(grid.nz))
        self.dx = dx = float(grid.dx)
        c, rho = float(medium.sound_speed), float(medium.density)
        self.c, self.rho = c, rho
        self.dt = dt = courant * (dx / (c * math.sqrt(3)))
        self.step_index = 0
        self.p = np.zeros(shape, dtype=dt_)
        self.velocity = []
        for axis in range(3):
            s = list(shape)
            s[axis] += 1
            self.velocity.append(np.zeros(s, dtype=dt_))
        processes = oracle_processes(air_absorption, c, dt) if air_absorption is not None else []
        self.psi = np.zeros((len(processes), *shape), dtype=dt_)
        relaxed = c**2 / (1.0 + sum(s for s, _ in processes))
        self.decay = np.zeros(MAX_RELAX)
        self.mean = np.zeros(MAX_RELAX)
        self.gain = np.zeros(MAX_RELAX)
        for r, (strength, tau) in enumerate(processes):        # c_backend.py:210-221
            decay = math.exp(-dt / tau)
            self.decay[r] = decay
            self.mean[r] = dt * (tau / dt) * (1.0 - decay)
            self.gain[r] = rho * relaxed * strength / dx
        self.relax_scale = dt * float(self.gain.sum())
        xi = tuple(walls.values) if walls is not None else (0.0,) * 6
        index, a = oracle_wall_list(shape, c, dt, dx, xi)
        self.wall_index = np.ascontiguousarray(index, dtype=np.int64)
        self.wall_fu = (1.0 / (1.0 + a)).astype(dt_)
        self.wall_fp = (a / (1.0 + a)).astype(dt_)
        self.wall_scratch = np.zeros(self.wall_index.size, dtype=dt_)
        self.has_layer = absorbing_layer is not None
        if self.has_layer:
            cells, faces = oracle_layer_factors(shape, dx, c, dt, absorbing_layer)
            self.cell = [x.astype(dt_) for x in cells]
            self.face = [x.astype(dt_) for x in faces]
        else:
            self.cell = [np.ones(n, dtype=dt_) for n in shape]
            self.face = [np.ones(n + 1, dtype=dt_) for n in shape]
        self.source_index = np.zeros(0, dtype=np.int64)
        self.source_signal = np.zeros((0, 0), dtype=dt_)
        self.receiver_index = np.zeros(0, dtype=np.int64)
        self.recordings = []

    def add_volume_source(self, point, signal):                   # c_backend.py:265-281
        flat = int(np.ravel_multi_index(oracle_cell_index(self.dx, self.shape, point), self.shape))
        signal = np.asarray(signal, dtype=self.dtype)
        length = max(self.source_signal.shape[1], signal.size)
        padded = np.zeros((self.source_signal.shape[0] + 1, length), dtype=self.dtype)
        padded[:-1, : self.source_signal.shape[1]] = self.source_signal
        padded[-1, : signal.size] = signal
        self.source_index = np.append(self.source_index, flat)
        self.source_signal = padded

    def add_pressure_receiver(self, point):
        flat = int(np.ravel_multi_index(oracle_cell_index(self.dx, self.shape, point), self.shape))
        self.receiver_index = np.append(self.receiver_index, flat)
        return self.receiver_index.size - 1

    @property
    def recorded_pressure(self):
        if not self.recordings:
            return np.zeros((self.receiver_index.size, 0))
        return np.concatenate(self.recordings, axis=1)

    def run(self, n_steps):                                       # c_backend.py:302-356
        if n_steps <= 0:
            return
        State, real = _struct(self.dtype)
        rp = ctypes.POINTER(real)

        def ptr(a):
            return a.ctypes.data_as(rp)

        def iptr(a):
            return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))

        recording = np.zeros((self.receiver_index.size, n_steps), dtype=self.dtype)
        state = State(
            nx=self.shape[0], ny=self.shape[1], nz=self.shape[2], n_relax=self.psi.shape[0],
            n_wall=self.wall_index.size, n_sources=self.source_index.size,
            n_receivers=self.receiver_index.size, n_steps=n_steps,
            source_length=self.source_signal.shape[1],
            vel_coef=self.dt / (self.rho * self.dx),
            pres_coef=self.rho * self.c**2 * self.dt / self.dx,
            src_coef=self.rho * self.c**2 * self.dt, relax_scale=self.relax_scale,
            p=ptr(self.p), vx=ptr(self.velocity[0]), vy=ptr(self.velocity[1]),
            vz=ptr(self.velocity[2]), psi=ptr(self.psi),
            relax_decay=(real * MAX_RELAX)(*self.decay), relax_mean=(real * MAX_RELAX)(*self.mean),
            relax_gain=(real * MAX_RELAX)(*self.gain),
            cell=(rp * 3)(*[ptr(x) for x in self.cell]), face=(rp * 3)(*[ptr(x) for x in self.face]),
            has_layer=int(self.has_layer), wall_index=iptr(self.wall_index),
            wall_from_updated=ptr(self.wall_fu), wall_from_previous=ptr(self.wall_fp),
            wall_scratch=ptr(self.wall_scratch), source_index=iptr(self.source_index),
            source_signal=ptr(self.source_signal), receiver_index=iptr(self.receiver_index),
            recording=ptr(recording),
        )
        self.lib.acfdtd_run(ctypes.byref(state), ctypes.c_int64(self.step_index))
        self.step_index += n_steps
        if self.receiver_index.size:
            self.recordings.append(recording)


def host_cores() -> int:
    return os.cpu_count() or 1
