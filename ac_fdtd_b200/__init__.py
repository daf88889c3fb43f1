"""B200-native staggered pressure-velocity FDTD: a ``cuda`` backend for ac-fdtd's solver API.

``CudaAcousticFDTD`` takes the same arguments and offers the same methods as ac-fdtd's
``AcousticFDTD`` (``src/ac_fdtd/scheme.py``); ``AcousticFDTD`` below is an alias so that
``from ac_fdtd_b200 import AcousticFDTD`` is a one-line switch. The value types (``Grid``,
``WallAdmittances`` ...) mirror the reference's, and the reference's own instances are
accepted too.
"""

from .air import AirAbsorption, RelaxationProcess
from .batch import RoomBatch
from .boundaries import (
    FACES,
    AbsorbingLayer,
    WallAdmittances,
    admittance_from_absorption,
    reflection_coefficient,
)
from .grid import Grid, max_stable_time_step
from .io import resample, write_wav
from .medium import AIR, Medium
from .room import ImpulseResponse, Room, simulate_impulse_response
from .solver import CudaAcousticFDTD, pinned_array
from .sources import band_limited_impulse, deconvolve, gaussian_derivative_pulse, gaussian_pulse

AcousticFDTD = CudaAcousticFDTD

__all__ = [
    "AIR",
    "FACES",
    "AbsorbingLayer",
    "AcousticFDTD",
    "AirAbsorption",
    "CudaAcousticFDTD",
    "Grid",
    "ImpulseResponse",
    "Medium",
    "RelaxationProcess",
    "Room",
    "RoomBatch",
    "WallAdmittances",
    "admittance_from_absorption",
    "band_limited_impulse",
    "deconvolve",
    "gaussian_derivative_pulse",
    "gaussian_pulse",
    "max_stable_time_step",
    "pinned_array",
    "reflection_coefficient",
    "resample",
    "simulate_impulse_response",
    "write_wav",
]
