"""Room impulse responses on the CUDA backend: the caller of the leapfrog, and what follows it.

``simulate_impulse_response`` is ac-fdtd's workflow (``src/ac_fdtd/room.py:121-176``) with the
solver class as a parameter, defaulting to ``CudaAcousticFDTD``: grid from the bandwidth at ten
points per wavelength, run length 1.5 Sabine times, a band-limited impulse injected at the
source, recordings deconvolved. With ``dtype=float64`` its recordings are bit-identical to the
reference's NumPy solver. The statistical formulae and decay metrics it relies on are here too
(``src/ac_fdtd/metrics.py``, ``boundaries.py:97-117``); the energy-decay integration runs in
FP64.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .air import AirAbsorption
from .boundaries import WallAdmittances, admittance_from_absorption
from .grid import Grid
from .medium import AIR, Medium
from .solver import CudaAcousticFDTD
from .sources import band_limited_impulse, deconvolve

__all__ = [
    "Room",
    "ImpulseResponse",
    "simulate_impulse_response",
    "random_incidence_absorption",
    "air_absorption_coefficient",
    "sabine_time",
    "eyring_time",
    "schroeder_decay",
    "reverberation_time",
    "early_decay_time",
    "clarity",
    "schroeder_frequency",
]

DEFAULT_POINTS_PER_WAVELENGTH = 10.0
DEFAULT_DURATION_FACTOR = 1.5
#: 24 ln(10) / c at 343 m/s, the constant of Sabine's formula.
_SABINE_NUMERATOR = 24.0 * np.log(10.0) / 343.0


def random_incidence_absorption(normalised_admittance: float, n_angles: int = 1024) -> float:
    """Paris integral of alpha(theta) sin(2 theta) over a quarter turn (midpoint angles)."""
    angles = (np.arange(n_angles) + 0.5) * (math.pi / 2.0) / n_angles
    cosines = np.cos(angles)
    reflection = (cosines - normalised_admittance) / (cosines + normalised_admittance)
    absorption = 1.0 - reflection**2
    return float(np.trapezoid(absorption * np.sin(2.0 * angles), angles))


def air_absorption_coefficient(attenuation_db_per_metre: float) -> float:
    """Energy coefficient m (1/m) of Sabine's 4 m V term from a pressure attenuation in dB/m."""
    return attenuation_db_per_metre / (10.0 * np.log10(np.e))


def sabine_time(volume, surface, absorption, air_coefficient=0.0) -> float:
    return _SABINE_NUMERATOR * volume / (surface * absorption + 4.0 * air_coefficient * volume)


def eyring_time(volume, surface, absorption, air_coefficient=0.0) -> float:
    return (_SABINE_NUMERATOR * volume
            / (-surface * np.log(1.0 - absorption) + 4.0 * air_coefficient * volume))


def schroeder_frequency(volume: float, reverberation: float) -> float:
    return 2000.0 * np.sqrt(reverberation / volume)


def schroeder_decay(response, floor_db: float = -120.0) -> np.ndarray:
    """Backward-integrated energy decay in dB (FP64), 0 at the start."""
    energy = np.asarray(response, dtype=np.float64) ** 2
    integrated = np.cumsum(energy[..., ::-1], axis=-1)[..., ::-1]
    with np.errstate(divide="ignore"):
        decay = 10.0 * np.log10(np.maximum(integrated / integrated[..., :1], 1e-300))
    return np.maximum(decay, floor_db)


def _decay_slope(decay, sample_rate, upper, lower) -> float:
    start = int(np.argmax(decay <= upper))
    end = int(np.argmax(decay <= lower))
    if end <= start:
        raise ValueError(f"the decay never reaches {lower} dB: the response is too short")
    slope, _ = np.polyfit(np.arange(start, end) / sample_rate, decay[start:end], 1)
    return -60.0 / slope


def reverberation_time(response, sample_rate: float, evaluation_range: float = 20.0) -> float:
    """T20 (or T30), fitted from -5 dB and extrapolated to 60 dB."""
    return _decay_slope(schroeder_decay(response), sample_rate, -5.0, -5.0 - evaluation_range)


def early_decay_time(response, sample_rate: float) -> float:
    return _decay_slope(schroeder_decay(response), sample_rate, 0.0, -10.0)


def clarity(response, sample_rate: float, split: float = 0.05) -> float:
    boundary = int(round(split * sample_rate))
    energy = np.asarray(response, dtype=np.float64) ** 2
    return 10.0 * np.log10(float(np.sum(energy[..., :boundary])) / float(np.sum(energy[..., boundary:])))


@dataclass(frozen=True)
class Room:
    """A rectangular room with one normal-incidence absorption on every wall."""

    dimensions: tuple[float, float, float]
    absorption: float = 0.1
    air: AirAbsorption | None = field(default_factory=AirAbsorption)
    medium: Medium = AIR

    @property
    def volume(self) -> float:
        return float(np.prod(self.dimensions))

    @property
    def surface(self) -> float:
        x, y, z = self.dimensions
        return 2.0 * (x * y + y * z + z * x)

    @property
    def wall_admittance(self) -> float:
        return admittance_from_absorption(self.absorption)

    @property
    def diffuse_absorption(self) -> float:
        return random_incidence_absorption(self.wall_admittance)

    def air_coefficient(self, frequency: float) -> float:
        if self.air is None:
            return 0.0
        return air_absorption_coefficient(float(self.air.attenuation(frequency)))

    def sabine_reverberation_time(self, frequency: float = 1000.0) -> float:
        return sabine_time(self.volume, self.surface, self.diffuse_absorption,
                           self.air_coefficient(frequency))

    def eyring_reverberation_time(self, frequency: float = 1000.0) -> float:
        return eyring_time(self.volume, self.surface, self.diffuse_absorption,
                           self.air_coefficient(frequency))


@dataclass(frozen=True)
class ImpulseResponse:
    signals: np.ndarray        # (receiver, sample), deconvolved
    recorded: np.ndarray       # raw pressure, same shape
    excitation: np.ndarray
    sample_rate: float
    max_frequency: float
    grid: Grid

    def decay_metrics(self, device: bool = True) -> dict:
        """T20, T30, EDT (seconds), C50 and C80 (dB) of every receiver's response, computed in
        FP64 on the GPU (``ac_fdtd_b200.postprocess``) or, with ``device=False``, on the host
        in the reference's arithmetic. A response too short for a fit, or for a clarity split,
        gives NaN there (the reference's functions raise for it)."""
        if device:
            from . import postprocess as where
        else:
            where = _HostMetrics
        out = {}
        for name, fit in (("t20", lambda s: where.reverberation_time(s, self.sample_rate, 20.0)),
                          ("t30", lambda s: where.reverberation_time(s, self.sample_rate, 30.0)),
                          ("edt", lambda s: where.early_decay_time(s, self.sample_rate))):
            values = []
            for signal in self.signals:
                try:
                    values.append(float(fit(signal)))
                except ValueError:
                    values.append(float("nan"))
            out[name] = np.array(values)
        n = self.signals.shape[-1]
        for name, split in (("c50", 0.05), ("c80", 0.08)):
            if not 0 < int(round(split * self.sample_rate)) < n:   # no early or no late part
                out[name] = np.full(len(self.signals), np.nan)
                continue
            out[name] = np.array([float(where.clarity(signal, self.sample_rate, split))
                                  for signal in self.signals])
        return out


class _HostMetrics:
    reverberation_time = staticmethod(lambda *a: reverberation_time(*a))
    early_decay_time = staticmethod(lambda *a: early_decay_time(*a))
    clarity = staticmethod(lambda *a: clarity(*a))


def simulate_impulse_response(room: Room, source, receivers, max_frequency: float,
                              duration: float | None = None,
                              points_per_wavelength: float = DEFAULT_POINTS_PER_WAVELENGTH,
                              courant: float = 1.0, *, dtype=np.float64,
                              solver_class=CudaAcousticFDTD, postprocess: str | None = None,
                              **solver_options) -> ImpulseResponse:
    """Excite ``room`` at ``source`` and return the impulse responses at ``receivers``.

    Same steps and defaults as ac-fdtd's ``simulate_impulse_response``; ``dtype`` defaults to
    float64 as there, and float32 is the fast setting. ``solver_class`` may be any class with
    the reference solver's constructor and methods (the reference's own ``AcousticFDTD``
    included). ``postprocess``: ``"device"`` deconvolves on the GPU in FP64 from the recordings
    in device memory (the default with the CUDA solver; equal to the reference's host
    arithmetic to rounding), ``"host"`` in the reference's NumPy arithmetic (bit for bit).
    """
    if postprocess is None:
        postprocess = "device" if issubclass(solver_class, CudaAcousticFDTD) else "host"
    if postprocess not in ("device", "host"):
        raise ValueError(f"postprocess must be 'device' or 'host', got {postprocess!r}")
    grid = Grid.from_max_frequency(room.dimensions, max_frequency=max_frequency,
                                   sound_speed=room.medium.sound_speed,
                                   points_per_wavelength=points_per_wavelength)
    solver = solver_class(grid, medium=room.medium, courant=courant, dtype=dtype,
                          walls=WallAdmittances.from_absorption(room.absorption),
                          air_absorption=room.air, **solver_options)
    if duration is None:
        duration = DEFAULT_DURATION_FACTOR * room.sabine_reverberation_time()
    n_steps = int(round(duration / solver.dt))
    excitation = band_limited_impulse(n_steps, solver.dt, max_frequency)
    solver.add_volume_source(source, excitation)
    for receiver in receivers:
        solver.add_pressure_receiver(receiver)
    solver.run(n_steps)
    if postprocess == "device":
        from . import postprocess as device

        on_device = solver.recorded_pressure_device()
        signals = device.deconvolve(on_device, excitation, solver.dt, max_frequency)
        recorded = on_device.cpu().numpy()
    else:
        recorded = solver.recorded_pressure
        signals = deconvolve(recorded, excitation, solver.dt, max_frequency)
    return ImpulseResponse(
        signals=signals, recorded=recorded, excitation=excitation, sample_rate=1.0 / solver.dt,
        max_frequency=max_frequency, grid=grid,
    )
