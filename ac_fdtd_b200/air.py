"""ISO 9613-1 air absorption as relaxation processes for the time-domain scheme.

Mirrors ac-fdtd ``src/ac_fdtd/air.py:67-237``: each ISO relaxation term (oxygen, nitrogen) is
a relaxing bulk modulus with strength ``Delta = C c / pi`` and time ``tau = 1/(2 pi F_r)``, and
the classical ``f^2`` term is a third process placed at the Nyquist frequency of ``dt``. The
standard's formulas are evaluated in the same order as the reference so the FP64 process
parameters, and everything the solver derives from them, are bit-identical.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

__all__ = ["AirAbsorption", "RelaxationProcess"]

_P_REF = 101325.0          # Pa
_T_REF = 293.15            # K
_T_TRIPLE = 273.16         # K
_KELVIN = 273.15
_DB_PER_NEPER = 8.685889638065035


@dataclass(frozen=True)
class RelaxationProcess:
    """One relaxation mechanism: ``strength`` Delta and ``relaxation_time`` tau (s)."""

    strength: float
    relaxation_time: float

    @property
    def frequency(self) -> float:
        return 1.0 / (2.0 * math.pi * self.relaxation_time)

    def attenuation(self, frequencies, sound_speed: float):
        fr = self.frequency
        f = np.asarray(frequencies, dtype=float)
        return self.strength * math.pi / sound_speed * f**2 * fr / (fr**2 + f**2)


@dataclass(frozen=True)
class AirAbsorption:
    """Atmospheric conditions (Celsius, percent RH, Pa) and which ISO terms to include."""

    temperature: float = 20.0
    relative_humidity: float = 50.0
    static_pressure: float = _P_REF
    classical: bool = True
    relaxation: bool = True

    def __post_init__(self) -> None:
        if not 0.0 <= self.relative_humidity <= 100.0:
            raise ValueError(f"relative_humidity is a percentage, got {self.relative_humidity}")
        if self.temperature <= -_KELVIN:
            raise ValueError(f"temperature must be above absolute zero, got {self.temperature}")

    @property
    def kelvin(self) -> float:
        return self.temperature + _KELVIN

    def _pa(self) -> float:
        return self.static_pressure / _P_REF

    def _tr(self) -> float:
        return self.kelvin / _T_REF

    @property
    def molar_water_concentration(self) -> float:
        exponent = -6.8346 * (_T_TRIPLE / self.kelvin) ** 1.261 + 4.6151
        return self.relative_humidity * 10.0**exponent / self._pa()

    @property
    def oxygen_relaxation_frequency(self) -> float:
        h = self.molar_water_concentration
        return self._pa() * (24.0 + 4.04e4 * h * (0.02 + h) / (0.391 + h))

    @property
    def nitrogen_relaxation_frequency(self) -> float:
        h = self.molar_water_concentration
        tr = self._tr()
        return self._pa() * tr**-0.5 * (9.0 + 280.0 * h * math.exp(-4.170 * (tr ** (-1 / 3) - 1.0)))

    def _coefficients(self) -> tuple[float, float, float]:
        """ISO coefficients (classical B, oxygen, nitrogen) in Np/m per the standard's terms."""
        tr = self._tr()
        classical = 1.84e-11 / self._pa() * tr**0.5
        oxygen = tr**-2.5 * 0.01275 * math.exp(-2239.1 / self.kelvin)
        nitrogen = tr**-2.5 * 0.1068 * math.exp(-3352.0 / self.kelvin)
        return classical, oxygen, nitrogen

    def attenuation(self, frequencies):
        """ISO 9613-1 attenuation in dB/m (the target the model reproduces)."""
        f = np.asarray(frequencies, dtype=float)
        classical, oxygen, nitrogen = self._coefficients()
        total = np.zeros_like(f)
        if self.classical:
            total += classical * f**2
        if self.relaxation:
            for coefficient, fr in ((oxygen, self.oxygen_relaxation_frequency),
                                    (nitrogen, self.nitrogen_relaxation_frequency)):
                total += coefficient * f**2 * fr / (fr**2 + f**2)
        return _DB_PER_NEPER * total

    def processes(self, sound_speed: float, dt: float) -> tuple[RelaxationProcess, ...]:
        """Relaxation fields for this air at this time step: O2, N2, then classical."""
        classical, oxygen, nitrogen = self._coefficients()
        out = []
        if self.relaxation:
            for coefficient, fr in ((oxygen, self.oxygen_relaxation_frequency),
                                    (nitrogen, self.nitrogen_relaxation_frequency)):
                out.append(RelaxationProcess(strength=coefficient * sound_speed / math.pi,
                                             relaxation_time=1.0 / (2.0 * math.pi * fr)))
        if self.classical:
            nyquist = 0.5 / dt
            out.append(RelaxationProcess(strength=classical * nyquist * sound_speed / math.pi,
                                         relaxation_time=1.0 / (2.0 * math.pi * nyquist)))
        return tuple(out)

    def model_attenuation(self, frequencies, sound_speed: float, dt: float):
        f = np.asarray(frequencies, dtype=float)
        total = np.zeros_like(f)
        for process in self.processes(sound_speed, dt):
            total += process.attenuation(f, sound_speed)
        return _DB_PER_NEPER * total

    def total_strength(self, sound_speed: float, dt: float) -> float:
        return sum(p.strength for p in self.processes(sound_speed, dt))
