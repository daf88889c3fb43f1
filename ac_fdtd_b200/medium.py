"""The propagation medium: sound speed and density.

Mirrors ac-fdtd ``src/ac_fdtd/medium.py:20-61``. ``Medium.air`` evaluates the same ideal-gas
expressions in the same order, so ``AIR`` here is bit-identical to the reference's ``AIR``
(c = 343.2 m/s, rho = 1.204 kg/m^3 at 20 C).
"""

from __future__ import annotations

from dataclasses import dataclass

__all__ = ["Medium", "AIR"]

_GAS_CONSTANT_DRY_AIR = 287.058   # J/(kg K)
_KELVIN_OFFSET = 273.15


@dataclass(frozen=True)
class Medium:
    sound_speed: float
    density: float

    @property
    def impedance(self) -> float:
        return self.density * self.sound_speed

    @classmethod
    def air(cls, temperature: float = 20.0, static_pressure: float = 101325.0) -> Medium:
        kelvin = temperature + _KELVIN_OFFSET
        speed = 331.3 * (kelvin / _KELVIN_OFFSET) ** 0.5
        return cls(sound_speed=speed, density=static_pressure / (_GAS_CONSTANT_DRY_AIR * kelvin))


AIR = Medium.air()
