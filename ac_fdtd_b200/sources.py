"""Excitation signals (ac-fdtd ``src/ac_fdtd/sources.py:40-77``) and deconvolution (:80-108)."""

from __future__ import annotations

import numpy as np

__all__ = ["gaussian_pulse", "gaussian_derivative_pulse", "band_limited_impulse", "deconvolve"]

_BANDWIDTH_LEVEL_DB = 40.0


def gaussian_pulse(n_steps: int, dt: float, max_frequency: float) -> np.ndarray:
    """exp(-((t - 4w)/w)^2) at t = (n + 1/2) dt, 40 dB down at ``max_frequency``."""
    decay = np.log(10.0 ** (_BANDWIDTH_LEVEL_DB / 20.0))
    width = np.sqrt(decay) / (np.pi * max_frequency)
    centre = 4.0 * width
    t = (np.arange(n_steps) + 0.5) * dt
    return np.exp(-(((t - centre) / width) ** 2))


def gaussian_derivative_pulse(n_steps: int, dt: float, max_frequency: float) -> np.ndarray:
    """Time derivative of :func:`gaussian_pulse`, -2 (t - 4w)/w^2 times the pulse.

    The reference has no such signal; its solver takes any sample array, and this one has no
    DC component, so a closed room does not accumulate a static pressure offset.
    """
    decay = np.log(10.0 ** (_BANDWIDTH_LEVEL_DB / 20.0))
    width = np.sqrt(decay) / (np.pi * max_frequency)
    centre = 4.0 * width
    t = (np.arange(n_steps) + 0.5) * dt
    return -2.0 * (t - centre) / width**2 * np.exp(-(((t - centre) / width) ** 2))


def band_limited_impulse(n_steps: int, dt: float, max_frequency: float) -> np.ndarray:
    """Hann-windowed sinc flat to ``max_frequency`` (``sources.py:54-77``)."""
    if max_frequency >= 0.5 / dt:
        raise ValueError(
            f"max_frequency {max_frequency} is at or above the Nyquist frequency {0.5 / dt}"
        )
    half = int(np.ceil(4.0 / (max_frequency * dt)))
    if 2 * half + 1 > n_steps:
        raise ValueError(
            f"a pulse band-limited to {max_frequency} Hz needs {2 * half + 1} steps, "
            f"but only {n_steps} were asked for"
        )
    offsets = np.arange(-half, half + 1)
    kernel = 2.0 * max_frequency * dt * np.sinc(2.0 * max_frequency * dt * offsets)
    kernel *= np.hanning(kernel.size)
    signal = np.zeros(n_steps)
    signal[: kernel.size] = kernel
    return signal


def deconvolve(recorded, excitation, dt: float, max_frequency: float,
               regularisation: float = 1e-6) -> np.ndarray:
    """Regularised spectral division of the excitation out of the recording (``sources.py:80-108``)."""
    recorded = np.asarray(recorded, dtype=float)
    spectrum = np.fft.rfft(recorded, axis=-1)
    source = np.fft.rfft(np.asarray(excitation, dtype=float))
    frequencies = np.fft.rfftfreq(recorded.shape[-1], dt)
    power = np.abs(source) ** 2
    response = spectrum * np.conjugate(source) / (power + regularisation * power.max())
    response[..., frequencies > max_frequency] = 0.0
    return np.fft.irfft(response, n=recorded.shape[-1], axis=-1)
