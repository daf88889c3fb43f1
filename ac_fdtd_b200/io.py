"""Impulse responses out of the grid's sample rate and into a WAV file (host side).

The solver samples at 1/dt, which the Courant condition sets from the cell size (a 2 cm grid
runs at 29.7 kHz), so a response is resampled to an audio rate before it is written. As in
ac-fdtd (``src/ac_fdtd/io.py:27-69``) the resampling is polyphase at an exact rational ratio --
the rate ratio approximated by a fraction with denominator at most 1000 -- and the file holds
32-bit float samples, one channel per response, normalised to a peak of 1 by default.
"""

from __future__ import annotations

from fractions import Fraction
from pathlib import Path

import numpy as np

__all__ = ["resample", "write_wav"]

#: Largest denominator of the rational approximation of target_rate / source_rate: exact to
#: about a part in 10^4 while keeping the polyphase filter short.
MAX_DENOMINATOR = 1000


def rational_ratio(source_rate: float, target_rate: float) -> tuple[int, int]:
    """(up, down) with up / down the closest fraction to target / source, down <= 1000."""
    if not (source_rate > 0.0 and target_rate > 0.0):
        raise ValueError(f"sample rates must be positive, got {source_rate} and {target_rate}")
    fraction = Fraction(target_rate / source_rate).limit_denominator(MAX_DENOMINATOR)
    return fraction.numerator, fraction.denominator


def resample(signal, source_rate: float, target_rate: float) -> np.ndarray:
    """Resample along the last axis (float64) from ``source_rate`` to ``target_rate``."""
    from scipy.signal import resample_poly

    up, down = rational_ratio(source_rate, target_rate)
    return resample_poly(np.asarray(signal, dtype=np.float64), up, down, axis=-1)


def write_wav(path, signal, sample_rate: float, target_rate: float | None = 48000.0,
              normalise: bool = True) -> Path:
    """Write one response, or a stack of them (time along the last axis), as float32 channels.

    ``sample_rate`` is the rate the signal is at (``solver.sample_rate`` for a raw recording);
    ``target_rate=None`` keeps it. The file's rate is the (resampled) rate rounded to an integer.
    Parent directories are created. Returns the path written.
    """
    from scipy.io import wavfile

    channels = np.atleast_2d(np.asarray(signal, dtype=np.float64))
    rate = float(sample_rate)
    if target_rate is not None:
        channels = resample(channels, rate, target_rate)
        rate = float(target_rate)
    if normalise:
        peak = float(np.max(np.abs(channels)))
        if peak > 0.0:
            channels = channels / peak
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    wavfile.write(path, int(round(rate)), np.ascontiguousarray(channels.T, dtype=np.float32))
    return path
