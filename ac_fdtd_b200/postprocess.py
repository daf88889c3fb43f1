"""The room workflow's steps after the time loop, in FP64 on the GPU.

The reference turns receiver recordings into room-acoustics figures on the host
(``src/ac_fdtd/sources.py:80-108`` deconvolution; ``src/ac_fdtd/metrics.py:57-111`` Schroeder
decay, T20/T30, EDT, clarity). Here the same steps run where the recordings already are:

* ``deconvolve`` -- real-to-complex FFT of the recordings and the excitation (cuFFT through
  ``torch.fft``: a library FFT, off the leapfrog's path), the regularised spectral division
  and band limit in this library's kernel (``acf_spectral_divide``), inverse FFT;
* ``schroeder_decay`` -- the backward integral of the squared signal as a CTA-wide scan
  (``acf_schroeder_decay``);
* ``reverberation_time`` / ``early_decay_time`` -- the least-squares slope between two levels of
  the decay curve (``acf_decay_fit``);
* ``clarity`` -- the early-to-late energy split (``acf_clarity``).

Inputs are NumPy arrays or CUDA tensors of shape ``(samples,)`` or ``(channels, samples)``;
every sum is FP64. Results agree with the reference to rounding (its sums are sequential,
these are tree-shaped), within about 1e-13 relative. There is no CPU path: without the library
or a GPU these raise.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _native

__all__ = ["deconvolve", "schroeder_decay", "reverberation_time", "early_decay_time", "clarity"]


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device is visible; the device post-processing has no CPU path")
    return torch


def _signals(response, torch):
    """(channels, samples) contiguous float64 CUDA tensor, and whether the input was 1-D."""
    t = response if isinstance(response, torch.Tensor) else torch.as_tensor(np.asarray(response, dtype=float))
    one = t.dim() == 1
    t = t.reshape(1, -1) if one else t.reshape(-1, t.shape[-1])
    return t.to(device="cuda", dtype=torch.float64).contiguous(), one


def _stream(torch) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _out(value, one: bool, as_numpy: bool):
    if as_numpy:
        value = value.cpu().numpy()
    return value[0] if one else value


def deconvolve(recorded, excitation, dt: float, max_frequency: float,
               regularisation: float = 1e-6, *, as_numpy: bool = True):
    """The impulse response: the excitation divided back out of the recordings, band-limited
    to ``max_frequency`` (``sources.py:80-108``)."""
    torch = _torch()
    lib = _native.library()
    x, one = _signals(recorded, torch)
    n = x.shape[-1]
    s, _ = _signals(excitation, torch)
    if s.shape[-1] != n:
        raise ValueError(f"excitation has {s.shape[-1]} samples, the recordings {n}")
    spectra = torch.fft.rfft(x, dim=-1).contiguous()
    source = torch.fft.rfft(s[0], dim=-1).contiguous()
    out = torch.empty_like(spectra)
    scratch = torch.empty(1, dtype=torch.float64, device="cuda")
    bins = spectra.shape[-1]
    bin_hz = 1.0 / (n * dt)            # numpy.fft.rfftfreq: bin k at k * (1 / (n d))
    _native.check(lib.acf_spectral_divide(spectra.data_ptr(), source.data_ptr(), x.shape[0], bins,
                                          bin_hz, float(max_frequency), float(regularisation),
                                          scratch.data_ptr(), out.data_ptr(), _stream(torch)),
                  "acf_spectral_divide")
    response = torch.fft.irfft(out, n=n, dim=-1)
    return _out(response, one, as_numpy)


def schroeder_decay(response, floor_db: float = -120.0, *, as_numpy: bool = True):
    """Backward-integrated energy decay curve in dB, starting at 0 (``metrics.py:57-69``)."""
    torch = _torch()
    lib = _native.library()
    x, one = _signals(response, torch)
    decay = torch.empty_like(x)
    _native.check(lib.acf_schroeder_decay(x.data_ptr(), x.shape[0], x.shape[1], float(floor_db),
                                          decay.data_ptr(), _stream(torch)), "acf_schroeder_decay")
    return _out(decay, one, as_numpy)


def _decay_slope(response, sample_rate: float, upper: float, lower: float):
    torch = _torch()
    lib = _native.library()
    x, one = _signals(response, torch)
    decay = torch.empty_like(x)
    stream = _stream(torch)
    _native.check(lib.acf_schroeder_decay(x.data_ptr(), x.shape[0], x.shape[1], -120.0,
                                          decay.data_ptr(), stream), "acf_schroeder_decay")
    seconds = torch.empty(x.shape[0], dtype=torch.float64, device="cuda")
    failed = torch.empty(x.shape[0], dtype=torch.int32, device="cuda")
    _native.check(lib.acf_decay_fit(decay.data_ptr(), x.shape[0], x.shape[1], float(sample_rate),
                                    float(upper), float(lower), seconds.data_ptr(),
                                    failed.data_ptr(), stream), "acf_decay_fit")
    if bool(failed.any()):
        raise ValueError(f"the decay never reaches {lower} dB: the response is too short, or the "
                         "room is too live for the run length")
    values = seconds.cpu().numpy()
    return float(values[0]) if one else values


def reverberation_time(response, sample_rate: float, evaluation_range: float = 20.0):
    """T20 (or T30), extrapolated to 60 dB, in seconds (``metrics.py:87-97``)."""
    return _decay_slope(response, sample_rate, -5.0, -5.0 - evaluation_range)


def early_decay_time(response, sample_rate: float):
    """EDT: the first 10 dB, extrapolated to 60 (``metrics.py:100-103``)."""
    return _decay_slope(response, sample_rate, 0.0, -10.0)


def clarity(response, sample_rate: float, split: float = 0.05):
    """C50 (or C80 with ``split=0.08``): early-to-late energy ratio in dB (``metrics.py:104-110``)."""
    torch = _torch()
    lib = _native.library()
    x, one = _signals(response, torch)
    boundary = int(round(split * sample_rate))
    db = torch.empty(x.shape[0], dtype=torch.float64, device="cuda")
    _native.check(lib.acf_clarity(x.data_ptr(), x.shape[0], x.shape[1], boundary, db.data_ptr(),
                                  _stream(torch)), "acf_clarity")
    values = db.cpu().numpy()
    return float(values[0]) if one else values
