"""Export of impulse responses (host side): resampling and WAV files, against fixtures made by
running the reference's own ``resample`` and ``write_wav`` (tests/golden/make_golden.py, part
``io``)."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest
from scipy.io import wavfile

from ac_fdtd_b200.io import rational_ratio, resample, write_wav

GOLDEN = Path(__file__).parent / "golden"


@pytest.fixture(scope="module")
def io_golden():
    data = np.load(GOLDEN / "io.npz")
    meta = json.loads((GOLDEN / "golden.json").read_text())["io"]
    return data, meta


def test_resampling_matches_the_reference(io_golden):
    data, meta = io_golden
    for n, (source_rate, target_rate) in enumerate(meta["cases"]):
        got = resample(data["signal"], source_rate, target_rate)
        want = data[f"resampled_{n}"]
        assert got.shape == want.shape
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-14 * np.max(np.abs(want)))


def test_wav_files_match_the_reference(io_golden, tmp_path):
    data, meta = io_golden
    path = write_wav(tmp_path / "nested" / "ir.wav", data["signal"], 29716.4)
    rate, written = wavfile.read(path)
    assert rate == meta["wav_rate"] and written.dtype == np.float32
    np.testing.assert_array_equal(written, data["wav"])
    assert np.max(np.abs(written)) == pytest.approx(1.0)
    path = write_wav(tmp_path / "raw.wav", data["signal"][0], 29716.4, target_rate=None,
                     normalise=False)
    rate, written = wavfile.read(path)
    assert rate == meta["wav_raw_rate"]
    np.testing.assert_array_equal(written, data["wav_raw"])


def test_ratio_and_edge_cases(tmp_path):
    assert rational_ratio(29716.4, 48000.0)[1] <= 1000
    assert rational_ratio(48000.0, 48000.0) == (1, 1)
    with pytest.raises(ValueError):
        resample(np.ones(10), 0.0, 48000.0)
    with pytest.raises(ValueError):
        rational_ratio(48000.0, -1.0)
    silent = write_wav(tmp_path / "silent.wav", np.zeros(64), 48000.0, target_rate=None)
    rate, written = wavfile.read(silent)
    assert rate == 48000 and not np.any(written)          # zero peak: left unnormalised
