"""Audio output (results/generate_audio.py:14-42): the oracle's restatement of
scipy.signal.butter / lfilter pinned against SciPy (the reference script's own
calls), the library's filter design against SciPy, and the WAV writer
against scipy.io.wavfile.write, byte for byte.  No GPU needed."""
import os

import numpy as np
import pytest

import audio_oracle as OA
import vocalsim_b200.audio as VA

signal = pytest.importorskip("scipy.signal")
wavfile = pytest.importorskip("scipy.io.wavfile")

MULS = [2, 3, 15, 30, 64]


def reference_pipeline(p, mul):
    """The steps of generate_audio.py:14-42 with SciPy."""
    p = np.asarray(p, np.float64)
    audio = np.clip(p / np.max(np.abs(p)), -1.0, 1.0)
    if mul == 1:
        return audio.astype(np.float32)
    b, a = signal.butter(2, 5050.0 / (44100 * mul / 2.0), btype="low")
    return signal.lfilter(b, a, audio)[::mul].astype(np.float32)


@pytest.mark.parametrize("mul", MULS)
def test_oracle_filter_design_matches_scipy(mul):
    wn = 5050.0 / (44100 * mul / 2.0)
    b, a = signal.butter(2, wn, btype="low")
    ob, oa = OA.butter2_lowpass(wn)
    assert np.allclose(ob, b, rtol=1e-15, atol=0) and np.allclose(oa, a, rtol=1e-15, atol=0)


@pytest.mark.parametrize("mul", MULS)
def test_library_filter_design_matches_scipy(mul):
    b, a = signal.butter(2, 5050.0 / (44100 * mul / 2.0), btype="low")
    lb, la = VA.audio_filter(mul)
    assert np.allclose(lb, b, rtol=1e-15, atol=0) and np.allclose(la, a, rtol=1e-15, atol=0)


def test_oracle_recursion_is_scipy_lfilter_bit_for_bit():
    rng = np.random.default_rng(3)
    x = rng.standard_normal(4000)
    for mul in (2, 15, 30):
        b, a = signal.butter(2, 5050.0 / (44100 * mul / 2.0), btype="low")
        assert np.array_equal(OA.lfilter_df2t(b, a, x), signal.lfilter(b, a, x))


@pytest.mark.parametrize("mul", [1, 2, 15, 30])
def test_oracle_pipeline_matches_reference_steps(mul):
    rng = np.random.default_rng(mul)
    p = (rng.standard_normal(3000) * 40.0).astype(np.float32)
    got, want = OA.audio(p, mul), reference_pipeline(p, mul)
    assert got.shape == want.shape == ((3000 + mul - 1) // mul,)
    assert np.max(np.abs(got - want)) <= 1e-7


def test_wav_bytes_match_scipy_writer(tmp_path):
    x = np.random.default_rng(0).standard_normal(777).astype(np.float32)
    wavfile.write(os.fspath(tmp_path / "ref.wav"), 44100, x)
    VA.write_wav(os.fspath(tmp_path / "ours.wav"), x)
    assert (tmp_path / "ref.wav").read_bytes() == (tmp_path / "ours.wav").read_bytes()


def test_audio_filter_rejects_bad_rates():
    with pytest.raises(Exception):
        VA.audio_filter(1)
    with pytest.raises(Exception):
        VA.audio_filter(65)
