"""RFI oracle (oracle/rfi_oracle.py) pinned to the reference's own tests of
rfi.rs (rfi.rs:201-296), and the --rfi JSON layout of tga_rfi_json."""
import ctypes
import json
import math

import numpy as np
import pytest

import rfi_oracle as RO
import tga
from testutil import _xs, quantize_bipolar_demean

FS = 16.368e6
N = 64 * 16368  # 64 ms, as the reference tests


def square_243(i):
    per = FS / 2.43e6
    return np.where(np.mod(i.astype(np.float64), per) < per / 2.0, 1.0, -1.0)


def bipolar(sig):
    return quantize_bipolar_demean(sig).astype(np.float64)


@pytest.fixture(scope="module")
def idx():
    return np.arange(N)


def test_square_wave_detected(idx):
    sig = 2.0 * square_243(idx) + _xs("oracle_xorshift_gaussian", 42, N)
    ch = RO.analyze_channel(0, bipolar(sig), FS)
    assert not ch["dead"]
    top = ch["lines"][0]
    assert abs(top["frequency"] - 2.43e6) < 1e3
    assert top["excess_db"] > 15.0
    assert abs(ch["period_samples"] - FS / 2.43e6) < 0.2
    assert ch["acf_lag1"] > 0.3 and ch["acf_lag3"] < -0.4 and ch["acf_lag16"] < 0.0


def test_white_noise_no_lines():
    ch = RO.analyze_channel(0, bipolar(_xs("oracle_xorshift_gaussian", 7, N)), FS)
    assert not ch["dead"] and ch["lines"] == []


def test_line_excess_scales_with_amplitude(idx):
    g = _xs("oracle_xorshift_gaussian", 9, N)
    w = RO.analyze_channel(0, bipolar(0.1 * square_243(idx) + g), FS)
    s = RO.analyze_channel(0, bipolar(2.0 * square_243(idx) + g), FS)
    assert s["lines"][0]["excess_db"] > w["lines"][0]["excess_db"] + 10.0


def test_gps_signal_not_flagged(idx):
    period = 16368
    code = tga.code_resampled(tga.GPS, 1, float(period), 2 * period)
    a = 2.0 * math.sqrt(10.0 ** 4.0 / FS)
    g = _xs("oracle_xorshift_gaussian", 11, N)
    cp = (idx + 137) % period
    sig = code[cp] * np.cos(2 * np.pi * 100e3 * idx / FS) * a + g
    assert RO.analyze_channel(0, bipolar(sig), FS)["lines"] == []


def test_dead_channel():
    ch = RO.analyze_channel(17, np.zeros(N), FS)
    assert ch["dead"] and ch["lines"] == [] and ch["acf_lag1"] is None


def test_rfi_json_layout_matches_serde_pretty():
    chans = (tga.RfiChannel * 2)()
    chans[0].antenna, chans[0].dead = 0, 0
    chans[0].acf_lag1, chans[0].acf_lag3, chans[0].acf_lag16 = 0.4125, -0.71, -0.5
    chans[0].period_samples = FS / 2.43e6
    chans[0].n_lines = 2
    chans[0].lines[0].frequency, chans[0].lines[0].excess_db = 2430000.0, 41.25
    chans[0].lines[1].frequency, chans[0].lines[1].excess_db = 4860015.625, 22.5
    chans[1].antenna, chans[1].dead = 1, 1
    chans[1].acf_lag1 = chans[1].acf_lag3 = chans[1].acf_lag16 = chans[1].period_samples = float("nan")
    p = ctypes.c_char_p()
    assert tga.lib().tga_rfi_json(chans, 2, ctypes.byref(p)) == 0
    text = ctypes.string_at(p).decode()
    tga.lib().tga_free(p)
    want = {"antenna_numbers": [0, 1], "channels": [
        {"antenna": 0, "dead": False, "acf_lag1": 0.4125, "acf_lag3": -0.71, "acf_lag16": -0.5,
         "period_samples": FS / 2.43e6,
         "lines": [{"frequency": 2430000.0, "excess_db": 41.25}, {"frequency": 4860015.625, "excess_db": 22.5}]},
        {"antenna": 1, "dead": True, "acf_lag1": None, "acf_lag3": None, "acf_lag16": None, "period_samples": None,
         "lines": []}]}
    assert text == json.dumps(want, indent=2)
