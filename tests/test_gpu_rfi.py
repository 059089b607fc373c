"""GPU RFI scan (tga_rfi_scan) against the FP64 oracle of rfi.rs on the same
packed rows: synthetic square-wave interferers, white noise, a GPS signal, a
dead channel, and the real TART recording (first 40920 bytes per antenna)."""
import math
import os

import numpy as np
import pytest

import rfi_oracle as RO
import tga
from testutil import _xs

pytestmark = pytest.mark.gpu

FS = 16.368e6
N = 64 * 16368


def _compare(got, want):
    assert len(got) == len(want)
    for g, w in zip(got, want):
        assert g["antenna"] == w["antenna"] and g["dead"] == w["dead"]
        for k in ("acf_lag1", "acf_lag3", "acf_lag16"):
            if w[k] is None:
                assert g[k] is None
            else:
                assert abs(g[k] - w[k]) <= 1e-12, (k, g[k], w[k])
        assert len(g["lines"]) == len(w["lines"]), (g["lines"], w["lines"])
        for gl, wl in zip(g["lines"], w["lines"]):
            assert gl["frequency"] == wl["frequency"]
            assert abs(gl["excess_db"] - wl["excess_db"]) <= 1e-9 * abs(wl["excess_db"])
        if w["period_samples"] is None:
            assert g["period_samples"] is None
        else:
            assert abs(g["period_samples"] - w["period_samples"]) <= 1e-12 * w["period_samples"]


def test_rfi_scan_matches_oracle_synthetic():
    i = np.arange(N)
    per = FS / 2.43e6
    sq = np.where(np.mod(i.astype(np.float64), per) < per / 2.0, 1.0, -1.0)
    period = 16368
    code = tga.code_resampled(tga.GPS, 1, float(period), 2 * period)
    gps = code[(i + 137) % period] * np.cos(2 * np.pi * 100e3 * i / FS) * 2.0 * math.sqrt(1e4 / FS)
    two = np.where(np.mod(i.astype(np.float64), FS / 1.1e6) < FS / 2.2e6, 1.0, -1.0)
    rows = [2.0 * sq + _xs("oracle_xorshift_gaussian", 42, N),
            _xs("oracle_xorshift_gaussian", 7, N),
            0.1 * sq + _xs("oracle_xorshift_gaussian", 9, N),
            gps + _xs("oracle_xorshift_gaussian", 11, N),
            np.full(N, -1.0),
            0.5 * sq + 0.7 * two + _xs("oracle_xorshift_gaussian", 13, N)]
    bits = np.packbits(np.stack(rows) >= 0.0, axis=1)
    with tga.Context(0) as ctx:
        got = ctx.rfi_scan(bits, FS)
        text = ctx.rfi_scan(bits, FS, as_json=True)
    want = RO.run(bits, FS)
    _compare(got, want)
    assert got[0]["lines"] and abs(got[0]["lines"][0]["frequency"] - 2.43e6) < 1e3
    assert got[1]["lines"] == [] and got[3]["lines"] == [] and got[4]["dead"]
    assert len(got[5]["lines"]) >= 2
    assert text.startswith('{\n  "antenna_numbers": [\n    0,')


def test_rfi_scan_matches_oracle_real_recording():
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "tart_head.npz"))
    bits = np.ascontiguousarray(z["head"])
    fs = float(z["sampling_frequency"])
    with tga.Context(0) as ctx:
        got = ctx.rfi_scan(bits, fs)
    _compare(got, RO.run(bits, fs))


@pytest.mark.parametrize("row_bytes", [1000, 1031, 3069], ids=["2^5x5^3", "bluestein-1031", "3x11x31"])
def test_rfi_spectrum_any_length(row_bytes):
    """Record lengths whose half length L = 4 row_bytes has odd radices
    (5^3; 3 x 11 x 31) or a prime factor above the largest pass radix (1031:
    Bluestein's chirp-z over a power-of-two convolution): the f64 spectrum,
    lines and floor match the oracle as at the usual lengths."""
    n = row_bytes * 8
    i = np.arange(n)
    sq = np.where(np.mod(i.astype(np.float64), FS / 1.5e6) < FS / 3.0e6, 1.0, -1.0)
    rows = [3.0 * sq + _xs("oracle_xorshift_gaussian", 21, n), _xs("oracle_xorshift_gaussian", 22, n)]
    bits = np.packbits(np.stack(rows) >= 0.0, axis=1)
    assert bits.shape[1] == row_bytes
    with tga.Context(0) as ctx:
        got = ctx.rfi_scan(bits, FS)
    _compare(got, RO.run(bits, FS))
    assert got[0]["lines"]
