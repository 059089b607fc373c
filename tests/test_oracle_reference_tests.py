"""The reference's correlation and driver unit tests, run on the CPU oracle.

Restates (file:line in tart-gnss-acquire):
* correlate.rs:213-295     delay recovery, [c,-c] flip recovery, noise bound
* acquisition.rs:425-515   GPS recovery, contrast, period-boundary sweep
* galileo.rs:400-466, beidou.rs:351-414, l1c.rs:360-425, sbas.rs:457-520,
  qzss.rs:456-520          per-constellation recovery / contrast / sweep
* acquisition.rs:551-595, galileo.rs:466-512, beidou.rs:415-470,
  l1c.rs:426-480           production-rate one-bit ACR C/N0 end to end
* acquisition.rs:517-549   acquire_all PRN and antenna filters
Passing these pins the oracle's correlator to the reference's behaviour.
"""
import numpy as np
import pytest

import acq_oracle as O
from testutil import (expected_recovered_sample, phasepoints, quantize_bipolar_demean,
                      synth_signal, synth_signal_cn0)


def _spectra(code, period=None):
    a, b = O.code_spectra(code, period if period is not None else len(code))
    return a, b


def test_correlate_code_recovers_delay():
    period, fs = 256, 1.023e6
    code = O.resampled_code(O.GPS, 1, float(period), period)
    cc, _ = _spectra(code)
    for delay in (0, 50, 128, 200):
        sig = synth_signal(code, period, delay, 0.0, fs, 0.05, 42)
        pk = O.correlate_code(sig, phasepoints(fs, period), cc, cc, np.array([0.0]), period, period, fs)
        assert pk["best_codephase"] % period == expected_recovered_sample(period, delay)
        assert pk["best_freq_idx"] == 0 and pk["best_peak"] > 0.0


def test_correlate_code_recovers_flipped_second_period():
    period, fs, delay = 256, 1.023e6, 50
    code = O.resampled_code(O.GPS, 1, float(period), 2 * period)
    cc, cc_alt = _spectra(code, period)
    sig = synth_signal_cn0(code, period, delay, 0.0, fs, 60.0, 42, True)
    pk = O.correlate_code(sig, phasepoints(fs, 2 * period), cc, cc_alt, np.array([0.0]),
                          2 * period, period, fs)
    assert pk["best_codephase"] % period == expected_recovered_sample(period, delay)
    assert pk["best_peak"] > 0.0


def test_correlate_code_noise_only_bounded():
    period, fs = 256, 1.023e6
    code = O.resampled_code(O.GPS, 1, float(period), period)
    cc, _ = _spectra(code)
    sig = synth_signal(code, period, 0, 0.0, fs, 0.0, 7)
    pk = O.correlate_code(sig, phasepoints(fs, period), cc, cc, np.array([0.0]), period, period, fs)
    assert pk["best_peak"] > 0.0 and np.isfinite(pk["best_peak"])
    assert pk["second_peak"] > 0.0 and pk["best_codephase"] < period


# (constellation, fs, period, prn, delay, seed, contrast_delay, contrast_seed, sin_step)
DRIVER_CASES = [
    (O.GPS, 2.046e6, 2046, 1, 500, 1, 123, 2, 3.3),
    (O.GALILEO, 1.023e6, 4092, 1, 900, 11, 600, 12, 2.7),
    (O.BEIDOU, 1.023e6, 10230, 1, 3000, 21, 1000, 22, 1.9),
    (O.L1C, 1.023e6, 10230, 1, 2500, 31, 700, 32, 1.3),
    (O.SBAS, 1.023e6, 1023, 120, 400, 41, 100, 42, 2.1),
    (O.QZSS, 1.023e6, 1023, 184, 250, 51, 300, 52, 3.9),
]


@pytest.mark.parametrize("case", DRIVER_CASES, ids=lambda c: O.NAMES[c[0]])
def test_driver_recovers_delay(case):
    c, fs, period, prn, delay, seed = case[:6]
    code = O.resampled_code(c, prn, float(period), 2 * period)
    f0 = 1200.0 if c == O.GPS else 0.0
    sig = synth_signal(code, period, delay, f0, fs, 0.05, seed)
    r = O.acquire_single(c, sig, phasepoints(fs, len(sig)), fs, 0.0, 3000.0, prn, period)
    assert int(round(r["codephase_frac"] * period)) == expected_recovered_sample(period, delay)
    assert 0.0 <= r["codephase_frac"] < 1.0 and r["signal_strength"] > 0.0
    if c == O.GPS:
        assert abs(abs(r["frequency"]) - abs(f0)) <= 250.0


@pytest.mark.parametrize("case", DRIVER_CASES, ids=lambda c: O.NAMES[c[0]])
def test_driver_noise_contrast(case):
    c, fs, period, prn = case[:4]
    cdelay, cseed, step = case[6:]
    code = O.resampled_code(c, prn, float(period), 2 * period)
    n = len(code)
    inj = synth_signal(code, period, cdelay, 0.0, fs, 0.05, cseed)
    noise = (np.sin(np.arange(n) * step) * 0.05).astype(np.float32)
    r1 = O.acquire_single(c, inj, phasepoints(fs, n), fs, 0.0, 3000.0, prn, period)
    r2 = O.acquire_single(c, noise, phasepoints(fs, n), fs, 0.0, 3000.0, prn, period)
    assert r1["signal_strength"] > 10.0 * r2["signal_strength"]


@pytest.mark.parametrize("case", [DRIVER_CASES[0], DRIVER_CASES[4]], ids=["gps", "sbas"])
def test_driver_sweep_period_boundary(case):
    c, fs, period, prn = case[:4]
    delay = 100
    lengths = list(range(period - 3, period + 13)) + list(range(2 * period - 3, 2 * period + 5))
    for n in lengths:
        code = O.resampled_code(c, prn, float(period), n)
        assert len(code) == n
        sig = np.array([code[(i + delay) % n] for i in range(n)], dtype=np.float32)
        r = O.acquire_single(c, sig, phasepoints(fs, n), fs, 0.0, 3000.0, prn, period)
        assert 0.0 <= r["codephase_frac"] < 1.0 and r["signal_strength"] > 0.0, n


# (constellation, period, delay step, seed base, trials (no flip, flip), table)
CN0_CASES = [
    (O.GPS, 16368, 137, 0xACE0, (80, 120), 0),
    (O.GALILEO, 65472, 251, 0xEA11, (60, 120), 1),
    (O.BEIDOU, 163680, 379, 0xB011, (50, 120), 2),
]


@pytest.mark.parametrize("case", CN0_CASES, ids=lambda c: O.NAMES[c[0]])
def test_cn0_acr_end_to_end(case):
    c, period, step, seed0, trials, table = case
    fs, f0, cn0 = 16.368e6, 100e3, 45.0
    code = O.resampled_code(c, 1, float(period), 2 * period)
    pp = phasepoints(fs, 2 * period)
    for flip, n_trials, lo, hi in ((False, trials[0], -1.0, 1.0), (True, trials[1], -4.0, -0.5)):
        ests = []
        for t in range(n_trials):
            delay = (t * step) % period
            cont = synth_signal_cn0(code, period, delay, f0, fs, cn0, seed0 + t, flip).astype(np.float64)
            sig = quantize_bipolar_demean(cont)
            r = O.acquire_single(c, sig, pp, fs, f0, 0.0, 1, period)
            v = O.estimate_cn0((r["signal_strength"] / r["second_peak"]) ** 2, table)
            if v is not None:
                ests.append(v)
        assert ests
        d = O.median(ests) - cn0
        assert lo <= d <= hi, (flip, d)


def test_acquire_all_prn_and_antenna_filters():
    fs = 2.046e6
    samples = 2 * int(fs / 1000.0)
    bits = np.array([[(i + a * 31) % 2 for i in range(samples)] for a in range(2)], dtype=np.uint8)
    out = O.acquire_all(bits, fs, O.GPS, ant_filter=[0], prn_filter=[2, 5, 9])
    assert out["antenna_numbers"] == [0]
    assert [r["sv"] for r in out["results"]] == ["GPS02", "GPS05", "GPS09"]
    assert len(out["results"][0]["strengths"]) == 1
    assert "phase_median" not in out["results"][0] and "freq_mad" not in out["results"][0]
