"""GPU tests of the tensor-core search (TGA_PRECISION_FP16_TC).

The inverse transforms of the search run on tcgen05 tensor cores with FP16
operands; every row whose FP16 key lies within the FP16 error bound of its
(antenna, PRN)'s best is re-evaluated in FP32, and the bins are reduced over
those FP32 keys.  Checks: every cell identical to the FP32 mode's (code
phase, Doppler bin, hypothesis, peak, second peak, C/N0); the FP16 keys'
error inside the bound the candidate rule assumes; reported values within
the FP32 tolerance of the oracle and 1e-3 of the FP64 oracle.
"""
import os

import numpy as np
import pytest

import acq_oracle as O
import tga
from parity import REL_TOL, assert_cell_parity, detected, rel
from testutil import phasepoints, quantize_bipolar_demean, synth_signal_cn0

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctxs():
    a, b = tga.Context(0), tga.Context(0)
    b.set_precision(tga.PRECISION_FP16_TC)
    yield a, b
    a.close()
    b.close()


def _sig(c, prn, cn0, flip, seed, dop=1234.5):
    fs = 16.368e6
    period = O.period_samples(c, fs)
    code = O.resampled_code(c, prn, float(period), 2 * period)
    cont = synth_signal_cn0(code, period, (prn * 7919) % period, 4.092e6 + dop, fs, cn0, seed, flip)
    sig = quantize_bipolar_demean(cont.astype(np.float64))
    return sig, phasepoints(fs, len(sig)), period, fs


@pytest.mark.parametrize("c,prn", [(O.GPS, 7), (O.SBAS, 133), (O.QZSS, 195), (O.GALILEO, 19), (O.BEIDOU, 30),
                                   (O.L1C, 12)], ids=["gps", "sbas", "qzss", "galileo", "beidou", "l1c"])
@pytest.mark.parametrize("flip", [False, True], ids=["noflip", "flip"])
def test_tc_single_matches_fp32_and_oracle(ctxs, c, prn, flip):
    f32, tc = ctxs
    sig, pp, period, fs = _sig(c, prn, 50.0 if flip else 47.0, flip, 0xC0DE + prn)
    a = f32.acquire_single(c, sig, pp, fs, 4.092e6, 6000.0, prn, period)
    b = tc.acquire_single(c, sig, pp, fs, 4.092e6, 6000.0, prn, period)
    assert (b.best_codephase, b.best_freq_idx, b.hypothesis) == (a.best_codephase, a.best_freq_idx, a.hypothesis)
    assert b.signal_strength == a.signal_strength and b.second_peak == a.second_peak
    r = O.acquire_single(c, sig, pp, fs, 4.092e6, 6000.0, prn, period, threads=8, grid=True)
    assert_cell_parity(dict(signal_strength=b.signal_strength, second_peak=b.second_peak,
                            best_codephase=b.best_codephase, best_freq_idx=b.best_freq_idx,
                            frequency=b.frequency, codephase_frac=b.codephase_frac), r, "tc")


def test_tc_peak_error_vs_fp64(ctxs):
    _, tc = ctxs
    for c, prn in [(O.GPS, 3), (O.GALILEO, 5), (O.BEIDOU, 9)]:
        sig, pp, period, fs = _sig(c, prn, 46.0, False, 0xF64 + prn, dop=-2100.0)
        b = tc.acquire_single(c, sig, pp, fs, 4.092e6, 6000.0, prn, period)
        r = O.acquire_single(c, sig, pp, fs, 4.092e6, 6000.0, prn, period, precision="f64", threads=8)
        assert rel(b.signal_strength, r["signal_strength"]) <= 1e-3
        assert b.best_codephase == r["best_codephase"] and b.best_freq_idx == r["best_freq_idx"]


CELL_FIELDS = ("best_codephase", "best_freq_idx", "hypothesis", "signal_strength", "second_peak", "codephase_frac",
               "frequency", "cn0_valid", "cn0_acr")
# amplitude error bound of the FP16 row keys, relative to the largest row
# amplitude of the (antenna, PRN), that the candidate rule of the library
# assumes (kTcKeyKeep = (1 - 2 d)^2, d = 2^-8)
KEY_BOUND = 2.0 ** -8
GROUPS = [(1 << tga.GPS | 1 << tga.SBAS | 1 << tga.QZSS, 1023), (1 << tga.GALILEO, 4092),
          (1 << tga.BEIDOU | 1 << tga.L1C, 10230)]


def _real_rows():
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "tart_head.npz"))
    head, ones, row_bytes, fs = z["head"], z["ones"], int(z["row_bytes"]), float(z["sampling_frequency"])
    from test_gpu_parity import _real_bits_for_gpu
    return _real_bits_for_gpu(head, ones, row_bytes), fs


def _check_keys(f32, tc, chips, n_ant, n_bins, n_prn):
    a, _ = f32.row_peaks(chips)
    b, refined = tc.row_peaks(chips)
    a = a.reshape(n_ant, n_bins * 2, n_prn)
    b = b.reshape(n_ant, n_bins * 2, n_prn)
    err = (np.abs(b - a).max(axis=1) / b.max(axis=1)).max()
    return float(err), refined


def test_tc_real_recording_equals_fp32(ctxs):
    """Every cell of the real TART recording, detected or not, identical to
    the FP32 search, and the FP16 keys inside the assumed error bound."""
    f32, tc = ctxs
    rows, fs = _real_rows()
    ants = list(range(0, 24, 3))
    for mask, chips in GROUPS:
        a = f32.acquire_cells(rows, fs, mask=mask, ant_filter=ants, cn0=True)
        b = tc.acquire_cells(rows, fs, mask=mask, ant_filter=ants, cn0=True)
        for k in CELL_FIELDS:
            assert np.array_equal(a[k], b[k]), (chips, k)
        n_prn = len(a) // len(ants)
        err, refined = _check_keys(f32, tc, chips, len(ants), 41, n_prn)
        print("\nLc=%d: FP16 key error %.2e of the row maximum (bound %.2e), %d of %d rows re-evaluated"
              % (chips, err, KEY_BOUND, refined, len(ants) * 82 * n_prn))
        assert err < KEY_BOUND
        assert len(a) <= refined < len(a) * 82


def test_tc_noise_cells_equal_fp32(ctxs):
    """Signal-free cells, where the best rows of an (antenna, PRN) are close
    to each other: the choice still equals the FP32 search's on every cell."""
    f32, tc = ctxs
    rng = np.random.default_rng(0xA015E)
    fs, n_ant = 16.368e6, 6
    bits = np.packbits(rng.integers(0, 2, size=(n_ant, 2 * 163680), dtype=np.uint8), axis=1)
    for mask, chips in GROUPS:
        a = f32.acquire_cells(bits, fs, mask=mask, cn0=True)
        b = tc.acquire_cells(bits, fs, mask=mask, cn0=True)
        for k in CELL_FIELDS:
            assert np.array_equal(a[k], b[k]), (chips, k)
        err, refined = _check_keys(f32, tc, chips, n_ant, 41, len(a) // n_ant)
        print("\nnoise Lc=%d: FP16 key error %.2e, %d rows re-evaluated for %d cells" % (chips, err, refined, len(a)))
        assert err < KEY_BOUND


def test_tc_wait_expiry_reports_timeout_and_context_survives():
    """Failure detection without a fault: with the test hook the correlator
    issues no MMA for its first batch, its bounded wait (1 s) expires, the
    kernel flags it, drains, frees TMEM and returns; the call fails with
    TGA_ERR_TIMEOUT and the same context then searches normally."""
    sig, pp, period, fs = _sig(tga.GPS, 7, 47.0, False, 0x7E57)
    with tga.Context(0) as c:
        c.set_precision(tga.PRECISION_FP16_TC)
        c.set_test_flags(tga.TEST_TC_SKIP_COMMIT)
        with pytest.raises(tga.TgaError) as ei:
            c.acquire_single(tga.GPS, sig, pp, fs, 4.092e6, 6000.0, 7, period)
        assert ei.value.code == 6  # TGA_ERR_TIMEOUT
        c.set_test_flags(0)
        r = c.acquire_single(tga.GPS, sig, pp, fs, 4.092e6, 6000.0, 7, period)
        c.set_precision(tga.PRECISION_FP32)
        f = c.acquire_single(tga.GPS, sig, pp, fs, 4.092e6, 6000.0, 7, period)
    assert (r.best_codephase, r.best_freq_idx) == (f.best_codephase, f.best_freq_idx)


@pytest.mark.parametrize("fs", [2.046e6, 4.092e6, 8.184e6], ids=["S2", "S4", "S8"])
@pytest.mark.parametrize("c,prn", [(O.GPS, 11), (O.GALILEO, 4), (O.BEIDOU, 21)], ids=["gps", "galileo", "beidou"])
def test_tc_other_integer_rates_match_fp32(ctxs, fs, c, prn):
    """Rates with 2, 4 and 8 samples per chip take the fused polyphase front
    end with fewer residues (and smaller folded magnitudes before the FP16
    scaling); the tensor-core search keeps the FP32 mode's answer there too.
    The IF sits at fs/4 so the carrier is below Nyquist at every rate."""
    f32, tc = ctxs
    fc = fs / 4
    period = O.period_samples(c, fs)
    code = O.resampled_code(c, prn, float(period), 2 * period)
    cont = synth_signal_cn0(code, period, (prn * 7919) % period, fc + 1734.0, fs, 47.0, 0x5A7E + prn, False)
    sig = quantize_bipolar_demean(cont.astype(np.float64))
    pp = phasepoints(fs, len(sig))
    a = f32.acquire_single(c, sig, pp, fs, fc, 6000.0, prn, period)
    b = tc.acquire_single(c, sig, pp, fs, fc, 6000.0, prn, period)
    assert (b.best_codephase, b.best_freq_idx, b.hypothesis) == (a.best_codephase, a.best_freq_idx, a.hypothesis)
    assert rel(b.signal_strength, a.signal_strength) <= REL_TOL
    assert rel(b.second_peak, a.second_peak) <= REL_TOL
    assert detected(a.signal_strength, a.second_peak)
    assert int(round(a.codephase_frac * period)) % period == (period - (prn * 7919) % period) % period
