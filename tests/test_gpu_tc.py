"""GPU tests of the tensor-core search (TGA_PRECISION_FP16_TC).

The DFT-31 stage of the search runs on tcgen05 tensor cores with FP16
operands; the row selected for each (antenna, PRN) is re-evaluated in FP32.
Checks: same detections, code phase, Doppler bin and hypothesis as the FP32
mode; reported values within the FP32 tolerance of the oracle; peak metric
within 1e-3 of the FP64 oracle.
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
    assert rel(b.signal_strength, a.signal_strength) <= REL_TOL
    assert b.second_peak == a.second_peak
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


def test_tc_real_recording_same_detections(ctxs):
    f32, tc = ctxs
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "tart_head.npz"))
    head, ones, row_bytes, fs = z["head"], z["ones"], int(z["row_bytes"]), float(z["sampling_frequency"])
    from test_gpu_parity import _real_bits_for_gpu
    rows = _real_bits_for_gpu(head, ones, row_bytes)
    ants = list(range(0, 24, 3))
    for mask in (1 << tga.GPS | 1 << tga.SBAS | 1 << tga.QZSS, 1 << tga.GALILEO, 1 << tga.BEIDOU | 1 << tga.L1C):
        a = f32.acquire_cells(rows, fs, mask=mask, ant_filter=ants, cn0=True)
        b = tc.acquire_cells(rows, fs, mask=mask, ant_filter=ants, cn0=True)
        da = np.array([detected(x, y) for x, y in zip(a["signal_strength"], a["second_peak"])])
        db = np.array([detected(x, y) for x, y in zip(b["signal_strength"], b["second_peak"])])
        assert np.array_equal(da, db)
        sel = da
        for k in ("best_codephase", "best_freq_idx", "hypothesis"):
            assert np.array_equal(a[k][sel], b[k][sel]), k
        same_row = (a["best_freq_idx"] == b["best_freq_idx"]) & (a["hypothesis"] == b["hypothesis"])
        assert np.all(np.abs(b["signal_strength"][same_row] - a["signal_strength"][same_row])
                      <= REL_TOL * a["signal_strength"][same_row])
        # the same row in the same FP32 arithmetic: the second peak read from
        # the re-evaluated row equals the FP32 search's second-peak pass
        assert np.array_equal(b["second_peak"][same_row], a["second_peak"][same_row])
        assert np.array_equal(b["best_codephase"][same_row], a["best_codephase"][same_row])
        # over all cells the selected row agrees almost everywhere
        assert same_row.mean() > 0.9


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
