"""GPU parity: the CUDA path, called through the C ABI, against the CPU oracle.

Covers the reference's driver tests at their own small sampling rates, the
production rate (16.368 MHz, one-bit samples) for all six constellations with
and without a sign flip between the two periods, the real TART recording,
and edge cases (dead channel, single bin, noise only)."""
import os

import numpy as np
import pytest

import acq_oracle as O
import tga
from parity import DETECT_RATIO, REL_TOL, assert_cell_parity, detected, rel
from testutil import phasepoints, quantize_bipolar_demean, synth_signal, synth_signal_cn0

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = tga.Context(0)
    yield c
    c.close()


def _as_dict(r):
    return dict(signal_strength=r.signal_strength, second_peak=r.second_peak, best_codephase=r.best_codephase,
                best_freq_idx=r.best_freq_idx, frequency=r.frequency, codephase_frac=r.codephase_frac)


DRIVER_CASES = [
    (O.GPS, 2.046e6, 2046, 1, 500, 1),
    (O.GALILEO, 1.023e6, 4092, 1, 900, 11),
    (O.BEIDOU, 1.023e6, 10230, 1, 3000, 21),
    (O.L1C, 1.023e6, 10230, 1, 2500, 31),
    (O.SBAS, 1.023e6, 1023, 120, 400, 41),
    (O.QZSS, 1.023e6, 1023, 184, 250, 51),
]


@pytest.mark.parametrize("case", DRIVER_CASES, ids=lambda c: O.NAMES[c[0]])
def test_driver_cases_match_oracle(ctx, case):
    # acquisition.rs:426, galileo.rs:401, beidou.rs:352, l1c.rs:361, sbas.rs:458, qzss.rs:457
    c, fs, period, prn, delay, seed = case
    code = O.resampled_code(c, prn, float(period), 2 * period)
    f0 = 1200.0 if c == O.GPS else 0.0
    sig = synth_signal(code, period, delay, f0, fs, 0.05, seed)
    pp = phasepoints(fs, len(sig))
    g = ctx.acquire_single(c, sig, pp, fs, 0.0, 3000.0, prn, period)
    r = O.acquire_single(c, sig, pp, fs, 0.0, 3000.0, prn, period, grid=True)
    assert g.path == 0
    assert int(round(g.codephase_frac * period)) == (period - delay) % period
    assert_cell_parity(_as_dict(g), r, O.NAMES[c])


PROD = [(O.GPS, 7), (O.SBAS, 133), (O.QZSS, 195), (O.GALILEO, 19), (O.BEIDOU, 30), (O.L1C, 12)]


@pytest.mark.parametrize("flip", [False, True], ids=["noflip", "flip"])
@pytest.mark.parametrize("c,prn", PROD, ids=[O.NAMES[c] for c, _ in PROD])
def test_production_rate_one_bit(ctx, c, prn, flip):
    fs = 16.368e6
    period = O.period_samples(c, fs)
    code = O.resampled_code(c, prn, float(period), 2 * period)
    delay = (prn * 7919) % period
    f0 = 4.092e6 + 1234.5
    cont = synth_signal_cn0(code, period, delay, f0, fs, 50.0 if flip else 47.0, 0xC0DE + prn,
                            flip).astype(np.float64)
    sig = quantize_bipolar_demean(cont)
    pp = phasepoints(fs, len(sig))
    g = ctx.acquire_single(c, sig, pp, fs, 4.092e6, 6000.0, prn, period)
    r = O.acquire_single(c, sig, pp, fs, 4.092e6, 6000.0, prn, period, threads=8, grid=True)
    if not flip:
        assert detected(r["signal_strength"], r["second_peak"])
    assert_cell_parity(_as_dict(g), r, (O.NAMES[c], flip))
    assert g.hypothesis == r["hypothesis"]


@pytest.mark.parametrize("c", [O.GPS, O.GALILEO, O.BEIDOU], ids=["ca", "e1", "boc"])
def test_noise_only_values(ctx, c):
    fs = 16.368e6
    period = O.period_samples(c, fs)
    rng = np.random.default_rng(5)
    sig = quantize_bipolar_demean(rng.standard_normal(2 * period))
    pp = phasepoints(fs, len(sig))
    prn = O.PRN_RANGE[c][0] + 4
    g = ctx.acquire_single(c, sig, pp, fs, 4.092e6, 6000.0, prn, period)
    r = O.acquire_single(c, sig, pp, fs, 4.092e6, 6000.0, prn, period, threads=8)
    assert rel(g.signal_strength, r["signal_strength"]) <= REL_TOL
    assert rel(g.second_peak, r["second_peak"]) <= REL_TOL


def test_dead_channel_and_single_bin(ctx):
    # all-zero samples: every correlation is 0 -> last index wins, second = 1e-6
    fs, period = 2.046e6, 2046
    sig = np.zeros(2 * period, np.float32)
    pp = phasepoints(fs, len(sig))
    g = ctx.acquire_single(O.GPS, sig, pp, fs, 0.0, 0.0, 3, period)
    r = O.acquire_single(O.GPS, sig, pp, fs, 0.0, 0.0, 3, period)
    assert g.signal_strength == r["signal_strength"] == 0.0
    assert g.second_peak == r["second_peak"] == float(np.float32(1e-6))
    assert g.best_codephase == r["best_codephase"] == period - 1
    assert g.best_freq_idx == r["best_freq_idx"] == 0


def _real():
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "tart_head.npz"))
    return z["head"], z["ones"], int(z["row_bytes"]), float(z["sampling_frequency"])


def _real_bits_for_gpu(head, ones, row_bytes):
    """Rebuild rows of the original length whose one-count equals the full
    record's (so the de-mean is identical) and whose head is the real data."""
    n_ant, hb = head.shape
    rows = np.zeros((n_ant, row_bytes), np.uint8)
    rows[:, :hb] = head
    for a in range(n_ant):
        need = int(ones[a]) - int(np.unpackbits(head[a]).sum())
        full, rem = divmod(need, 8)
        rows[a, hb:hb + full] = 0xFF
        if rem:
            rows[a, hb + full] = (0xFF << (8 - rem)) & 0xFF
    return rows


@pytest.mark.parametrize("c,prns", [(O.GPS, [6, 19, 9, 1]), (O.SBAS, [127, 129, 144, 120]),
                                    (O.GALILEO, [34, 15]), (O.BEIDOU, [1, 20]), (O.L1C, [4]),
                                    (O.QZSS, [206, 195])], ids=lambda x: O.NAMES[x] if isinstance(x, int) else "p")
def test_real_recording_acquire_all(ctx, c, prns):
    head, ones, row_bytes, fs = _real()
    rows = _real_bits_for_gpu(head, ones, row_bytes)
    ants = [0, 7, 23]
    out = ctx.acquire_all(rows, fs, mask=1 << c, ant_filter=ants, prn_filter=prns, cn0=True)[O.NAMES[c]]
    bits = np.unpackbits(rows, axis=1)
    ref = O.acquire_all(bits, fs, c, ant_filter=ants, prn_filter=prns, cn0=True, threads=8, grid=True)
    assert out["antenna_numbers"] == ref["antenna_numbers"]
    assert [r["sv"] for r in out["results"]] == [r["sv"] for r in ref["results"]]
    for go, ro in zip(out["results"], ref["results"]):
        for a in range(len(ants)):
            cell = ro["cells"][a]
            g = dict(signal_strength=go["strengths"][a], second_peak=go["second_peaks"][a],
                     best_codephase=go["best_codephase"][a], best_freq_idx=go["best_freq_idx"][a],
                     frequency=go["freqs"][a], codephase_frac=go["phases"][a])
            assert_cell_parity(g, cell, (ro["sv"], ants[a]))
        if ro.get("cn0_acr") is None:
            assert go.get("cn0_acr") is None
        else:
            for x, y in zip(go["cn0_acr"], ro["cn0_acr"]):
                assert (x is None) == (y is None)
                if x is not None:
                    assert abs(x - y) <= REL_TOL * abs(y)
        if all(detected(cl["signal_strength"], cl["second_peak"]) for cl in ro["cells"]):
            for k in ("phase_median", "freq_median", "phase_mad", "freq_mad"):
                assert go[k] == ro[k], k


def test_acr_batch_matches_oracle(ctx):
    for tid in range(4):
        t = O.acr_table(tid)
        ra = np.concatenate([t[:, 0], np.geomspace(0.5, t[-1, 0] * 3, 400), [1.0, np.nan, np.inf]])
        got = ctx.estimate_cn0_batch(ra, tid)
        for r, gv in zip(ra, got):
            ov = O.estimate_cn0(r, tid)
            assert (gv is None) == (ov is None), r
            if gv is not None:
                assert abs(gv - ov) <= 1e-12 * abs(ov), (r, gv, ov)


def test_antenna_xcorr_bit_exact(ctx):
    head, ones, row_bytes, fs = _real()
    rows = _real_bits_for_gpu(head, ones, row_bytes)
    bits = np.unpackbits(rows, axis=1)
    m = ctx.correlation_matrix(rows)
    for i, j in [(0, 1), (3, 17), (5, 5), (23, 0)]:
        exp = O.correlate_antennas(bits[i], bits[j])
        assert m[i, j] == exp and ctx.correlate(rows, i, j) == exp


@pytest.mark.parametrize("case", [DRIVER_CASES[0], DRIVER_CASES[4], DRIVER_CASES[1]], ids=["gps", "sbas", "galileo"])
def test_generic_path_period_boundary_sweep(ctx, case):
    # acquisition.rs:487-515, sbas.rs:491, galileo.rs:436: lengths around the
    # period boundaries, most of them not 2 periods -> generic (Bluestein) path
    c, fs, period, prn = case[:4]
    delay = 100
    lengths = list(range(period - 3, period + 13, 3)) + list(range(2 * period - 3, 2 * period + 5))
    for n in lengths:
        code = O.resampled_code(c, prn, float(period), n)
        sig = code[(np.arange(n) + delay) % n].astype(np.float32)
        pp = phasepoints(fs, n)
        g = ctx.acquire_single(c, sig, pp, fs, 0.0, 3000.0, prn, period)
        r = O.acquire_single(c, sig, pp, fs, 0.0, 3000.0, prn, period, grid=True)
        assert g.path == (0 if n == 2 * period else 1), n
        assert 0.0 <= g.codephase_frac < 1.0 and g.signal_strength > 0.0, n
        assert_cell_parity(_as_dict(g), r, ("n", n))


def test_generic_path_16mhz_one_bit(ctx):
    # 16 MHz sampling (the reference's --benchmark rate): 15.64 samples per
    # chip, so the code is not a fixed polyphase pattern -> generic path
    fs, c, prn = 16e6, O.GPS, 17
    period = O.period_samples(c, fs)
    code = O.resampled_code(c, prn, float(period), 2 * period)
    cont = synth_signal_cn0(code, period, 777, 4.092e6 - 2345.0, fs, 48.0, 99, False).astype(np.float64)
    sig = quantize_bipolar_demean(cont)
    pp = phasepoints(fs, len(sig))
    g = ctx.acquire_single(c, sig, pp, fs, 4.092e6, 6000.0, prn, period)
    r = O.acquire_single(c, sig, pp, fs, 4.092e6, 6000.0, prn, period, threads=8, grid=True)
    assert g.path == 1
    assert_cell_parity(_as_dict(g), r, "16MHz")
