"""GPU non-coherent search on the tensor cores (TGA_PRECISION_FP16_TC, Lc =
1023): the FP16 two-stage transform picks the bin of every (antenna, PRN),
the FP32 engine re-evaluates that row, so the selected bins and code phases
must be the FP32 search's wherever a satellite is present and every reported
power must be the FP32 power of the selected row; other code lengths run the
FP32 search in either precision; an expired wait is reported as a timeout."""
import numpy as np
import pytest

import acq_oracle as O
import nc_oracle as NC
import tga
from parity import REL_TOL
from test_nc_cpu import FS, synth

pytestmark = pytest.mark.gpu

P = 16368


@pytest.fixture(scope="module")
def ctx():
    c = tga.Context(0)
    yield c
    c.close()


def _both(ctx, bits, constellation, **kw):
    ctx.set_precision(tga.PRECISION_FP32)
    f32 = ctx.search_noncoherent(bits, FS, constellation, **kw)
    ctx.set_precision(tga.PRECISION_FP16_TC)
    try:
        tc = ctx.search_noncoherent(bits, FS, constellation, **kw)
    finally:
        ctx.set_precision(tga.PRECISION_FP32)
    return f32, tc


def _same_row_same_power(f32, tc):
    same = (f32["best_freq_idx"] == tc["best_freq_idx"]) & (f32["best_codephase"] == tc["best_codephase"])
    np.testing.assert_allclose(tc["power"][same], f32["power"][same], rtol=REL_TOL)
    np.testing.assert_allclose(tc["second_power"][same], f32["second_power"][same], rtol=REL_TOL, atol=1e-30)
    return same


def test_weak_10ms_coherent_matches_fp32_and_oracle(ctx):
    sats = [(O.GPS, 2, 4321, 620.0, 34.0), (O.GPS, 11, 9000, -310.0, 34.0), (O.GPS, 23, 222, 45.0, 34.0)]
    bits = synth(sats, 30 * P + 5000, seed=33, n_ant=2)
    prns = [2, 11, 23, 31]
    kw = dict(prns=prns, center_freq=4.092e6, bin_step_hz=50.0, n_bins=41, coherent_periods=10, blocks=3,
              start=5000)
    f32, tc = _both(ctx, bits, tga.GPS, **kw)
    same = _same_row_same_power(f32, tc)
    present = f32["prn"] != 31
    assert np.all(same[present])
    want = NC.search_nc(bits, FS, O.GPS, prns, [0, 1], 4.092e6, 50.0, 41, 10, 3, 5000)
    for g, w in zip(tc[present], [w for w in want if w["prn"] != 31]):
        assert g["best_codephase"] == w["best_codephase"] and g["best_freq_idx"] == w["best_freq_idx"]
        assert abs(g["power"] - w["power"]) <= REL_TOL * w["power"]


@pytest.mark.parametrize("blocks", [1, 2, 5])
def test_block_counts(ctx, blocks):
    sats = [(O.GPS, 5, 700, -1200.0, 40.0), (O.GPS, 19, 16000, 2400.0, 40.0)]
    bits = synth(sats, blocks * 4 * P, seed=50 + blocks, n_ant=3)
    kw = dict(prns=[5, 19, 30], bin_step_hz=250.0, n_bins=41, coherent_periods=4, blocks=blocks)
    f32, tc = _both(ctx, bits, tga.GPS, **kw)
    same = _same_row_same_power(f32, tc)
    assert np.all(same[f32["prn"] != 30])


def test_sbas_and_qzss_codes(ctx):
    sats = [(O.SBAS, 133, 3000, 800.0, 42.0)]
    bits = synth(sats, 20 * P, seed=7)
    f32, tc = _both(ctx, bits, tga.SBAS, prns=[133, 135], bin_step_hz=100.0, n_bins=21, coherent_periods=10,
                    blocks=2)
    same = _same_row_same_power(f32, tc)
    assert same[0]


def test_other_code_lengths_run_fp32(ctx):
    bits = synth([(O.GALILEO, 12, 20000, 500.0, 45.0)], 2 * 65472, seed=8)
    kw = dict(prns=[12, 13], bin_step_hz=250.0, n_bins=9, coherent_periods=1, blocks=2)
    f32, tc = _both(ctx, bits, tga.GALILEO, **kw)
    for k in ("best_freq_idx", "best_codephase", "power", "second_power"):
        np.testing.assert_array_equal(tc[k], f32[k])


def test_expired_wait_is_a_timeout(ctx):
    bits = synth([(O.GPS, 3, 100, 0.0, 45.0)], 2 * P, seed=9)
    ctx.set_precision(tga.PRECISION_FP16_TC)
    ctx.set_test_flags(tga.TEST_TC_SKIP_COMMIT)
    try:
        with pytest.raises(tga.TgaError) as e:
            ctx.search_noncoherent(bits, FS, tga.GPS, prns=[3], bin_step_hz=500.0, n_bins=3, coherent_periods=1,
                                   blocks=2)
        assert e.value.code == 6  # TGA_ERR_TIMEOUT
    finally:
        ctx.set_test_flags(0)
        ctx.set_precision(tga.PRECISION_FP32)
    f32, tc = _both(ctx, bits, tga.GPS, prns=[3], bin_step_hz=500.0, n_bins=3, coherent_periods=1, blocks=2)
    assert tc["best_codephase"][0] == f32["best_codephase"][0] == (P - 100) % P


@pytest.mark.parametrize("fs", [4.092e6, 8.184e6], ids=["S4", "S8"])
def test_other_integer_rates(ctx, fs):
    """4 and 8 samples per chip: fewer polyphase residues in the front end and
    smaller folded magnitudes ahead of the FP16 scaling; IF at fs/4."""
    import math
    Pf = O.period_samples(O.GPS, fs)
    n = 12 * Pf
    rng = np.random.default_rng(int(fs) % 997)
    t = np.arange(n)
    x = rng.standard_normal((2, n))
    sats = [(9, 1234, 900.0), (27, Pf - 3, -1750.0)]
    for prn, delay, dop in sats:
        code = O.resampled_code(O.GPS, prn, float(Pf), Pf).astype(np.float64)
        amp = 2.0 * math.sqrt(10.0 ** (40.0 / 10.0) / fs)
        for a in range(2):
            x[a] += amp * code[(t + delay) % Pf] * np.cos(2 * np.pi * (fs / 4 + dop) / fs * t + rng.uniform(0, 6.28))
    bits = np.packbits(x >= 0, axis=1)
    kw = dict(prns=[9, 27, 14], center_freq=fs / 4, bin_step_hz=250.0, n_bins=21, coherent_periods=4, blocks=3)
    ctx.set_precision(tga.PRECISION_FP32)
    f32 = ctx.search_noncoherent(bits, fs, tga.GPS, **kw)
    ctx.set_precision(tga.PRECISION_FP16_TC)
    try:
        tc = ctx.search_noncoherent(bits, fs, tga.GPS, **kw)
    finally:
        ctx.set_precision(tga.PRECISION_FP32)
    same = _same_row_same_power(f32, tc)
    present = f32["prn"] != 14
    assert np.all(same[present])
    for g in tc[present]:
        delay = dict((p, d) for p, d, _ in sats)[int(g["prn"])]
        assert int(g["best_codephase"]) == (Pf - delay) % Pf
