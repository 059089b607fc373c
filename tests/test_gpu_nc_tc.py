"""GPU non-coherent search on the tensor cores (TGA_PRECISION_FP16_TC) at
every code length: the FP16 transform's summed keys pick the rows of every
(antenna, PRN) worth re-evaluating (within the FP16 error bound of the
best), the FP32 engine re-evaluates those rows and the bins are reduced over
the FP32 keys, so every cell -- bin, code phase, power and second power --
must equal the FP32 search's.  Lc = 1023 (GPS, SBAS) runs PRN pairs as the
two chains, Lc = 4092 (Galileo) too, Lc = 10230 (BeiDou, L1C) runs pairs of
blocks of one PRN (odd block counts included); satellites present must be
found where the oracle finds them; an expired wait is reported as a
timeout."""
import numpy as np
import pytest

import acq_oracle as O
import nc_oracle as NC
import tga
from parity import REL_TOL
from test_nc_cpu import FS, synth

pytestmark = pytest.mark.gpu

P = 16368
FIELDS = ("prn", "antenna", "best_freq_idx", "best_codephase", "power", "second_power", "frequency")
# amplitude error bound of the FP16 keys relative to the (antenna, PRN)'s
# largest, assumed by the library's candidate rule (kTcKeyKeep)
KEY_BOUND = 2.0 ** -8


@pytest.fixture(scope="module")
def ctx():
    c = tga.Context(0)
    yield c
    c.close()


def _both(ctx, bits, constellation, **kw):
    """FP32 and tensor-core searches, with both arithmetics' row peaks and
    the number of rows the tensor-core search re-evaluated."""
    chips = {tga.GPS: 1023, tga.SBAS: 1023, tga.QZSS: 1023, tga.GALILEO: 4092, tga.BEIDOU: 10230,
             tga.L1C: 10230}[constellation]
    ctx.set_precision(tga.PRECISION_FP32)
    f32 = ctx.search_noncoherent(bits, FS, constellation, **kw)
    rows32, _ = ctx.row_peaks(chips)
    ctx.set_precision(tga.PRECISION_FP16_TC)
    try:
        tc = ctx.search_noncoherent(bits, FS, constellation, **kw)
        rows16, refined = ctx.row_peaks(chips)
    finally:
        ctx.set_precision(tga.PRECISION_FP32)
    return f32, tc, (rows32, rows16, refined)


def _identical(f32, tc, rows, n_bins):
    for k in FIELDS:
        np.testing.assert_array_equal(tc[k], f32[k], err_msg=k)
    rows32, rows16, refined = rows
    n_prn = len(np.unique(f32["prn"]))
    a = np.sqrt(rows32.reshape(-1, n_bins, n_prn))
    b = np.sqrt(rows16.reshape(-1, n_bins, n_prn))
    err = float((np.abs(b - a).max(axis=1) / b.max(axis=1)).max())
    assert err < KEY_BOUND, err
    assert len(f32) <= refined <= len(f32) * n_bins
    return err, refined


def _oracle_agrees(tc, want, absent):
    for g, w in zip(tc, want):
        assert (g["prn"], g["antenna"]) == (w["prn"], w["antenna"])
        if g["prn"] in absent:
            continue
        assert g["best_codephase"] == w["best_codephase"] and g["best_freq_idx"] == w["best_freq_idx"], (g, w)
        assert abs(g["power"] - w["power"]) <= REL_TOL * w["power"]


def test_weak_10ms_coherent_matches_fp32_and_oracle(ctx):
    sats = [(O.GPS, 2, 4321, 620.0, 34.0), (O.GPS, 11, 9000, -310.0, 34.0), (O.GPS, 23, 222, 45.0, 34.0)]
    bits = synth(sats, 30 * P + 5000, seed=33, n_ant=2)
    prns = [2, 11, 23, 31]
    kw = dict(prns=prns, center_freq=4.092e6, bin_step_hz=50.0, n_bins=41, coherent_periods=10, blocks=3,
              start=5000)
    f32, tc, rows = _both(ctx, bits, tga.GPS, **kw)
    _identical(f32, tc, rows, 41)
    want = NC.search_nc(bits, FS, O.GPS, prns, [0, 1], 4.092e6, 50.0, 41, 10, 3, 5000)
    _oracle_agrees(tc, want, {31})


@pytest.mark.parametrize("blocks", [1, 2, 5])
def test_block_counts(ctx, blocks):
    sats = [(O.GPS, 5, 700, -1200.0, 40.0), (O.GPS, 19, 16000, 2400.0, 40.0)]
    bits = synth(sats, blocks * 4 * P, seed=50 + blocks, n_ant=3)
    kw = dict(prns=[5, 19, 30], bin_step_hz=250.0, n_bins=41, coherent_periods=4, blocks=blocks)
    f32, tc, rows = _both(ctx, bits, tga.GPS, **kw)
    _identical(f32, tc, rows, 41)


def test_sbas_codes(ctx):
    sats = [(O.SBAS, 133, 3000, 800.0, 42.0)]
    bits = synth(sats, 20 * P, seed=7)
    f32, tc, rows = _both(ctx, bits, tga.SBAS, prns=[133, 135], bin_step_hz=100.0, n_bins=21, coherent_periods=10,
                          blocks=2)
    _identical(f32, tc, rows, 21)
    assert tc["best_codephase"][0] == (P - 3000) % P


@pytest.mark.parametrize("blocks", [2, 3], ids=["even", "odd"])
def test_galileo_e1c(ctx, blocks):
    """Lc = 4092 (E1-C, 4 ms periods, BOC(1,1) pulse in the front end): the
    three-stage tensor-core transform with PRN-pair chains."""
    Pg = 65472
    sats = [(O.GALILEO, 12, 20000, 500.0, 44.0), (O.GALILEO, 30, 777, -2250.0, 44.0)]
    bits = synth(sats, blocks * Pg, seed=8 + blocks, n_ant=2)
    prns = [12, 30, 5]
    kw = dict(prns=prns, bin_step_hz=125.0, n_bins=41, coherent_periods=1, blocks=blocks)
    f32, tc, rows = _both(ctx, bits, tga.GALILEO, **kw)
    _identical(f32, tc, rows, 41)
    want = NC.search_nc(bits, FS, O.GALILEO, prns, [0, 1], 4.092e6, 125.0, 41, 1, blocks, 0)
    _oracle_agrees(tc, want, {5})


@pytest.mark.parametrize("c,prns", [(tga.BEIDOU, [21, 40, 7]), (tga.L1C, [3, 61, 30])], ids=["beidou", "l1c"])
@pytest.mark.parametrize("blocks", [2, 3], ids=["even", "odd"])
def test_boc_10230(ctx, c, prns, blocks):
    """Lc = 10230 (B1C / L1C pilots, 10 ms periods): the chains take the
    blocks of one PRN two at a time (an odd count leaves chain b a zero
    block in the last round)."""
    Pb = 163680
    sats = [(c, prns[0], 100000, 250.0, 42.0), (c, prns[1], 3333, -1950.0, 42.0)]
    bits = synth(sats, blocks * Pb, seed=60 + blocks + c, n_ant=2)
    kw = dict(prns=prns, bin_step_hz=50.0, n_bins=21, coherent_periods=1, blocks=blocks)
    f32, tc, rows = _both(ctx, bits, c, **kw)
    _identical(f32, tc, rows, 21)
    want = NC.search_nc(bits, FS, c, prns, [0, 1], 4.092e6, 50.0, 21, 1, blocks, 0)
    _oracle_agrees(tc, want, {prns[2]})


def test_noise_only_cells_identical(ctx):
    """No satellite: the best rows of an (antenna, PRN) are close to each
    other, the case the FP16 bound exists for."""
    rng = np.random.default_rng(0x5EED)
    for c, per, blocks in ((tga.GPS, P, 4), (tga.GALILEO, 65472, 2), (tga.BEIDOU, 163680, 2)):
        bits = np.packbits(rng.integers(0, 2, size=(3, blocks * per), dtype=np.uint8), axis=1)
        kw = dict(prns=[1, 2, 3, 4], bin_step_hz=100.0, n_bins=31, coherent_periods=1, blocks=blocks)
        f32, tc, rows = _both(ctx, bits, c, **kw)
        err, refined = _identical(f32, tc, rows, 31)
        print("\nnoise, constellation %d: FP16 key error %.2e, %d rows re-evaluated for %d cells"
              % (c, err, refined, len(f32)))


def test_expired_wait_is_a_timeout(ctx):
    for c, per in ((tga.GPS, P), (tga.BEIDOU, 163680)):
        bits = synth([(c, 3, 100, 0.0, 45.0)], 2 * per, seed=9)
        ctx.set_precision(tga.PRECISION_FP16_TC)
        ctx.set_test_flags(tga.TEST_TC_SKIP_COMMIT)
        try:
            with pytest.raises(tga.TgaError) as e:
                ctx.search_noncoherent(bits, FS, c, prns=[3], bin_step_hz=500.0, n_bins=3, coherent_periods=1,
                                       blocks=2)
            assert e.value.code == 6  # TGA_ERR_TIMEOUT
        finally:
            ctx.set_test_flags(0)
            ctx.set_precision(tga.PRECISION_FP32)
        f32, tc, _ = _both(ctx, bits, c, prns=[3], bin_step_hz=500.0, n_bins=3, coherent_periods=1, blocks=2)
        assert tc["best_codephase"][0] == f32["best_codephase"][0] == (per - 100) % per


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
    for k in FIELDS:
        np.testing.assert_array_equal(tc[k], f32[k], err_msg=k)
    for g in tc[tc["prn"] != 14]:
        delay = dict((p, d) for p, d, _ in sats)[int(g["prn"])]
        assert int(g["best_codephase"]) == (Pf - delay) % Pf
