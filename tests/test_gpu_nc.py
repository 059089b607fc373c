"""GPU non-coherent search (tga_search_noncoherent) against the oracle:
the 1 ms x 10 GPS C/A search with 21 x 500 Hz bins, a weak-signal search with
10 ms coherent blocks and 50 Hz bins (reduced in antennas, blocks and bins),
a BOC class, and the two-period single block against the drop-in search."""
import numpy as np
import pytest

import acq_oracle as O
import nc_oracle as NC
import tga
from parity import REL_TOL
from test_nc_cpu import FS, synth

pytestmark = pytest.mark.gpu


def _compare(got, want):
    assert len(got) == len(want)
    for g, w in zip(got, want):
        assert (g["prn"], g["antenna"]) == (w["prn"], w["antenna"])
        assert g["best_codephase"] == w["best_codephase"] and g["best_freq_idx"] == w["best_freq_idx"], (g, w)
        assert abs(g["power"] - w["power"]) <= REL_TOL * w["power"]
        assert abs(g["second_power"] - w["second_power"]) <= REL_TOL * max(w["second_power"], 1e-30)
        assert abs(g["frequency"] - w["frequency"]) <= 1e-9


@pytest.fixture(scope="module")
def ctx():
    c = tga.Context(0)
    yield c
    c.close()


def test_ca_1ms_x10_21_bins(ctx):
    P = 16368
    sats = [(O.GPS, 4, 1234, -3300.0, 45.0), (O.GPS, 9, 8000, 2100.0, 45.0), (O.GPS, 17, 15000, 450.0, 45.0),
            (O.GPS, 28, 77, -4900.0, 45.0)]
    bits = synth(sats, 10 * P, seed=21)
    prns = [4, 9, 17, 28, 30]
    got = ctx.search_noncoherent(bits, FS, tga.GPS, prns=prns, bin_step_hz=500.0, n_bins=21, coherent_periods=1,
                                 blocks=10)
    want = NC.search_nc(bits, FS, O.GPS, prns, [0], 4.092e6, 500.0, 21, 1, 10, 0)
    _compare(got, want)
    for g, (c, prn, d, dop, _) in zip(got[:4], sats):
        assert g["best_codephase"] == (P - d) % P and abs(g["frequency"] - dop) <= 250.0


def test_weak_10ms_coherent_50hz(ctx):
    P = 16368
    sats = [(O.GPS, 2, 4321, 620.0, 34.0), (O.GPS, 11, 9000, -310.0, 34.0), (O.GPS, 23, 222, 45.0, 34.0)]
    bits = synth(sats, 30 * P + 5000, seed=33, n_ant=2)
    prns = [2, 11, 23, 31]
    kw = dict(center_freq=4.092e6, bin_step_hz=50.0, n_bins=41, coherent_periods=10, blocks=3, start=5000)
    got = ctx.search_noncoherent(bits, FS, tga.GPS, prns=prns, **kw)
    want = NC.search_nc(bits, FS, O.GPS, prns, [0, 1], 4.092e6, 50.0, 41, 10, 3, 5000)
    _compare(got, want)
    det = got[got["prn"] != 31]
    assert np.all(det["power"] > 2.0 * det["second_power"])


def test_boc_class(ctx):
    P = 163680
    bits = synth([(O.BEIDOU, 19, 70000, 900.0, 45.0)], 2 * P, seed=4)
    got = ctx.search_noncoherent(bits, FS, tga.BEIDOU, prns=[19, 20], bin_step_hz=100.0, n_bins=5,
                                 coherent_periods=1, blocks=2, center_freq=4.092e6 + 900.0)
    want = NC.search_nc(bits, FS, O.BEIDOU, [19, 20], [0], 4.092e6 + 900.0, 100.0, 5, 1, 2, 0)
    _compare(got, want)


def test_single_two_period_block_matches_dropin(ctx):
    P = 16368
    bits = synth([(O.GPS, 7, 3000, 1200.0, 50.0)], 2 * P, seed=5)
    grid = O.freq_grid(4.092e6, 6000.0)
    d = ctx.acquire_cells(bits, FS, mask=1 << tga.GPS, prn_filter=[7])[0]
    g = ctx.search_noncoherent(bits, FS, tga.GPS, prns=[7], bin_step_hz=grid[1] - grid[0], n_bins=len(grid),
                               coherent_periods=2, blocks=1)[0]
    assert d["hypothesis"] == 0
    assert g["best_codephase"] == d["best_codephase"] % P and g["best_freq_idx"] == d["best_freq_idx"]
    assert abs(g["power"] - d["signal_strength"] ** 2) <= 2 * REL_TOL * g["power"]


def test_multi_call_equals_single_calls(ctx):
    """tga_search_noncoherent_multi: GPS and SBAS (one shared front end),
    Galileo with its own blocks and grid, in one call, equal to the three
    searches run one by one, in both arithmetics."""
    P = 16368
    sats = [(O.GPS, 6, 4000, 900.0, 44.0), (O.SBAS, 127, 123, -1400.0, 44.0), (O.GALILEO, 8, 30000, 375.0, 44.0)]
    bits = synth(sats, 8 * P, seed=71, n_ant=2)
    searches = [dict(constellation=tga.GPS, prns=[6, 9], bin_step_hz=500.0, n_bins=21, coherent_periods=1, blocks=8),
                dict(constellation=tga.SBAS, prns=[127, 140], bin_step_hz=500.0, n_bins=21, coherent_periods=1,
                     blocks=8),
                dict(constellation=tga.GALILEO, prns=[8, 2], bin_step_hz=125.0, n_bins=41, coherent_periods=1,
                     blocks=2)]
    for prec in (tga.PRECISION_FP32, tga.PRECISION_FP16_TC):
        ctx.set_precision(prec)
        try:
            multi = ctx.search_noncoherent_multi(bits, FS, searches)
            for sd, m in zip(searches, multi):
                kw = {k: v for k, v in sd.items() if k != "constellation"}
                one = ctx.search_noncoherent(bits, FS, sd["constellation"], **kw)
                for k in ("prn", "antenna", "best_freq_idx", "best_codephase", "power", "second_power", "frequency"):
                    np.testing.assert_array_equal(m[k], one[k], err_msg=k)
        finally:
            ctx.set_precision(tga.PRECISION_FP32)
    assert multi[0]["best_codephase"][0] == (P - 4000) % P
    assert multi[1]["best_codephase"][0] == (P - 123) % P
    assert multi[2]["best_codephase"][0] == (4 * P - 30000) % (4 * P)
