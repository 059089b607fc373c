"""Edge cases of the batched search: results independent of the batch they
are computed in (all antennas and constellations at once versus one antenna
and one constellation), rows whose length is not a multiple of 8 bytes, GPS
PRNs 34 / 37 (shared G2 delay) and 38 (delay 0), recordings shorter than the
search window, and the error paths (out-of-range filters) returning status
codes."""
import numpy as np
import pytest

import acq_oracle as O
import tga
from parity import assert_cell_parity
from testutil import make_observation

pytestmark = pytest.mark.gpu

FS = 16.368e6
N = 327360 + 4000  # two 10 ms periods and some


@pytest.fixture(scope="module")
def rec():
    sats = []
    for c, prn, delay, dop in ((O.GPS, 34, 1200, 800.0), (O.GPS, 38, 9000, -1500.0), (O.GALILEO, 7, 30000, 2500.0),
                               (O.BEIDOU, 21, 100000, -300.0), (O.L1C, 5, 5000, 1800.0)):
        P = O.period_samples(c, FS)
        sats.append(dict(code=O.resampled_code(c, prn, float(P), P), period=P, delay=delay, doppler=dop, cn0=48.0))
    packed, _ = make_observation(6, N, FS, sats, seed=404)
    return packed


def _key(cells):
    return {(int(c["constellation"]), int(c["prn"]), int(c["antenna"])): c for c in cells}


@pytest.mark.parametrize("precision", [tga.PRECISION_FP32, tga.PRECISION_FP16_TC], ids=["fp32", "fp16tc"])
def test_results_do_not_depend_on_the_batch(rec, precision):
    with tga.Context(0) as ctx:
        ctx.set_precision(precision)
        full = _key(ctx.acquire_cells(rec, FS, mask=tga.ALL, cn0=True))
        for c in (tga.GPS, tga.GALILEO, tga.BEIDOU):
            for ant in (1, 4):
                part = _key(ctx.acquire_cells(rec, FS, mask=1 << c, ant_filter=[ant], cn0=True))
                for k, v in part.items():
                    w = full[k]
                    for f in ("best_codephase", "best_freq_idx", "hypothesis", "signal_strength", "second_peak",
                              "cn0_acr", "cn0_valid"):
                        assert v[f] == w[f], (k, f, v[f], w[f])


def test_row_length_not_a_multiple_of_8(rec):
    bits = np.ascontiguousarray(rec[:, : 40921])  # odd byte count: rows start unaligned
    with tga.Context(0) as ctx:
        cells = ctx.acquire_cells(bits, FS, mask=1 << tga.GPS, prn_filter=[34, 37, 38], ant_filter=[0, 3])
    ub = np.unpackbits(bits, axis=1)
    for cell in cells:
        r = O.acquire_all(ub, FS, O.GPS, ant_filter=[int(cell["antenna"])], prn_filter=[int(cell["prn"])],
                          threads=4, grid=True)["results"][0]["cells"][0]
        g = {k: cell[k].item() for k in cell.dtype.names}
        assert_cell_parity(g, r, ("odd-row", int(cell["prn"]), int(cell["antenna"])))


def test_short_recording_searches_the_samples_it_has(rec):
    """8 ms of data, less than two BeiDou periods: like the reference
    (acquisition.rs:288, len = num_samples.min(raw.len())) the search window
    is the whole recording (the generic path)."""
    bits = np.ascontiguousarray(rec[:, :16368])
    with tga.Context(0) as ctx:
        cell = ctx.acquire_cells(bits, FS, mask=1 << tga.BEIDOU, prn_filter=[21], ant_filter=[2])[0]
    r = O.acquire_all(np.unpackbits(bits, axis=1), FS, O.BEIDOU, ant_filter=[2], prn_filter=[21], threads=8,
                      grid=True)["results"][0]["cells"][0]
    assert_cell_parity({k: cell[k].item() for k in cell.dtype.names}, r, "short")


def test_error_paths_return_status_codes(rec):
    with tga.Context(0) as ctx:
        with pytest.raises(tga.TgaError) as e:
            ctx.acquire_cells(rec, FS, mask=1 << tga.GPS, ant_filter=[9])
        assert e.value.code == 1
        with pytest.raises(tga.TgaError) as e:
            ctx.acquire_cells(rec, FS, mask=1 << tga.GPS, prn_filter=[39])
        assert e.value.code == 1
        # the context is still usable
        ok = ctx.acquire_cells(rec, FS, mask=1 << tga.GPS, prn_filter=[38], ant_filter=[0])
        assert len(ok) == 1 and ok[0]["prn"] == 38
