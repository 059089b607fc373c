"""Launch-shape variants of the FP32 correlation kernels (tga_set_variant)
and their autotuner (tga_autotune).  The variant is per context: a context
with the alternative shapes returns the same cells, field for field, as a
default context on the same bits, for every code length; the autotuner
reports every code length of the search, with both variants' results equal
to variant 0's, keeps its choice on the context, and a search after it
(graphs on) still equals the default context's."""
import numpy as np
import pytest
import torch

import acq_oracle as O
import tga
from testutil import make_observation

pytestmark = pytest.mark.gpu

FS = 16.368e6
N = 327360 + 2000
FIELDS = ("constellation", "prn", "antenna", "best_codephase", "best_freq_idx", "hypothesis", "signal_strength",
          "second_peak", "codephase_frac", "frequency", "cn0_acr", "cn0_valid")


def _obs(seed, n_ant=2):
    sats = []
    rng = np.random.default_rng(seed)
    for c, prn in ((O.GPS, 7), (O.QZSS, 190), (O.GALILEO, 4), (O.BEIDOU, 12), (O.L1C, 40)):
        P = O.period_samples(c, FS)
        sats.append(dict(code=O.resampled_code(c, prn, float(P), P), period=P, delay=int(rng.integers(P)),
                         doppler=float(rng.uniform(-4000, 4000)), cn0=46.0))
    packed, _ = make_observation(n_ant, N, FS, sats, seed=seed)
    return packed


def _same(a, b):
    assert len(a) == len(b)
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f


@pytest.mark.parametrize("precision", [tga.PRECISION_FP32, tga.PRECISION_FP16_TC], ids=["fp32", "fp16tc"])
def test_variant_is_per_context_and_exact(precision):
    bits = _obs(81)
    with tga.Context(0) as base, tga.Context(0) as alt:
        base.set_precision(precision)
        alt.set_precision(precision)
        for lc in (1023, 4092, 10230):
            alt.set_variant(lc, 1)
        want = base.acquire_cells(bits, FS, mask=tga.ALL, cn0=True)
        got = alt.acquire_cells(bits, FS, mask=tga.ALL, cn0=True)
        _same(got, want)
        # the default context is unaffected by the other context's variants
        _same(base.acquire_cells(bits, FS, mask=tga.ALL, cn0=True), want)


def test_set_variant_rejects_bad_arguments():
    with tga.Context(0) as ctx:
        for lc, v in ((1000, 0), (1023, 2), (4092, -1)):
            with pytest.raises(tga.TgaError):
                ctx.set_variant(lc, v)


def test_autotune_keeps_an_exact_variant():
    bits = _obs(82)
    d_bits = torch.from_numpy(bits).cuda()
    n_ant, row_bytes = bits.shape
    with tga.Context(0) as base, tga.Context(0) as ctx:
        want = base.acquire_cells(bits, FS, mask=tga.ALL, cn0=True)
        tuned = ctx.autotune(d_bits.data_ptr(), n_ant, row_bytes, FS, mask=tga.ALL, cn0=True, reps=2)
        assert [e["lc"] for e in tuned] == [1023, 4092, 10230]
        for e in tuned:
            assert e["same_results"] == [True, True]
            assert e["variant"] in (0, 1)
            assert all(m > 0.0 for m in e["ms"])
            assert e["ms"][e["variant"]] == min(e["ms"])
        # graphs back on: eager, captured, replayed, all equal to the default context
        states = []
        for _ in range(3):
            got = ctx.acquire_cells(None, FS, mask=tga.ALL, cn0=True, device_bits=d_bits.data_ptr(), n_ant=n_ant,
                                    row_bytes=row_bytes)
            _same(got, want)
            states.append(ctx.last_graph())
        assert states == [tga.GRAPH_NONE, tga.GRAPH_CAPTURED, tga.GRAPH_REPLAYED]


def test_autotune_only_reports_searched_lengths():
    bits = _obs(83)
    d_bits = torch.from_numpy(bits).cuda()
    with tga.Context(0) as ctx:
        tuned = ctx.autotune(d_bits.data_ptr(), bits.shape[0], bits.shape[1], FS, mask=1 << tga.GALILEO, reps=1)
        assert [e["lc"] for e in tuned] == [4092]
        with pytest.raises(tga.TgaError):
            ctx.autotune(d_bits.data_ptr(), bits.shape[0], bits.shape[1], FS, mask=1 << tga.GALILEO, reps=0)
