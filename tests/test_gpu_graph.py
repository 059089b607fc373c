"""CUDA-graph capture and replay of the batched search (tga_set_graphs):
a plan runs eagerly on its first call, is captured on its second and
replayed after that; every call returns exactly what an eager context
returns on the same bits, including after the bits change under a replayed
graph, after the plan changes (antenna filter, precision) and after the
context's buffers grow (the graph is rebuilt)."""
import numpy as np
import pytest

import acq_oracle as O
import tga
from testutil import make_observation

pytestmark = pytest.mark.gpu

FS = 16.368e6
N = 327360 + 2000
FIELDS = ("constellation", "prn", "antenna", "best_codephase", "best_freq_idx", "hypothesis", "signal_strength",
          "second_peak", "codephase_frac", "frequency", "cn0_acr", "cn0_valid")


def _obs(seed, n_ant=3):
    sats = []
    rng = np.random.default_rng(seed)
    for c, prn in ((O.GPS, 5), (O.SBAS, 133), (O.GALILEO, 11), (O.BEIDOU, 30), (O.L1C, 9)):
        P = O.period_samples(c, FS)
        sats.append(dict(code=O.resampled_code(c, prn, float(P), P), period=P, delay=int(rng.integers(P)),
                         doppler=float(rng.uniform(-4000, 4000)), cn0=47.0))
    packed, _ = make_observation(n_ant, N, FS, sats, seed=seed)
    return packed


def _same(a, b):
    assert len(a) == len(b)
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f


@pytest.fixture(scope="module")
def eager():
    with tga.Context(0) as c:
        c.set_graphs(False)
        yield c


@pytest.mark.parametrize("precision", [tga.PRECISION_FP32, tga.PRECISION_FP16_TC], ids=["fp32", "fp16tc"])
def test_capture_then_replay_equals_eager(eager, precision):
    bits1, bits2 = _obs(71), _obs(72)
    eager.set_precision(precision)
    want1 = eager.acquire_cells(bits1, FS, mask=tga.ALL, cn0=True)
    want2 = eager.acquire_cells(bits2, FS, mask=tga.ALL, cn0=True)
    with tga.Context(0) as ctx:
        ctx.set_precision(precision)
        states, launches = [], []
        for bits, want in ((bits1, want1), (bits1, want1), (bits1, want1), (bits2, want2), (bits1, want1)):
            got = ctx.acquire_cells(bits, FS, mask=tga.ALL, cn0=True)
            _same(got, want)
            states.append(ctx.last_graph())
            launches.append(ctx.last_stats()["kernel_launches"])
        assert states == [tga.GRAPH_NONE, tga.GRAPH_CAPTURED, tga.GRAPH_REPLAYED, tga.GRAPH_REPLAYED,
                          tga.GRAPH_REPLAYED]
        # a replay reports the kernels it ran, like the eager call
        assert len(set(launches)) == 1 and launches[0] > 0
        # a new plan (antenna filter) starts eager again, then is captured
        sub = [ctx.acquire_cells(bits2, FS, mask=tga.ALL, cn0=True, ant_filter=[2, 0]) for _ in range(2)]
        assert ctx.last_graph() == tga.GRAPH_CAPTURED
        want_sub = eager.acquire_cells(bits2, FS, mask=tga.ALL, cn0=True, ant_filter=[2, 0])
        for s in sub:
            _same(s, want_sub)
        # the first plan is still cached
        _same(ctx.acquire_cells(bits1, FS, mask=tga.ALL, cn0=True), want1)
        assert ctx.last_graph() == tga.GRAPH_REPLAYED
    eager.set_precision(tga.PRECISION_FP32)


def test_buffer_growth_rebuilds_the_graph(eager):
    """Bits resident on the device keep the plan's key fixed; a larger search
    in between reallocates the context's shared buffers, so the next call of
    the plan captures a new graph instead of replaying stale pointers."""
    import torch
    small, big = _obs(81, n_ant=2), _obs(82, n_ant=5)
    small_d, big_d = torch.from_numpy(small).cuda(), torch.from_numpy(big).cuda()
    mask = 1 << tga.GPS | 1 << tga.GALILEO

    def run(ctx, t):
        return ctx.acquire_cells(None, FS, mask=mask, device_bits=t.data_ptr(), n_ant=t.shape[0],
                                 row_bytes=t.shape[1])

    want = eager.acquire_cells(small, FS, mask=mask)
    with tga.Context(0) as ctx:
        for _ in range(3):
            _same(run(ctx, small_d), want)
        assert ctx.last_graph() == tga.GRAPH_REPLAYED
        run(ctx, big_d)
        _same(run(ctx, small_d), want)
        assert ctx.last_graph() == tga.GRAPH_CAPTURED
        _same(run(ctx, small_d), want)
        assert ctx.last_graph() == tga.GRAPH_REPLAYED


def test_profiling_and_generic_plans_run_eagerly():
    bits = _obs(91, n_ant=1)
    with tga.Context(0) as ctx:
        ctx.set_profiling(True)
        for _ in range(3):
            ctx.acquire_cells(bits, FS, mask=1 << tga.GPS)
            assert ctx.last_graph() == tga.GRAPH_NONE
        ctx.set_profiling(False)
        # 16 MHz: no integer number of samples per chip, the generic path
        short = np.ascontiguousarray(bits[:, : 2 * 16000 // 8 + 64])
        for _ in range(3):
            ctx.acquire_cells(short, 16.0e6, mask=1 << tga.GPS, prn_filter=[5])
            assert ctx.last_graph() == tga.GRAPH_NONE


def test_timeout_reported_through_captured_and_replayed_graphs():
    """The tensor-core wait-expiry hook (no MMA issued, every wait bounded to
    1 s, nothing faults) under graph capture and replay: each call fails with
    TGA_ERR_TIMEOUT, and with the hook off the next plan runs normally."""
    bits = _obs(95, n_ant=1)
    mask = 1 << tga.GPS
    with tga.Context(0) as ctx:
        ctx.set_precision(tga.PRECISION_FP16_TC)
        ctx.set_test_flags(tga.TEST_TC_SKIP_COMMIT)
        states = []
        for _ in range(3):
            with pytest.raises(tga.TgaError) as ei:
                ctx.acquire_cells(bits, FS, mask=mask, prn_filter=[5])
            assert ei.value.code == 6  # TGA_ERR_TIMEOUT
            states.append(ctx.last_graph())
        assert states == [tga.GRAPH_NONE, tga.GRAPH_CAPTURED, tga.GRAPH_REPLAYED]
        ctx.set_test_flags(0)
        got = ctx.acquire_cells(bits, FS, mask=mask, prn_filter=[5])
    with tga.Context(0) as ref:
        ref.set_graphs(False)
        ref.set_precision(tga.PRECISION_FP16_TC)
        _same(got, ref.acquire_cells(bits, FS, mask=mask, prn_filter=[5]))


def test_stream_of_observations_equals_single_calls():
    """tga_acquire_all_stream: four observations (two distinct recordings,
    each twice, so both alternated buffers serve a cached graph plan) in
    one call, the copy of each overlapping the previous search; every
    observation's cells equal a separate tga_acquire_all call, in both
    arithmetics."""
    import torch
    rng = np.random.default_rng(404)
    obs = []
    for _ in range(2):
        host = torch.from_numpy(rng.integers(0, 256, size=(4, 40920), dtype=np.uint8)).pin_memory().numpy()
        obs.append(host)
    seq = [obs[0], obs[1], obs[0], obs[1]]
    with tga.Context(0) as ctx:
        for prec in (tga.PRECISION_FP32, tga.PRECISION_FP16_TC):
            ctx.set_precision(prec)
            want = [ctx.acquire_cells(o, 16.368e6, mask=tga.ALL, cn0=True) for o in obs]
            got = ctx.acquire_cells_stream(seq, 16.368e6, mask=tga.ALL, cn0=True)
            assert len(got) == 4
            for i, g in enumerate(got):
                assert np.array_equal(g, want[i % 2]), (prec, i)
