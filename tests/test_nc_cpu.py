"""Non-coherent search oracle (oracle/nc_oracle.py): with one block of two
periods it reproduces the drop-in oracle's [c,c] result exactly (same lag,
bin and metric squared), and it finds weak injected satellites."""
import math

import numpy as np

import acq_oracle as O
import nc_oracle as NC

FS = 16.368e6


def synth(sats, n, seed, n_ant=1):
    rng = np.random.default_rng(seed)
    t = np.arange(n)
    x = rng.standard_normal((n_ant, n))
    for c, prn, delay, dop, cn0 in sats:
        P = O.period_samples(c, FS)
        code = O.resampled_code(c, prn, float(P), P).astype(np.float64)
        amp = 2.0 * math.sqrt(10.0 ** (cn0 / 10.0) / FS)
        for a in range(n_ant):
            x[a] += amp * code[(t + delay) % P] * np.cos(2 * np.pi * (4.092e6 + dop) / FS * t + rng.uniform(0, 6.28))
    return np.packbits(x >= 0, axis=1)


def test_one_two_period_block_is_the_dropin_cc_hypothesis():
    P = 16368
    bits = synth([(O.GPS, 7, 3000, 1200.0, 50.0)], 2 * P, seed=5)
    ub = np.unpackbits(bits, axis=1)[0].astype(np.float64)
    s = 2 * ub - 1
    sig = (s - s.mean()).astype(np.float32)
    pp = 2 * np.pi / FS * np.arange(2 * P)
    r = O.acquire_single(O.GPS, sig, pp, FS, 4.092e6, 6000.0, 7, P, precision="f64")
    grid = O.freq_grid(4.092e6, 6000.0)
    step = grid[1] - grid[0]
    nc = NC.search_nc(bits, FS, O.GPS, [7], [0], 4.092e6, step, len(grid), 2, 1, 0)[0]
    assert nc["best_codephase"] == r["best_codephase"] % P
    assert nc["best_freq_idx"] == r["best_freq_idx"]
    # the drop-in rounds the carrier phase to f32 (up to 0.002 rad over two
    # periods), the non-coherent mode uses the exact phase: ~1e-4 in power
    assert abs(nc["power"] - r["signal_strength"] ** 2) <= 2e-4 * nc["power"]


def test_weak_satellite_found_with_noncoherent_sums():
    P = 16368
    sats = [(O.GPS, 3, 5000, 1500.0, 40.0)]
    bits = synth(sats, 10 * P, seed=8)
    out = NC.search_nc(bits, FS, O.GPS, [3], [0], 4.092e6, 500.0, 21, 1, 10, 0)[0]
    assert out["best_codephase"] == (P - 5000) % P
    assert abs(out["frequency"] - 1500.0) <= 250.0
    assert out["power"] > 2.0 * out["second_power"]
