"""Test-signal helpers, restating the reference's test utilities.

* phasepoints ............... src/testutil.rs:10-13
* synth_signal .............. src/testutil.rs:21-40
* expected_recovered_sample . src/testutil.rs:45-47
* synth_signal_cn0 .......... src/testutil.rs:60-81 (Box-Muller xorshift64)
* quantize_bipolar_demean ... src/simulator.rs:237-244
* pack_row .................. src/simulator.rs:280-293 (numpy.packbits)
* make_observation .......... seeded synthetic multi-satellite 1-bit
                              recording in the same signal model, used by
                              the parity tests and the benchmark.
"""
import math

import numpy as np

TAU = 6.283185307179586
MASK64 = (1 << 64) - 1


class XorShift:
    """testutil.rs:84-100 (xorshift64, 53-bit uniform, Box-Muller)."""

    def __init__(self, seed):
        self.s = seed & MASK64

    def next_f64(self):
        x = self.s
        x ^= (x << 13) & MASK64
        x ^= x >> 7
        x ^= (x << 17) & MASK64
        self.s = x
        return (x >> 11) / float(1 << 53)

    def gaussian(self):
        u1 = max(self.next_f64(), 1e-12)
        u2 = self.next_f64()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(TAU * u2)


def xorshift_stream(seed, n):
    """Vectorised xorshift64: n consecutive raw outputs (uint64)."""
    out = np.empty(n, dtype=np.uint64)
    s = seed & MASK64
    # Sequential by nature; do it in Python only for modest n.
    for i in range(n):
        s ^= (s << 13) & MASK64
        s ^= s >> 7
        s ^= (s << 17) & MASK64
        out[i] = s
    return out


def phasepoints(fs, n):
    pc = TAU / fs
    return pc * np.arange(n, dtype=np.float64)


def _xs(fn, seed, n):
    import ctypes
    import acq_oracle
    out = np.empty(n)
    f = getattr(acq_oracle.lib(), fn)
    f.argtypes = [ctypes.c_uint64, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double)]
    f(seed & MASK64, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


def synth_signal(code, code_period, delay, f0, fs, noise_amp, seed):
    n = len(code)
    u = _xs("oracle_xorshift_uniform", seed, n)
    i = np.arange(n)
    cp = (i + delay) % code_period
    carrier = np.cos(TAU * f0 * i.astype(np.float64) / fs)
    noise = noise_amp * (2.0 * u - 1.0)
    return (np.asarray(code, dtype=np.float64)[cp] * carrier + noise).astype(np.float32)


def expected_recovered_sample(period, delay):
    return (period - delay) % period


def synth_signal_cn0(code, period, delay, f0, fs, cn0_db, seed, flip):
    """Returns float32 like the reference (callers widen to f64 before quantizing)."""
    a = 2.0 * math.sqrt(10.0 ** (cn0_db / 10.0) / fs)
    epoch = period + (period - delay) % period
    n = len(code)
    g = _xs("oracle_xorshift_gaussian", seed, n)
    i = np.arange(n)
    cp = (i + delay) % period
    sign = np.where(flip & (i >= epoch), -1.0, 1.0)
    carrier = a * np.cos(TAU * f0 * i.astype(np.float64) / fs)
    return (sign * np.asarray(code)[cp] * carrier + g).astype(np.float32)


def quantize_bipolar_demean(signal):
    bip = np.where(np.asarray(signal, dtype=np.float64) >= 0.0, 1.0, -1.0)
    mean = float(np.sum(bip)) / len(bip)
    return (bip - mean).astype(np.float32)


def pack_row(bits):
    return np.packbits(np.asarray(bits, dtype=np.uint8))


def make_observation(n_ant, n_samples, fs, sats, seed, noise_sigma=1.0):
    """Seeded 1-bit multi-satellite recording.

    sats: list of dicts {code: +-1 array of one period P (resampled at fs),
    period: P, delay: samples, doppler: Hz (carrier at IF+doppler), cn0: dB-Hz,
    flips: optional list of +-1 per code epoch}.  Signal model of
    testutil.rs:60-81 (A = 2 sqrt(C/N0 / fs), real carrier, unit Gaussian
    noise) summed over satellites, sign-quantised (v >= 0 -> 1) and packed
    MSB-first.  Each antenna gets its own noise and carrier phase.
    Returns (packed [n_ant, ceil(n/8)] uint8, bits [n_ant, n]).
    """
    rng = np.random.default_rng(seed)
    t = np.arange(n_samples, dtype=np.float64)
    bits = np.empty((n_ant, n_samples), dtype=np.uint8)
    for a in range(n_ant):
        v = rng.standard_normal(n_samples) * noise_sigma
        for s in sats:
            P = s["period"]
            amp = 2.0 * math.sqrt(10.0 ** (s["cn0"] / 10.0) / fs)
            idx = (np.arange(n_samples) + s["delay"]) % P
            chip = np.asarray(s["code"], dtype=np.float64)[idx]
            if s.get("flips") is not None:
                ep = (np.arange(n_samples) + s["delay"]) // P
                chip = chip * np.asarray(s["flips"], dtype=np.float64)[ep % len(s["flips"])]
            ph = rng.uniform(0, TAU)
            v += amp * chip * np.cos(TAU * (s.get("if", 4.092e6) + s["doppler"]) * t / fs + ph)
        bits[a] = (v >= 0.0).astype(np.uint8)
    packed = np.packbits(bits, axis=1)
    return packed, bits


# code period (s) and primary chips per constellation (GPS, Galileo, BeiDou,
# SBAS, L1C, QZSS), for the band-limited fine-acquisition front end
CODE_PERIOD_S = {0: 1e-3, 1: 4e-3, 2: 10e-3, 3: 1e-3, 4: 10e-3, 5: 1e-3}
PRIMARY_CHIPS = {0: 1023, 1: 4092, 2: 10230, 3: 1023, 4: 10230, 5: 1023}


def synth_fine(sats, n_ant, n_samples, fs, sigma_chips, seed, if_hz=4.092e6):
    """Band-limited 1-bit recording for fine acquisition: every satellite
    (dict c, prn, tau (continuous delay, samples), dop (Hz), cn0 (dB-Hz))
    reaches every antenna with the same delay and Doppler and its own random
    carrier phase; its code edges are smoothed by the same Gaussian front end
    the fine-acquisition replica models (sigma_chips).  Unit Gaussian noise,
    sign-quantised, packed MSB-first.  Returns (bits, per-satellite phases)."""
    import fine_oracle as FO
    import tga
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n_ant, n_samples))
    n = np.arange(n_samples, dtype=np.float64)
    phases = []
    for s in sats:
        seq = tga.code_chips(s["c"], s["prn"]).astype(np.float64)
        T, sigma = FO.model_geometry(len(seq), CODE_PERIOD_S[s["c"]], PRIMARY_CHIPS[s["c"]], fs, sigma_chips)
        code = FO.band_limited_signal(seq, T, sigma, n, s["tau"])
        amp = 2.0 * math.sqrt(10.0 ** (s["cn0"] / 10.0) / fs)
        th = rng.uniform(0, 2 * np.pi, size=n_ant)
        phases.append(th)
        cyc = np.mod((if_hz + s["dop"]) / fs * n, 1.0)
        for a in range(n_ant):
            x[a] += amp * code * np.cos(2 * np.pi * cyc + th[a])
    bits = np.packbits(x >= 0.0, axis=1)
    return bits, phases
