"""FP64 CPU restatement of the narrowband RFI scan (test infrastructure).

Follows rfi.rs (tart-gnss-acquire --rfi): analyze_channel (rfi.rs:145-168),
detect_lines (rfi.rs:91-140) and autocorrelation (rfi.rs:84-87), with the
reference's constants: 15 dB minimum excess over the median bin power,
10 kHz clustering, at most 3 lines.  The FFT is numpy's (pocketfft) in f64;
the reference's is rustfft 6.4.1 in f64 (absent here).  Only tests/ import
this module; it checks tga_rfi_scan.
"""
import numpy as np

MIN_EXCESS_DB = 15.0
CLUSTER_HZ = 10_000.0
MAX_LINES = 3


def autocorrelation(z, lag):
    n = len(z)
    return float(np.dot(z[: n - lag], z[lag:]) / (n - lag))


def detect_lines(z, fs):
    n = len(z)
    if n < 8:
        return []
    X = np.fft.fft(np.asarray(z, dtype=np.float64))
    half = n // 2
    p = X[:half].real ** 2 + X[:half].imag ** 2
    floor = np.sort(p)[half // 2]
    k = np.arange(1, half - 1)
    peak = (p[k] > p[k - 1]) & (p[k] >= p[k + 1])
    k = k[peak]
    with np.errstate(divide="ignore", invalid="ignore"):
        ex = 10.0 * np.log10(p[k] / floor)
    keep = ex > MIN_EXCESS_DB
    lines = [dict(frequency=float(kk) * (fs / n), excess_db=float(e)) for kk, e in zip(k[keep], ex[keep])]
    lines.sort(key=lambda l: -l["excess_db"])  # stable, like Rust's sort_by
    out = []
    for line in lines:
        if all(abs(c["frequency"] - line["frequency"]) > CLUSTER_HZ for c in out):
            out.append(line)
            if len(out) == MAX_LINES:
                break
    return out


def analyze_channel(antenna, bipolar, fs):
    """bipolar: the +-1 samples of one antenna (Observation::get_antenna)."""
    bipolar = np.asarray(bipolar, dtype=np.float64)
    mean = float(np.sum(bipolar)) / len(bipolar)
    z = bipolar - mean
    var = float(np.dot(z, z)) / len(z)
    if var < 1e-9:
        return dict(antenna=antenna, dead=True, acf_lag1=None, acf_lag3=None, acf_lag16=None,
                    period_samples=None, lines=[])
    lines = detect_lines(z, fs)
    return dict(antenna=antenna, dead=False, acf_lag1=autocorrelation(z, 1), acf_lag3=autocorrelation(z, 3),
                acf_lag16=autocorrelation(z, 16), period_samples=(fs / lines[0]["frequency"]) if lines else None,
                lines=lines)


def run(bits, fs):
    """rfi::run over packed MSB-first rows [n_ant, row_bytes]."""
    ub = np.unpackbits(np.asarray(bits, dtype=np.uint8), axis=1)
    return [analyze_channel(a, 2.0 * ub[a].astype(np.float64) - 1.0, fs) for a in range(ub.shape[0])]
