"""FP64 CPU restatement of the fine-acquisition model (test infrastructure).

This module is the checker of tart-gnss_b200's fine acquisition
(tga_fine_eval / tga_fine_acquire); only tests/ may import it.  The model
has no counterpart in the reference's Rust crate; its only precedent is
optimize_fit (junk/acquisition.py:403-445), which refines the frequency by a
scalar search and the code phase by a Gaussian fit.  Here, for one satellite
and A antennas,

    R_a(tau, f) = (1/N) sum_n s_a[n] exp(+i 2 pi f (n - n0) / fs) c(n - tau)
    P(tau, f, phi) = | sum_a exp(-i phi_a) R_a |^2

with s_a the de-meaned +-1 samples (mean over the whole row, as
acquisition.rs:281-294), the wipe-off sign of correlate.rs:110-115, n0 the
window centre, and c the code as rectangular (sub)chips of T samples whose
edges are smoothed by a Gaussian of standard deviation sigma samples (a
front-end filter model):

    c(t) = seq[k] + sum_m d_m (Phi((t - m T) / sigma) - [t >= m T]),
    k = floor(t / T), d_m = seq[m] - seq[m - 1] over the four edges around t.

The gradient and Hessian of P are written out analytically; the tests check
them against central finite differences of P and the GPU against all three.
"""
import math

import numpy as np
from scipy.special import ndtr

SQRT_2PI_INV = 1.0 / math.sqrt(2.0 * math.pi)


def replica(seq, T, sigma, t):
    """c(t), c'(t), c''(t) for an array of continuous times t (samples)."""
    seq = np.asarray(seq, dtype=np.float64)
    L = len(seq)
    t = np.asarray(t, dtype=np.float64)
    k = np.floor(t / T).astype(np.int64)
    c = seq[np.mod(k, L)].copy()
    c1 = np.zeros_like(t)
    c2 = np.zeros_like(t)
    for dm in (-1, 0, 1, 2):
        m = k + dm
        d = seq[np.mod(m, L)] - seq[np.mod(m - 1, L)]
        u = (t - m * T) / sigma
        pdf = SQRT_2PI_INV * np.exp(-0.5 * u * u)
        c += d * (ndtr(u) - (u >= 0))
        c1 += d * pdf / sigma
        c2 -= d * u * pdf / sigma ** 2
    return c, c1, c2


def model_geometry(seq_len, code_period_s, primary_chips, fs, sigma_chips):
    """(T, sigma) in samples, as the library derives them."""
    T = fs * code_period_s / seq_len
    sigma = sigma_chips * fs * code_period_s / primary_chips
    return T, sigma


def pm_rows(bits):
    """Packed MSB-first rows -> de-meaned +-1 float64 rows (whole-row mean)."""
    ub = np.unpackbits(np.asarray(bits, dtype=np.uint8), axis=1).astype(np.float64)
    s = 2.0 * ub - 1.0
    return s - s.mean(axis=1, keepdims=True)


def sums(rows, start, length, tau, f, fs, seq, T, sigma):
    """[A, 6] complex: R, dR/dtau, dR/df, d2R/dtau2, d2R/df2, d2R/dtau df,
    normalised by the window length."""
    n = np.arange(start, start + length, dtype=np.float64)
    dn = n - (start + 0.5 * length)
    cyc = np.mod(f / fs * dn, 1.0)
    w = np.exp(2j * np.pi * cyc)
    x = 2.0 * np.pi * dn / fs
    c, c1, c2 = replica(seq, T, sigma, n - tau)
    s = rows[:, start:start + length]
    cols = [w * c, w * (-c1), 1j * x * w * c, w * c2, -(x * x) * w * c, 1j * x * w * (-c1)]
    return np.stack([s @ v for v in cols], axis=1) / length


def assemble(R, phi):
    """P, gradient and Hessian in the order (tau, f, phi_0 .. phi_{A-1})."""
    A = R.shape[0]
    u = np.exp(-1j * np.asarray(phi, dtype=np.float64))
    S, St, Sf, Stt, Sff, Stf = (u @ R[:, k] for k in range(6))
    P = abs(S) ** 2
    D = 2 + A
    g = np.zeros(D)
    H = np.zeros((D, D))
    Q = -1j * u * R[:, 0]
    Qt = -1j * u * R[:, 1]
    Qf = -1j * u * R[:, 2]
    cS = np.conj(S)
    g[0] = 2 * (cS * St).real
    g[1] = 2 * (cS * Sf).real
    g[2:] = 2 * (cS * Q).real
    H[0, 0] = 2 * (np.conj(St) * St + cS * Stt).real
    H[1, 1] = 2 * (np.conj(Sf) * Sf + cS * Sff).real
    H[0, 1] = H[1, 0] = 2 * (np.conj(St) * Sf + cS * Stf).real
    H[0, 2:] = H[2:, 0] = 2 * (np.conj(St) * Q + cS * Qt).real
    H[1, 2:] = H[2:, 1] = 2 * (np.conj(Sf) * Q + cS * Qf).real
    H[2:, 2:] = 2 * (np.conj(Q)[:, None] * Q[None, :]).real
    H[2:, 2:] += np.diag(2 * (cS * (-u * R[:, 0])).real)
    return P, g, H


def power(rows, start, length, tau, f, fs, seq, T, sigma, phi):
    R = sums(rows, start, length, tau, f, fs, seq, T, sigma)
    return abs(np.exp(-1j * np.asarray(phi)) @ R[:, 0]) ** 2


def band_limited_signal(seq, T, sigma, n, tau):
    """The same smoothed code evaluated as a received waveform c(n - tau):
    the synthetic front end of the fine-acquisition tests."""
    return replica(seq, T, sigma, np.asarray(n, dtype=np.float64) - tau)[0]
