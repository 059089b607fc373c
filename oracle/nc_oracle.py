"""CPU restatement of the engine's non-coherent search (test infrastructure).

The reference crate has no non-coherent mode; this restates the extension
implemented by tga_search_noncoherent on top of the reference's own steps:
antenna prep (acquisition.rs:281-294: +-1, mean over the whole row,
(v - mean) as f32), wipe-off by the carrier exp(+i 2 pi f (n - n0) / fs)
with n0 the first sample of the block (the sign convention of
correlate.rs:110-115; the phase is exact, not the reference's f32-rounded
absolute phase, whose rounding step reaches 0.25 rad over 100 ms), circular
correlation with the code as
IFFT(FFT(x) conj(FFT(code))) (correlate.rs:118-133), here of each coherent
block folded into one code period and accumulated as N |corr|^2 over the
blocks (N samples per block, the square of the reference's |IFFT_N| /
sqrt(N) metric); last maximum over lags, then over bins; second peak at a
circular distance of more than ceil(fs / 1.023 MHz) (correlate.rs:157-175).
Only tests/ import this module.
"""
import math

import numpy as np

import acq_oracle as O


def search_nc(bits, fs, c, prns, ants, center, step, nb, K, B, start):
    ub = np.unpackbits(np.asarray(bits, dtype=np.uint8), axis=1).astype(np.float64)
    s = 2.0 * ub - 1.0
    v = (s - s.mean(axis=1, keepdims=True)).astype(np.float32)
    P = O.period_samples(c, fs)
    N = K * P
    fc = [center + (i - (nb - 1) // 2) * step for i in range(nb)]
    cw = math.ceil(fs / 1.023e6)
    out = []
    for prn in prns:
        code = O.resampled_code(c, prn, float(P), P).astype(np.float64)
        Cc = np.conj(np.fft.fft(code))
        for a in ants:
            accs = []
            for f in fc:
                acc = np.zeros(P)
                for b in range(B):
                    n0 = start + b * N
                    n = n0 + np.arange(N)
                    x = v[a, n].astype(np.float64)
                    iq = x * np.exp(2j * np.pi * (f * np.arange(N, dtype=np.float64) / fs))
                    fold = iq.reshape(K, P).sum(axis=0)
                    corr = np.fft.ifft(np.fft.fft(fold) * Cc)
                    acc += N * np.abs(corr) ** 2
                accs.append(acc)
            best_bin, best_lag, best_p = 0, 0, -1.0
            for i, acc in enumerate(accs):
                lag = len(acc) - 1 - int(np.argmax(acc[::-1]))  # last maximum
                if i == 0 or acc[lag] >= best_p:
                    best_bin, best_lag, best_p = i, lag, acc[lag]
            acc = accs[best_bin]
            d = np.abs(np.arange(P) - best_lag)
            d = np.minimum(d, P - d)
            far = acc[d > cw]
            out.append(dict(prn=prn, antenna=a, best_freq_idx=best_bin, best_codephase=best_lag, power=best_p,
                            second_power=float(far.max()) if far.size else 0.0, frequency=fc[best_bin] - center))
    return out
