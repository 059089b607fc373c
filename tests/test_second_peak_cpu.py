"""The second peak from four values per polyphase residue (CPU model of the
tensor-core search's FP32 re-evaluation, pfa_kernel mode CAND with p2rows).

The reference's second peak (correlate.rs:157-175) is the largest |y|^2 of
the chosen row more than chip_width lags (circularly) from its peak.  The
re-evaluation keeps only the four largest |y|^2 of each residue rho of the
row (lags rho + S n) and takes the second peak from those 4 S values.  That
is exact while at most three lags of a residue lie within chip_width of the
peak, i.e. ceil((2 chip_width + 1) / S) <= 3, which holds at every fused
rate (chip_width = S).  These cases check the rule against the full scan on
random rows, on rows with the largest values of a residue packed around the
peak, and with ties."""
import numpy as np
import pytest


def second_full(pw, cw):
    P = len(pw)
    tau = int(np.flatnonzero(pw == pw.max())[-1])  # the reference keeps the last maximum
    d = np.abs(np.arange(P) - tau)
    dist = np.minimum(d, P - d)
    out = pw[dist > cw]
    return tau, (float(out.max()) if len(out) else 0.0)


def second_top4(pw, S, cw):
    P = len(pw)
    tau, _ = second_full(pw, cw)
    best = 0.0
    for rho in range(S):
        lags = np.arange(rho, P, S)
        keep = lags[np.argsort(-pw[lags], kind="stable")[:4]]
        for t in keep:
            d = abs(int(t) - tau)
            if min(d, P - d) > cw:
                best = max(best, float(pw[t]))
    return tau, best


@pytest.mark.parametrize("S", [1, 2, 4, 8, 16])
def test_random_rows(S):
    rng = np.random.default_rng(S)
    cw = S
    assert (2 * cw + S) // S <= 3
    for trial in range(200):
        L = int(rng.integers(8, 60))
        pw = rng.exponential(size=S * L).astype(np.float32)
        assert second_top4(pw, S, cw) == second_full(pw, cw)


@pytest.mark.parametrize("S", [1, 4, 16])
def test_largest_values_around_the_peak(S):
    """Each residue's three largest values sit at its three lags closest to
    the peak (all inside the window): the fourth kept value is the answer."""
    rng = np.random.default_rng(100 + S)
    cw = S
    for trial in range(100):
        L = int(rng.integers(8, 40))
        P = S * L
        pw = rng.uniform(0.0, 1.0, size=P).astype(np.float32)
        tau = int(rng.integers(0, P))
        for off in range(-cw, cw + 1):
            pw[(tau + off) % P] = 5.0 + rng.uniform()
        pw[tau] = 10.0
        assert second_top4(pw, S, cw) == second_full(pw, cw)


def test_ties():
    S, cw, L = 16, 16, 30
    pw = np.ones(S * L, dtype=np.float32)
    pw[100] = 4.0
    assert second_top4(pw, S, cw) == second_full(pw, cw) == (100, 1.0)
    pw = np.zeros(S * L, dtype=np.float32)
    assert second_top4(pw, S, cw) == second_full(pw, cw)
