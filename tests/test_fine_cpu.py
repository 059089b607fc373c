"""Fine-acquisition oracle: the analytic gradient and Hessian of the coherent
multi-antenna power against central finite differences (FP64, CPU)."""
import numpy as np
import pytest

import fine_oracle as FO
import tga
from testutil import CODE_PERIOD_S, PRIMARY_CHIPS, synth_fine

FS = 16.368e6


@pytest.mark.parametrize("c,prn", [(tga.GPS, 5), (tga.BEIDOU, 19)], ids=["gps", "beidou-boc"])
def test_oracle_gradient_and_hessian_match_finite_differences(c, prn):
    P0 = int(FS * CODE_PERIOD_S[c])
    n = min(2 * P0, 65472)
    sats = [dict(c=c, prn=prn, tau=1234.37, dop=812.5, cn0=52.0)]
    bits, _ = synth_fine(sats, 2, n, FS, 0.1, seed=7)
    rows = FO.pm_rows(bits)
    seq = tga.code_chips(c, prn).astype(np.float64)
    T, sigma = FO.model_geometry(len(seq), CODE_PERIOD_S[c], PRIMARY_CHIPS[c], FS, 0.1)
    theta = np.array([1234.2, 4.092e6 + 800.0, 0.3, -1.1])

    def P_of(th):
        return FO.power(rows, 0, n, th[0], th[1], FS, seq, T, sigma, th[2:])

    def g_of(th):
        R = FO.sums(rows, 0, n, th[0], th[1], FS, seq, T, sigma)
        return FO.assemble(R, th[2:])[1]

    R = FO.sums(rows, 0, n, theta[0], theta[1], FS, seq, T, sigma)
    P, g, H = FO.assemble(R, theta[2:])
    assert np.isclose(P, P_of(theta))
    h = np.array([1e-3, 1e-2, 1e-4, 1e-4])
    for i in range(4):
        e = np.zeros(4)
        e[i] = h[i]
        gfd = (P_of(theta + e) - P_of(theta - e)) / (2 * h[i])
        assert abs(gfd - g[i]) <= 1e-5 * max(abs(g[i]), np.abs(g).max() * 1e-3), (i, gfd, g[i])
        Hfd = (g_of(theta + e) - g_of(theta - e)) / (2 * h[i])
        assert np.allclose(Hfd, H[:, i], rtol=1e-4, atol=1e-6 * np.abs(H[:, i]).max()), (i, Hfd, H[:, i])


def test_replica_derivatives_match_finite_differences():
    seq = np.array([1, -1, -1, 1, 1, 1, -1, 1], dtype=np.float64)
    t = np.linspace(-3.0, 70.0, 997)
    c, c1, c2 = FO.replica(seq, 8.0, 1.3, t)
    h = 1e-4
    cp = FO.replica(seq, 8.0, 1.3, t + h)
    cm = FO.replica(seq, 8.0, 1.3, t - h)
    assert np.allclose((cp[0] - cm[0]) / (2 * h), c1, atol=1e-6)
    assert np.allclose((cp[1] - cm[1]) / (2 * h), c2, atol=1e-5)
    # five sigma from the nearest edge the replica is the chip value
    far = FO.replica(seq, 8.0, 0.8, np.array([4.0, 12.0, 20.0]))[0]
    assert np.allclose(far, [1, -1, -1], atol=1e-6)
