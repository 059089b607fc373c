"""GPU tests of fine acquisition (tga_fine_eval / tga_fine_acquire).

The kernel's coherent power, gradient and Hessian are checked against the
FP64 oracle and against central finite differences of the GPU power; the
Newton refinement is checked on a band-limited 24-antenna recording of GPS
C/A and Galileo E1-C satellites at off-grid delays and Dopplers, against the
grid estimate of the acquisition search (integer code phase, 300 Hz bins).
"""
import numpy as np
import pytest

import fine_oracle as FO
import tga
from testutil import CODE_PERIOD_S, PRIMARY_CHIPS, synth_fine

pytestmark = pytest.mark.gpu

FS = 16.368e6
IF = 4.092e6


@pytest.fixture(scope="module")
def ctx():
    c = tga.Context(0)
    yield c
    c.close()


def _model(c, prn):
    seq = tga.code_chips(c, prn).astype(np.float64)
    T, sigma = FO.model_geometry(len(seq), CODE_PERIOD_S[c], PRIMARY_CHIPS[c], FS, 0.1)
    return seq, T, sigma


@pytest.mark.parametrize("c,prn", [(tga.GPS, 5), (tga.GALILEO, 11), (tga.BEIDOU, 19)],
                         ids=["gps", "galileo", "beidou-boc"])
def test_fine_eval_matches_fp64_oracle(ctx, c, prn):
    P0 = int(FS * CODE_PERIOD_S[c])
    n = min(2 * P0, 65472)
    sats = [dict(c=c, prn=prn, tau=2345.61, dop=-1530.0, cn0=50.0)]
    bits, _ = synth_fine(sats, 3, n + 4003, FS, 0.1, seed=11 + prn)
    start, length = 1003, n  # window not byte aligned
    phases = np.array([0.4, -2.0, 1.1])
    tau, f = 2345.61 + 0.3, IF - 1530.0 + 20.0
    P, g, H = ctx.fine_eval(bits, FS, c, prn, tau, f, start, length, phases)
    seq, T, sigma = _model(c, prn)
    R = FO.sums(FO.pm_rows(bits), start, length, tau, f, FS, seq, T, sigma)
    Po, go, Ho = FO.assemble(R, phases)
    assert abs(P - Po) <= 1e-4 * Po
    assert np.abs(g - go).max() <= 1e-3 * np.abs(go).max()
    assert np.abs(H - Ho).max() <= 1e-3 * np.abs(Ho).max()
    # no phases: every antenna aligned to its own correlation phase
    Pa, _, _ = ctx.fine_eval(bits, FS, c, prn, tau, f, start, length, None)
    assert abs(Pa - np.abs(R[:, 0]).sum() ** 2) <= 1e-4 * Pa


def test_fine_gradient_matches_gpu_finite_differences(ctx):
    c, prn = tga.GPS, 9
    sats = [dict(c=c, prn=prn, tau=777.25, dop=2210.0, cn0=48.0)]
    bits, ph = synth_fine(sats, 4, 163680, FS, 0.1, seed=3)
    theta = np.array([777.25 + 0.2, IF + 2210.0 - 15.0, 0.1, 0.9, -0.4, 2.0])

    def P_at(th):
        return ctx.fine_eval(bits, FS, c, prn, th[0], th[1], 0, 163680, th[2:])[0]

    _, g, _ = ctx.fine_eval(bits, FS, c, prn, theta[0], theta[1], 0, 163680, theta[2:])
    h = np.array([0.02, 0.5, 1e-3, 1e-3, 1e-3, 1e-3])
    for i in range(len(theta)):
        e = np.zeros(len(theta))
        e[i] = h[i]
        gfd = (P_at(theta + e) - P_at(theta - e)) / (2 * h[i])
        assert abs(gfd - g[i]) <= 2e-2 * abs(g[i]) + 1e-3 * np.abs(g).max(), (i, gfd, g[i])


def _wrap(x, P):
    return (x + 0.5 * P) % P - 0.5 * P


def test_fine_acquire_beats_grid_estimate(ctx, capsys):
    """24 antennas, 6 GPS C/A + 6 Galileo E1-C satellites, 10 ms window,
    C/N0 45 dB-Hz, delays and Dopplers off-grid.  The refined delay and
    Doppler (one joint estimate per satellite over all antennas) against
    the grid estimates of the acquisition search on the antennas where it
    found the satellite."""
    rng = np.random.default_rng(2026)
    n = 163680
    sats = []
    for c, lo, hi in ((tga.GPS, 1, 32), (tga.GALILEO, 1, 36)):
        for prn in rng.choice(np.arange(lo, hi + 1), size=6, replace=False):
            P0 = int(FS * CODE_PERIOD_S[c])
            sats.append(dict(c=c, prn=int(prn), tau=float(rng.uniform(0, P0)), dop=float(rng.uniform(-4000, 4000)),
                             cn0=45.0))
    bits, _ = synth_fine(sats, 24, n, FS, 0.1, seed=99)
    grid_tau, grid_f, tasks = [], [], []
    for s in sats:
        P0 = int(FS * CODE_PERIOD_S[s["c"]])
        cells = ctx.acquire_cells(bits, FS, mask=1 << s["c"], prn_filter=[s["prn"]])
        tau_g = cells["best_codephase"] % P0
        f_g = cells["frequency"] + IF
        et, ef = _wrap(tau_g - s["tau"], P0), f_g - (IF + s["dop"])
        # grid quantisation error where the search found the satellite (its
        # peak in the right cell); at 45 dB-Hz a 2 ms C/A search misses it on
        # some antennas, and those misses are not grid error
        hit = (np.abs(et) <= 2.0) & (np.abs(ef) <= 300.0)
        assert hit.any()
        grid_tau.append(et[hit])
        grid_f.append(ef[hit])
        best = int(np.argmax(cells["signal_strength"]))  # start from the strongest antenna
        tasks.append((s["c"], s["prn"], float(tau_g[best]), float(f_g[best]), 0, n))
    res, _ = ctx.fine_acquire(bits, FS, tasks)
    ref_tau = np.array([_wrap(r["code_phase"] - s["tau"], int(FS * CODE_PERIOD_S[s["c"]])) for r, s in zip(res, sats)])
    ref_f = np.array([r["frequency"] - (IF + s["dop"]) for r, s in zip(res, sats)])
    grid_tau = np.concatenate(grid_tau)
    grid_f = np.concatenate(grid_f)
    rms = lambda x: float(np.sqrt(np.mean(np.square(x))))
    with capsys.disabled():
        print("\nfine acquisition: delay RMS grid %.3f -> refined %.4f samples (mean %+.4f); Doppler RMS grid %.1f -> "
              "refined %.2f Hz (mean %+.2f); converged %d/%d; acquired antenna-cells %d/%d"
              % (rms(grid_tau), rms(ref_tau), ref_tau.mean(), rms(grid_f), rms(ref_f), ref_f.mean(),
                 sum(r["converged"] for r in res), len(res), len(grid_tau), 24 * len(sats)))
        for c, name in ((tga.GPS, "GPS C/A"), (tga.GALILEO, "Galileo E1-C")):
            k = np.array([s["c"] == c for s in sats])
            print("  %s: refined delay RMS %.4f samples, Doppler RMS %.2f Hz" % (name, rms(ref_tau[k]), rms(ref_f[k])))
    assert all(r["power"] >= r["power_start"] for r in res)
    assert rms(ref_f) * 5 <= rms(grid_f)
    assert rms(ref_tau) * 5 <= rms(grid_tau)
