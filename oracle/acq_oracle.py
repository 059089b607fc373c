"""CPU ORACLE for the acquisition search -- test infrastructure, not product.

A numpy/scipy restatement of tart-gnss-acquire v0.4.0's FFT acquisition
path.  Only tests/, __graft_entry__.smoke() and bench.py (its CPU-baseline
and reference legs) may import it.  It follows the reference step by step,
including the work the reference repeats (wipe-off and forward FFT per PRN,
code spectra per antenna), so that timing it is timing the reference
algorithm:

* frequency grid ............ acquisition.rs:188-198 (same in every driver)
* code_spectra .............. correlate.rs:47-68
* correlate_code ............ correlate.rs:91-183 (f32, 3 FFTs of N per bin,
                              |.|/sqrt(N), last-max argmax, strict '>' between
                              hypotheses, last-max over bins, second peak)
* acquire_full & siblings ... acquisition.rs:176-248 (+ sbas/qzss/galileo/
                              beidou/l1c twins)
* acquire_all_* ............. acquisition.rs:261-396 (antenna prep :281-294,
                              ACR :341-357, median/MAD :365-377, sort :393)

Third-party arithmetic: the reference's FFT is rustfft 6.4.1 (f32,
unnormalised); here scipy.fft (pocketfft) in complex64 with the same
normalisation.  The two libraries round differently, so FP32 peak *values*
agree only to ~1e-6 relative; argmax positions and bins agree except where
two candidates tie to that level.  Pinned by the reference's own tests
(tests/test_oracle_reference_tests.py) and code KATs.  `precision="f64"`
runs the same algorithm in float64 (FP64 accuracy oracle).

Code chips come from the C restatement in codes_oracle.c (liboracle.so).
"""
import ctypes
import math
import os
import concurrent.futures as cf

import numpy as np
import scipy.fft as sfft

HERE = os.path.dirname(os.path.abspath(__file__))
TAU = 6.283185307179586  # std::f64::consts::TAU

GPS, GALILEO, BEIDOU, SBAS, L1C, QZSS = range(6)
NAMES = ["gps", "galileo", "beidou", "sbas", "l1c", "qzss"]
PRN_RANGE = {GPS: (1, 38), GALILEO: (1, 50), BEIDOU: (1, 63), SBAS: (120, 158), L1C: (1, 63), QZSS: (184, 206)}
SV_FMT = {GPS: "GPS{:02d}", GALILEO: "GSAT{:02d}", BEIDOU: "BEIDOU{:02d}", SBAS: "SBAS{:03d}",
          L1C: "GPSL1C{:02d}", QZSS: "QZSS{:03d}"}
ACR_TABLE_ID = {GPS: 0, SBAS: 0, QZSS: 0, GALILEO: 1, BEIDOU: 2, L1C: 3}
GNSS_IF = 4.092e6
SEARCH_BAND = 6000.0

_lib = None


def lib():
    """Load (building if needed) the oracle's C part."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", HERE])
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        L.oracle_base_sequence.argtypes = [ctypes.c_int, ctypes.c_int, dp]
        L.oracle_resampled.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_size_t, dp]
        L.oracle_estimate_cn0.argtypes = [ctypes.c_double, ctypes.c_int, dp]
        L.oracle_acr_table.argtypes = [ctypes.c_int, dp, ctypes.c_int]
        L.oracle_median.argtypes = [dp, ctypes.c_size_t]
        L.oracle_median.restype = ctypes.c_double
        L.oracle_mad.argtypes = [dp, ctypes.c_size_t, ctypes.c_double]
        L.oracle_mad.restype = ctypes.c_double
        L.oracle_b1cp_bits.argtypes = [ctypes.c_int, ctypes.c_char_p]
        L.oracle_l1cp_bits.argtypes = [ctypes.c_int, ctypes.c_char_p]
        L.oracle_ca_from_delay.argtypes = [ctypes.c_int, dp]
        _load_tables(L)
        _lib = L
    return _lib


TABLES = os.path.join(os.path.dirname(HERE), "tests", "golden", "tables.json")


def tables():
    """The oracle's own copy of the reference's data tables (read from its
    sources by tests/golden/make_golden.py)."""
    import json
    with open(TABLES) as f:
        return json.load(f)


def _load_tables(L):
    t = tables()
    ip = lambda v: (ctypes.c_int * len(v))(*v)
    L.oracle_set_ca_delays(ip(t["gps_g2_delay"]), ip(t["sbas_g2_delay"]), ip(t["qzss_g2_delay"]))
    L.oracle_set_weil(ip([x for p in t["b1cp_weil_wp"] for x in p]), ip([x for p in t["l1cp_weil_wp"] for x in p]))
    for i, h in enumerate(t["galileo_e1c_hex"]):
        L.oracle_set_e1c_hex(i + 1, h.encode())
    for tid, key in enumerate(("acr_gps_l1_ca", "acr_galileo_e1c", "acr_beidou_b1c", "acr_gps_l1c")):
        rows = [x for p in t[key] for x in p]
        if not L.oracle_set_acr(tid, (ctypes.c_double * len(rows))(*rows), len(t[key])):
            raise ValueError("ACR table %s does not fit the oracle" % key)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


# ---------------------------------------------------------------------------
# codes, ACR, stats (C part)
# ---------------------------------------------------------------------------
def base_sequence(constellation, prn):
    out = np.zeros(20460)
    n = lib().oracle_base_sequence(constellation, prn, _dp(out))
    if n == 0:
        raise ValueError("PRN %d out of range for %s" % (prn, NAMES[constellation]))
    return out[:n].copy()


def resampled_code(constellation, prn, samples_per_code, num_samples):
    out = np.zeros(num_samples)
    if lib().oracle_resampled(constellation, prn, float(samples_per_code), num_samples, _dp(out)) == 0:
        raise ValueError("PRN %d out of range for %s" % (prn, NAMES[constellation]))
    return out


def weil_bits(constellation, prn):
    buf = ctypes.create_string_buffer(10230)
    (lib().oracle_b1cp_bits if constellation == BEIDOU else lib().oracle_l1cp_bits)(prn, buf)
    return np.frombuffer(buf.raw, dtype=np.uint8).copy()


def estimate_cn0(r_a, table_id):
    v = ctypes.c_double()
    ok = lib().oracle_estimate_cn0(float(r_a), table_id, ctypes.byref(v))
    return v.value if ok else None


def acr_table(table_id):
    buf = np.zeros(2 * 100)
    n = lib().oracle_acr_table(table_id, _dp(buf), 100)
    return buf[:2 * n].reshape(n, 2)


def median(x):
    a = np.ascontiguousarray(x, dtype=np.float64)
    return lib().oracle_median(_dp(a), len(a))


def mad(x, med):
    a = np.ascontiguousarray(x, dtype=np.float64)
    return lib().oracle_mad(_dp(a), len(a), float(med))


# ---------------------------------------------------------------------------
# observation helpers (observation.rs)
# ---------------------------------------------------------------------------
def unpack_bits(packed):
    """observation.rs:232-240 (MSB-first)."""
    return np.unpackbits(np.asarray(packed, dtype=np.uint8), axis=-1)


def correlate_antennas(bits_i, bits_j):
    """observation.rs:175-195, exact in f64 (sums of +-1 are integers)."""
    a = np.asarray(bits_i).astype(np.int64) * 2 - 1
    b = np.asarray(bits_j).astype(np.int64) * 2 - 1
    return float(np.sum(a * b)) / len(a)


def antenna_prep(bits_row, num_samples, fs):
    """acquisition.rs:281-294: +-1, mean over the full record, de-mean, first
    num_samples as f32, phasepoints TAU/fs*i."""
    bip = bits_row.astype(np.float64) * 2.0 - 1.0
    # Sum of +-1 values is an exact integer in f64 (order-independent).
    mean = float(np.sum(bip)) / len(bip)
    n = min(num_samples, len(bip))
    sig = (bip[:n] - mean).astype(np.float32)
    pc = TAU / fs
    pp = pc * np.arange(n, dtype=np.float64)
    return sig, pp


# ---------------------------------------------------------------------------
# correlation core (correlate.rs)
# ---------------------------------------------------------------------------
def freq_grid(center_freq, search_band):
    """acquisition.rs:188-198."""
    n = 2.0 * search_band / 300.0
    n = int(math.floor(abs(n) + 0.5)) * (1 if n >= 0 else -1)  # f64::round
    n_bins = max(n, 0) + 1
    if n_bins == 1:
        return np.array([center_freq])
    return np.array([(center_freq - search_band) + (i * (2.0 * search_band)) / (n_bins - 1.0)
                     for i in range(n_bins)])


def _types(precision):
    return (np.float32, np.complex64) if precision == "f32" else (np.float64, np.complex128)


def code_spectra(code, period, precision="f32"):
    """correlate.rs:47-68: conj(FFT([c,c])), conj(FFT([c,-c]))."""
    ft, ct = _types(precision)
    alt = np.array(code, dtype=np.float64)
    split = min(period, len(alt))
    alt[split:] = -alt[split:]
    a = np.conj(sfft.fft(np.asarray(code).astype(ft).astype(ct)))
    b = np.conj(sfft.fft(alt.astype(ft).astype(ct)))
    return a.astype(ct), b.astype(ct)


def _last_argmax(v):
    """Rust Iterator::max_by with partial_cmp returns the LAST maximal element."""
    return len(v) - 1 - int(np.argmax(v[::-1]))


def _bin_work(sig, pp, freq, cc, cc_alt, ft, ct):
    phase = (pp * freq).astype(np.float32)           # (p * freq) as f32
    if ft is np.float32:
        # f32::cos/sin (glibc cosf/sinf are correctly rounded in practice):
        # evaluate in f64 and round once.
        c = np.cos(phase.astype(np.float64)).astype(np.float32)
        s = np.sin(phase.astype(np.float64)).astype(np.float32)
    else:
        c, s = np.cos(phase.astype(np.float64)), np.sin(phase.astype(np.float64))
    iq = np.empty(len(sig), dtype=ct)
    iq.real = c * sig.astype(ft)
    iq.imag = s * sig.astype(ft)
    spec = sfft.fft(iq)
    n = len(sig)
    scale = ft(1.0) / np.sqrt(ft(n))
    best = None
    corrs = []
    for hyp, rep in enumerate((cc, cc_alt)):
        prod = spec * rep
        corr = (np.abs(sfft.ifft(prod, norm="forward")) * scale).astype(ft)
        corrs.append(corr)
        idx = _last_argmax(corr)
        val = corr[idx]
        if best is None or val > best[1]:
            best = (idx, val, corr, hyp)
    return best + (corrs[1 - best[3]],)


def _fold_grid(res, period):
    """Per bin, the larger of the two hypotheses' |corr| at each code phase
    (index mod period).  Used by the parity tests to recognise exact ties,
    where the reference's own choice depends on FP rounding order."""
    rows = []
    for r in res:
        c = np.asarray(r[2], dtype=np.float64)
        other = np.asarray(r[4], dtype=np.float64)
        m = np.maximum(c, other)
        g = np.full(period, -np.inf)
        idx = np.arange(len(m)) % period
        np.maximum.at(g, idx, m)
        rows.append(g)
    return np.array(rows)


def correlate_code(sig, pp, cc, cc_alt, fc, num_samples, period, fs, precision="f32", threads=1, grid=False):
    """correlate.rs:91-183.  Returns dict(best_peak, second_peak, best_freq_idx,
    best_codephase, hypothesis[, grid])."""
    if len(fc) == 0:
        raise ValueError("frequency bin list must be non-empty")
    ft, ct = _types(precision)
    if threads > 1:
        with cf.ThreadPoolExecutor(threads) as ex:
            res = list(ex.map(lambda f: _bin_work(sig, pp, f, cc, cc_alt, ft, ct), fc))
    else:
        res = [_bin_work(sig, pp, f, cc, cc_alt, ft, ct) for f in fc]
    vals = np.array([r[1] for r in res])
    bi = _last_argmax(vals)
    idx, peak, corr, hyp, _ = res[bi]
    chip_width = int(math.ceil(fs / 1.023e6))
    main = idx % period
    icp = np.arange(len(corr)) % period
    dist = np.where(icp >= main, np.minimum(icp - main, period - icp + main),
                    np.minimum(main - icp, period - main + icp))
    cand = corr[dist > chip_width]
    second = ft(cand.max()) if len(cand) else ft(-np.inf)
    if second <= 0.0:
        second = ft(1e-6)
    out = dict(best_peak=ft(peak), second_peak=ft(second), best_freq_idx=bi,
               best_codephase=int(idx), hypothesis=hyp)
    if grid:
        out["grid"] = _fold_grid(res, period)
    return out


def acquire_single(constellation, sig, pp, fs, center_freq, search_band, prn, period,
                   precision="f32", threads=1, grid=False):
    """acquire_full (acquisition.rs:176-248) and its five twins."""
    n = len(sig)
    fc = freq_grid(center_freq, search_band)
    code = resampled_code(constellation, prn, float(period), n)
    cc, cc_alt = code_spectra(code, period, precision)
    pk = correlate_code(np.asarray(sig, np.float32), np.asarray(pp, np.float64), cc, cc_alt, fc, n,
                        period, fs, precision, threads, grid)
    cp = pk["best_codephase"] % period
    out = dict(prn=prn, signal_strength=float(pk["best_peak"]), second_peak=float(pk["second_peak"]),
               codephase_frac=cp / float(period), frequency=float(fc[pk["best_freq_idx"]] - center_freq),
               best_freq_idx=pk["best_freq_idx"], best_codephase=cp, hypothesis=pk["hypothesis"])
    if grid:
        out["grid"] = pk["grid"]
    return out


def period_samples(constellation, fs):
    """(fs/1000) as usize for C/A; (fs*period) as usize otherwise."""
    if constellation in (GPS, SBAS, QZSS):
        return int(fs / 1000.0)
    return int(fs * (0.004 if constellation == GALILEO else 0.010))


def acquire_all(bits, fs, constellation, center_freq=GNSS_IF, search_band=SEARCH_BAND,
                ant_filter=None, prn_filter=None, cn0=False, precision="f32", threads=1, grid=False):
    """acquire_all_* (acquisition.rs:261-396).  bits: [n_ant, n_samples] 0/1."""
    bits = np.asarray(bits)
    period = period_samples(constellation, fs)
    num_samples = 2 * period
    ants = list(ant_filter) if ant_filter is not None else list(range(bits.shape[0]))
    ant_data = [antenna_prep(bits[a], num_samples, fs) for a in ants]
    lo, hi = PRN_RANGE[constellation]
    prns = list(prn_filter) if prn_filter is not None else list(range(lo, hi + 1))
    results = []
    for prn in prns:
        cells = [acquire_single(constellation, s, p, fs, center_freq, search_band, prn, period,
                                precision, threads, grid) for (s, p) in ant_data]
        strengths = [c["signal_strength"] for c in cells]
        seconds = [c["second_peak"] for c in cells]
        phases = [c["codephase_frac"] for c in cells]
        freqs = [c["frequency"] for c in cells]
        r = dict(sv=SV_FMT[constellation].format(prn), strengths=strengths, phases=phases,
                 freqs=freqs, cells=cells)
        if cn0:
            vals = []
            for vm, vs in zip(strengths, seconds):
                vals.append(estimate_cn0((vm / vs) ** 2, ACR_TABLE_ID[constellation])
                            if (vs > 0.0 and vm > vs) else None)
            r["cn0_acr"] = None if all(v is None for v in vals) else vals
        if len(phases) > 1:
            pm, fm = median(phases), median(freqs)
            r.update(phase_median=pm, phase_mad=mad(phases, pm), freq_median=fm, freq_mad=mad(freqs, fm))
        results.append(r)
    results.sort(key=lambda r: r["sv"])
    return dict(antenna_numbers=ants, results=results)
