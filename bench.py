#!/usr/bin/env python3
"""Benchmark: acquisition cells/s of the --all search over 24 antennas.

Workload (one "step"): tart-gnss-acquire's `--all` search (GPS, Galileo,
BeiDou, SBAS, L1C, QZSS: 276 PRNs) with `--cn0`, over 24 antennas of
synthetic 1-bit data at 16.368 MHz, 100 ms per antenna, reference semantics
(two code periods coherent, dual [c,c]/[c,-c] hypothesis, 41 x 300 Hz Doppler
bins around 4.092 MHz).  cells = sum over (antenna, PRN) of n_bins * period.

Synthetic data: 10 satellites per constellation (random PRNs, code phase
uniform, Doppler uniform +-4 kHz, random +-1 sign per code epoch, C/N0 uniform
38-50 dB-Hz), unit Gaussian noise, sign-quantised, packed MSB-first; seeded
(0x5EED2026 + 1 + rank).

Output: one JSON line (rank 0).  `value` is device time with the packed bits
already in HBM, for the tensor-core search (FP16 tcgen05 transform, FP32
accumulation, selected rows re-evaluated in FP32) unless --precision fp32;
`compare` holds the same measurement for the other arithmetic (the FP32
fused search by default) and whether both detect the same cells with the same
code phase, Doppler bin and hypothesis.  `e2e` goes through the C ABI
(tga_acquire_all) from pinned host memory with the H2D copy and the result
D2H inside the timed region.
`--impl reference` times the CPU restatement of the reference algorithm (the
reference itself is Rust and cannot be built here) on a bounded sample.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tart-gnss_b200"))

FS = 16.368e6
N_ANT = 24
SAMPLES = 1636800  # 100 ms
SEED = 0x5EED2026 + 1
METRIC = "acq cells/s, --all x 24 ant: BF16-TC vs FP32 fused on B200, same detections"
WORKLOAD = ("--all x 24 ant, 16.368 MHz 1-bit, 100 ms synthetic, 276 PRNs x 41 bins x 300 Hz, "
            "2-period coherent dual-hypothesis, --cn0")
# PRNs of each code length in the --all search (GPS 38 + SBAS 39 + QZSS 23;
# Galileo 50; BeiDou 63 + L1C 63) and the samples per chip at 16.368 MHz
GROUP_PRNS = {1023: 100, 4092: 50, 10230: 126}
SAMPLES_PER_CHIP = 16


def workload_config(n_ant, sharded=False, world=1):
    """The `config` object of both arms: the workload only, nothing of the
    arithmetic or the implementation that runs it."""
    cells = sum(n_ant * 41 * n * SAMPLES_PER_CHIP * lc for lc, n in GROUP_PRNS.items())
    par = ("antenna shards (strong scaling: the antennas of one %d-antenna observation split over %d GPUs, cells "
           "all-gathered)" % (n_ant, world) if sharded else
           "replicas (weak scaling: one %d-antenna observation per GPU)" % n_ant)
    return {"workload": WORKLOAD, "n_ant": n_ant,
            "cells_per_step_per_gpu": float(cells) / (world if sharded else 1),
            "l2": "256 MB buffer written between timed steps; 3.9 GB intermediate per step", "parallelism": par}


def tga_codes(c, prn, period):
    """One period of a PRN's resampled code from the library (GPU arm)."""
    import tga
    return tga.code_resampled(c, int(prn), float(period), period).astype(np.float32)


def oracle_codes(c, prn, period):
    """The same code from the oracle's C restatement (reference arm, so that
    arm never loads the library; tests/test_lib_cpu.py pins the two equal)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import acq_oracle as O
    return O.resampled_code(c, int(prn), float(period), period).astype(np.float32)


def synth_observation(seed, n_ant=N_ANT, n_samples=SAMPLES, chunk=163680, codes=tga_codes):
    """Seeded synthetic 1-bit recording (see module docstring).  `codes`
    makes one period of a PRN's code; both generators give identical bits."""
    rng = np.random.default_rng(seed)
    sats = []
    for c in range(6):
        lo, hi = {0: (1, 38), 1: (1, 50), 2: (1, 63), 3: (120, 158), 4: (1, 63), 5: (184, 206)}[c]
        P = int(FS / 1000.0) if c in (0, 3, 5) else int(FS * (0.004 if c == 1 else 0.010))
        for prn in rng.choice(np.arange(lo, hi + 1), size=10, replace=False):
            code = codes(c, prn, P)
            n_ep = n_samples // P + 2
            sats.append(dict(c=c, prn=int(prn), P=P, code=code, delay=int(rng.integers(0, P)),
                             dop=float(rng.uniform(-4000, 4000)), cn0=float(rng.uniform(38, 50)),
                             flips=rng.choice([-1.0, 1.0], size=n_ep).astype(np.float32)))
    phase = np.exp(1j * rng.uniform(0, 2 * np.pi, size=(n_ant, len(sats)))).astype(np.complex64)
    bits = np.empty((n_ant, n_samples // 8), np.uint8)
    for t0 in range(0, n_samples, chunk):
        n = min(chunk, n_samples - t0)
        t = np.arange(t0, t0 + n)
        U = np.empty((len(sats), n), np.complex64)
        for k, s in enumerate(sats):
            amp = 2.0 * math.sqrt(10.0 ** (s["cn0"] / 10.0) / FS)
            idx = t + s["delay"]
            chip = s["code"][idx % s["P"]] * s["flips"][idx // s["P"]]
            ph = (2 * np.pi * ((4.092e6 + s["dop"]) / FS) * t) % (2 * np.pi)
            U[k] = (amp * chip) * np.exp(1j * ph).astype(np.complex64)
        v = (phase @ U).real + rng.standard_normal((n_ant, n), dtype=np.float32)
        bits[:, t0 // 8:(t0 + n) // 8] = np.packbits(v >= 0.0, axis=1)
    return bits, sats


def synth_weak_observation(seed, n_ant=N_ANT, n_samples=SAMPLES, n_sats=8, chunk=163680, cn0=(28.0, 36.0)):
    """Weak-signal recording: n_sats GPS C/A satellites (PRNs 1-32) at C/N0
    uniform in cn0 (28-36 dB-Hz), code phase uniform, Doppler uniform +-4 kHz, random
    +-1 navigation bits of 20 ms with a random bit-edge offset, per-antenna
    carrier phases, unit Gaussian noise, sign-quantised.  Returns (bits,
    satellites)."""
    import tga
    rng = np.random.default_rng(seed)
    P = int(FS / 1000.0)
    sats = []
    for prn in rng.choice(np.arange(1, 33), size=n_sats, replace=False):
        code = tga.code_resampled(0, int(prn), float(P), P).astype(np.float32)
        sats.append(dict(prn=int(prn), code=code, delay=int(rng.integers(0, P)), dop=float(rng.uniform(-4000, 4000)),
                         cn0=float(rng.uniform(*cn0)), edge=int(rng.integers(0, 20)),
                         bits=rng.choice([-1.0, 1.0], size=n_samples // (20 * P) + 3).astype(np.float32)))
    phase = np.exp(1j * rng.uniform(0, 2 * np.pi, size=(n_ant, len(sats)))).astype(np.complex64)
    bits = np.empty((n_ant, n_samples // 8), np.uint8)
    for t0 in range(0, n_samples, chunk):
        n = min(chunk, n_samples - t0)
        t = np.arange(t0, t0 + n)
        U = np.empty((len(sats), n), np.complex64)
        for k, s in enumerate(sats):
            amp = 2.0 * math.sqrt(10.0 ** (s["cn0"] / 10.0) / FS)
            idx = t + s["delay"]
            chip = s["code"][idx % P] * s["bits"][(idx // P + s["edge"]) // 20]
            ph = (2 * np.pi * ((4.092e6 + s["dop"]) / FS) * t) % (2 * np.pi)
            U[k] = (amp * chip) * np.exp(1j * ph).astype(np.complex64)
        v = (phase @ U).real + rng.standard_normal((n_ant, n), dtype=np.float32)
        bits[:, t0 // 8:(t0 + n) // 8] = np.packbits(v >= 0.0, axis=1)
    return bits, sats


def synth_fine_observation(seed, n_ant=24, n=163680, sigma_chips=0.1):
    """Band-limited 1-bit recording for the fine-acquisition measurement: 6
    GPS C/A and 6 Galileo E1-C satellites at 45 dB-Hz, continuous delays and
    Dopplers, chip edges smoothed by a Gaussian of sigma_chips (the front-end
    model of the refinement), per-antenna carrier phases, unit noise.
    Returns (bits, satellites)."""
    import tga
    from scipy.special import ndtr
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n_ant, n))
    t_all = np.arange(n, dtype=np.float64)
    sats = []
    for c, hi, per_s, chips in ((0, 32, 1e-3, 1023), (1, 36, 4e-3, 4092)):
        for prn in rng.choice(np.arange(1, hi + 1), size=6, replace=False):
            P0 = int(FS * per_s)
            s = dict(c=c, prn=int(prn), P=P0, tau=float(rng.uniform(0, P0)), dop=float(rng.uniform(-4000, 4000)))
            seq = tga.code_chips(c, int(prn)).astype(np.float64)
            L = len(seq)
            T, sig = FS * per_s / L, sigma_chips * FS * per_s / chips
            t = t_all - s["tau"]
            k = np.floor(t / T).astype(np.int64)
            code = seq[np.mod(k, L)].copy()
            for dm in (-1, 0, 1, 2):
                m = k + dm
                d = seq[np.mod(m, L)] - seq[np.mod(m - 1, L)]
                u = (t - m * T) / sig
                code += d * (ndtr(u) - (u >= 0))
            amp = 2.0 * math.sqrt(10.0 ** 4.5 / FS)
            cyc = np.mod((4.092e6 + s["dop"]) / FS * t_all, 1.0)
            for a in range(n_ant):
                x[a] += amp * code * np.cos(2 * np.pi * cyc + rng.uniform(0, 2 * np.pi))
            sats.append(s)
    return np.packbits(x >= 0.0, axis=1), sats


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.path = os.path.join("/tmp", "tga_clocks_%d_%d.csv" % (os.getpid(), index))

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i] and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


CPU_SAMPLE_REPEATS = 16  # ~10 s of oracle work per sample on a 16-core host


def cpu_sample_baseline(threads, repeats=CPU_SAMPLE_REPEATS):
    """CPU restatement of the reference algorithm (oracle) on a bounded sample
    of the same workload: antenna 0, a PRN subset of every constellation, all
    41 bins.  Returns (cells/s, seconds, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import acq_oracle as O
    bits, _ = synth_observation(SEED, n_ant=1, codes=oracle_codes)
    ub = np.unpackbits(bits, axis=1)
    sample = {O.GPS: [1, 2, 3, 4], O.SBAS: [120, 121], O.QZSS: [184], O.GALILEO: [1, 2], O.BEIDOU: [1, 2],
              O.L1C: [1, 2]}
    cells = 0.0
    t0 = time.perf_counter()
    for _ in range(repeats):
        for c, prns in sample.items():
            P = O.period_samples(c, FS)
            O.acquire_all(ub, FS, c, prn_filter=prns, cn0=True, threads=threads)
            cells += len(prns) * 41 * P
    dt = time.perf_counter() - t0
    desc = ("antenna 0 of the workload, PRNs GPS 1-4, SBAS 120-121, QZSS 184, Galileo 1-2, BeiDou 1-2, "
            "L1C 1-2, all 41 bins, x%d; numpy/scipy (pocketfft complex64) restatement of correlate_code, "
            "3 FFTs of 2P per bin as the reference" % repeats)
    return cells / dt, dt, desc


def fp64_peak_errors(bits, runs, threads):
    """Peak-metric error of the GPU searches against the oracle in float64 on
    a bounded sample of the benchmark recording (antenna 0, the PRNs of the
    CPU baseline sample, all 41 bins): per constellation, the largest
    relative error of signal_strength, the largest C/N0 (ACR, dB-Hz) error
    and whether code phase, bin, hypothesis and C/N0 validity equal the FP64
    result.  runs: {arithmetic: cells}."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import acq_oracle as O
    names = {O.GPS: "GPS L1 C/A", O.SBAS: "SBAS", O.QZSS: "QZSS", O.GALILEO: "Galileo E1-C",
             O.BEIDOU: "BeiDou B1C", O.L1C: "GPS L1C"}
    sample = {O.GPS: [1, 2, 3, 4], O.SBAS: [120, 121], O.QZSS: [184], O.GALILEO: [1, 2], O.BEIDOU: [1, 2],
              O.L1C: [1, 2]}
    ub = np.unpackbits(bits[:1], axis=1)
    out = {}
    for c, prns in sample.items():
        ref = O.acquire_all(ub, FS, c, prn_filter=prns, cn0=True, precision="f64", threads=threads)
        per = {}
        for arith, cells in runs.items():
            worst, worst_cn0, same = 0.0, 0.0, True
            for r in ref["results"]:
                rc = r["cells"][0]
                g = cells[(cells["constellation"] == c) & (cells["prn"] == rc["prn"]) & (cells["antenna"] == 0)][0]
                worst = max(worst, abs(g["signal_strength"] - rc["signal_strength"]) / rc["signal_strength"])
                rcn0 = (r.get("cn0_acr") or [None])[0]
                same &= (int(g["best_codephase"]) == int(rc["best_codephase"]) and
                         int(g["best_freq_idx"]) == int(rc["best_freq_idx"]) and
                         int(g["hypothesis"]) == int(rc["hypothesis"]) and
                         bool(g["cn0_valid"]) == (rcn0 is not None))
                if rcn0 is not None and g["cn0_valid"]:
                    worst_cn0 = max(worst_cn0, abs(float(g["cn0_acr"]) - rcn0))
            per[arith] = {"max_rel_peak_error": worst, "max_cn0_error_db": worst_cn0, "same_cell": bool(same)}
        out[names[c]] = per
    return out


# tensor-core MMA FLOPs per complex output point of the inverse transform,
# by code length: the Good-Thomas stages 31 x 33 (Lc = 1023), 31 x 12 x 11
# (4092) and 31 x 30 x 11 (10230) as real 2R x 2R GEMMs, 8 R per stage
TC_MMA_FLOPS_PER_POINT = {1023: 8 * (31 + 33), 4092: 8 * (31 + 12 + 11), 10230: 8 * (31 + 30 + 11)}


# index of a constellation's PRN inside its code-length group's row-peak
# array (the group's constellations in mask order)
GROUP_OF = {0: (1023, 0, 1), 3: (1023, 38, 120), 5: (1023, 77, 184), 1: (4092, 0, 1), 2: (10230, 0, 1),
            4: (10230, 63, 1)}


def fp64_key_errors(bits, tc_rows, threads):
    """Error of the tensor-core search's FP16 row keys against the oracle in
    float64 on the bounded sample (antenna 0, the PRNs of the CPU baseline
    sample, all 41 bins x 2 hypotheses): per constellation, the largest
    |FP16 row peak - FP64 row peak| relative to the largest FP64 row peak of
    the (antenna, PRN) (the normalisation of the library's candidate bound,
    2^-8), and the largest relative error of the best row's peak.
    tc_rows: {chips: array [n_ant, 82, n_prn]} from Context.row_peaks."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import acq_oracle as O
    import concurrent.futures as cf
    names = {O.GPS: "GPS L1 C/A", O.SBAS: "SBAS", O.QZSS: "QZSS", O.GALILEO: "Galileo E1-C",
             O.BEIDOU: "BeiDou B1C", O.L1C: "GPS L1C"}
    sample = {O.GPS: [1, 2, 3, 4], O.SBAS: [120, 121], O.QZSS: [184], O.GALILEO: [1, 2], O.BEIDOU: [1, 2],
              O.L1C: [1, 2]}
    ub = np.unpackbits(bits[:1], axis=1)[0]
    fc = O.freq_grid(4.092e6, 6000.0)
    out = {}
    for c, prns in sample.items():
        P = O.period_samples(c, FS)
        sig, pp = O.antenna_prep(ub, 2 * P, FS)
        chips, off, first = GROUP_OF[c]
        worst_rows, worst_best = 0.0, 0.0
        for prn in prns:
            code = O.resampled_code(c, prn, float(P), 2 * P)
            cc, ca = O.code_spectra(code, P, "f64")

            def rowmax(f):
                r = O._bin_work(sig, pp, f, cc, ca, np.float64, np.complex128)
                m = [0.0, 0.0]
                m[r[3]], m[1 - r[3]] = float(r[2].max()), float(r[4].max())
                return m
            with cf.ThreadPoolExecutor(threads) as ex:
                ref = np.array(list(ex.map(rowmax, fc))).reshape(-1)  # [bin * 2 + hyp]
            got = tc_rows[chips][0, :, off + prn - first]
            worst_rows = max(worst_rows, float(np.abs(got - ref).max() / ref.max()))
            b = int(np.argmax(ref))
            worst_best = max(worst_best, abs(got[b] - ref[b]) / ref[b])
        out[names[c]] = {"max_row_error_of_row_max": worst_rows, "max_rel_error_best_row": worst_best}
    return out


def fp32_peak_tflops(sm_mhz, n_sm=148):
    return n_sm * 128 * 2 * sm_mhz * 1e6 / 1e12


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    times, vals = [], []
    for i in range(args.warmup + args.steps):
        v, dt, desc = cpu_sample_baseline(threads)
        if i >= args.warmup:
            times.append(dt)
            vals.append(v)
    value = statistics.mean(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(N_ANT),
            "cpu_baseline": {"value": value, "unit": "cells/s", "cores": threads, "kind": "port",
                             "sample": "bounded sample of the workload: " + desc},
            "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# The --all search non-coherently over the whole 100 ms: one code period per
# coherent block and bins of 1 / (2 T) per code length over +-5 kHz
CONFIG2 = [  # (constellation, PRN range, blocks, bins, bin step Hz)
    (0, (1, 38), 100, 21, 500.0), (3, (120, 158), 100, 21, 500.0), (5, (184, 206), 100, 21, 500.0),
    (1, (1, 50), 25, 81, 125.0), (2, (1, 63), 10, 201, 50.0), (4, (1, 63), 10, 201, 50.0)]


def run_config2(ctx, bits, sats, args, world, stream, flush, kernel_times, prec_id):
    """Every constellation of the --all search over the full 100 ms of the
    benchmark recording, non-coherently: coherent blocks of one code period
    (1 / 4 / 10 ms), |y|^2 summed over the 100 / 25 / 10 blocks, Doppler
    +-5 kHz in 500 / 125 / 50 Hz bins, 24 antennas.  Both arithmetics end to
    end through tga_search_noncoherent_multi from pinned host bits (GPS /
    SBAS / QZSS and BeiDou / L1C share their front ends); cell-blocks count
    (antenna, PRN, bin, lag, block).  Detection against the injected
    satellites: summed peak > 1.5 x second peak, code phase within one
    sample, frequency within one bin."""
    import torch
    import tga
    if world > 1:
        import torch.distributed as dist
    searches = [dict(constellation=c, prns=list(range(lo, hi + 1)), center_freq=4.092e6, bin_step_hz=step,
                     n_bins=nb, coherent_periods=1, blocks=B) for c, (lo, hi), B, nb, step in CONFIG2]
    n_ant = bits.shape[0]
    period = {0: 16368, 3: 16368, 5: 16368, 1: 65472, 2: 163680, 4: 163680}
    cells = float(sum(n_ant * (hi - lo + 1) * nb * period[c] * B for c, (lo, hi), B, nb, _ in CONFIG2))
    host = torch.from_numpy(bits).pin_memory().numpy()
    steps, warm = min(args.steps, 3), min(args.warmup, 1)
    runs, peaks = {}, {}
    for prec in ("fp16tc", "fp32"):
        ctx.set_precision(prec_id[prec])
        for _ in range(warm):
            out = ctx.search_noncoherent_multi(host, FS, searches)
        if world > 1:
            dist.barrier()
        times = []
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = ctx.search_noncoherent_multi(host, FS, searches)
            times.append(time.perf_counter() - t0)
        t = statistics.mean(times)
        if world > 1:
            tt = torch.tensor([t], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        refined = sum(ctx.row_peaks(lc)[1] for lc in (1023, 4092, 10230)) if prec == "fp16tc" else 0
        peaks[prec] = {lc: ctx.row_peaks(lc)[0] for lc in (1023, 4092, 10230)}
        # one more, untimed call with per-kernel events for the breakdown
        tga.lib().tga_set_profiling(ctx._h, 1)
        ctx.search_noncoherent_multi(host, FS, searches)
        kt = {k: round(v[0], 3) for k, v in kernel_times().items()}
        tga.lib().tga_set_profiling(ctx._h, 0)
        runs[prec] = (t, out, kt, refined)
    truth = {}
    for sv in sats:
        truth[(sv["c"], sv["prn"])] = sv

    def detect(outs):
        det_all, stats = [], {}
        for (c, (lo, hi), B, nb, step), o in zip(CONFIG2, outs):
            P = period[c]
            det = o["power"] > 1.5 * o["second_power"]
            present = np.array([(c, int(x["prn"])) in truth for x in o])
            hit = np.zeros(len(o), bool)
            for i, x in enumerate(o):
                sv = truth.get((c, int(x["prn"])))
                if sv is not None:
                    d = abs(int(x["best_codephase"]) - (P - sv["delay"]) % P)
                    hit[i] = min(d, P - d) <= 1 and abs(x["frequency"] - sv["dop"]) <= step
            stats[tga.NAMES[c]] = {"p_detect": float(np.mean(det[present] & hit[present])),
                                   "p_false_alarm": float(np.mean(det[~present])) if (~present).any() else None}
            det_all.append(det)
        return det_all, stats
    # the FP16 keys' error against the FP32 ones on the whole workload:
    # largest amplitude difference over the bins of an (antenna, PRN),
    # relative to its largest FP16 row amplitude (the candidate bound's
    # normalisation; powers are sums over the blocks)
    key_err = {}
    for lc, nb in ((1023, 21), (4092, 81), (10230, 201)):
        a = np.sqrt(peaks["fp32"][lc].reshape(n_ant, nb, -1))
        b = np.sqrt(peaks["fp16tc"][lc].reshape(n_ant, nb, -1))
        key_err[str(lc)] = float((np.abs(b - a).max(axis=1) / b.max(axis=1)).max())
    fields = ("best_freq_idx", "best_codephase", "power", "second_power")
    identical = all(np.array_equal(a[k], b[k]) for a, b in zip(runs["fp16tc"][1], runs["fp32"][1]) for k in fields)
    _, st16 = detect(runs["fp16tc"][1])
    _, st32 = detect(runs["fp32"][1])
    t16, t32 = runs["fp16tc"][0], runs["fp32"][0]
    return {"workload": "--all x %d ant, 100 ms, non-coherent: one code period per coherent block (GPS/SBAS/QZSS "
                        "1 ms x 100, Galileo 4 ms x 25, BeiDou/L1C 10 ms x 10), Doppler +-5 kHz in 500 / 125 / 50 Hz "
                        "bins (1 / 2T), 276 PRNs; the benchmark recording (10 satellites per constellation, "
                        "38-50 dB-Hz, random sign per code epoch); tga_search_noncoherent_multi from pinned host "
                        "bits (end to end)" % n_ant,
            "unit": "cell-blocks/s", "cells_per_step_per_gpu": cells, "steps": steps, "warmup": warm,
            "fp16tc": {"value": cells * world / t16, "ms_per_step": t16 * 1e3, "kernels_ms": runs["fp16tc"][2],
                       "rows_reevaluated_fp32": runs["fp16tc"][3], "detection": st16},
            "fp32": {"value": cells * world / t32, "ms_per_step": t32 * 1e3, "kernels_ms": runs["fp32"][2],
                     "detection": st32},
            "speedup_fp16tc_over_fp32": t32 / t16, "identical_cells": bool(identical),
            "fp16_key_error_vs_fp32": {"per_code_length": key_err, "bound": 2.0 ** -8}}


def load_peaks():
    """Measured peaks of this GPU pool (driver-written), or None."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(path))
    except Exception:
        return None


def detections(cells):
    """Detected cells (strength / second >= 2, i.e. r_A >= 4) and their
    (code phase, Doppler bin, hypothesis)."""
    det = cells["signal_strength"] >= 2.0 * cells["second_peak"]
    return det, np.stack([cells["best_codephase"], cells["best_freq_idx"], cells["hypothesis"]], axis=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--n-ant", type=int, default=N_ANT, help="antennas per GPU (profiling runs use fewer)")
    ap.add_argument("--variant10", type=int, default=None, help="launch-shape variant of the Lc=10230 kernels "
                    "(skips the autotuner)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--precision", default="fp16tc", choices=["fp32", "fp16tc"],
                    help="search arithmetic of the headline: FP16 tensor-core transform with FP32 refinement "
                         "(default), or FP32 CUDA cores")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the second arithmetic (the FP32 fused search beside the tensor-core one)")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain GPS C/A search (1 antenna, 1 ms coherent x 10, 21 x 500 Hz bins)")
    ap.add_argument("--no-weak", action="store_true",
                    help="skip the weak-signal non-coherent search (10 ms coherent x 10, 201 x 50 Hz bins)")
    ap.add_argument("--no-fine", action="store_true", help="skip the fine-acquisition measurement")
    ap.add_argument("--no-config2", action="store_true",
                    help="skip the non-coherent --all search (per-code-length bins over 100 ms)")
    ap.add_argument("--config2-only", action="store_true",
                    help="run only the non-coherent --all search of --n-ant antennas and print its object "
                         "(profiling runs)")
    ap.add_argument("--sharded", action="store_true",
                    help="with N GPUs, split the antennas of one observation over the ranks (strong scaling, "
                         "multi_gpu.py) instead of one observation per rank")
    ap.add_argument("--no-split", action="store_true", help="skip the --benchmark-style setup/search split")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    import tga

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    bits_np, sats_np = synth_observation(SEED + rank, n_ant=args.n_ant)
    n_ant, row_bytes = bits_np.shape
    pinned = torch.empty((n_ant, row_bytes), dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = bits_np
    d_bits = pinned.to("cuda", non_blocking=False)
    ctx = tga.Context(local)
    if args.variant10 is not None:
        tga.lib().tga_set_variant(ctx._h, 10230, args.variant10)
    stream = torch.cuda.ExternalStream(tga.lib().tga_stream(ctx._h))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    lib = tga.lib()
    import ctypes
    prec_id = {"fp32": tga.PRECISION_FP32, "fp16tc": tga.PRECISION_FP16_TC}

    # --sharded: this rank's antennas of the one observation (all of them at N = 1)
    from multi_gpu import acquire_cells_sharded, shard_antennas
    shard = shard_antennas(range(n_ant), world, rank) if args.sharded else None

    def step_device():
        return ctx.acquire_cells(None, FS, mask=tga.ALL, cn0=True, device_bits=d_bits.data_ptr(), n_ant=n_ant,
                                 row_bytes=row_bytes, ant_filter=shard)

    def kernel_times():
        cap = 64
        names = (ctypes.c_char_p * cap)()
        ms = (ctypes.c_double * cap)()
        la = (ctypes.c_int32 * cap)()
        fl = (ctypes.c_double * cap)()
        n = ctypes.c_int()
        lib.tga_kernel_times.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        lib.tga_kernel_times(ctx._h, cap, names, ms, la, fl, ctypes.byref(n))
        return {names[i].decode(): (ms[i], la[i], fl[i]) for i in range(min(n.value, cap))}

    tuned = {}

    def measure(precision):
        """W warm-up and K timed device steps of one arithmetic; every rank
        takes the same collective steps.  Returns ms/step (max over ranks),
        cells, per-kernel times, launches and the last step's cells."""
        ctx.set_precision(prec_id[precision])
        if args.variant10 is None and not args.no_autotune:
            # launch shapes picked on this workload, before the warm-up
            tuned[precision] = ctx.autotune(d_bits.data_ptr(), n_ant, row_bytes, FS, mask=tga.ALL, cn0=True, reps=3)
        for _ in range(args.warmup):
            step_device()
        torch.cuda.synchronize()
        lib.tga_set_profiling(ctx._h, 1)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        total_ms, launches, agg, out = 0.0, 0, {}, None
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)  # evict L2 between steps (outside the timed events)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            out = step_device()
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
            launches += ctx.last_stats()["kernel_launches"]
            for k, (ms, la, fl) in kernel_times().items():
                a = agg.setdefault(k, [0.0, 0, 0.0])
                a[0] += ms
                a[1] += la
                a[2] += fl
        torch.cuda.synchronize()
        lib.tga_set_profiling(ctx._h, 0)
        cells = ctx.last_stats()["cells"]
        ms_step = total_ms / args.steps
        if world > 1:
            t = torch.tensor([ms_step], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_step = float(t.item())
            dist.barrier()
        return ms_step, cells, agg, launches, out

    def roofline(agg, precision, sm_mhz):
        """Dominant kernel of a run against its roofline.  `achieved` counts
        the algorithmic FLOPs the library reports per launch (5 P log2 P + 9 P
        per correlation row of P lags: product, inverse FFT, power; the
        executed arithmetic is larger).  The tensor-core correlator is held
        against the measured sustained dense FP16/BF16 rate (it is timed
        inside a long step), the FP32 kernels against the FP32 pipe.  For the
        tensor-core kernel `tensor_pipe_util` is the fraction of that rate its
        executed MMAs take (the DFT stages as dense real 2R x 2R GEMMs)."""
        dname, (dms, dl, dfl) = max(agg.items(), key=lambda kv: kv[1][0])
        avg_launch_s = dms / dl / 1e3
        achieved = dfl / dl / avg_launch_s / 1e12
        peaks = load_peaks()
        extra = {}
        if precision == "fp16tc" and dname.startswith("correlate_tc"):
            if peaks and peaks.get("bf16_tflops_sustained"):
                peak, src = float(peaks["bf16_tflops_sustained"]), "of measured: MEASURED_PEAKS.json bf16_tflops_sustained"
            else:
                peak, src = 1400.0, "of fallback: sustained dense bf16 figure of the profiling recipe"
            bound = "tensor"
            lc = int(dname.split("Lc=")[1].rstrip("]"))
            rows = n_ant * 41 * 2 * GROUP_PRNS[lc]
            executed = rows * SAMPLES_PER_CHIP * lc * TC_MMA_FLOPS_PER_POINT[lc]
            extra = {"tensor_pipe_util": executed / avg_launch_s / 1e12 / peak,
                     "executed_tflops": executed / avg_launch_s / 1e12,
                     "executed_flops": "the DFT stages as dense real 2R x 2R GEMMs, 8 x (sum of the radices) per "
                                       "complex output point (%d at Lc = %d)" % (TC_MMA_FLOPS_PER_POINT[lc], lc)}
        else:
            peak = fp32_peak_tflops(sm_mhz)
            src = ("148 SM x 128 FP32 lanes x 2 flop x median SM clock under load (%.0f MHz); "
                   "MEASURED_PEAKS.json has no FP32 SIMT figure" % sm_mhz)
            bound = "fp32"
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tp):
            traffic = json.load(open(tp)).get(dname.split("[")[0], {}).get("bytes_per_launch")
        return dict({"bound": bound, "kernel": dname, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": src,
                     "flops": "algorithmic: 5 P log2 P + 9 P per correlation row of P lags (two hypotheses per "
                              "(antenna, bin, PRN))",
                     "flops_per_launch": dfl / dl, "avg_launch_ms": dms / dl}, **extra)

    def kernels(agg):
        tot = sum(x[0] for x in agg.values())
        return {k: {"ms_per_step": v[0] / args.steps, "share": v[0] / tot, "launches_per_step": v[1] / args.steps}
                for k, v in agg.items()}

    if args.config2_only:
        c2 = run_config2(ctx, bits_np, sats_np, args, world, stream, flush, kernel_times, prec_id)
        if rank == 0:
            print(json.dumps({"config2": c2}), flush=True)
        ctx.close()
        if world > 1:
            dist.destroy_process_group()
        return
    clk = Clocks(local)
    clk.start()
    ms_step, cells, agg, launches, out = measure(args.precision)
    # the last timed step's row keys and, in tensor-core mode, how many rows
    # the FP16 key bound sent to the FP32 re-evaluation
    head_rows, refined_rows = {}, {}
    for chips in GROUP_PRNS:
        r, nref = ctx.row_peaks(chips)
        head_rows[chips] = r.reshape(n_ant, 82, -1)
        refined_rows[chips] = nref
    other = None
    if not args.no_compare:
        oprec = "fp32" if args.precision == "fp16tc" else "fp16tc"
        other = (oprec,) + measure(oprec)
    plain = None
    if not args.no_plain:
        # plain GPS C/A acquisition: 1 antenna, 10 ms (1 ms coherent x 10
        # non-coherent sums), PRNs 1-32, 21 x 500 Hz bins, 4 satellites at
        # 45 dB-Hz with navigation bits; both arithmetics, and (rank 0) the
        # oracle on the same bits: PRN set, code phase and bin compared
        pbits, psats = synth_weak_observation(SEED + 2000 + rank, n_ant=1, n_samples=163680, n_sats=4,
                                              cn0=(45.0, 45.0))
        pkw = dict(prns=list(range(1, 33)), bin_step_hz=500.0, n_bins=21, coherent_periods=1, blocks=10)
        pcells = 1 * 32 * 21 * 16368.0 * 10
        pres = {}
        for prec in ("fp16tc", "fp32"):
            ctx.set_precision(prec_id[prec])
            for _ in range(args.warmup):
                pout = ctx.search_noncoherent(pbits, FS, tga.GPS, **pkw)
            pt = []
            for _ in range(args.steps):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                pout = ctx.search_noncoherent(pbits, FS, tga.GPS, **pkw)
                pt.append(time.perf_counter() - t0)
            pres[prec] = (statistics.mean(pt), pout)
        ctx.set_precision(prec_id[args.precision])
        ptruth = {s["prn"]: s for s in psats}

        def pdet(out):
            return {int(c["prn"]): (int(c["best_codephase"]), int(c["best_freq_idx"]))
                    for c in out if c["power"] > 1.5 * c["second_power"]}

        plain = {"workload": "GPS C/A PRNs 1-32 x 1 antenna, 1 ms coherent x 10 blocks (10 ms), 21 x 500 Hz bins, "
                             "4 satellites at 45 dB-Hz with navigation bits; tga_search_noncoherent end to end",
                 "unit": "cell-blocks/s", "cells_per_step": pcells}
        for prec, (t_s, pout) in pres.items():
            d = pdet(pout)
            found = sum(1 for prn, s in ptruth.items() if prn in d and d[prn][0] == (16368 - s["delay"]) % 16368)
            plain[prec] = {"value": pcells / t_s, "ms_per_step": t_s * 1e3, "detected_prns": sorted(d),
                           "injected_found": "%d of %d" % (found, len(ptruth))}
        plain["same_detections"] = pdet(pres["fp16tc"][1]) == pdet(pres["fp32"][1])
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import nc_oracle
            ref = nc_oracle.search_nc(pbits, FS, tga.GPS, list(range(1, 33)), [0], 4.092e6, 500.0, 21, 1, 10, 0)
            rdet = {int(r["prn"]): (int(r["best_codephase"]), int(r["best_freq_idx"])) for r in ref
                    if r["power"] > 1.5 * r["second_power"]}
            plain["oracle_equal"] = {prec: pdet(pout) == rdet for prec, (t_s, pout) in pres.items()}

    weak = None
    if not args.no_weak:
        # weak-signal search: GPS C/A PRNs 1-32, 10 ms coherent blocks x 10
        # (100 ms), 201 bins of 50 Hz, on its own recording (8 satellites at
        # 28-36 dB-Hz with navigation-bit transitions); both arithmetics, end
        # to end through tga_search_noncoherent; cells count (antenna, PRN,
        # bin, code phase, block)
        wbits, wsats = synth_weak_observation(SEED + 1000 + rank, n_ant=n_ant)
        whost = torch.from_numpy(wbits).pin_memory().numpy()
        kw = dict(prns=list(range(1, 33)), bin_step_hz=50.0, n_bins=201, coherent_periods=10, blocks=10)
        wcells = n_ant * 32 * 201 * 16368.0 * 10
        runs = {}
        for prec in (args.precision, "fp32" if args.precision == "fp16tc" else "fp16tc"):
            ctx.set_precision(prec_id[prec])
            for _ in range(args.warmup):
                wout = ctx.search_noncoherent(whost, FS, tga.GPS, **kw)
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            wt = []
            for _ in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                wout = ctx.search_noncoherent(whost, FS, tga.GPS, **kw)
                wt.append(time.perf_counter() - t0)
            w_s = statistics.mean(wt)
            if world > 1:
                t = torch.tensor([w_s], device="cuda", dtype=torch.float64)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                w_s = float(t.item())
            # one more, untimed call with per-kernel events for the breakdown
            lib.tga_set_profiling(ctx._h, 1)
            ctx.search_noncoherent(whost, FS, tga.GPS, **kw)
            kt = {k: v[0] for k, v in kernel_times().items()}
            lib.tga_set_profiling(ctx._h, 0)
            runs[prec] = (w_s, wout, kt)
        ctx.set_precision(prec_id[args.precision])
        dtype_name = {"fp32": "f32", "fp16tc": "f16-tc+f32"}
        truth = {s["prn"]: s for s in wsats}
        thr = 1.5  # detection: summed peak power > 1.5 x the second peak

        def detect(out):
            det = out["power"] > thr * out["second_power"]
            hit = np.zeros(len(out), bool)
            for i, c in enumerate(out):
                s = truth.get(int(c["prn"]))
                if s is not None:
                    d = abs(int(c["best_codephase"]) - (16368 - s["delay"]) % 16368)
                    hit[i] = min(d, 16368 - d) <= 1 and abs(c["frequency"] - s["dop"]) <= 50.0
            present = np.array([int(c["prn"]) in truth for c in out])
            return det, {"p_detect": float(np.mean(det[present] & hit[present])),
                         "p_false_alarm": float(np.mean(det[~present])),
                         "present_cells": int(present.sum()), "absent_cells": int((~present).sum())}

        w_head, out_head, kt_head = runs[args.precision]
        other_prec = "fp32" if args.precision == "fp16tc" else "fp16tc"
        w_other, out_other, _ = runs[other_prec]
        det_h, stats_h = detect(out_head)
        det_o, stats_o = detect(out_other)
        same_rows = bool(np.array_equal(out_head["best_codephase"][det_h], out_other["best_codephase"][det_o])
                         and np.array_equal(out_head["best_freq_idx"][det_h], out_other["best_freq_idx"][det_o]))
        weak = {"workload": "GPS C/A PRNs 1-32 x %d ant, 10 ms coherent x 10 blocks (100 ms), 201 x 50 Hz bins; "
                            "8 satellites at C/N0 28-36 dB-Hz with navigation-bit transitions; "
                            "tga_search_noncoherent from pinned host bits (end to end)" % n_ant,
                "arithmetic": dtype_name[args.precision], "value": wcells * world / w_head,
                "unit": "cell-blocks/s", "ms_per_step": w_head * 1e3, "cells_per_step_per_gpu": wcells,
                "detection": dict(stats_h, threshold="power > %.1f x second_power, code phase within 1 sample "
                                                     "and frequency within 50 Hz of the truth" % thr),
                "kernels_ms": {k: v for k, v in kt_head.items() if k.startswith("nc_")},
                "compare": {"arithmetic": dtype_name[other_prec], "value": wcells * world / w_other,
                            "ms_per_step": w_other * 1e3, "speedup_of_weak": w_other / w_head,
                            "detection": stats_o,
                            "same_detections": bool(np.array_equal(det_h, det_o)) and same_rows}}
    config2 = None
    if not args.no_config2:
        config2 = run_config2(ctx, bits_np, sats_np, args, world, stream, flush, kernel_times, prec_id)
        ctx.set_precision(prec_id[args.precision])
    clocks = clk.stop()
    sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0
    # whole-job cells per step: every rank's (one observation per rank), or
    # the one observation split over the ranks (--sharded)
    job_cells = cells * world
    if args.sharded and world > 1:
        t = torch.tensor([cells], device="cuda", dtype=torch.float64)
        dist.all_reduce(t)
        job_cells = float(t.item())
    value = job_cells / (ms_step / 1e3)

    # end to end through the C ABI from pinned host memory
    ctx.set_precision(prec_id[args.precision])
    host = pinned.numpy()
    e2e_times = []
    for i in range(0 if args.no_e2e else args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if args.sharded and world > 1:
            acquire_cells_sharded(ctx, host, FS, mask=tga.ALL, cn0=True)
        else:
            ctx.acquire_cells(host, FS, mask=tga.ALL, cn0=True)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_times.append(dt)
    h2d, d2h = ctypes.c_uint64(), ctypes.c_uint64()
    lib.tga_last_transfer_bytes.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                                            ctypes.POINTER(ctypes.c_uint64)]
    lib.tga_last_transfer_bytes(ctx._h, ctypes.byref(h2d), ctypes.byref(d2h))
    # the same searches as a stream of observations (tga_acquire_all_stream):
    # the copy of observation i + 1 overlaps the search of observation i
    stream_s = None
    if not args.no_e2e and not (args.sharded and world > 1):
        seq = [host] * max(args.steps, 2)
        ctx.acquire_cells_stream(seq, FS, mask=tga.ALL, cn0=True)  # warm-up: both buffers' plans
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.acquire_cells_stream(seq, FS, mask=tga.ALL, cn0=True)
        stream_s = (time.perf_counter() - t0) / len(seq)
    e2e_s = statistics.mean(e2e_times) if e2e_times else float("nan")
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())

    dtype = {"fp32": "f32", "fp16tc": "f16-tc+f32"}
    line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "strong" if args.sharded else "weak",
            "vs_baseline": None, "dtype": dtype[args.precision], "data": "synthetic",
            "config": workload_config(n_ant, args.sharded, world),
            "arithmetic": ("FP16 tensor-core (tcgen05) transform, FP32 accumulation, selected rows "
                           "re-evaluated in FP32" if args.precision == "fp16tc" else "FP32 CUDA-core transform"),
            "e2e": {"value": job_cells / e2e_s, "unit": "cells/s", "h2d_bytes_per_step": h2d.value,
                    "d2h_bytes_per_step": d2h.value, "ms_per_step": e2e_s * 1e3},
            "gpu_launches": launches,
            "e2e_stream": None if stream_s is None else {
                "value": job_cells / stream_s, "unit": "cells/s", "ms_per_observation": stream_s * 1e3,
                "observations": max(args.steps, 2),
                "how": "tga_acquire_all_stream over the steps' observations from pinned host memory: each copy "
                       "overlaps the previous search"},
            "roofline": roofline(agg, args.precision, sm_mhz),
            "kernels": kernels(agg),
            "clocks": clocks}
    if tuned:
        # tga_autotune on this workload before each arithmetic's warm-up: the
        # launch shape kept per code length and the step time of each variant
        line["autotune"] = {dtype[p]: [{"lc": e["lc"], "variant": e["variant"],
                                        "ms_per_variant": [round(m, 3) for m in e["ms"]],
                                        "same_results": e["same_results"]} for e in v]
                            for p, v in tuned.items()}
    if other is not None:
        oprec, oms, ocells, oagg, olaunch, oout = other
        da, ka = detections(out)
        db, kb = detections(oout)
        same = bool(np.array_equal(da, db) and np.array_equal(ka[da], kb[db]))
        # every field of every cell, detected or not
        identical = all(np.array_equal(out[k], oout[k]) for k in
                        ("best_codephase", "best_freq_idx", "hypothesis", "signal_strength", "second_peak",
                         "cn0_valid", "cn0_acr"))
        ovalue = ocells * world / (oms / 1e3)
        line["compare"] = {"arithmetic": dtype[oprec], "value": ovalue, "ms_per_step": oms,
                           "speedup_of_headline": value / ovalue, "same_detections": same,
                           "identical_cells": bool(identical),
                           "detected_cells": int(da.sum()), "cells": int(len(da)),
                           "roofline": roofline(oagg, oprec, sm_mhz), "gpu_launches": olaunch}
    if rank == 0 and world == 1 and other is not None and not args.no_cpu_baseline:
        line["peak_error_vs_fp64"] = {
            "sample": "antenna 0, PRNs GPS 1-4, SBAS 120-121, QZSS 184, Galileo 1-2, BeiDou 1-2, L1C 1-2, 41 bins; "
                      "oracle (reference algorithm) in float64",
            "per_constellation": fp64_peak_errors(bits_np, {dtype[args.precision]: out, dtype[other[0]]: other[5]},
                                                  os.cpu_count() or 1)}
    if args.precision == "fp16tc":
        line["rows_reevaluated_fp32"] = {
            str(chips): {"rows": refined_rows[chips], "of_rows": int(head_rows[chips].size),
                         "per_cell": refined_rows[chips] / (head_rows[chips].size / 82)} for chips in GROUP_PRNS}
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            line["fp16_key_error_vs_fp64"] = {
                "sample": "antenna 0, PRNs GPS 1-4, SBAS 120-121, QZSS 184, Galileo 1-2, BeiDou 1-2, L1C 1-2, "
                          "41 bins x 2 hypotheses; oracle (reference algorithm) in float64",
                "bound": 2.0 ** -8,
                "per_constellation": fp64_key_errors(bits_np, head_rows, os.cpu_count() or 1)}
    if config2 is not None:
        line["config2"] = config2
    if plain is not None:
        line["plain_gps"] = plain
    if weak is not None:
        line["weak_signal"] = weak
    if not args.no_fine:
        # fine acquisition: grid estimates of the search, then the joint
        # multi-antenna Newton refinement, timed end to end through the C ABI
        fbits, fsats = synth_fine_observation(SEED + 7 + rank, n_ant=n_ant)
        IF = 4.092e6
        tasks, gt, gf = [], [], []
        for sv in fsats:
            cells = ctx.acquire_cells(fbits, FS, mask=1 << sv["c"], prn_filter=[sv["prn"]])
            tau_g = cells["best_codephase"] % sv["P"]
            f_g = cells["frequency"] + IF
            et = (tau_g - sv["tau"] + 0.5 * sv["P"]) % sv["P"] - 0.5 * sv["P"]
            ef = f_g - (IF + sv["dop"])
            hit = (np.abs(et) <= 2.0) & (np.abs(ef) <= 300.0)
            gt.append(et[hit])
            gf.append(ef[hit])
            b = int(np.argmax(cells["signal_strength"]))
            tasks.append((sv["c"], sv["prn"], float(tau_g[b]), float(f_g[b]), 0, fbits.shape[1] * 8))
        ft = []
        for i in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res, _ = ctx.fine_acquire(fbits, FS, tasks)
            if i >= args.warmup:
                ft.append(time.perf_counter() - t0)
        rt = np.array([(r["code_phase"] - sv["tau"] + 0.5 * sv["P"]) % sv["P"] - 0.5 * sv["P"]
                       for r, sv in zip(res, fsats)])
        rf = np.array([r["frequency"] - (IF + sv["dop"]) for r, sv in zip(res, fsats)])
        rms = lambda v: float(np.sqrt(np.mean(np.square(v))))
        gt, gf = np.concatenate(gt), np.concatenate(gf)
        line["fine_acquisition"] = {
            "workload": "%d antennas x 12 satellites (6 GPS C/A, 6 Galileo E1-C), 10 ms window, 45 dB-Hz, band-limited "
                        "synthetic, joint Newton refinement of delay, Doppler and per-antenna phase" % n_ant,
            "ms_per_call": 1e3 * statistics.mean(ft),
            "delay_rms_samples": {"grid": rms(gt), "refined": rms(rt)},
            "doppler_rms_hz": {"grid": rms(gf), "refined": rms(rf)},
            "converged": int(sum(r["converged"] for r in res))}
    if rank == 0 and not args.no_split:
        # --benchmark (main.rs:482-694) through tga_benchmark: one PRN per
        # constellation on antenna 0 of the benchmark observation, setup
        # (host extraction of every antenna's window) and search timed apart
        ctx.benchmark(bits_np, FS)  # warm-up
        entries = ctx.benchmark(bits_np, FS)
        names = {tga.GPS: "GPS", tga.GALILEO: "Galileo", tga.BEIDOU: "BeiDou", tga.SBAS: "SBAS", tga.QZSS: "QZSS",
                 tga.L1C: "L1C"}
        total_search = sum(e["search_s"] for e in entries)
        line["benchmark_split"] = {
            "per_constellation": [{"constellation": names[e["constellation"]], "prn": e["prn"],
                                   "setup_s": e["setup_s"], "search_s": e["search_s"]} for e in entries],
            "setup_s": sum(e["setup_s"] for e in entries), "search_s": total_search,
            "acq_per_s": len(entries) / total_search, "arithmetic": dtype[args.precision]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, dt, desc = cpu_sample_baseline(os.cpu_count() or 1)
        line["cpu_baseline"] = {"value": v, "unit": "cells/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": desc, "seconds": dt}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
