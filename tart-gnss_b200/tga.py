"""Python binding of libtga.so (ctypes), mirroring tart-gnss-acquire's API.

Function names, arguments and results follow the reference crate:

* acquire_full / acquire_sbas / acquire_qzss / acquire_galileo_single /
  acquire_beidou_single / acquire_l1c_single  (acquisition.rs:176,
  sbas.rs:132, qzss.rs:135, galileo.rs:133, beidou.rs:85, l1c.rs:94)
  -> AcquisitionResult(prn, signal_strength, second_peak, codephase_frac,
     frequency)
* acquire_all(...) -> {constellation: {"antenna_numbers", "results"}} with the
  per-PRN result dicts of acquire_all_* (acquisition.rs:261-396): sv,
  strengths, phases, freqs, cn0_acr (only with cn0), phase_median,
  phase_mad, freq_median, freq_mad (only with >1 antenna), sorted by sv.
* estimate_cn0_batch (acr.rs:49), correlate (observation.rs:175),
  code generators (generate_*_code / *_resampled).

The compute runs in libtga.so on the GPU; there is no CPU fallback.  A
missing library or device raises.
"""
import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtga.so")

GPS, GALILEO, BEIDOU, SBAS, L1C, QZSS = range(6)
NAMES = ["gps", "galileo", "beidou", "sbas", "l1c", "qzss"]
# PRN range of each constellation, in constellation order
PRN_RANGE = [(1, 38), (1, 50), (1, 63), (120, 158), (1, 63), (184, 206)]
ALL = 0x3F
GPS_IF = 4.092e6
GPS_SEARCH_BAND = 6000.0
ACR_TABLE = {GPS: 0, SBAS: 0, QZSS: 0, GALILEO: 1, BEIDOU: 2, L1C: 3}
PRECISION_FP32, PRECISION_FP16_TC = 0, 1
TEST_TC_SKIP_COMMIT = 1
GRAPH_NONE, GRAPH_CAPTURED, GRAPH_REPLAYED = 0, 1, 2

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "no sm_100 device", 4: "out of memory",
          5: "unsupported", 6: "timeout", 7: "capacity"}


class TgaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (STATUS.get(code, "error"), code, msg))
        self.code = code


class Result(ctypes.Structure):
    _fields_ = [("prn", ctypes.c_int32), ("best_freq_idx", ctypes.c_int32), ("best_codephase", ctypes.c_int64),
                ("signal_strength", ctypes.c_double), ("second_peak", ctypes.c_double),
                ("codephase_frac", ctypes.c_double), ("frequency", ctypes.c_double),
                ("hypothesis", ctypes.c_int32), ("path", ctypes.c_int32)]


class BenchEntry(ctypes.Structure):
    _fields_ = [("constellation", ctypes.c_int32), ("prn", ctypes.c_int32), ("setup_s", ctypes.c_double),
                ("search_s", ctypes.c_double), ("result", Result)]


class TuneEntry(ctypes.Structure):
    """tga_tune_entry: one code length tuned by tga_autotune."""
    _fields_ = [("lc", ctypes.c_int32), ("variant", ctypes.c_int32), ("ms", ctypes.c_double * 2),
                ("same_results", ctypes.c_int32 * 2)]


class Cell(ctypes.Structure):
    _fields_ = [("constellation", ctypes.c_int32), ("prn", ctypes.c_int32), ("antenna", ctypes.c_int32),
                ("best_freq_idx", ctypes.c_int32), ("best_codephase", ctypes.c_int64),
                ("signal_strength", ctypes.c_double), ("second_peak", ctypes.c_double),
                ("codephase_frac", ctypes.c_double), ("frequency", ctypes.c_double),
                ("cn0_acr", ctypes.c_double), ("cn0_valid", ctypes.c_int32), ("hypothesis", ctypes.c_int32)]


class AllOptions(ctypes.Structure):
    _fields_ = [("constellation_mask", ctypes.c_uint32), ("ant_filter", ctypes.POINTER(ctypes.c_int32)),
                ("n_ant_filter", ctypes.c_size_t), ("prn_filter", ctypes.POINTER(ctypes.c_int32)),
                ("n_prn_filter", ctypes.c_size_t), ("center_freq", ctypes.c_double),
                ("search_band", ctypes.c_double), ("cn0", ctypes.c_int32), ("debug", ctypes.c_int32)]


CELL_DTYPE = np.dtype([("constellation", "<i4"), ("prn", "<i4"), ("antenna", "<i4"), ("best_freq_idx", "<i4"),
                       ("best_codephase", "<i8"), ("signal_strength", "<f8"), ("second_peak", "<f8"),
                       ("codephase_frac", "<f8"), ("frequency", "<f8"), ("cn0_acr", "<f8"),
                       ("cn0_valid", "<i4"), ("hypothesis", "<i4")])
assert CELL_DTYPE.itemsize == ctypes.sizeof(Cell)

_lib = None
class FineTask(ctypes.Structure):
    """tga_fine_task: start point and window of one satellite's refinement."""
    _fields_ = [("constellation", ctypes.c_int32), ("prn", ctypes.c_int32), ("code_phase", ctypes.c_double),
                ("frequency", ctypes.c_double), ("start", ctypes.c_int64), ("length", ctypes.c_int64)]


class FineOptions(ctypes.Structure):
    _fields_ = [("edge_sigma_chips", ctypes.c_double), ("scan_half_width_hz", ctypes.c_double),
                ("max_iter", ctypes.c_int32), ("tol_code_phase", ctypes.c_double), ("tol_frequency", ctypes.c_double)]


class FineResult(ctypes.Structure):
    _fields_ = [("code_phase", ctypes.c_double), ("frequency", ctypes.c_double), ("power", ctypes.c_double),
                ("power_start", ctypes.c_double), ("iterations", ctypes.c_int32), ("converged", ctypes.c_int32)]


class RfiLine(ctypes.Structure):
    _fields_ = [("frequency", ctypes.c_double), ("excess_db", ctypes.c_double)]


class RfiChannel(ctypes.Structure):
    """tga_rfi_channel: RfiChannel of rfi.rs (NaN for None)."""
    _fields_ = [("antenna", ctypes.c_int32), ("dead", ctypes.c_int32), ("acf_lag1", ctypes.c_double),
                ("acf_lag3", ctypes.c_double), ("acf_lag16", ctypes.c_double), ("period_samples", ctypes.c_double),
                ("n_lines", ctypes.c_int32), ("lines", RfiLine * 3)]


class NcOptions(ctypes.Structure):
    _fields_ = [("constellation", ctypes.c_int32), ("prn_filter", ctypes.POINTER(ctypes.c_int32)),
                ("n_prn_filter", ctypes.c_size_t), ("ant_filter", ctypes.POINTER(ctypes.c_int32)),
                ("n_ant_filter", ctypes.c_size_t), ("center_freq", ctypes.c_double), ("bin_step_hz", ctypes.c_double),
                ("n_bins", ctypes.c_int32), ("coherent_periods", ctypes.c_int32), ("blocks", ctypes.c_int32),
                ("start", ctypes.c_int64)]


NC_CELL_DTYPE = np.dtype([("prn", np.int32), ("antenna", np.int32), ("best_freq_idx", np.int32),
                          ("reserved", np.int32), ("best_codephase", np.int64), ("power", np.float64),
                          ("second_power", np.float64), ("frequency", np.float64)])


class Observation(ctypes.Structure):
    """tga_observation (Observation::from_hdf5, observation.rs:48-92)."""
    _fields_ = [("num_antenna", ctypes.c_uint32), ("sampling_frequency", ctypes.c_double),
                ("row_bytes", ctypes.c_size_t), ("timestamp", ctypes.c_char * 64),
                ("config_json", ctypes.c_void_p), ("data", ctypes.c_void_p), ("error", ctypes.c_char * 256)]


_P = ctypes.c_void_p


def lib():
    """Load libtga.so (built in-tree by __graft_entry__.build() / make)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libtga.so not built at %s (run `make -C tart-gnss_b200`)" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    i32, sz, dbl = ctypes.c_int, ctypes.c_size_t, ctypes.c_double
    L.tga_create.argtypes = [i32, ctypes.POINTER(_P)]
    L.tga_destroy.argtypes = [_P]
    L.tga_last_error.argtypes = [_P]
    L.tga_last_error.restype = ctypes.c_char_p
    L.tga_version.restype = ctypes.c_char_p
    single = [_P, i32, _P, _P, sz, dbl, dbl, dbl, i32, sz, ctypes.POINTER(Result)]
    L.tga_acquire_single.argtypes = single
    for nm in ("tga_acquire_full", "tga_acquire_sbas", "tga_acquire_qzss", "tga_acquire_galileo_single",
               "tga_acquire_beidou_single", "tga_acquire_l1c_single"):
        getattr(L, nm).argtypes = [_P, _P, _P, sz, dbl, dbl, dbl, i32, sz, ctypes.POINTER(Result)]
    L.tga_acquire_all.argtypes = [_P, _P, sz, sz, dbl, ctypes.POINTER(AllOptions), _P, sz, ctypes.POINTER(sz)]
    L.tga_acquire_all_device.argtypes = L.tga_acquire_all.argtypes
    L.tga_acquire_all_stream.argtypes = [_P, _P, sz, sz, sz, dbl, ctypes.POINTER(AllOptions), _P, sz,
                                         ctypes.POINTER(sz)]
    L.tga_all_cell_count.argtypes = [sz, ctypes.POINTER(AllOptions), ctypes.POINTER(sz)]
    L.tga_last_search_stats.argtypes = [_P, ctypes.POINTER(dbl), ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(dbl)]
    L.tga_acr_cn0.argtypes = [_P, _P, sz, i32, _P, _P]
    L.tga_antenna_xcorr.argtypes = [_P, _P, sz, sz, i32, i32, ctypes.POINTER(dbl)]
    L.tga_antenna_xcorr_matrix.argtypes = [_P, _P, sz, sz, _P]
    L.tga_code_chips.argtypes = [i32, i32, _P, sz, ctypes.POINTER(sz)]
    L.tga_code_resampled.argtypes = [i32, i32, dbl, sz, _P]
    L.tga_stream.argtypes = [_P]
    L.tga_stream.restype = ctypes.c_void_p
    L.tga_set_profiling.argtypes = [_P, i32]
    L.tga_set_graphs.argtypes = [_P, i32]
    L.tga_benchmark.argtypes = [_P, _P, sz, sz, dbl, _P]
    L.tga_autotune.argtypes = [_P, _P, sz, sz, dbl, _P, i32, _P, _P]
    L.tga_last_graph.argtypes = [_P, ctypes.POINTER(ctypes.c_int)]
    L.tga_set_variant.argtypes = [_P, i32, i32]
    L.tga_set_precision.argtypes = [_P, i32]
    L.tga_set_test_flags.argtypes = [_P, i32]
    L.tga_rfi_scan.argtypes = [_P, _P, sz, sz, dbl, _P]
    L.tga_search_noncoherent.argtypes = [_P, _P, sz, sz, dbl, _P, _P, sz, _P]
    L.tga_search_noncoherent_multi.argtypes = [_P, _P, sz, sz, dbl, _P, sz, _P, sz, _P]
    L.tga_results_json.argtypes = [_P, sz, _P, sz, ctypes.c_uint32, i32, dbl, dbl, _P, _P]
    L.tga_observation_read_hdf5.argtypes = [ctypes.c_char_p, _P]
    L.tga_observation_free.argtypes = [_P]
    L.tga_acr_table.argtypes = [_P, i32, i32, dbl, dbl, dbl, dbl, i32, _P, sz, _P]
    L.tga_rfi_json.argtypes = [_P, sz, _P]
    L.tga_fine_eval.argtypes = [_P, _P, sz, sz, dbl, _P, _P, dbl, _P, _P, _P]
    L.tga_fine_acquire.argtypes = [_P, _P, sz, sz, dbl, _P, sz, _P, _P, _P]
    L.tga_acquire_single_static.argtypes = [i32, _P, _P, sz, dbl, dbl, dbl, i32, sz, _P, _P]
    L.tga_last_transfer_bytes.argtypes = [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    L.tga_kernel_times.argtypes = [_P, i32, _P, _P, _P, _P, ctypes.POINTER(ctypes.c_int)]
    L.tga_last_row_peaks.argtypes = [_P, i32, _P, sz, ctypes.POINTER(sz), ctypes.POINTER(ctypes.c_int64)]
    _lib = L
    return L


def read_hdf5(path):
    """TART HDF5 observation: dict(num_antenna, sampling_frequency, row_bytes,
    timestamp, config (str), data [num_antenna, row_bytes] packed bits)."""
    obs = Observation()
    rc = lib().tga_observation_read_hdf5(str(path).encode(), ctypes.byref(obs))
    if rc:
        raise TgaError(rc, obs.error.decode(errors="replace"))
    try:
        n = obs.num_antenna * obs.row_bytes
        data = np.ctypeslib.as_array(ctypes.cast(obs.data, ctypes.POINTER(ctypes.c_uint8)), shape=(n,)).copy()
        out = dict(num_antenna=obs.num_antenna, sampling_frequency=obs.sampling_frequency, row_bytes=obs.row_bytes,
                   timestamp=obs.timestamp.decode(), config=ctypes.string_at(obs.config_json).decode(),
                   data=data.reshape(obs.num_antenna, obs.row_bytes))
    finally:
        lib().tga_observation_free(ctypes.byref(obs))
    return out


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


# ---------------------------------------------------------------------------
# host-side code tables (no GPU needed)
# ---------------------------------------------------------------------------
def code_chips(constellation, prn):
    """generate_*_code: +-1 chips (BOC half-chips for BeiDou / L1C)."""
    n = ctypes.c_size_t()
    rc = lib().tga_code_chips(constellation, prn, None, 0, ctypes.byref(n))
    if rc:
        raise TgaError(rc, "bad constellation/PRN")
    out = np.empty(n.value, dtype=np.int8)
    lib().tga_code_chips(constellation, prn, _ptr(out), n.value, ctypes.byref(n))
    return out


def code_resampled(constellation, prn, samples_per_code, num_samples):
    out = np.empty(num_samples, dtype=np.float32)
    rc = lib().tga_code_resampled(constellation, prn, float(samples_per_code), num_samples, _ptr(out))
    if rc:
        raise TgaError(rc, "bad constellation/PRN")
    return out


@dataclass
class AcquisitionResult:
    prn: int
    signal_strength: float
    second_peak: float
    codephase_frac: float
    frequency: float
    best_freq_idx: int = 0
    best_codephase: int = 0
    hypothesis: int = 0
    path: int = 0


def _median(x):
    """stats.rs:10-20."""
    s = sorted(x)
    m = len(s) // 2
    return (s[m - 1] + s[m]) / 2.0 if len(s) % 2 == 0 else s[m]


def _mad(x, med):
    return _median([abs(v - med) for v in x])


SV_FMT = {GPS: "GPS{:02d}", GALILEO: "GSAT{:02d}", BEIDOU: "BEIDOU{:02d}", SBAS: "SBAS{:03d}",
          L1C: "GPSL1C{:02d}", QZSS: "QZSS{:03d}"}


class Context:
    """One engine context on one GPU (tga_create / tga_destroy)."""

    def __init__(self, device=0):
        self._h = _P()
        rc = lib().tga_create(device, ctypes.byref(self._h))
        if rc:
            raise TgaError(rc, "tga_create(device=%d) failed" % device)

    def close(self):
        if self._h:
            lib().tga_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc:
            raise TgaError(rc, lib().tga_last_error(self._h).decode())

    # ---- single PRN --------------------------------------------------------
    def acquire_single(self, constellation, signal_f32, phasepoints, sampling_freq, center_freq, search_band, prn,
                       samples_per_chunk):
        sig = np.ascontiguousarray(signal_f32, dtype=np.float32)
        pp = np.ascontiguousarray(phasepoints, dtype=np.float64)
        if len(pp) < len(sig):
            raise ValueError("phasepoints shorter than signal")
        r = Result()
        self._check(lib().tga_acquire_single(self._h, constellation, _ptr(sig), _ptr(pp), len(sig),
                                             float(sampling_freq), float(center_freq), float(search_band), int(prn),
                                             int(samples_per_chunk), ctypes.byref(r)))
        return AcquisitionResult(r.prn, r.signal_strength, r.second_peak, r.codephase_frac, r.frequency,
                                 r.best_freq_idx, r.best_codephase, r.hypothesis, r.path)

    def acquire_full(self, *a):
        return self.acquire_single(GPS, *a)

    def acquire_sbas(self, *a):
        return self.acquire_single(SBAS, *a)

    def acquire_qzss(self, *a):
        return self.acquire_single(QZSS, *a)

    def acquire_galileo_single(self, *a):
        return self.acquire_single(GALILEO, *a)

    def acquire_beidou_single(self, *a):
        return self.acquire_single(BEIDOU, *a)

    def acquire_l1c_single(self, *a):
        return self.acquire_single(L1C, *a)

    # ---- all PRNs, all antennas -------------------------------------------
    def _options(self, mask, ant_filter, prn_filter, center_freq, search_band, cn0, debug):
        o = AllOptions()
        o.constellation_mask = mask
        keep = []
        if ant_filter is not None:
            a = np.ascontiguousarray(ant_filter, dtype=np.int32)
            keep.append(a)
            o.ant_filter = a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            o.n_ant_filter = len(a)
        if prn_filter is not None:
            p = np.ascontiguousarray(prn_filter, dtype=np.int32)
            keep.append(p)
            o.prn_filter = p.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            o.n_prn_filter = len(p)
        o.center_freq = center_freq
        o.search_band = search_band
        o.cn0 = 1 if cn0 else 0
        o.debug = 1 if debug else 0
        return o, keep

    def acquire_cells(self, packed_bits, sampling_freq, mask=ALL, ant_filter=None, prn_filter=None,
                      center_freq=GPS_IF, search_band=GPS_SEARCH_BAND, cn0=False, device_bits=None, n_ant=None,
                      row_bytes=None):
        """Raw per-(constellation, prn, antenna) cells as a numpy record array.

        packed_bits: [n_ant, row_bytes] uint8 host array, or pass device_bits
        (an integer device pointer, e.g. torch tensor .data_ptr()) with
        n_ant and row_bytes."""
        o, keep = self._options(mask, ant_filter, prn_filter, center_freq, search_band, cn0, False)
        if device_bits is None:
            bits = np.ascontiguousarray(packed_bits, dtype=np.uint8)
            n_ant, row_bytes = bits.shape
        n = ctypes.c_size_t()
        self._check(lib().tga_all_cell_count(n_ant, ctypes.byref(o), ctypes.byref(n)))
        out = np.zeros(n.value, dtype=CELL_DTYPE)
        fn = lib().tga_acquire_all if device_bits is None else lib().tga_acquire_all_device
        src = _ptr(bits) if device_bits is None else ctypes.c_void_p(device_bits)
        self._check(fn(self._h, src, n_ant, row_bytes, float(sampling_freq), ctypes.byref(o), _ptr(out),
                       len(out), ctypes.byref(n)))
        del keep
        return out

    def acquire_cells_stream(self, observations, sampling_freq, mask=ALL, ant_filter=None, prn_filter=None,
                             center_freq=GPS_IF, search_band=GPS_SEARCH_BAND, cn0=False):
        """tga_acquire_all_stream: a list of host observations of one shape
        [n_ant, row_bytes] searched in turn, the copy of the next one
        overlapping the search of the current one.  Returns one cell array
        per observation."""
        obs = [np.ascontiguousarray(o, dtype=np.uint8) for o in observations]
        n_ant, row_bytes = obs[0].shape
        if any(o.shape != (n_ant, row_bytes) for o in obs):
            raise ValueError("observations of different shapes")
        o, keep = self._options(mask, ant_filter, prn_filter, center_freq, search_band, cn0, False)
        ptrs = (ctypes.c_void_p * len(obs))(*[x.ctypes.data for x in obs])
        n = ctypes.c_size_t()
        self._check(lib().tga_acquire_all_stream(self._h, ptrs, len(obs), n_ant, row_bytes, float(sampling_freq),
                                                 ctypes.byref(o), None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=CELL_DTYPE)
        self._check(lib().tga_acquire_all_stream(self._h, ptrs, len(obs), n_ant, row_bytes, float(sampling_freq),
                                                 ctypes.byref(o), _ptr(out), len(out), ctypes.byref(n)))
        del keep
        per = len(out) // len(obs)
        return [out[i * per:(i + 1) * per] for i in range(len(obs))]

    def acquire_all(self, packed_bits, sampling_freq, mask=ALL, ant_filter=None, prn_filter=None,
                    center_freq=GPS_IF, search_band=GPS_SEARCH_BAND, cn0=False, debug=False):
        """acquire_all_* for every constellation in mask, grouped like the
        reference's *AllAcquisitionOutput (per-PRN results sorted by sv)."""
        cells = self.acquire_cells(packed_bits, sampling_freq, mask, ant_filter, prn_filter, center_freq,
                                   search_band, cn0)
        n_ant = np.asarray(packed_bits).shape[0]
        ants = list(ant_filter) if ant_filter is not None else list(range(n_ant))
        out = {}
        for c in range(6):
            if not (mask >> c) & 1:
                continue
            sel = cells[cells["constellation"] == c]
            results = []
            for prn in dict.fromkeys(sel["prn"].tolist()):
                rows = sel[sel["prn"] == prn]
                r = {"sv": SV_FMT[c].format(prn), "strengths": rows["signal_strength"].tolist(),
                     "phases": rows["codephase_frac"].tolist(), "freqs": rows["frequency"].tolist(),
                     "second_peaks": rows["second_peak"].tolist(),
                     "best_freq_idx": rows["best_freq_idx"].tolist(),
                     "best_codephase": rows["best_codephase"].tolist()}
                if cn0:
                    vals = [float(v) if ok else None for v, ok in zip(rows["cn0_acr"], rows["cn0_valid"])]
                    r["cn0_acr"] = None if all(v is None for v in vals) else vals
                if len(rows) > 1:
                    pm, fm = _median(r["phases"]), _median(r["freqs"])
                    r.update(phase_median=pm, phase_mad=_mad(r["phases"], pm), freq_median=fm,
                             freq_mad=_mad(r["freqs"], fm))
                results.append(r)
            results.sort(key=lambda r: r["sv"])
            out[NAMES[c]] = {"antenna_numbers": ants, "results": results}
        return out

    def row_peaks(self, chips):
        """Row peaks of the last acquire_cells call for its group of `chips`-chip
        codes as the search's arithmetic computed them (tga_last_row_peaks):
        array [n_ant, n_bins, 2 hypotheses, n_prn] in signal_strength units,
        and the number of rows the tensor-core search re-evaluated in FP32."""
        n = ctypes.c_size_t()
        refined = ctypes.c_int64()
        self._check(lib().tga_last_row_peaks(self._h, int(chips), None, 0, ctypes.byref(n), ctypes.byref(refined)))
        out = np.zeros(n.value, dtype=np.float64)
        self._check(lib().tga_last_row_peaks(self._h, int(chips), _ptr(out), len(out), ctypes.byref(n), None))
        return out, int(refined.value)

    def set_test_flags(self, flags):
        """Test hooks (TGA_TEST_*); 0 in normal use."""
        self._check(lib().tga_set_test_flags(self._h, int(flags)))

    def set_precision(self, precision):
        """0 = FP32 (default), 1 = FP16 tensor-core search with FP32 refinement."""
        self._check(lib().tga_set_precision(self._h, int(precision)))

    def benchmark(self, packed_bits, sampling_freq):
        """--benchmark: one PRN per constellation on antenna 0, setup and
        search timed separately; list of dicts in the reference's order."""
        bits = np.ascontiguousarray(packed_bits, dtype=np.uint8)
        out = (BenchEntry * 6)()
        self._check(lib().tga_benchmark(self._h, _ptr(bits), bits.shape[0], bits.shape[1], float(sampling_freq),
                                        out))
        return [{"constellation": e.constellation, "prn": e.prn, "setup_s": e.setup_s, "search_s": e.search_s,
                 "result": e.result} for e in out]

    def autotune(self, device_bits, n_ant, row_bytes, sampling_freq, mask=ALL, ant_filter=None,
                 prn_filter=None, center_freq=GPS_IF, search_band=GPS_SEARCH_BAND, cn0=False, reps=3):
        """tga_autotune: time each launch-shape variant on this search (bits
        on the device, an integer pointer) and keep the fastest per code
        length on the context.  Returns one dict per code length searched:
        lc, variant (kept), ms [variant 0, variant 1], same_results."""
        o, keep = self._options(mask, ant_filter, prn_filter, center_freq, search_band, cn0, False)
        out = (TuneEntry * 3)()
        n = ctypes.c_size_t()
        self._check(lib().tga_autotune(self._h, ctypes.c_void_p(device_bits), n_ant, row_bytes,
                                       float(sampling_freq), ctypes.byref(o), int(reps), out, ctypes.byref(n)))
        del keep
        return [{"lc": e.lc, "variant": e.variant, "ms": list(e.ms), "same_results": [bool(x) for x in e.same_results]}
                for e in out[:n.value]]

    def set_variant(self, lc, variant):
        """Launch-shape variant (0 or 1) of the FP32 correlation kernels for chip count lc."""
        self._check(lib().tga_set_variant(self._h, int(lc), int(variant)))

    def set_profiling(self, enable):
        """Per-kernel CUDA-event timing of later calls (tga_kernel_times)."""
        self._check(lib().tga_set_profiling(self._h, 1 if enable else 0))

    def set_graphs(self, enable):
        """CUDA-graph capture and replay of repeated acquire_all plans (on by default)."""
        self._check(lib().tga_set_graphs(self._h, 1 if enable else 0))

    def last_graph(self):
        """GRAPH_NONE (eager), GRAPH_CAPTURED or GRAPH_REPLAYED for the last acquire_all call."""
        v = ctypes.c_int()
        self._check(lib().tga_last_graph(self._h, ctypes.byref(v)))
        return v.value

    def last_stats(self):
        cells, launches, ms = ctypes.c_double(), ctypes.c_int32(), ctypes.c_double()
        lib().tga_last_search_stats(self._h, ctypes.byref(cells), ctypes.byref(launches), ctypes.byref(ms))
        return {"cells": cells.value, "kernel_launches": launches.value, "device_ms": ms.value}

    # ---- ACR and antenna correlation ---------------------------------------
    def estimate_cn0_batch(self, r_a, table):
        ra = np.ascontiguousarray(r_a, dtype=np.float64)
        cn0 = np.zeros(len(ra))
        valid = np.zeros(len(ra), dtype=np.uint8)
        self._check(lib().tga_acr_cn0(self._h, _ptr(ra), len(ra), table, _ptr(cn0), _ptr(valid)))
        return [float(c) if v else None for c, v in zip(cn0, valid)]

    def correlate(self, packed_bits, i, j):
        bits = np.ascontiguousarray(packed_bits, dtype=np.uint8)
        out = ctypes.c_double()
        self._check(lib().tga_antenna_xcorr(self._h, _ptr(bits), bits.shape[0], bits.shape[1], i, j,
                                            ctypes.byref(out)))
        return out.value

    def acquire_json(self, packed_bits, sampling_freq, mask=ALL, cn0=False, filter_phase_mad=float("nan"),
                     filter_freq_mad=float("nan")):
        """The CLI's acquisition JSON (CombinedOutput, main.rs:893) for every
        antenna: the cells of acquire_cells through tga_results_json; a MAD
        filter of NaN is off (--filter-phase-mad / --filter-freq-mad)."""
        cells = self.acquire_cells(packed_bits, sampling_freq, mask=mask, cn0=cn0)
        n_ant = np.asarray(packed_bits).shape[0]
        ants = np.arange(n_ant, dtype=np.int32)
        p = ctypes.c_char_p()
        nf = ctypes.c_size_t()
        self._check(lib().tga_results_json(_ptr(cells), len(cells), _ptr(ants), n_ant, mask, int(cn0),
                                           float(filter_phase_mad), float(filter_freq_mad), ctypes.byref(p),
                                           ctypes.byref(nf)))
        text = ctypes.string_at(p).decode()
        lib().tga_free(p)
        return text

    def fine_eval(self, packed_bits, sampling_freq, constellation, prn, code_phase, frequency, start, length,
                  phases=None, edge_sigma_chips=0.1):
        """Coherent power P, gradient and Hessian at one point, parameter order
        (code_phase, frequency, phi_0 .. phi_{A-1}); phases None = aligned."""
        bits = np.ascontiguousarray(packed_bits, dtype=np.uint8)
        A = bits.shape[0]
        t = FineTask(constellation, prn, float(code_phase), float(frequency), int(start), int(length))
        ph = None if phases is None else np.ascontiguousarray(phases, dtype=np.float64)
        P = ctypes.c_double()
        g = np.zeros(2 + A)
        H = np.zeros((2 + A, 2 + A))
        self._check(lib().tga_fine_eval(self._h, _ptr(bits), A, bits.shape[1], float(sampling_freq), ctypes.byref(t),
                                        None if ph is None else _ptr(ph), float(edge_sigma_chips), ctypes.byref(P),
                                        _ptr(g), _ptr(H)))
        return P.value, g, H

    def fine_acquire(self, packed_bits, sampling_freq, tasks, edge_sigma_chips=0.1, scan_half_width_hz=0.0,
                     max_iter=0):
        """Newton refinement of (code_phase, frequency) per task, tasks being
        (constellation, prn, code_phase, frequency, start, length) tuples.
        Returns (list of dicts, phases [n_tasks, n_ant])."""
        bits = np.ascontiguousarray(packed_bits, dtype=np.uint8)
        A = bits.shape[0]
        arr = (FineTask * len(tasks))(*[FineTask(int(c), int(p), float(cp), float(f), int(s0), int(n))
                                        for c, p, cp, f, s0, n in tasks])
        out = (FineResult * len(tasks))()
        phases = np.zeros((len(tasks), A))
        opt = FineOptions(float(edge_sigma_chips), float(scan_half_width_hz), int(max_iter), 0.0, 0.0)
        self._check(lib().tga_fine_acquire(self._h, _ptr(bits), A, bits.shape[1], float(sampling_freq), arr,
                                           len(tasks), ctypes.byref(opt), out, _ptr(phases)))
        res = [{k: getattr(r, k) for k, _ in FineResult._fields_} for r in out]
        return res, phases

    def search_noncoherent(self, packed_bits, sampling_freq, constellation, prns=None, ants=None,
                           center_freq=GPS_IF, bin_step_hz=500.0, n_bins=21, coherent_periods=1, blocks=10, start=0):
        """Non-coherent search: record array of NC_CELL_DTYPE in (PRN, antenna) order."""
        bits = np.ascontiguousarray(packed_bits, dtype=np.uint8)
        pr = None if prns is None else np.ascontiguousarray(prns, dtype=np.int32)
        an = None if ants is None else np.ascontiguousarray(ants, dtype=np.int32)
        i32p = ctypes.POINTER(ctypes.c_int32)
        o = NcOptions(int(constellation), None if pr is None else pr.ctypes.data_as(i32p), 0 if pr is None else len(pr),
                      None if an is None else an.ctypes.data_as(i32p), 0 if an is None else len(an),
                      float(center_freq), float(bin_step_hz), int(n_bins), int(coherent_periods), int(blocks),
                      int(start))
        n = ctypes.c_size_t()
        self._check(lib().tga_search_noncoherent(self._h, _ptr(bits), bits.shape[0], bits.shape[1],
                                                 float(sampling_freq), ctypes.byref(o), None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=NC_CELL_DTYPE)
        self._check(lib().tga_search_noncoherent(self._h, _ptr(bits), bits.shape[0], bits.shape[1],
                                                 float(sampling_freq), ctypes.byref(o), _ptr(out), len(out),
                                                 ctypes.byref(n)))
        return out

    def search_noncoherent_multi(self, packed_bits, sampling_freq, searches):
        """Several non-coherent searches of one recording in one call
        (tga_search_noncoherent_multi).  searches: list of dicts with the
        keyword arguments of search_noncoherent plus `constellation`.  Returns
        one record array per search, in order."""
        bits = np.ascontiguousarray(packed_bits, dtype=np.uint8)
        i32p = ctypes.POINTER(ctypes.c_int32)
        keep, opts = [], (NcOptions * len(searches))()
        for i, sd in enumerate(searches):
            pr = sd.get("prns")
            an = sd.get("ants")
            pr = None if pr is None else np.ascontiguousarray(pr, dtype=np.int32)
            an = None if an is None else np.ascontiguousarray(an, dtype=np.int32)
            keep += [pr, an]
            opts[i] = NcOptions(int(sd["constellation"]), None if pr is None else pr.ctypes.data_as(i32p),
                                0 if pr is None else len(pr), None if an is None else an.ctypes.data_as(i32p),
                                0 if an is None else len(an), float(sd.get("center_freq", GPS_IF)),
                                float(sd.get("bin_step_hz", 500.0)), int(sd.get("n_bins", 21)),
                                int(sd.get("coherent_periods", 1)), int(sd.get("blocks", 10)), int(sd.get("start", 0)))
        n = ctypes.c_size_t()
        self._check(lib().tga_search_noncoherent_multi(self._h, _ptr(bits), bits.shape[0], bits.shape[1],
                                                       float(sampling_freq), opts, len(searches), None, 0,
                                                       ctypes.byref(n)))
        out = np.zeros(n.value, dtype=NC_CELL_DTYPE)
        self._check(lib().tga_search_noncoherent_multi(self._h, _ptr(bits), bits.shape[0], bits.shape[1],
                                                       float(sampling_freq), opts, len(searches), _ptr(out), len(out),
                                                       ctypes.byref(n)))
        del keep
        res, k = [], 0
        for sd in searches:
            n_ant = bits.shape[0] if sd.get("ants") is None else len(sd["ants"])
            n_prn = len(sd["prns"]) if sd.get("prns") is not None else PRN_RANGE[int(sd["constellation"])][1] - \
                PRN_RANGE[int(sd["constellation"])][0] + 1
            res.append(out[k:k + n_ant * n_prn])
            k += n_ant * n_prn
        return res

    def acr_table(self, constellation, prn=1, sampling_freq=16.368e6, cn0_lo=33.0, cn0_hi=62.0, cn0_step=0.5,
                  trials=100):
        """gen_acr_tables Monte Carlo on the GPU: [n, 2] array of (r_A, C/N0)."""
        n = ctypes.c_size_t()
        self._check(lib().tga_acr_table(self._h, constellation, prn, float(sampling_freq), float(cn0_lo),
                                        float(cn0_hi), float(cn0_step), int(trials), None, 0, ctypes.byref(n)))
        out = np.zeros((n.value, 2))
        self._check(lib().tga_acr_table(self._h, constellation, prn, float(sampling_freq), float(cn0_lo),
                                        float(cn0_hi), float(cn0_step), int(trials), _ptr(out), n.value,
                                        ctypes.byref(n)))
        return out

    def rfi_scan(self, packed_bits, sampling_freq, as_json=False):
        """rfi::run on packed rows: list of dicts shaped like rfi.rs's RfiChannel
        (None where the reference has None), or the --rfi JSON text."""
        bits = np.ascontiguousarray(packed_bits, dtype=np.uint8)
        out = (RfiChannel * bits.shape[0])()
        self._check(lib().tga_rfi_scan(self._h, _ptr(bits), bits.shape[0], bits.shape[1], float(sampling_freq), out))
        if as_json:
            p = ctypes.c_char_p()
            self._check(lib().tga_rfi_json(out, len(out), ctypes.byref(p)))
            text = ctypes.string_at(p).decode()
            lib().tga_free(p)
            return text
        opt = lambda v: None if np.isnan(v) else float(v)
        return [dict(antenna=c.antenna, dead=bool(c.dead), acf_lag1=opt(c.acf_lag1), acf_lag3=opt(c.acf_lag3),
                     acf_lag16=opt(c.acf_lag16), period_samples=opt(c.period_samples),
                     lines=[dict(frequency=c.lines[k].frequency, excess_db=c.lines[k].excess_db)
                            for k in range(c.n_lines)]) for c in out]

    def correlation_matrix(self, packed_bits):
        bits = np.ascontiguousarray(packed_bits, dtype=np.uint8)
        out = np.zeros((bits.shape[0], bits.shape[0]))
        self._check(lib().tga_antenna_xcorr_matrix(self._h, _ptr(bits), bits.shape[0], bits.shape[1], _ptr(out)))
        return out
