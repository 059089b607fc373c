/*
 * tga.h -- C ABI of the B200 acquisition engine (libtga.so).
 *
 * Drop-in replacement for the parallel code-phase / Doppler acquisition
 * search of tart-gnss-acquire v0.4.0 (tmolteno/tart-gnss).  The reference is
 * a Rust crate with no FFI; every entry point below names the Rust function
 * it replaces (file:line in the reference crate) so that a thin Rust
 * `extern "C"` shim can bind it.
 *
 * Conventions
 *  - Every function returns an int status (TGA_OK == 0).  Nothing aborts the
 *    process; on failure tga_last_error() describes the problem.
 *  - All buffers are caller-allocated.  Pointers named h_* are host memory,
 *    d_* are device memory on the context's GPU.
 *  - A context owns one CUDA stream, device scratch buffers and captured
 *    graphs.  A context is not thread-safe: use one context per host thread
 *    (contexts on the same device may coexist).
 *  - Results follow the reference semantics exactly: dual hypothesis
 *    ([c,c] and [c,-c]) over two code periods, 300 Hz Doppler bins over
 *    +-search_band, last-maximum tie rule over bins, strict ">" between
 *    hypotheses, second peak > 1 chip away from the main peak.
 */
#ifndef TGA_H
#define TGA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define TGA_OK 0
#define TGA_ERR_INVALID_ARG 1   /* bad size, PRN out of range, empty grid ... */
#define TGA_ERR_CUDA 2          /* a CUDA runtime call failed                  */
#define TGA_ERR_NO_DEVICE 3     /* no usable sm_100 device                      */
#define TGA_ERR_OUT_OF_MEMORY 4
#define TGA_ERR_UNSUPPORTED 5
#define TGA_ERR_TIMEOUT 6       /* host watchdog expired waiting for the GPU    */
#define TGA_ERR_CAPACITY 7      /* caller's output buffer is too small          */

/* ---- constellations (order and names of CombinedOutput, lib.rs:32-45) ---- */
#define TGA_GPS 0      /* GPS L1 C/A, PRN 1-38     (acquisition.rs)  */
#define TGA_GALILEO 1  /* Galileo E1-C, PRN 1-50   (galileo.rs)      */
#define TGA_BEIDOU 2   /* BeiDou B1C pilot, 1-63   (beidou.rs)       */
#define TGA_SBAS 3     /* SBAS L1 C/A, PRN 120-158 (sbas.rs)         */
#define TGA_L1C 4      /* GPS L1C pilot, PRN 1-63  (l1c.rs)          */
#define TGA_QZSS 5     /* QZSS L1 C/A, PRN 184-206 (qzss.rs)         */
#define TGA_N_CONSTELLATIONS 6
#define TGA_ALL_CONSTELLATIONS 0x3Fu

/* ---- ACR tables (acr_tables.rs) ------------------------------------------ */
#define TGA_ACR_GPS_L1_CA 0  /* GPS / SBAS / QZSS C/A, 2 ms */
#define TGA_ACR_GALILEO_E1C 1
#define TGA_ACR_BEIDOU_B1C 2
#define TGA_ACR_GPS_L1C 3

typedef struct tga_ctx tga_ctx;

/* Single-antenna, single-PRN result.  Mirrors AcquisitionResult
 * (acquisition.rs:18-30) and its per-constellation twins, plus the raw
 * CorrelationPeak fields (correlate.rs:28-38). */
typedef struct {
  int32_t prn;
  int32_t best_freq_idx;      /* CorrelationPeak.best_freq_idx                */
  int64_t best_codephase;     /* sample index of the peak, in [0, period)     */
  double signal_strength;     /* CorrelationPeak.best_peak as f64             */
  double second_peak;         /* CorrelationPeak.second_peak as f64           */
  double codephase_frac;      /* (best_codephase % period) / period           */
  double frequency;           /* fc[best_freq_idx] - center_freq (Hz)         */
  int32_t hypothesis;         /* 0: [c,c] won, 1: [c,-c] won                  */
  int32_t path;               /* 0: fused polyphase kernels, 1: generic path  */
} tga_result;

/* One (constellation, antenna, PRN) cell of an all-PRN search.  The per-PRN
 * vectors of *PrnResult (acquisition.rs:32-59) are these cells grouped by
 * (constellation, prn) in antenna order. */
typedef struct {
  int32_t constellation;
  int32_t prn;
  int32_t antenna;
  int32_t best_freq_idx;
  int64_t best_codephase;
  double signal_strength;
  double second_peak;
  double codephase_frac;
  double frequency;
  double cn0_acr;             /* valid only when cn0_valid != 0                */
  int32_t cn0_valid;          /* 0 mirrors the `null` entries of cn0_acr      */
  int32_t hypothesis;
} tga_cell;

/* Options of an all-PRN search: the arguments of acquire_all_* (for example
 * acquisition.rs:261-269) shared by all selected constellations. */
typedef struct {
  uint32_t constellation_mask;  /* bit TGA_x selects constellation x          */
  const int32_t* ant_filter;    /* NULL: every antenna (ant_filter == None)   */
  size_t n_ant_filter;
  const int32_t* prn_filter;    /* NULL: every PRN of each constellation      */
  size_t n_prn_filter;
  double center_freq;           /* reference CLI passes 4.092e6 for all six   */
  double search_band;           /* reference CLI passes 6000.0 for all six    */
  int32_t cn0;                  /* estimate ACR C/N0 per antenna (--cn0)      */
  int32_t debug;                /* per-PRN stderr lines (--debug)             */
} tga_all_options;

/* ---- context ------------------------------------------------------------- */
/* Replaces nothing in the reference (its state is a thread-local FftPlanner,
 * acquisition.rs:201-212, and LazyLock code caches, beidou_codes.rs:89-98). */
int tga_create(int device, tga_ctx** out);
int tga_destroy(tga_ctx* ctx);
const char* tga_last_error(const tga_ctx* ctx);
const char* tga_version(void);

/* ---- single-PRN search ----------------------------------------------------
 * Replaces acquire_full (acquisition.rs:176), acquire_sbas (sbas.rs:132),
 * acquire_qzss (qzss.rs:135), acquire_galileo_single (galileo.rs:133),
 * acquire_beidou_single (beidou.rs:85) and acquire_l1c_single (l1c.rs:94):
 * same arguments (host slices of de-meaned f32 samples and f64 phase
 * points), same AcquisitionResult.  When num_samples == 2 * samples_per_chunk
 * and the resampled code is a whole number of samples per chip the fused
 * polyphase kernels run; any other length runs the generic GPU path
 * (Bluestein FFTs of length num_samples). */
int tga_acquire_single(tga_ctx* ctx, int constellation, const float* h_signal_f32,
                       const double* h_phasepoints, size_t num_samples, double sampling_freq,
                       double center_freq, double search_band, int prn,
                       size_t samples_per_chunk, tga_result* out);
int tga_acquire_full(tga_ctx* ctx, const float* h_signal_f32, const double* h_phasepoints,
                     size_t num_samples, double sampling_freq, double center_freq,
                     double search_band, int prn, size_t samples_per_chunk, tga_result* out);
int tga_acquire_sbas(tga_ctx* ctx, const float* h_signal_f32, const double* h_phasepoints,
                     size_t num_samples, double sampling_freq, double center_freq,
                     double search_band, int prn, size_t samples_per_chunk, tga_result* out);
int tga_acquire_qzss(tga_ctx* ctx, const float* h_signal_f32, const double* h_phasepoints,
                     size_t num_samples, double sampling_freq, double center_freq,
                     double search_band, int prn, size_t samples_per_chunk, tga_result* out);
int tga_acquire_galileo_single(tga_ctx* ctx, const float* h_signal_f32,
                               const double* h_phasepoints, size_t num_samples,
                               double sampling_freq, double center_freq, double search_band,
                               int prn, size_t samples_per_chunk, tga_result* out);
int tga_acquire_beidou_single(tga_ctx* ctx, const float* h_signal_f32,
                              const double* h_phasepoints, size_t num_samples,
                              double sampling_freq, double center_freq, double search_band,
                              int prn, size_t samples_per_chunk, tga_result* out);
int tga_acquire_l1c_single(tga_ctx* ctx, const float* h_signal_f32, const double* h_phasepoints,
                           size_t num_samples, double sampling_freq, double center_freq,
                           double search_band, int prn, size_t samples_per_chunk,
                           tga_result* out);

/* ---- single-PRN search without allocation ------------------------------------
 * Has no counterpart in the reference.  For callers that cannot call
 * cudaMalloc while they run: a real-time receiver loop (cudaMalloc can
 * synchronise the device and take unbounded time), a process whose device
 * memory is already held by another framework's caching allocator, or a
 * host that only allows memory reserved when the library was loaded.  Same
 * search and result as tga_acquire_single on the fused path, but inputs and
 * the result are DEVICE pointers (n samples, n phase points, one
 * tga_result) and the work is queued on `stream` (a cudaStream_t; NULL =
 * default stream) without synchronising.  It needs no context.
 *
 * Scratch comes from one fixed 16 MiB array in the library's device memory
 * (held on every GPU that loads the library until the process exits).  A
 * search fits when, with every term rounded up to a multiple of 256 bytes,
 *   n_bins * 2 * samples_per_chunk * 8  +  2 * chips * 8  +  n_bins * 16
 *   + n_bins * 8  +  (chips + 1)  +  about 800 bytes
 * is at most 16 MiB (chips = 1023, 4092 or 10230): for example GPS / SBAS /
 * QZSS at 16.368 MHz with up to 63 bins (the reference's +-6 kHz / 300 Hz
 * grid has 41), Galileo at 4.092 MHz, or BeiDou / L1C at 2.046 MHz.  Larger
 * searches return TGA_ERR_CAPACITY.  Only the fused polyphase search is
 * built in: a window of exactly two periods with a whole number of samples
 * per chip (samples_per_chunk a multiple of the chip count).  There is no
 * generic fallback, so inputs that tga_acquire_single serves through its
 * generic path (e.g. 16 MHz sampling) return TGA_ERR_UNSUPPORTED here.  The
 * first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and uploads constant tables: make it before any
 * stream capture.  Host threads may make their first calls at once (the
 * set-up is serialised).  Every call shares the array and leaves its
 * contents behind (each call writes every part it reads first); calls that
 * overlap on the GPU race on it, so serialise them. */
int tga_acquire_single_static(int constellation, const float* d_signal_f32,
                              const double* d_phasepoints, size_t num_samples,
                              double sampling_freq, double center_freq, double search_band,
                              int prn, size_t samples_per_chunk, tga_result* d_out, void* stream);

/* ---- all-PRN, all-antenna search ------------------------------------------
 * Replaces acquire_all_gps (acquisition.rs:261), acquire_all_sbas
 * (sbas.rs:216), acquire_all_qzss (qzss.rs:219), acquire_all_galileo
 * (galileo.rs:219), acquire_all_beidou (beidou.rs:171), acquire_all_l1c
 * (l1c.rs:180), and the per-constellation loop of main.rs:719-819.
 *
 * Input is the observation's packed 1-bit data exactly as stored in the
 * HDF5 `data` dataset (observation.rs:62-75): n_ant rows of row_bytes bytes,
 * MSB-first (numpy.packbits).  The antenna mean is taken over the whole row
 * (acquisition.rs:285); the search uses the first 2 code periods.
 *
 * out receives one tga_cell per (constellation, PRN, antenna), ordered by
 * constellation (TGA_x order), then PRN in the order searched (prn_filter
 * order, or ascending), then antenna (ant_filter order).  *n_out is set to
 * the count; TGA_ERR_CAPACITY if out_capacity is too small (then *n_out is
 * the required count).
 *
 * tga_acquire_all takes host bits and copies them to the device;
 * tga_acquire_all_device takes bits already resident on the context's GPU. */
int tga_acquire_all(tga_ctx* ctx, const uint8_t* h_packed_bits, size_t n_ant, size_t row_bytes,
                    double sampling_freq, const tga_all_options* opt, tga_cell* out,
                    size_t out_capacity, size_t* n_out);
/* A stream of observations: n_obs recordings of the same shape searched one
 * after the other with the same options, each exactly as tga_acquire_all
 * would search it (the cells of observation i at out + i * C, C the count
 * of tga_all_cell_count; *n_out = n_obs * C), while the host-to-device copy
 * of observation i + 1 runs on a second stream during the search of
 * observation i (two device buffers, alternated).  The host rows should be
 * pinned for the copies to overlap.  No counterpart in the reference: it
 * serves a receiver that acquires on a stream of recordings. */
int tga_acquire_all_stream(tga_ctx* ctx, const uint8_t* const* h_packed_bits, size_t n_obs, size_t n_ant,
                           size_t row_bytes, double sampling_freq, const tga_all_options* opt, tga_cell* out,
                           size_t out_capacity, size_t* n_out);
int tga_acquire_all_device(tga_ctx* ctx, const uint8_t* d_packed_bits, size_t n_ant,
                           size_t row_bytes, double sampling_freq, const tga_all_options* opt,
                           tga_cell* out, size_t out_capacity, size_t* n_out);

/* --benchmark (main.rs:482-694): for GPS, Galileo, BeiDou, SBAS, QZSS and
 * L1C in that order, one PRN (1, 1, 1, 120, 184, 1) on antenna 0 of the
 * observation.  setup_s = host extraction of every antenna's de-meaned f32
 * window and phasepoints (main.rs:497-517), search_s = the single-PRN
 * acquisition through tga_acquire_single (wall clock, result read back).
 * out receives 6 entries. */
typedef struct {
  int32_t constellation;
  int32_t prn;
  double setup_s;
  double search_s;
  tga_result result;
} tga_bench_entry;
int tga_benchmark(tga_ctx* ctx, const uint8_t* h_packed_bits, size_t n_ant, size_t row_bytes,
                  double sampling_freq, tga_bench_entry out[6]);

/* Number of cells tga_acquire_all would produce for these options. */
int tga_all_cell_count(size_t n_ant, const tga_all_options* opt, size_t* n_cells);

/* Search work of the last tga_acquire_all* call on this context:
 * cells = sum over (constellation, antenna, PRN) of n_bins * period, and the
 * kernels launched.  Used by benchmarks to report cells/s. */
int tga_last_search_stats(const tga_ctx* ctx, double* cells, int32_t* kernel_launches,
                          double* device_ms);
/* Host<->device bytes moved by the last call (inputs in, results out). */
int tga_last_transfer_bytes(const tga_ctx* ctx, uint64_t* h2d_bytes, uint64_t* d2h_bytes);
/* The CUDA stream (cudaStream_t) every kernel of this context runs on, so a
 * caller can time calls with CUDA events on it. */
void* tga_stream(tga_ctx* ctx);
/* Per-kernel device timing of later calls (CUDA events around each launch,
 * on the context stream).  tga_kernel_times returns, for the last call, up
 * to cap entries of (kernel name, total ms, launches, algorithmic FLOPs).
 * Algorithmic FLOPs count 5 N log2 N per complex FFT of N points, 6 per
 * complex product, 3 per |y|^2 and 10 per wiped-off sample, whatever the
 * kernel executes. */
int tga_set_profiling(tga_ctx* ctx, int enable);
/* Arithmetic of the correlation search.
 *  TGA_PRECISION_FP32 (default): every transform stage in FP32 on the CUDA
 *    cores; results within 1e-4 of the reference algorithm.
 *  TGA_PRECISION_FP16_TC: the inverse transforms of the search run on the
 *    tensor cores (tcgen05, FP16 operands, FP32 accumulation); the row chosen for
 *    every (antenna, PRN) is then re-evaluated in FP32, so reported peak, lag
 *    and second peak are FP32 values; only the choice of Doppler bin and
 *    hypothesis among near-equal candidates can differ from the FP32 mode. */
/* Test hooks (0 in normal use).  TGA_TEST_TC_SKIP_COMMIT: the tensor-core
 * correlator issues no MMA for its first batch, so its bounded wait (1 s)
 * expires with nothing in flight; the call then fails with TGA_ERR_TIMEOUT
 * and the context stays usable.  It exists to test that failure path. */
#define TGA_TEST_TC_SKIP_COMMIT 1
int tga_set_test_flags(tga_ctx* ctx, int flags);
#define TGA_PRECISION_FP32 0
#define TGA_PRECISION_FP16_TC 1
int tga_set_precision(tga_ctx* ctx, int precision);
/* Launch-shape variant of this context's FP32 correlation kernels, for its
 * current precision (each precision keeps its own), for chip
 * count lc (1023, 4092, 10230): 0 = default; 1 = twice the polyphase
 * branches per CTA (16, 4, 2) at one CTA per SM, sharing the code spectrum
 * in L1.  Results are identical; only speed varies.  (The tensor-core
 * search takes the variant in its FP32 re-evaluation of the selected row.) */
int tga_set_variant(tga_ctx* ctx, int lc, int variant);

/* One code length tuned by tga_autotune. */
typedef struct {
  int32_t lc;            /* chip count: 1023, 4092 or 10230 */
  int32_t variant;       /* the variant kept (now set on the context) */
  double ms[2];          /* median device time of the whole search per variant */
  int32_t same_results[2]; /* 1 if that variant's cells equal variant 0's */
} tga_tune_entry;

/* Autotuner of the launch shapes: runs the search tga_acquire_all_device
 * would run (packed bits on the device) once untimed and `reps` times timed
 * per candidate variant of each code length in the search, one length at a
 * time with the others fixed, and keeps on the context (for its current
 * precision) the fastest variant whose cells equal variant 0's.  The search's code lengths come out in
 * out[0..*n_out), ascending.  Graphs are off while it runs; later searches
 * build their graphs with the kept variants.  reps: 1-100. */
int tga_autotune(tga_ctx* ctx, const uint8_t* d_packed_bits, size_t n_ant, size_t row_bytes,
                 double sampling_freq, const tga_all_options* opt, int reps, tga_tune_entry out[3],
                 size_t* n_out);
/* CUDA graphs for tga_acquire_all / tga_acquire_all_device (enabled by
 * default).  A search plan (bits buffer, shapes, options, precision,
 * variant) runs eagerly on its first call, is captured into a CUDA graph on
 * its second and is replayed from that graph after that; a reallocation of
 * the context's buffers rebuilds it.  Results are the same either way.
 * Calls with profiling enabled, and plans with constellations on the
 * generic path, run eagerly.  No counterpart in the reference (a CPU
 * library); it serves the batched search's launch path. */
int tga_set_graphs(tga_ctx* ctx, int enable);
/* Row peaks of the last search call.  After tga_acquire_all*, for its fused
 * group of `chips`-chip codes (1023: GPS, SBAS, QZSS; 4092: Galileo; 10230:
 * BeiDou, L1C): out[((ant * n_bins + bin) * 2 + hyp) * n_prn + i] is the
 * largest |IFFT_2P| / sqrt(2P) of that (bin, hypothesis) row -- the
 * reference's signal_strength units.  After tga_search_noncoherent (chips =
 * its code length): out[(ant * n_bins + bin) * n_prn + i] is the row's
 * largest summed power in tga_nc_cell.power units.  Values are as the
 * search's own arithmetic computed them: the FP16 tensor-core row maxima in
 * TGA_PRECISION_FP16_TC, FP32 otherwise.  ant and i index the call's antenna
 * list and the group's PRNs (its constellations in mask order).  *n_out =
 * the row count; out may be NULL to query it (TGA_ERR_CAPACITY if cap is
 * smaller).  *n_rows_refined (may be NULL) = rows the tensor-core search
 * re-evaluated in FP32 (0 in FP32 mode).  No counterpart in the reference;
 * it serves the measurement of the reduced-precision keys' error. */
int tga_last_row_peaks(tga_ctx* ctx, int chips, double* out, size_t cap, size_t* n_out,
                       int64_t* n_rows_refined);
/* How the last tga_acquire_all* call ran: eagerly, captured then launched,
 * or replayed from a graph captured earlier. */
#define TGA_GRAPH_NONE 0
#define TGA_GRAPH_CAPTURED 1
#define TGA_GRAPH_REPLAYED 2
int tga_last_graph(const tga_ctx* ctx, int* state);
int tga_kernel_times(const tga_ctx* ctx, int cap, const char** names, double* ms,
                     int32_t* launches, double* flops, int* n);

/* ---- ACR C/N0 --------------------------------------------------------------
 * Replaces estimate_cn0 (acr.rs:49-84) over a batch, on the GPU:
 * cn0[i] = estimate_cn0(r_a[i], table), valid[i] = 0 where it returns None. */
int tga_acr_cn0(tga_ctx* ctx, const double* h_r_a, size_t n, int table, double* h_cn0,
                uint8_t* h_valid);

/* ---- antenna cross-correlation ---------------------------------------------
 * Replaces Observation::correlate (observation.rs:175-195): zero-lag mean of
 * the +-1 products of antennas i and j over the whole record, on the GPU. */
int tga_antenna_xcorr(tga_ctx* ctx, const uint8_t* h_packed_bits, size_t n_ant,
                      size_t row_bytes, int i, int j, double* out);
/* All n_ant x n_ant pairs at once (row-major out[i*n_ant + j]). */
int tga_antenna_xcorr_matrix(tga_ctx* ctx, const uint8_t* h_packed_bits, size_t n_ant,
                             size_t row_bytes, double* out);

/* ---- result aggregation and JSON (host) --------------------------------------
 * Groups the cells of tga_acquire_all into the reference's output structs
 * and serialises them as serde_json::to_string_pretty does for
 * CombinedOutput (lib.rs:32-45; per-PRN fields acquisition.rs:32-66, ACR
 * :341-357, median/MAD :365-377, sort by sv :393).  filter_phase_mad /
 * filter_freq_mad (NaN = off) drop results whose MAD exceeds the threshold,
 * like apply_mad_filters (main.rs:242-256); *n_filtered counts them.
 * *json is malloc'd: release it with tga_free. */
int tga_results_json(const tga_cell* cells, size_t n_cells, const int32_t* antenna_numbers,
                     size_t n_ant, uint32_t constellation_mask, int cn0, double filter_phase_mad,
                     double filter_freq_mad, char** json, size_t* n_filtered);
/* One f64 in the JSON number format above (shortest round-trip digits). */
int tga_format_f64(double v, char* out, size_t capacity);
void tga_free(void* p);

/* ---- observation files (host) -----------------------------------------------
 * Replaces Observation::from_hdf5 (observation.rs:48-92): reads the
 * `config` JSON (num_antenna, sampling_frequency; config.rs:10-19), the
 * `timestamp` string and the packed `data` rows of a TART HDF5 file.  The
 * bits stay packed (the kernels unpack in registers), unlike the reference
 * which expands them to one byte per sample (observation.rs:232-240). */
typedef struct {
  uint32_t num_antenna;
  double sampling_frequency;
  size_t row_bytes;          /* packed bytes per antenna row                  */
  char timestamp[64];
  char* config_json;         /* malloc'd; freed by tga_observation_free       */
  uint8_t* data;             /* malloc'd num_antenna * row_bytes packed bits  */
  char error[256];           /* message when the call fails                   */
} tga_observation;
int tga_observation_read_hdf5(const char* path, tga_observation* out);
void tga_observation_free(tga_observation* obs);

/* ---- code tables (host) -----------------------------------------------------
 * +-1 primary chips of one PRN: generate_ca_code (acquisition.rs:130),
 * generate_sbas_ca_code (sbas.rs:111), generate_qzss_ca_code (qzss.rs:111),
 * generate_e1c_code (galileo.rs:99), generate_b1c_pilot_code
 * (beidou_codes.rs:145, BOC(1,1) half-chips) and generate_l1c_pilot_code
 * (l1c_codes.rs:175, BOC(1,1) half-chips).  Returns the length in *n. */
int tga_code_chips(int constellation, int prn, int8_t* out, size_t capacity, size_t* n);
/* The code resampled to num_samples samples: gold_code (acquisition.rs:162),
 * sbas_gold_code, qzss_gold_code, e1c_code_resampled (galileo.rs:112),
 * b1c_code_resampled (beidou_codes.rs:166), l1c_code_resampled
 * (l1c_codes.rs:197). */
int tga_code_resampled(int constellation, int prn, double samples_per_code,
                       size_t num_samples, float* out);

/* ---- non-coherent search (weak-signal mode) ------------------------------------
 * An extension of the drop-in search (no reference counterpart; the crate
 * searches one two-period window): `blocks` consecutive coherent blocks of
 * `coherent_periods` code periods starting at sample `start`; each block is
 * wiped off by the exact carrier phase measured from its first sample (the
 * sign convention of correlate.rs:110-115), folded into one period and
 * correlated cyclically with the code; |y|^2 is summed over the blocks before
 * the peak search.  With TGA_PRECISION_FP16_TC and a 1023-chip code (GPS,
 * SBAS, QZSS C/A) the bins are chosen on the tensor cores and the selected
 * row of every (antenna, PRN) is re-evaluated in FP32; other codes run the
 * FP32 search in either precision.  Doppler bins are centred:
 * center_freq + (i - (n_bins - 1) / 2) * bin_step_hz.  Ties: the later lag
 * within a bin, the later bin across bins; second peak at a circular
 * distance of more than ceil(fs / 1.023 MHz) samples from the peak.  Needs an
 * integer number of samples per chip (TGA_ERR_UNSUPPORTED otherwise). */
typedef struct tga_nc_options {
  int32_t constellation;
  const int32_t* prn_filter;   /* NULL = every PRN of the constellation     */
  size_t n_prn_filter;
  const int32_t* ant_filter;   /* NULL = every antenna                      */
  size_t n_ant_filter;
  double center_freq;          /* Hz                                        */
  double bin_step_hz;
  int32_t n_bins;
  int32_t coherent_periods;
  int32_t blocks;
  int64_t start;               /* first sample                              */
} tga_nc_options;
typedef struct tga_nc_cell {
  int32_t prn;
  int32_t antenna;
  int32_t best_freq_idx;
  int32_t reserved;
  int64_t best_codephase;      /* samples, [0, period)                     */
  double power;                /* sum over blocks of (|r| sqrt(N))^2, N = samples per block */
  double second_power;
  double frequency;            /* bin frequency - center_freq (Hz)          */
} tga_nc_cell;
/* Cells in (PRN, antenna) order; cap counts cells. */
int tga_search_noncoherent(tga_ctx* ctx, const uint8_t* h_packed_bits, size_t n_ant, size_t row_bytes, double fs,
                           const tga_nc_options* opt, tga_nc_cell* out, size_t cap, size_t* n_out);
/* Several non-coherent searches of one recording in one call, e.g. every
 * constellation of an --all search with its own blocks and Doppler grid:
 * opts[i] as for tga_search_noncoherent; the cells of opts[0], then those
 * of opts[1], ..., each in (PRN, antenna) order.  Searches with the same
 * code length and pulse (GPS / SBAS / QZSS; BeiDou / L1C), blocks, Doppler
 * grid and antennas share one front end and forward transform.  No
 * counterpart in the reference (an extension, like tga_search_noncoherent). */
int tga_search_noncoherent_multi(tga_ctx* ctx, const uint8_t* h_packed_bits, size_t n_ant, size_t row_bytes,
                                 double fs, const tga_nc_options* opts, size_t n_opts, tga_nc_cell* out, size_t cap,
                                 size_t* n_out);

/* ---- ACR table Monte Carlo (examples/gen_acr_tables.rs) ---------------------------
 * Regenerates a C/N0 lookup table for one constellation: for every C/N0 from
 * cn0_lo to cn0_hi in cn0_step, `trials` two-code-period signals of `prn` at
 * fs on a 100 kHz carrier (random code delay and carrier phase, unit noise,
 * the reference generator's xorshift64 streams and seeds), one-bit
 * quantised on the GPU and searched with the batched acquisition (one bin at
 * 100 kHz); r_A = sum peak^2 / sum second^2, forced strictly increasing like
 * the reference.  out receives (r_A, C/N0) pairs; cap counts pairs. */
int tga_acr_table(tga_ctx* ctx, int constellation, int prn, double fs, double cn0_lo, double cn0_hi,
                  double cn0_step, int trials, double* out, size_t cap, size_t* n_out);

/* ---- narrowband RFI scan (--rfi) ----------------------------------------------
 * rfi::analyze_channel (rfi.rs:145-168) for every antenna row: spectral lines
 * at least 15 dB above the median bin power of the whole record (f64 FFT),
 * clustered within 10 kHz, strongest first, at most 3 (rfi.rs:91-140); the
 * implied period fs / f of the strongest; the autocorrelation at lags 1, 3,
 * 16 (rfi.rs:84-87).  Dead channels (variance < 1e-9) carry NaN fields and no
 * lines.  NaN stands for the reference's None. */
typedef struct tga_rfi_line {
  double frequency;          /* Hz */
  double excess_db;          /* dB above the median bin power */
} tga_rfi_line;
typedef struct tga_rfi_channel {
  int32_t antenna;
  int32_t dead;
  double acf_lag1, acf_lag3, acf_lag16;
  double period_samples;
  int32_t n_lines;
  tga_rfi_line lines[3];
} tga_rfi_channel;
int tga_rfi_scan(tga_ctx* ctx, const uint8_t* h_packed_bits, size_t n_ant, size_t row_bytes, double fs,
                 tga_rfi_channel* out);
/* RfiReport as serde_json::to_string_pretty writes it (main.rs:439-478);
 * *json is malloc'd, release with tga_free. */
int tga_rfi_json(const tga_rfi_channel* channels, size_t n, char** json);

/* ---- fine acquisition --------------------------------------------------------
 * Refines a grid estimate (the search's code phase and Doppler bin) of one
 * satellite by Newton iteration on the coherent multi-antenna power
 *
 *   P = | sum_a exp(-i phi_a) R_a(tau, f) |^2,
 *   R_a = (1/N) sum_n s_a[n] exp(+i 2 pi f (n - n0) / fs) c(n - tau),
 *
 * over a window of N samples (n0 its centre), with per-antenna carrier phases
 * phi_a, continuous code delay tau (samples; the search's best_codephase
 * convention) and carrier frequency f (Hz, absolute, like the search's
 * Doppler grid).  c is the code with Gaussian-smoothed (sub)chip edges (a
 * front-end filter model, edge_sigma_chips), which makes P smooth in tau.
 * The window must hold no data-bit or secondary-code transition.
 * Reference counterpart: optimize_fit (junk/acquisition.py:403-445), a scalar
 * frequency search and a Gaussian fit of three code-phase samples. */
typedef struct tga_fine_task {
  int32_t constellation;     /* TGA_GPS ... TGA_QZSS                          */
  int32_t prn;
  double code_phase;         /* start delay, samples                          */
  double frequency;          /* start carrier frequency, Hz                   */
  int64_t start;             /* window: samples [start, start + length)       */
  int64_t length;
} tga_fine_task;
typedef struct tga_fine_options {
  double edge_sigma_chips;   /* replica edge smoothing, chips (0 -> 0.1)      */
  double scan_half_width_hz; /* frequency pre-scan +- this around the start
                                (0 -> 150 Hz + 1/window; < 0 -> no scan)      */
  int32_t max_iter;          /* Newton evaluations (0 -> 20)                  */
  double tol_code_phase;     /* convergence, samples (0 -> 1e-4)              */
  double tol_frequency;      /* convergence, Hz (0 -> 1e-3)                   */
} tga_fine_options;
typedef struct tga_fine_result {
  double code_phase;         /* refined delay, samples                         */
  double frequency;          /* refined carrier frequency, Hz                  */
  double power;              /* P at the solution                              */
  double power_start;        /* P at the start point with aligned phases       */
  int32_t iterations;        /* Newton evaluations used                        */
  int32_t converged;         /* 1 when the last accepted step met the tolerances */
} tga_fine_result;
/* Refine n_tasks satellites on host packed bits [n_ant][row_bytes]; phases
 * (n_tasks * n_ant, may be NULL) receives the fitted carrier phases. */
int tga_fine_acquire(tga_ctx* ctx, const uint8_t* h_packed_bits, size_t n_ant, size_t row_bytes, double fs,
                     const tga_fine_task* tasks, size_t n_tasks, const tga_fine_options* opt,
                     tga_fine_result* out, double* phases);
/* P, its gradient and Hessian at one point, in the parameter order
 * (code_phase, frequency, phi_0 .. phi_{n_ant-1}): grad has 2 + n_ant
 * entries, hess (2 + n_ant)^2 (row-major); either may be NULL. */
int tga_fine_eval(tga_ctx* ctx, const uint8_t* h_packed_bits, size_t n_ant, size_t row_bytes, double fs,
                  const tga_fine_task* task, const double* phases, double edge_sigma_chips, double* power,
                  double* grad, double* hess);

#ifdef __cplusplus
}
#endif
#endif /* TGA_H */
