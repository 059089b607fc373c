// Internal interface between the host orchestration (tga_api.cpp) and the
// CUDA kernels (acq_kernels.cu).  Plain C++ types only.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace tga {

constexpr int kMaxPulse = 64;  // samples per chip supported by the fused path
constexpr int kMaxBins = 4096;

// One polyphase class of the fused path: period P = S * Lc samples, a code
// that is a chip sequence of length Lc held for S samples per chip and
// shaped by pulse[0..S) (all +1, or the BOC(1,1) +1/-1 halves).
struct PolyClass {
  int P = 0, S = 0, Lc = 0, M = 0;  // M = Lc / 1023
  float pulse[kMaxPulse] = {};
  // launch shape of the FP32 correlation kernels (0 = default, 1 = twice the
  // polyphase branches per CTA at one CTA per SM); results do not depend on it
  int variant = 0;
};

// Sample source of the front end.
struct SampleSource {
  // bits mode: packed MSB-first rows, antenna mean in d_mean (f64)
  const uint8_t* bits = nullptr;
  size_t row_bytes = 0;
  const double* mean = nullptr;
  // float mode (single-PRN API): de-meaned f32 samples and f64 phase points
  const float* sig = nullptr;
  const double* pp = nullptr;
  size_t n_samples = 0;
  // rows searched (antenna index into bits / mean / sig rows)
  const int32_t* ant = nullptr;
  int n_ant = 0;
  double pc = 0.0;  // TAU / fs, bits mode phase points pc * n
};

// One fine-acquisition evaluation: a (sub)chip sequence of seq_len entries,
// T samples each, at continuous delay tau (samples) and carrier frequency
// f_over_fs (cycles per sample), over samples [start, start + length) with
// the carrier phase referred to sample n0; chip edges smoothed by a Gaussian
// of sigma samples.  Sums land in out[slot][antenna][12].
struct FineTask {
  const int8_t* seq;
  int seq_len;
  int slot;
  double T, tau, f_over_fs, two_pi_over_fs, n0, sigma;
  long long start, length;
};

struct SearchDims {
  int n_ant = 0, nb = 0, n_prn = 0;
  const double* fc = nullptr;  // device Doppler grid [nb]
};

// Per-(antenna, PRN) best row after the bin / hypothesis reduction.
struct BestRow {
  int32_t ab;      // antenna_slot * nb + bin
  int32_t hyp;     // 0 [c,c], 1 [c,-c]
  int32_t tau;     // lag in samples, [0, P)
  float p;         // |y|^2 at the peak
  float p2;        // second peak |y|^2 (second-peak pass, or the re-evaluated rows); 0 when none
};

// Finalised cell (device side); host converts to tga_cell.
struct CellOut {
  double strength, second, codephase_frac, frequency, cn0;
  int32_t bin, tau, hyp, cn0_valid;
};

// Launchers; all asynchronous on `st`.  Return the launch error.
cudaError_t launch_antenna_means(const uint8_t* d_bits, int n_rows, size_t row_bytes,
                                 double* d_mean, cudaStream_t st);
cudaError_t launch_frontend(const SampleSource& src, const SearchDims& dims, const PolyClass& pc,
                            float2* d_z, cudaStream_t st);
cudaError_t launch_forward_z(const PolyClass& pc, int n_ab, float2* d_z, int num_sms, cudaStream_t st);
// launch_forward_z that also writes the tensor-core FP16 operands of Z
// (launch_tc_pack's layout and scale, tc_z_scale) from shared memory
cudaError_t launch_forward_z_tc(const PolyClass& pc, int n_ab, float2* d_z, void* d_z16, const void* d_map,
                                float z16_scale, int num_sms, cudaStream_t st);
// d_map of launch_forward_z_tc for chip count 1023 M: per FP16 unit four
// 16-bit offsets into the transformed sequence (0xffff: zero), host-built
std::vector<uint16_t> tc_unit_map(int M);
// launch_forward_seqs that also writes the tensor-core FP16 operands
cudaError_t launch_forward_seqs_tc(const PolyClass& pc, long long n_seq, float2* d_z, void* d_z16, const void* d_map,
                                   float z16_scale, int num_sms, cudaStream_t st);
// FP16 scale of Z in the tensor-core operands
float tc_z_scale(const PolyClass& pc);
// |y| of a tensor-core key's row maximum is sqrt(key) x tc_key_amplitude
double tc_key_amplitude(const PolyClass& pc);
// forward transform of n_seq Lc-point sequences in place (any count)
cudaError_t launch_forward_seqs(const PolyClass& pc, long long n_seq, float2* d_z, int num_sms, cudaStream_t st);
cudaError_t launch_code_spectra(const PolyClass& pc, const int8_t* d_chips, int n_prn, float2* d_D,
                                int num_sms, cudaStream_t st);
cudaError_t launch_correlate(const PolyClass& pc, const SearchDims& dims, const float2* d_Z,
                             const float2* d_D, unsigned long long* d_keys, int num_sms,
                             cudaStream_t st);
// launch_correlate over the rows listed in d_cand (*d_count of them, at
// most capacity): each listed row's FP32 key is written where
// launch_correlate would write it; other keys are left as they are.  With
// d_p2rows, each listed row's second peak against its own maximum (what
// launch_second_peak computes for a chosen row) is written there as well.
cudaError_t launch_correlate_listed(const PolyClass& pc, const SearchDims& dims, const float2* d_Z,
                                    const float2* d_D, const int2* d_cand, const int* d_count, int capacity,
                                    unsigned long long* d_keys, int num_sms, cudaStream_t st,
                                    float* d_p2rows = nullptr, int chip_width = 0);
// d_best[w].p2 = d_p2rows at the row d_best[w] chose (the keys' layout:
// [ab][hyp][prn] with n_hyp hypotheses, 2 for the drop-in search, 1 for the
// non-coherent one).
cudaError_t launch_second_from_rows(const SearchDims& dims, int n_hyp, const float* d_p2rows, BestRow* d_best,
                                    cudaStream_t st);
// Lists, per (antenna, PRN), the rows whose reduced-precision key is at least
// keep x the largest of its nb * n_hyp rows (appended to d_cand, counted in
// *d_count, which must start at 0; d_cand holds up to n_ant * nb * n_hyp *
// n_prn rows).  Keys are [ant][bin][hyp][prn].
cudaError_t launch_tc_candidates(const SearchDims& dims, int n_hyp, const unsigned long long* d_keys, float keep,
                                 int2* d_cand, int* d_count, cudaStream_t st);
// Tensor-core search: FP16 operands in the (31, R2, R3) frequency layout
// (launch_tc_pack of Z and of the code spectra), then the three-stage tcgen05
// correlator (FP32 accumulation in TMEM).  Keys hold |y|^2 scaled by 2^-2k
// (comparisons only) and must be zeroed before the launch; *d_err is set
// non-zero when a bounded wait on the tensor cores expired.
size_t tc_operand_bytes(const PolyClass& pc, long long n_seq, bool code);
// the three inverse-DFT matrices of class M in the correlator's shared-memory
// layouts (FP16), to be uploaded once and passed as d_bmat
std::vector<unsigned char> tc_dft_matrices(int M);
cudaError_t launch_tc_pack(const PolyClass& pc, const float2* d_src, long long n_seq, bool code, void* d_dst,
                           int num_sms, cudaStream_t st);
// test_flags bit 0: skip the first MMA batch and its commit (test hook for
// the bounded-wait failure path; 0 in normal use)
cudaError_t launch_correlate_tc(const PolyClass& pc, const SearchDims& dims, const void* d_bmat, const void* d_z16,
                                const void* d_d16, unsigned long long* d_keys, int* d_err, int test_flags,
                                int num_sms, cudaStream_t st);
// the non-coherent search (Lc = 1023): per (antenna, bin) row and PRN the
// row maximum of |y|^2 summed over B coherent blocks; z16 holds the FP16 Z of
// [n_ant * nb][B][S] sequences
cudaError_t launch_correlate_tc_nc(const PolyClass& pc, const SearchDims& dims, int B, const void* d_bmat,
                                   const void* d_z16, const void* d_d16, unsigned long long* d_keys, int* d_err,
                                   int test_flags, int num_sms, cudaStream_t st);
cudaError_t launch_reduce_bins(const SearchDims& dims, const unsigned long long* d_keys,
                               BestRow* d_best, cudaStream_t st);
cudaError_t launch_second_peak(const PolyClass& pc, const SearchDims& dims, const float2* d_Z,
                               const float2* d_D, BestRow* d_best, int chip_width, int num_sms,
                               cudaStream_t st);
// d_tables: ACR table id (TGA_ACR_*) per PRN of the group.
cudaError_t launch_finalize(const PolyClass& pc, const SearchDims& dims, const BestRow* d_best,
                            double center_freq, const int8_t* d_tables, int want_cn0, CellOut* d_out,
                            cudaStream_t st);
cudaError_t launch_acr_batch(const double* d_ra, int n, int table, double* d_cn0, uint8_t* d_valid,
                             cudaStream_t st);
cudaError_t launch_xcorr_matrix(const uint8_t* d_bits, int n_ant, size_t row_bytes,
                                unsigned long long* d_counts, cudaStream_t st);

// Generic path (any length N): reference algorithm with Bluestein FFTs.
struct GenericPlan {
  int N = 0;        // signal length
  int Mpow2 = 0;    // Bluestein length (power of two >= 2N-1)
  int log2M = 0;
};
cudaError_t launch_generic(const GenericPlan& gp, const float* d_sig, const double* d_pp,
                           const double* d_fc, int nb, const float* d_code_a,
                           const float* d_code_b, int period, double fs, float2* d_work,
                           size_t work_elems, float* d_corr, int* d_result_i, float* d_result_f,
                           cudaStream_t st);
size_t generic_work_elems(const GenericPlan& gp, int nb);
cudaError_t launch_bits_to_signal(const uint8_t* d_bits, size_t row_bytes, int row, const double* d_mean, int n,
                                  double pc, float* d_sig, double* d_pp, cudaStream_t st);

// fine acquisition: per (task, antenna) the complex sums R, dR/dtau, dR/df,
// d2R/dtau2, d2R/df2, d2R/dtau df (un-normalised), zeroed and accumulated
cudaError_t launch_fine_sums(const uint8_t* d_bits, int n_ant, size_t row_bytes, const double* d_mean,
                             const FineTask* d_tasks, int n_tasks, long long max_length, double* d_out,
                             cudaStream_t st);

// narrowband RFI scan of every antenna row (rfi.rs:91-168): f64 spectrum,
// exact median bin power, local maxima above 15 dB (up to cap per antenna,
// d_count counts all), exact autocorrelation popcounts at lags 1, 3, 16
cudaError_t rfi_scan_device(const uint8_t* d_bits, int n_ant, size_t row_bytes, const double* d_mean, double* d_z,
                            void* d_X, void* d_work, double* d_p, unsigned* d_hist, unsigned long long* d_prefix,
                            unsigned long long* d_rank, int cap, unsigned* d_count, long long* d_bins,
                            double* d_excess, unsigned long long* d_acf, int num_sms, cudaStream_t st,
                            std::string* why);

// f64 spectrum of `batch` real records of n samples (n even) held as doubles
// in d_x (overwritten): p[a][k] = |X_a[k]|^2 for k < n / 2.  d_buf holds
// batch * n / 2 complex doubles, d_work fft64_workspace_bytes(n, batch).
size_t fft64_workspace_bytes(long long n, int batch);
cudaError_t real_power_spectrum(double* d_x, void* d_buf, void* d_work, long long n, int batch, double* d_p,
                                int num_sms, cudaStream_t st, std::string* why);

// ACR Monte Carlo synthesizer (examples/gen_acr_tables.rs): n_points x
// n_trials rows of 2 * period one-bit samples, packed MSB-first
cudaError_t launch_acr_synth(const int8_t* d_code, int period, int n_trials, double cn0_lo, double cn0_step,
                             int n_points, double fs, double f_carrier, uint8_t* d_bits, cudaStream_t st);

// non-coherent search: K-period cyclic blocks, |y|^2 summed over B blocks
cudaError_t launch_nc_frontend(const SampleSource& src, const SearchDims& dims, const PolyClass& pc, int K, int B,
                               long long start, float2* d_z, cudaStream_t st);
cudaError_t launch_nc_correlate(const PolyClass& pc, const SearchDims& dims, int B, const float2* d_z,
                                const float2* d_D, unsigned long long* d_keys, int num_sms, cudaStream_t st);
cudaError_t launch_nc_reduce(const SearchDims& dims, const unsigned long long* d_keys, BestRow* d_best,
                             cudaStream_t st);
// launch_nc_correlate over the (ab, prn) rows listed in d_cand (*d_count of
// them, at most capacity), as the FP32 re-evaluation of a reduced-precision
// search's candidates: each listed row's key is written where
// launch_nc_correlate would write it; with d_p2rows, also each listed row's
// second peak against its own maximum (what launch_nc_second computes for a
// chosen row)
cudaError_t launch_nc_correlate_listed(const PolyClass& pc, const SearchDims& dims, int B, const float2* d_z,
                                       const float2* d_D, const int2* d_cand, const int* d_count, int capacity,
                                       unsigned long long* d_keys, int num_sms, cudaStream_t st,
                                       float* d_p2rows = nullptr, int chip_width = 0);
cudaError_t launch_nc_second(const PolyClass& pc, const SearchDims& dims, int B, const float2* d_z,
                             const float2* d_D, BestRow* d_best, int chip_width, int num_sms, cudaStream_t st);

int kernel_launch_count_reset();
void kernel_launch_add(int n);
int kernel_launch_count();

}  // namespace tga
