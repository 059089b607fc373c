// Narrowband RFI scan per antenna (tart-gnss-acquire --rfi, rfi.rs:91-168).
//
// For every antenna row of packed bits:
//   * z = (+-1 samples) - mean over the whole row (rfi.rs:145-147);
//   * its spectrum in f64 (rfi.rs:100-106: FFT of the whole record, powers of
//     the first n/2 bins), with this library's own f64 FFT (fft64.cu) over
//     all antennas at once;
//   * the median bin power, exactly: a radix select over the bit patterns of
//     the non-negative powers (8 passes of 8 bits), no sorting;
//   * local maxima p[k] > p[k-1], p[k] >= p[k+1] with 10 log10(p / floor) >
//     15 dB (rfi.rs:113-123), appended to a per-antenna list that the host
//     clusters (10 kHz, strongest first, at most 3 lines; rfi.rs:125-139);
//   * the autocorrelation at lags 1, 3 and 16 (rfi.rs:84-87) exactly from
//     popcounts: sum z_i z_{i+L} = sum s s' - m (sum s_head + sum s_tail)
//     + (n - L) m^2 with sum s s' = (n - L) - 2 popcount(b_i xor b_{i+L}).
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "engine.h"

namespace tga {

namespace {

__global__ void rfi_prepare_kernel(const uint8_t* __restrict__ bits, size_t row_bytes, const double* __restrict__ mean,
                                   long long n, double* __restrict__ z) {
  const int a = blockIdx.y;
  const uint8_t* row = bits + (size_t)a * row_bytes;
  const double m = mean[a];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int bit = (__ldg(row + (i >> 3)) >> (7 - (int)(i & 7))) & 1;
    z[(size_t)a * n + i] = (bit ? 1.0 : -1.0) - m;
  }
}

// one radix-select pass: histogram of the 8-bit digit at `shift` over the
// elements whose higher digits equal the prefix found so far
__global__ void rfi_hist_kernel(const double* __restrict__ p, long long half, int shift,
                                const unsigned long long* __restrict__ prefix, unsigned* __restrict__ hist) {
  __shared__ unsigned sh[256];
  const int a = blockIdx.y;
  for (int i = threadIdx.x; i < 256; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const unsigned long long mask = shift >= 56 ? 0ull : (~0ull << (shift + 8));
  const unsigned long long pre = prefix[a] & mask;
  const double* row = p + (size_t)a * half;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < half; k += (long long)gridDim.x * blockDim.x) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(row[k]);
    if ((u & mask) == pre) atomicAdd(&sh[(u >> shift) & 255u], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[(size_t)a * 256 + i], sh[i]);
}

// picks the digit holding rank[a], narrows the prefix and the rank, clears
// the histogram for the next pass (one thread per antenna)
__global__ void rfi_select_kernel(int n_ant, int shift, unsigned* __restrict__ hist,
                                  unsigned long long* __restrict__ prefix, unsigned long long* __restrict__ rank) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n_ant) return;
  unsigned* h = hist + (size_t)a * 256;
  unsigned long long r = rank[a], cum = 0;
  int d = 255;
  for (int i = 0; i < 256; ++i) {
    if (cum + h[i] > r) {
      d = i;
      break;
    }
    cum += h[i];
  }
  for (int i = 0; i < 256; ++i) h[i] = 0;
  prefix[a] |= (unsigned long long)d << shift;
  rank[a] = r - cum;
}

__global__ void rfi_peaks_kernel(const double* __restrict__ p, long long half, const unsigned long long* __restrict__ floor_bits,
                                 double min_excess_db, int cap, unsigned* __restrict__ count,
                                 long long* __restrict__ bins, double* __restrict__ excess) {
  const int a = blockIdx.y;
  const double* row = p + (size_t)a * half;
  const double fl = __longlong_as_double((long long)floor_bits[a]);
  for (long long k = 1 + (long long)blockIdx.x * blockDim.x + threadIdx.x; k < half - 1;
       k += (long long)gridDim.x * blockDim.x) {
    const double v = row[k];
    if (v > row[k - 1] && v >= row[k + 1]) {
      const double ex = 10.0 * log10(v / fl);
      if (ex > min_excess_db) {
        const unsigned idx = atomicAdd(&count[a], 1u);
        if (idx < (unsigned)cap) {
          bins[(size_t)a * cap + idx] = k;
          excess[(size_t)a * cap + idx] = ex;
        }
      }
    }
  }
}

__device__ __forceinline__ unsigned long long be_word(const uint8_t* row, size_t row_bytes, long long w) {
  unsigned long long v = 0;
  const long long b0 = w * 8;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const long long b = b0 + i;
    v = (v << 8) | (b < (long long)row_bytes ? (unsigned long long)__ldg(row + b) : 0ull);
  }
  return v;
}

// per antenna and lag L in {1, 3, 16}: popcounts of b_i xor b_{i+L}, of b_i
// and of b_{i+L} over i < n - L (big-endian words: sample 64 w + j is bit 63 - j)
__global__ void rfi_acf_kernel(const uint8_t* __restrict__ bits, size_t row_bytes, long long n,
                               unsigned long long* __restrict__ out /* [a][3][3] */) {
  const int a = blockIdx.y;
  const uint8_t* row = bits + (size_t)a * row_bytes;
  const long long words = (n + 63) / 64;
  const int lags[3] = {1, 3, 16};
  unsigned long long acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += (long long)gridDim.x * blockDim.x) {
    const unsigned long long cur = be_word(row, row_bytes, w), nxt = be_word(row, row_bytes, w + 1);
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      const int L = lags[l];
      const unsigned long long sh = (cur << L) | (nxt >> (64 - L));
      const long long vb = n - L - 64 * w;  // valid positions in this word
      const unsigned long long mask = vb >= 64 ? ~0ull : (vb <= 0 ? 0ull : (~0ull << (64 - vb)));
      acc[3 * l] += __popcll((cur ^ sh) & mask);
      acc[3 * l + 1] += __popcll(cur & mask);
      acc[3 * l + 2] += __popcll(sh & mask);
    }
  }
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    unsigned long long v = acc[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(out + (size_t)a * 9 + j, v);
  }
}

}  // namespace

cudaError_t rfi_scan_device(const uint8_t* d_bits, int n_ant, size_t row_bytes, const double* d_mean, double* d_z,
                            void* d_X, void* d_work, double* d_p, unsigned* d_hist, unsigned long long* d_prefix,
                            unsigned long long* d_rank, int cap, unsigned* d_count, long long* d_bins,
                            double* d_excess, unsigned long long* d_acf, int num_sms, cudaStream_t st,
                            std::string* why) {
  const long long n = (long long)row_bytes * 8, half = n / 2;
  if (n_ant <= 0 || n < 8) return cudaSuccess;
  cudaError_t e;
  dim3 g1(256, n_ant);
  rfi_prepare_kernel<<<g1, 256, 0, st>>>(d_bits, row_bytes, d_mean, n, d_z);
  kernel_launch_add(1);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // powers of the first n/2 bins of every antenna's f64 spectrum
  if ((e = real_power_spectrum(d_z, d_X, d_work, n, n_ant, d_p, num_sms, st, why)) != cudaSuccess) return e;
  // median bin power: rank half / 2 (rfi.rs:110-111)
  if ((e = cudaMemsetAsync(d_hist, 0, (size_t)n_ant * 256 * sizeof(unsigned), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(d_prefix, 0, (size_t)n_ant * sizeof(unsigned long long), st)) != cudaSuccess) return e;
  {
    const unsigned long long r = (unsigned long long)(half / 2);
    std::vector<unsigned long long> rk((size_t)n_ant, r);
    if ((e = cudaMemcpyAsync(d_rank, rk.data(), rk.size() * sizeof(r), cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return e;
    for (int shift = 56; shift >= 0; shift -= 8) {
      rfi_hist_kernel<<<g1, 256, 0, st>>>(d_p, half, shift, d_prefix, d_hist);
      rfi_select_kernel<<<(n_ant + 63) / 64, 64, 0, st>>>(n_ant, shift, d_hist, d_prefix, d_rank);
      kernel_launch_add(2);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;  // rk is a host temporary
  }
  if ((e = cudaMemsetAsync(d_count, 0, (size_t)n_ant * sizeof(unsigned), st)) != cudaSuccess) return e;
  rfi_peaks_kernel<<<g1, 256, 0, st>>>(d_p, half, d_prefix, 15.0, cap, d_count, d_bins, d_excess);
  kernel_launch_add(1);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(d_acf, 0, (size_t)n_ant * 9 * sizeof(unsigned long long), st)) != cudaSuccess) return e;
  rfi_acf_kernel<<<dim3(64, n_ant), 256, 0, st>>>(d_bits, row_bytes, n, d_acf);
  kernel_launch_add(1);
  return cudaGetLastError();
}

}  // namespace tga
