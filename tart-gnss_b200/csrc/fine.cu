// Fine acquisition: correlation of a band-limited code replica at a
// continuous code delay and carrier frequency, with its first and second
// derivatives, over many antennas in one pass.
//
// The reference's only precedent is optimize_fit (junk/acquisition.py:403-445),
// which refines the frequency by a scalar search and the code phase by a
// Gaussian fit to three correlation samples.  Here the refinement is a Newton
// iteration on the coherent multi-antenna power
//
//   P(tau, f, phi) = | sum_a exp(-i phi_a) R_a(tau, f) |^2,
//   R_a(tau, f)    = (1/N) sum_n s_a[n] exp(+i 2 pi f (n - n0) / fs) c(n - tau),
//
// s_a the de-meaned +-1 samples of antenna a (the reference's wipe-off sign
// convention, correlate.rs:110-115), c the code as a sequence of
// rectangular (sub)chips of T samples whose edges are smoothed by a Gaussian
// of standard deviation sigma samples (a front-end filter model; without it a
// fractional delay is not observable at an integer number of samples per
// chip).  The kernel returns, per (task, antenna), the six complex sums
//
//   R, dR/dtau, dR/df, d2R/dtau2, d2R/df2, d2R/dtau df
//
// from which the host forms P, its gradient with respect to (tau, f, phi_a)
// and its Hessian: the gradient of |S|^2 is the adjoint contraction
// 2 Re(conj(S) dS), which needs exactly these tangents of S.
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.h"

namespace tga {

namespace {

constexpr int kFineThreads = 256;
constexpr int kFineChunk = 1024;  // samples per block

// replica value and its first two derivatives at continuous time t (samples)
// from the four edges around t: c(t) = seq[k] + sum_m d_m (Phi(u_m) - [u_m >= 0])
__device__ __forceinline__ void replica(const int8_t* __restrict__ seq, int L, double T, double inv_sigma, double t,
                                        float& c, float& c1, float& c2) {
  const double q = t / T;
  const long long k = (long long)floor(q);
  const int kk = (int)(((k % L) + L) % L);
  c = (float)__ldg(seq + kk);
  c1 = 0.f;
  c2 = 0.f;
  const float is = (float)inv_sigma;
#pragma unroll
  for (int dm = -1; dm <= 2; ++dm) {
    const int m = kk + dm;
    const int mi = ((m % L) + L) % L, mp = ((m - 1) % L + L) % L;
    const float d = (float)(__ldg(seq + mi) - __ldg(seq + mp));  // jump at edge m
    if (d == 0.f) continue;
    const float u = (float)((t - (double)(k + dm) * T) * inv_sigma);
    const float pdf = 0.3989422804014327f * __expf(-0.5f * u * u);
    c += d * (normcdff(u) - (u >= 0.f ? 1.f : 0.f));
    c1 += d * pdf * is;
    c2 -= d * u * pdf * is * is;
  }
}

__global__ void __launch_bounds__(kFineThreads) fine_sums_kernel(const uint8_t* __restrict__ bits, int n_ant,
                                                                 size_t row_bytes, const double* __restrict__ mean,
                                                                 const FineTask* __restrict__ tasks,
                                                                 double* __restrict__ out) {
  __shared__ float s_w[7][kFineChunk];  // per sample: a0 (2), a1 (2), a2 (2), x
  const FineTask tk = tasks[blockIdx.y];
  const long long c0 = (long long)blockIdx.x * kFineChunk;
  if (c0 >= tk.length) return;
  const int cn = (int)min((long long)kFineChunk, tk.length - c0);
  const double inv_sigma = 1.0 / tk.sigma;
  for (int i = threadIdx.x; i < kFineChunk; i += kFineThreads) {
    float a[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (i < cn) {
      const long long n = tk.start + c0 + i;
      const double dn = (double)n - tk.n0;
      // carrier phase reduced in f64 before the single-precision sincos
      double cyc = tk.f_over_fs * dn;
      cyc -= floor(cyc);
      float sn, cs;
      sincospif((float)(2.0 * cyc), &sn, &cs);
      float c, c1, c2;
      replica(tk.seq, tk.seq_len, tk.T, inv_sigma, (double)n - tk.tau, c, c1, c2);
      a[0] = cs * c;
      a[1] = sn * c;
      a[2] = -cs * c1;  // d/dtau of c(n - tau) = -c'
      a[3] = -sn * c1;
      a[4] = cs * c2;
      a[5] = sn * c2;
      a[6] = (float)(dn * tk.two_pi_over_fs);
    }
#pragma unroll
    for (int j = 0; j < 7; ++j) s_w[j][i] = a[j];
  }
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int ant = warp; ant < n_ant; ant += kFineThreads / 32) {
    const uint8_t* row = bits + (size_t)ant * row_bytes;
    const float m = (float)mean[ant];
    const float s_hi = 1.f - m, s_lo = -1.f - m;
    float acc[12];
#pragma unroll
    for (int j = 0; j < 12; ++j) acc[j] = 0.f;
    for (int i = lane; i < cn; i += 32) {
      const long long n = tk.start + c0 + i;
      const int bit = (__ldg(row + (n >> 3)) >> (7 - (int)(n & 7))) & 1;
      const float s = bit ? s_hi : s_lo;
      const float a0r = s_w[0][i], a0i = s_w[1][i], a1r = s_w[2][i], a1i = s_w[3][i];
      const float a2r = s_w[4][i], a2i = s_w[5][i], x = s_w[6][i];
      const float sx = s * x, sxx = sx * x;
      acc[0] = fmaf(s, a0r, acc[0]);  // R
      acc[1] = fmaf(s, a0i, acc[1]);
      acc[2] = fmaf(s, a1r, acc[2]);  // dR/dtau
      acc[3] = fmaf(s, a1i, acc[3]);
      acc[4] = fmaf(-sx, a0i, acc[4]);  // dR/df / (2 pi / fs) folded in x: i x a0
      acc[5] = fmaf(sx, a0r, acc[5]);
      acc[6] = fmaf(s, a2r, acc[6]);  // d2R/dtau2
      acc[7] = fmaf(s, a2i, acc[7]);
      acc[8] = fmaf(-sxx, a0r, acc[8]);  // d2R/df2: -x^2 a0
      acc[9] = fmaf(-sxx, a0i, acc[9]);
      acc[10] = fmaf(-sx, a1i, acc[10]);  // d2R/dtau df: i x a1
      acc[11] = fmaf(sx, a1r, acc[11]);
    }
#pragma unroll
    for (int j = 0; j < 12; ++j) {
      float v = acc[j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      acc[j] = v;
    }
    if (lane == 0) {
      double* dst = out + ((size_t)tk.slot * n_ant + ant) * 12;
#pragma unroll
      for (int j = 0; j < 12; ++j) atomicAdd(dst + j, (double)acc[j]);
    }
  }
}

}  // namespace

cudaError_t launch_fine_sums(const uint8_t* d_bits, int n_ant, size_t row_bytes, const double* d_mean,
                             const FineTask* d_tasks, int n_tasks, long long max_length, double* d_out,
                             cudaStream_t st) {
  if (n_tasks <= 0 || max_length <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(d_out, 0, (size_t)n_tasks * n_ant * 12 * sizeof(double), st);
  if (e != cudaSuccess) return e;
  const long long chunks = (max_length + kFineChunk - 1) / kFineChunk;
  if (chunks > 0x7fffffffLL || n_tasks > 65535) return cudaErrorInvalidValue;
  dim3 grid((unsigned)chunks, (unsigned)n_tasks);
  fine_sums_kernel<<<grid, kFineThreads, 0, st>>>(d_bits, n_ant, row_bytes, d_mean, d_tasks, d_out);
  kernel_launch_add(1);
  return cudaGetLastError();
}

}  // namespace tga
