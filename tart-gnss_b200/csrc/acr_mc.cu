// GPU signal synthesizer of the ACR table Monte Carlo
// (examples/gen_acr_tables.rs:63-83 and :134-160).
//
// One thread per (C/N0 point, trial) writes one row of packed bits: two code
// periods of the code circularly delayed by `delay`, on a 100 kHz carrier of
// phase theta with amplitude A = 2 sqrt(C/N0 / fs), plus unit Gaussian noise,
// one-bit quantised (v >= 0 -> 1, simulator.rs:237-244).  The trial's random
// numbers follow the reference generator exactly: xorshift64 (<<13, >>7,
// <<17; 53-bit doubles), seed = trial ^ (bits(cn0) << 33); delay and theta
// from the stream seeded with seed * 0x9E3779B97F4A7C15 + 1, the noise
// (Box-Muller with u1 clamped at 1e-12) from the stream seeded with seed.
// The rows then go through the batched acquisition search as if they were
// antennas of one observation.
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.h"

namespace tga {

namespace {

struct XorShift {
  unsigned long long s;
  __device__ __forceinline__ double next_f64() {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return (double)(s >> 11) / 9007199254740992.0;  // 2^53
  }
  __device__ __forceinline__ double gaussian() {
    const double u1 = fmax(next_f64(), 1e-12);
    const double u2 = next_f64();
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  }
};

__global__ void acr_synth_kernel(const int8_t* __restrict__ code, int period, int n_trials, double cn0_lo,
                                 double cn0_step, int n_points, double fs, double f_carrier,
                                 uint8_t* __restrict__ bits) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n_points * n_trials) return;
  const int j = row / n_trials, t = row - j * n_trials;
  const double cn0 = cn0_lo + (double)j * cn0_step;
  const unsigned long long seed = (unsigned long long)t ^ ((unsigned long long)__double_as_longlong(cn0) << 33);
  XorShift r1{seed * 0x9E3779B97F4A7C15ull + 1ull};
  const int delay = (int)((unsigned long long)(r1.next_f64() * (double)period) % (unsigned long long)period);
  const double theta = r1.next_f64() * 6.283185307179586;
  const double a = 2.0 * sqrt(pow(10.0, cn0 / 10.0) / fs);
  XorShift rn{seed};
  const int n = 2 * period;
  uint8_t* out = bits + (size_t)row * (n / 8);
  const double w = 6.283185307179586 * f_carrier;
  unsigned byte = 0;
  for (int i = 0; i < n; ++i) {
    int cp = i + delay;
    cp -= cp >= period ? period : 0;
    cp -= cp >= period ? period : 0;
    const double carrier = a * cos(w * (double)i / fs + theta);
    const double v = (double)code[cp] * carrier + rn.gaussian();
    byte = (byte << 1) | (v >= 0.0 ? 1u : 0u);
    if ((i & 7) == 7) {
      out[i >> 3] = (uint8_t)byte;
      byte = 0;
    }
  }
}

}  // namespace

cudaError_t launch_acr_synth(const int8_t* d_code, int period, int n_trials, double cn0_lo, double cn0_step,
                             int n_points, double fs, double f_carrier, uint8_t* d_bits, cudaStream_t st) {
  const int rows = n_points * n_trials;
  if (rows <= 0) return cudaSuccess;
  if ((2 * period) % 8) return cudaErrorInvalidValue;
  acr_synth_kernel<<<(rows + 63) / 64, 64, 0, st>>>(d_code, period, n_trials, cn0_lo, cn0_step, n_points, fs,
                                                      f_carrier, d_bits);
  kernel_launch_add(1);
  return cudaGetLastError();
}

}  // namespace tga
