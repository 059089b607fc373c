// Single-PRN acquisition that allocates nothing: tga_acquire_single_static.
//
// Who needs it: callers that must not call cudaMalloc during operation --
// a real-time receiver loop (cudaMalloc can synchronise the device and take
// unbounded time), a process whose device memory is already held by another
// framework's caching allocator, or an embedding host that only permits
// memory reserved when the library was loaded.  Such a caller passes device
// pointers for the samples, the phase points and the result, plus a stream,
// and this entry point uses only the fixed scratch array below.
//
// The scratch array is a file-scope __device__ array; every GPU that loads
// the library holds it (kNoAllocScratchBytes) until the process exits.  In
// host code its name is only a host-side stand-in for the symbol, not a
// device address, so its device address is fetched once per device with
// cudaGetSymbolAddress (with that device current) on the first call made on
// that device; make that first call before any stream capture.  All calls
// share the array and it keeps the previous call's contents: every buffer
// carved from it is fully written before it is read, and calls that overlap
// on the GPU (concurrent streams or host threads) race on it.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/tga.h"
#include "engine.h"
#include "gnss_tables.h"

namespace tga {

constexpr size_t kNoAllocScratchBytes = 16u << 20;  // 16 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
// Per-device address of the scratch array.  Set once per device under the
// mutex (host threads making their first calls at once wait for each
// other), then only read.
std::atomic<unsigned char*> g_scratch_ptr[kMaxDevices];
std::mutex g_scratch_mutex;

// Device address of the scratch array on the current device (set-up once).
cudaError_t scratch_for_current_device(unsigned char** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  unsigned char* ptr = g_scratch_ptr[dev].load(std::memory_order_acquire);
  if (!ptr) {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    ptr = g_scratch_ptr[dev].load(std::memory_order_relaxed);
    if (!ptr) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return e;
      ptr = static_cast<unsigned char*>(p);
      g_scratch_ptr[dev].store(ptr, std::memory_order_release);
    }
  }
  *out = ptr;
  return cudaSuccess;
}

// Doppler grid (acquisition.rs:188-198) evaluated on the device with the
// same IEEE double operations as the host.
__global__ void grid_kernel(double center, double band, int nb, double* fc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  if (nb == 1) {
    fc[0] = center;
    return;
  }
  const double lo = __dsub_rn(center, band);
  const double step = __ddiv_rn(__dmul_rn((double)i, __dmul_rn(2.0, band)), __dsub_rn((double)nb, 1.0));
  fc[i] = __dadd_rn(lo, step);
}

// +-1 primary chips of one PRN, generated on the device from the table
// parameters, so no host staging buffer is needed.
struct ChipParams {
  int constellation;
  int g2delay;         // C/A: G2 delay
  int weil_w, weil_p;  // B1C / L1C
  char hex[1024];      // Galileo E1-C memory code
};

__device__ int legendre_bit(int k, int n) {
  // 1 iff k is a non-zero quadratic residue mod the prime n (Euler's criterion)
  if (k == 0) return 0;
  unsigned r = 1, b = (unsigned)k, e = (unsigned)(n - 1) / 2;
  while (e) {
    if (e & 1u) r = (r * b) % (unsigned)n;
    b = (b * b) % (unsigned)n;
    e >>= 1;
  }
  return r == 1u ? 1 : 0;
}

__global__ void chips_kernel(ChipParams cp, int8_t* chips, int8_t* table) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = cp.constellation;
  if (c == TGA_GPS || c == TGA_SBAS || c == TGA_QZSS) {
    if (i != 0) return;
    // IS-GPS-200 G1 (taps 3,10) and G2 (taps 2,3,6,8,9,10), all-ones seed;
    // chip = +1 when the G1 output differs from the delayed G2 output.
    unsigned g1 = 0x3FF, g2 = 0x3FF;
    uint32_t g2bits[32] = {};
    uint32_t g1bits[32] = {};
    for (int n = 0; n < 1023; ++n) {
      const unsigned o1 = (g1 >> 9) & 1u, o2 = (g2 >> 9) & 1u;
      g1bits[n >> 5] |= o1 << (n & 31);
      g2bits[n >> 5] |= o2 << (n & 31);
      const unsigned f1 = ((g1 >> 2) ^ (g1 >> 9)) & 1u;
      const unsigned f2 = ((g2 >> 1) ^ (g2 >> 2) ^ (g2 >> 5) ^ (g2 >> 7) ^ (g2 >> 8) ^ (g2 >> 9)) & 1u;
      g1 = ((g1 << 1) | f1) & 0x3FF;
      g2 = ((g2 << 1) | f2) & 0x3FF;
    }
    for (int n = 0; n < 1023; ++n) {
      const int j = ((n - cp.g2delay) % 1023 + 1023) % 1023;
      const unsigned a = (g1bits[n >> 5] >> (n & 31)) & 1u, b = (g2bits[j >> 5] >> (j & 31)) & 1u;
      chips[n] = (a ^ b) ? 1 : -1;
    }
    table[0] = TGA_ACR_GPS_L1_CA;
  } else if (c == TGA_GALILEO) {
    if (i >= 1023) return;
    const char ch = cp.hex[i];
    const int v = (ch >= '0' && ch <= '9') ? ch - '0' : ((ch | 0x20) - 'a' + 10);
    for (int b = 0; b < 4; ++b) chips[4 * i + b] = ((v >> (3 - b)) & 1) ? 1 : -1;
    if (i == 0) table[0] = TGA_ACR_GALILEO_E1C;
  } else if (c == TGA_BEIDOU) {
    if (i >= 10230) return;
    const int N = 10243, k = (i + cp.weil_p - 1) % N;
    chips[i] = (legendre_bit(k, N) ^ legendre_bit((k + cp.weil_w) % N, N)) ? -1 : 1;
    if (i == 0) table[0] = TGA_ACR_BEIDOU_B1C;
  } else if (c == TGA_L1C) {
    if (i >= 10230) return;
    const int N = 10223, split = cp.weil_p - 1;
    int bit;
    if (i < split) {
      bit = legendre_bit(i, N) ^ legendre_bit((i + cp.weil_w) % N, N);
    } else if (i < split + 7) {
      const int ex[7] = {0, 1, 1, 0, 1, 0, 0};
      bit = ex[i - split];
    } else {
      const int k = i - 7;
      bit = legendre_bit(k, N) ^ legendre_bit((k + cp.weil_w) % N, N);
    }
    chips[i] = bit ? -1 : 1;
    if (i == 0) table[0] = TGA_ACR_GPS_L1C;
  }
}

__global__ void result_kernel(const CellOut* cell, int prn, tga_result* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const CellOut o = *cell;
  tga_result r;
  r.prn = prn;
  r.best_freq_idx = o.bin;
  r.best_codephase = o.tau;
  r.signal_strength = o.strength;
  r.second_peak = o.second;
  r.codephase_frac = o.codephase_frac;
  r.frequency = o.frequency;
  r.hypothesis = o.hyp;
  r.path = 0;
  *out = r;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Whether the reference's resampled code over 2P samples is
// chip((n/S) mod Lc) * pulse(n mod S) for every chip sequence: the index
// rule idx(n) = floor(n / (P / seq_len)) mod seq_len must map n to chip
// (n/S) mod Lc, with the BOC half-chip parity a function of n mod S only.
bool index_structure(int c, size_t P, int S, int Lc, float* pulse) {
  const bool boc = (c == TGA_BEIDOU || c == TGA_L1C);
  const size_t seq = boc ? 2 * (size_t)Lc : (size_t)Lc;
  const double spc = (double)P / (double)seq;
  for (int s = 0; s < S; ++s) pulse[s] = 0.f;
  for (size_t n = 0; n < 2 * P; ++n) {
    const double q = std::floor((double)n / spc);
    const size_t idx = (q > 0.0 ? (size_t)q : 0) % seq;
    const size_t chip = boc ? idx / 2 : idx;
    if (chip != (n / (size_t)S) % (size_t)Lc) return false;
    const float sign = (boc && (idx & 1)) ? -1.f : 1.f;
    float& ps = pulse[n % (size_t)S];
    if (ps == 0.f) ps = sign;
    else if (ps != sign) return false;
  }
  return true;
}

}  // namespace

}  // namespace tga

using namespace tga;

// See include/tga.h.  Allocates no device or host memory.
extern "C" int tga_acquire_single_static(int constellation, const float* d_signal_f32,
                                         const double* d_phasepoints, size_t num_samples,
                                         double sampling_freq, double center_freq, double search_band,
                                         int prn, size_t samples_per_chunk, tga_result* d_out,
                                         void* stream) {
  if (!d_signal_f32 || !d_phasepoints || !d_out) return TGA_ERR_INVALID_ARG;
  if (constellation < 0 || constellation >= TGA_N_CONSTELLATIONS) return TGA_ERR_INVALID_ARG;
  static const int kLo[6] = {1, 1, 1, 120, 1, 184}, kHi[6] = {38, 50, 63, 158, 63, 206};
  static const int kChips[6] = {1023, 4092, 10230, 1023, 10230, 1023};
  if (prn < kLo[constellation] || prn > kHi[constellation]) return TGA_ERR_INVALID_ARG;
  const size_t P = samples_per_chunk;
  const int Lc = kChips[constellation];
  // only the fused path: a window of exactly two periods, whole samples per chip
  if (P == 0 || num_samples != 2 * P || P % (size_t)Lc != 0) return TGA_ERR_UNSUPPORTED;
  const int S = (int)(P / (size_t)Lc);
  if (S > kMaxPulse || P > (size_t)1 << 30) return TGA_ERR_UNSUPPORTED;
  PolyClass pc;
  pc.P = (int)P;
  pc.S = S;
  pc.Lc = Lc;
  pc.M = Lc / 1023;
  if (!index_structure(constellation, P, S, Lc, pc.pulse)) return TGA_ERR_UNSUPPORTED;
  // Doppler bins (acquisition.rs:189-191)
  const double x = std::round(2.0 * search_band / 300.0);
  const size_t nb = (x > 0.0 ? (size_t)x : 0) + 1;
  if (nb > (size_t)kMaxBins) return TGA_ERR_INVALID_ARG;

  // carve the scratch array; reject anything that does not fit
  const size_t z_bytes = align256(nb * 2 * (size_t)S * Lc * sizeof(float2));
  const size_t d_bytes = align256((size_t)2 * Lc * sizeof(float2));
  const size_t k_bytes = align256(nb * 2 * sizeof(unsigned long long));
  const size_t small = align256(sizeof(BestRow)) + align256(sizeof(CellOut)) + align256(nb * sizeof(double)) +
                       align256((size_t)Lc + 1) + align256(sizeof(int32_t));
  if (z_bytes + d_bytes + k_bytes + small > kNoAllocScratchBytes) return TGA_ERR_CAPACITY;

  unsigned char* base = nullptr;
  if (scratch_for_current_device(&base) != cudaSuccess) return TGA_ERR_CUDA;
  unsigned char* p = base;
  float2* d_z = (float2*)p;
  p += z_bytes;
  float2* d_D = (float2*)p;
  p += d_bytes;
  unsigned long long* d_keys = (unsigned long long*)p;
  p += k_bytes;
  BestRow* d_best = (BestRow*)p;
  p += align256(sizeof(BestRow));
  CellOut* d_cell = (CellOut*)p;
  p += align256(sizeof(CellOut));
  double* d_fc = (double*)p;
  p += align256(nb * sizeof(double));
  int8_t* d_chips = (int8_t*)p;
  p += align256((size_t)Lc + 1);
  int32_t* d_ant = (int32_t*)p;

  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return TGA_ERR_CUDA;

  ChipParams cp;
  std::memset(&cp, 0, sizeof cp);
  cp.constellation = constellation;
  if (constellation == TGA_GPS) cp.g2delay = TGA_GPS_G2_DELAY[prn - 1];
  if (constellation == TGA_SBAS) cp.g2delay = TGA_SBAS_G2_DELAY[prn - 120];
  if (constellation == TGA_QZSS) cp.g2delay = TGA_QZSS_G2_DELAY[prn - 184];
  if (constellation == TGA_BEIDOU) {
    cp.weil_w = TGA_B1CP_WP[prn - 1][0];
    cp.weil_p = TGA_B1CP_WP[prn - 1][1];
  }
  if (constellation == TGA_L1C) {
    cp.weil_w = TGA_L1CP_WP[prn - 1][0];
    cp.weil_p = TGA_L1CP_WP[prn - 1][1];
  }
  if (constellation == TGA_GALILEO) std::memcpy(cp.hex, TGA_GALILEO_E1C_HEX[prn - 1], 1023);

  grid_kernel<<<((unsigned)nb + 127) / 128, 128, 0, st>>>(center_freq, search_band, (int)nb, d_fc);
  chips_kernel<<<(Lc + 255) / 256, 256, 0, st>>>(cp, d_chips, d_chips + Lc);
  if (cudaMemsetAsync(d_ant, 0, sizeof(int32_t), st) != cudaSuccess) return TGA_ERR_CUDA;

  SampleSource src;
  src.sig = d_signal_f32;
  src.pp = d_phasepoints;
  src.n_samples = num_samples;
  src.ant = d_ant;
  src.n_ant = 1;
  SearchDims dims;
  dims.n_ant = 1;
  dims.nb = (int)nb;
  dims.n_prn = 1;
  dims.fc = d_fc;
  const int chip_width = (int)std::ceil(sampling_freq / 1.023e6);
  cudaError_t e = launch_code_spectra(pc, d_chips, 1, d_D, sms, st);
  if (e == cudaSuccess) e = launch_frontend(src, dims, pc, d_z, st);
  if (e == cudaSuccess) e = launch_forward_z(pc, (int)nb, d_z, sms, st);
  if (e == cudaSuccess) e = launch_correlate(pc, dims, d_z, d_D, d_keys, sms, st);
  if (e == cudaSuccess) e = launch_reduce_bins(dims, d_keys, d_best, st);
  if (e == cudaSuccess) e = launch_second_peak(pc, dims, d_z, d_D, d_best, chip_width, sms, st);
  if (e == cudaSuccess) e = launch_finalize(pc, dims, d_best, center_freq, d_chips + Lc, 0, d_cell, st);
  if (e != cudaSuccess) return TGA_ERR_CUDA;
  result_kernel<<<1, 32, 0, st>>>(d_cell, prn, d_out);
  return cudaGetLastError() == cudaSuccess ? TGA_OK : TGA_ERR_CUDA;
}
