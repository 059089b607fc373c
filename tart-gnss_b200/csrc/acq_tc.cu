// Tensor-core correlator (sm_100a, tcgen05): reduced-precision search.
//
// Same transform as pfa_kernel<..,CORR> (acq_kernels.cu), but the DFT-31 stage
// -- half of the FP32 work -- runs on the 5th-generation tensor cores:
//
//   U[col][ta] = sum_ka X[col][ka] * W31^(ta*ka)        (inverse DFT, 31 points)
//
// is one GEMM per group of transform columns, D = A * B^T with
//   A = data, M = 128 columns per tile, K = 64 = 31 complex inputs as
//       interleaved (re, im) FP16 pairs + 2 zeros,
//   B = DFT-31 as a real 64 x 64 matrix (N = 31 complex outputs interleaved),
//   D = FP32 accumulator in tensor memory (TMEM), one lane per column.
// Both operands are K-major with the 128-byte swizzle in shared memory.  One
// elected thread issues 4 K-steps of tcgen05.mma (M128 N64 K16) per tile and
// commits to an mbarrier; each warp then reads its 32 TMEM lanes
// (tcgen05.ld 32x32b) straight into the FP32 shared buffer of the DFT-33 /
// DFT-M stages, which aliases the operand tiles (the MMA has completed).
//
// FP16 range: the complex products Z*conj(C) are scaled by 2^-k with
// 4 S Lc^2 2^-k <= 32768 (an upper bound on |Z*D|), so no operand overflows.
// Keys carry |y|^2 2^-2k and are only compared; the selected row of every
// (antenna, PRN) is re-evaluated in FP32 afterwards (launch_refine), so the
// reported peak, lag and second peak are FP32 values.
//
// Waits on the tensor cores are bounded: on expiry the kernel sets *err,
// drains (again bounded), frees its TMEM and returns.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "dft.cuh"
#include "engine.h"
#include "pfa_common.cuh"

namespace tga {

namespace {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ uint32_t mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done;
}
// D[tmem] (+)= A[smem desc] * B[smem desc]^T, kind::f16, no lanes masked.
__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 128-byte rows,
// 8-row groups 1024 bytes apart, sm_100 descriptor version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// Instruction descriptor: kind::f16, A = B = FP16, D = FP32, both K-major,
// N = 64, M = 128.
constexpr uint32_t kIdescF16 = (1u << 4) | (0u << 7) | (0u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

// byte offset of 16-byte chunk j of row r inside a 128B-swizzled K-major tile
__device__ __forceinline__ uint32_t sw128_off(int r, int j) {
  return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((j ^ (r & 7)) << 4));
}

__device__ __forceinline__ uint32_t pack_h2(float lo, float hi) {
  const __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}

constexpr int kTcThreads = 384;  // 12 warps: 3 tiles x 4 TMEM lane quadrants
constexpr int kTcTmemCols = 256;
constexpr long long kWaitPolls = 1LL << 22;

template <int M, int BC>
struct TcGeo {
  static constexpr int COLS = 33 * M, LC = 31 * COLS;
  static constexpr int NCOL = BC * COLS;                  // transform columns per group
  static constexpr int TILES = (NCOL + 127) / 128;         // 128-row MMA tiles
  static constexpr int A_BYTES = TILES * 16384;
  static constexpr int BUF_BYTES = BC * LC * 8;
  static constexpr int R_BYTES = ((A_BYTES > BUF_BYTES ? A_BYTES : BUF_BYTES) + 1023) / 1024 * 1024;
  // at least 80 KB so that no more than two CTAs (2 x 256 TMEM columns) share an SM
  static constexpr int SMEM_RAW = R_BYTES + 8192 + 1024;
  static constexpr int SMEM = SMEM_RAW > 81920 ? SMEM_RAW : 81920;
  static_assert(TILES <= 3, "TMEM budget: 3 tiles x 64 columns");
};

struct TcParams {
  PfaParams p;
  float in_scale;  // 2^-k applied to the products before FP16 conversion
  int* err;
};

template <int M, int BC>
__global__ void __launch_bounds__(kTcThreads, 2) pfa_tc_kernel(TcParams tp) {
  using G = Geo<M>;
  using T = TcGeo<M, BC>;
  constexpr int COLS = G::COLS, LC = G::LC, NC = G::NC, NT = kTcThreads;
  const PfaParams& p = tp.p;
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t s_bar;
  __shared__ uint32_t s_tmem;
  __shared__ unsigned long long s_key;
  // 1024-aligned regions: R (operand tiles / FP32 transform buffer), B (DFT-31)
  const uint32_t raw = smem_addr(smem_raw);
  unsigned char* R = smem_raw + ((1024 - (raw & 1023)) & 1023);
  unsigned char* Bm = R + T::R_BYTES;
  float2* buf = reinterpret_cast<float2*>(R);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int S = p.S;

  if (warp == 0) {
    tmem_alloc(&s_tmem, kTcTmemCols);
    tmem_relinquish();
  }
  if (tid == 0) mbar_init(&s_bar, 1);
  // B[n][k]: inverse DFT-31 as a real 64x64 matrix, n = 2 ta + (0 re | 1 im),
  // k = 2 ka + (0 re | 1 im); rows and columns 62, 63 are zero.
  for (int e = tid; e < 64 * 8; e += NT) {
    const int n = e >> 3, j = e & 7;
    uint32_t w[4];
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      float v[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int k = 8 * j + 2 * h + q;
        float val = 0.f;
        if (n < 62 && k < 62) {
          const int ta = n >> 1, u = n & 1, ka = k >> 1, vv = k & 1;
          const int m = (ta * ka) % 31;
          const float c = kCos31[m], sn = kSin31[m];
          val = (u == 0) ? (vv == 0 ? c : -sn) : (vv == 0 ? sn : c);
        }
        v[q] = val;
      }
      w[h] = pack_h2(v[0], v[1]);
    }
    *reinterpret_cast<uint4*>(Bm + sw128_off(n, j)) = make_uint4(w[0], w[1], w[2], w[3]);
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = s_tmem;
  const uint64_t db = sw128_desc(smem_addr(Bm));
  uint32_t phase = 0;
  bool failed = false;

  const int groups = (S + BC - 1) / BC;
  for (int w = blockIdx.x; w < p.n_items && !failed; w += gridDim.x) {
    const int ab_h = w / p.n_prn, prn = w - ab_h * p.n_prn, hyp = ab_h & 1;
    float pmax = -1.f;
    int cmax = 0;
    auto lag_of = [&](int code) -> int {
      const int c = code & 15, q = code >> 4;
      const int b = q % 33, q2 = q / 33;
      const int a = q2 % 31, rho = q2 / 31;
      return rho + S * G::natural(a, b, c);
    };
    if (tid == 0) s_key = 0ull;

    for (int g = 0; g < groups; ++g) {
      auto seq_of = [&](int s) -> int {
        const int rho = g * BC + s;
        return rho < S ? rho : -1;
      };
      auto epilogue = [&](int s, int a, int b, int c, float2 v) {
        const float pw = fmaf(v.x, v.x, v.y * v.y);
        const int code = ((seq_of(s) * 31 + a) * 33 + b) * 16 + c;
        if (pw == pmax) {
          if (lag_of(code) > lag_of(cmax)) cmax = code;
        }
        cmax = pw > pmax ? code : cmax;
        pmax = fmaxf(pw, pmax);
      };

      // ---- stage 1a: products -> FP16 operand rows (one row per column) ----
      for (int u = tid; u < T::NCOL; u += NT) {
        const int s = u / COLS, col = u - s * COLS;
        const int q = seq_of(s);
        if (q < 0) continue;
        const float2* zs = p.z + ((size_t)ab_h * S + q) * LC + col;
        const float2* ds = p.D + ((size_t)prn * 2 + hyp) * LC + col;
        uint32_t pk[32];
#pragma unroll
        for (int a = 0; a < 31; ++a) {
          const float2 x = cmul(__ldcg(zs + a * COLS), __ldg(ds + a * COLS));
          pk[a] = pack_h2(x.x * tp.in_scale, x.y * tp.in_scale);
        }
        pk[31] = 0u;
        unsigned char* rowp = R + (u >> 7) * 16384;
        const int r = u & 127;
#pragma unroll
        for (int j = 0; j < 8; ++j)
          *reinterpret_cast<uint4*>(rowp + sw128_off(r, j)) = make_uint4(pk[4 * j], pk[4 * j + 1], pk[4 * j + 2], pk[4 * j + 3]);
      }
      fence_async_smem();
      tc_fence_before();
      __syncthreads();

      // ---- stage 1b: DFT-31 on the tensor cores ----
      if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int t = 0; t < T::TILES; ++t) {
          const uint64_t da = sw128_desc(smem_addr(R + t * 16384));
#pragma unroll
          for (int ks = 0; ks < 4; ++ks)
            mma_f16(tmem_base + (uint32_t)(t * 64), da + (uint64_t)(2 * ks), db + (uint64_t)(2 * ks), kIdescF16,
                    ks > 0 ? 1u : 0u);
        }
        mma_commit(&s_bar);
      }
      uint32_t done = 0;
      for (long long it = 0; it < kWaitPolls && !done; ++it) done = mbar_try_wait(&s_bar, phase);
      if (__syncthreads_or(!done)) {
        failed = true;
        break;
      }
      phase ^= 1u;
      tc_fence_after();

      // ---- stage 1c: TMEM -> FP32 transform buffer (aliases the operand tiles) ----
      {
        const int t = warp >> 2, quad = warp & 3;
        if (t < T::TILES) {
          const int u = t * 128 + quad * 32 + lane;  // this thread's TMEM lane = column
          const int s = u / COLS, col = u - s * COLS;
          const bool valid = u < T::NCOL && seq_of(s) >= 0;
          const uint32_t taddr = tmem_base + ((uint32_t)(quad * 32) << 16) + (uint32_t)(t * 64);
#pragma unroll
          for (int chunk = 0; chunk < 4; ++chunk) {
            uint32_t r[16];
            tmem_ld16(taddr + (uint32_t)(16 * chunk), r);
            tmem_wait_ld();
            if (valid) {
              float2* dst = buf + s * LC + col;
#pragma unroll
              for (int h = 0; h < 8; ++h) {
                const int ta = chunk * 8 + h;
                if (ta < 31) dst[ta * COLS] = make_float2(__uint_as_float(r[2 * h]), __uint_as_float(r[2 * h + 1]));
              }
            }
          }
        }
      }
      tc_fence_before();
      __syncthreads();

      // ---- stage 2: DFT-33 over digit b (FP32) ----
      for (int u = tid; u < BC * 31 * NC; u += NT) {
        const int s = u / (31 * NC), r = u - s * 31 * NC;
        const int a = r / NC, c = r - a * NC;
        if (seq_of(s) < 0) continue;
        float2* base = buf + s * LC + a * COLS + c * 33;
        float2 x[33];
#pragma unroll
        for (int b = 0; b < 33; ++b) x[b] = base[b];
        if constexpr (NC == 1) {
          dft33<true>(x, [&](int tb, float2 v) { epilogue(s, a, tb, 0, v); });
        } else {
          dft33<true>(x, [&](int tb, float2 v) { base[tb] = v; });
        }
      }
      // ---- stage 3: DFT-M over digit c (FP32) ----
      if constexpr (NC > 1) {
        __syncthreads();
        for (int u = tid; u < BC * 1023; u += NT) {
          const int s = u / 1023, gi = u - s * 1023;
          const int a = gi / 33, b = gi - a * 33;
          if (seq_of(s) < 0) continue;
          const float2* base = buf + s * LC + a * COLS + b;
          float2 x[NC];
#pragma unroll
          for (int c = 0; c < NC; ++c) x[c] = base[c * 33];
          dft_small<NC, true>(x, [&](int tc, float2 v) { epilogue(s, a, b, tc, v); });
        }
      }
      __syncthreads();
    }
    if (failed) break;

    unsigned long long kbest =
        pmax < 0.f ? 0ull : (((unsigned long long)__float_as_uint(pmax) << 32) | (unsigned)lag_of(cmax));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, kbest, o);
      kbest = other > kbest ? other : kbest;
    }
    if (lane == 0) atomicMax(&s_key, kbest);
    __syncthreads();
    if (tid == 0) p.keys[w] = s_key;
    __syncthreads();
  }

  if (failed) {
    // the tensor cores did not answer in time: flag it, give the in-flight
    // MMAs a second bounded window to finish, then release TMEM
    if (tid == 0) atomicExch(tp.err, 1);
    uint32_t done = 0;
    for (long long it = 0; it < kWaitPolls && !done; ++it) done = mbar_try_wait(&s_bar, phase);
    __syncthreads();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, kTcTmemCols);
}

template <int M, int BC>
cudaError_t run_tc(const TcParams& tp, int num_sms, cudaStream_t st) {
  using T = TcGeo<M, BC>;
  auto kern = pfa_tc_kernel<M, BC>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, T::SMEM);
  if (e != cudaSuccess) return e;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTcThreads, T::SMEM);
  if (per_sm < 1) per_sm = 1;
  if (per_sm > 2) per_sm = 2;  // TMEM: 2 x 256 columns per SM
  int grid = num_sms * per_sm;
  if (grid > tp.p.n_items) grid = tp.p.n_items;
  if (grid < 1) return cudaSuccess;
  kern<<<grid, kTcThreads, T::SMEM, st>>>(tp);
  kernel_launch_add(1);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_correlate_tc(const PolyClass& pc, const SearchDims& dims, const float2* d_Z, const float2* d_D,
                                unsigned long long* d_keys, int* d_err, int num_sms, cudaStream_t st) {
  TcParams tp = {};
  tp.p.z = const_cast<float2*>(d_Z);
  tp.p.D = d_D;
  tp.p.keys = d_keys;
  tp.p.n_prn = dims.n_prn;
  tp.p.S = pc.S;
  tp.p.P = pc.P;
  tp.p.n_items = dims.n_ant * dims.nb * 2 * dims.n_prn;
  tp.err = d_err;
  // 2^-k with 4 S Lc^2 2^-k <= 32768
  const double bound = 4.0 * pc.S * (double)pc.Lc * (double)pc.Lc;
  int k = 0;
  while (bound / (double)(1ull << k) > 32768.0 && k < 60) ++k;
  tp.in_scale = (float)(1.0 / (double)(1ull << k));
  switch (pc.M) {
    case 1: return run_tc<1, 8>(tp, num_sms, st);
    case 4: return run_tc<4, 2>(tp, num_sms, st);
    case 10: return run_tc<10, 1>(tp, num_sms, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace tga
