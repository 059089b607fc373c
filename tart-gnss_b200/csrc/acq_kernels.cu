// CUDA kernels of the B200 acquisition engine (sm_100a).
//
// Fused path.  For a window of two code periods (N = 2P) the reference's
// dual-hypothesis correlation (correlate.rs:91-183) is rewritten exactly:
//
//  1. Fold:  f = x[0:P] + x[P:2P] gives the [c,c] correlation; the [c,-c]
//     correlation is the negacyclic correlation of g = x[0:P] - x[P:2P].
//  2. Polyphase: the resampled code is c(n) = chip((n / S) mod Lc) * pulse(n % S)
//     (S samples per chip, P = S * Lc).  Then for every lag tau = rho + S*t
//        r(tau) = sum_m chip(m) z_rho(m + t),   z_rho(j) = sum_s pulse(s) f(S j + rho + s)
//     i.e. S independent circular correlations of length Lc (the chip count,
//     1023 / 4092 / 10230) instead of one of length 2P.  The negacyclic
//     branch is made cyclic by the twist v(j) = exp(i pi j / Lc).
//  3. Every Lc is 31 * 33 * M (M = 1, 4, 10), pairwise coprime, so each
//     length-Lc DFT is a twiddle-free Good-Thomas transform: a DFT-31 stage
//     fed straight from global memory (Z * conj(D) formed in registers), a
//     DFT-33 stage and a DFT-M stage through shared memory.  The last stage
//     feeds |y|^2 straight into the argmax; no correlation vector ever
//     leaves the SM.
//
// Frequency-domain arrays use the digit layout [k31][kM][k33]; time-domain
// lag digits map to natural lags by the Chinese remainder theorem.
//
// Generic path (any N): the reference algorithm on the GPU, with Bluestein
// FFTs of length N built on a power-of-two Stockham FFT.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <vector>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "dft.cuh"
#include "engine.h"
#include "gnss_tables.h"
#include "pfa_common.cuh"

namespace tga {

// Launches of the calling host thread: a search runs on the thread that
// called the entry point, so a per-thread count is that call's count even
// when several contexts run on several threads at once.
static thread_local int g_launches = 0;
int kernel_launch_count_reset() {
  int v = g_launches;
  g_launches = 0;
  return v;
}
int kernel_launch_count() { return g_launches; }
void kernel_launch_add(int n) { g_launches += n; }

#define TGA_LAUNCHED() (++g_launches, cudaGetLastError())

// ---------------------------------------------------------------------------
// antenna means: mean of the +-1 samples over the whole row (acquisition.rs:285)
// ---------------------------------------------------------------------------
__global__ void antenna_means_kernel(const uint8_t* __restrict__ bits, size_t row_bytes,
                                     double* __restrict__ mean) {
  const uint8_t* row = bits + (size_t)blockIdx.x * row_bytes;
  unsigned long long ones = 0;
  const size_t n_words = row_bytes / 8;
  const bool aligned = (((uintptr_t)row) & 7) == 0;
  if (aligned) {
    const unsigned long long* w = reinterpret_cast<const unsigned long long*>(row);
    for (size_t i = threadIdx.x; i < n_words; i += blockDim.x) ones += __popcll(__ldg(w + i));
    for (size_t i = n_words * 8 + threadIdx.x; i < row_bytes; i += blockDim.x) ones += __popc(row[i]);
  } else {
    for (size_t i = threadIdx.x; i < row_bytes; i += blockDim.x) ones += __popc(row[i]);
  }
  for (int o = 16; o > 0; o >>= 1) ones += __shfl_xor_sync(0xffffffffu, ones, o);
  __shared__ unsigned long long part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = ones;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += part[i];
    const double n = (double)(row_bytes * 8);
    // sum of +-1 over the row is the exact integer 2*ones - n
    mean[blockIdx.x] = (double)(2.0 * (double)t - n) / n;
  }
}

cudaError_t launch_antenna_means(const uint8_t* d_bits, int n_rows, size_t row_bytes, double* d_mean,
                                 cudaStream_t st) {
  if (n_rows <= 0) return cudaSuccess;
  antenna_means_kernel<<<n_rows, 256, 0, st>>>(d_bits, row_bytes, d_mean);
  return TGA_LAUNCHED();
}

// ---------------------------------------------------------------------------
// front end: carrier wipe-off (correlate.rs:110-115), fold, polyphase boxcar
// ---------------------------------------------------------------------------
struct FrontParams {
  SampleSource src;
  const double* fc;
  int nb, P, S, Lc;
  float pulse[kMaxPulse];
  // pulse shape: 0 any, 1 constant w0, 2 w0 for the first S / 2 samples and
  // -w0 for the rest (BOC(1, 1)); 1 and 2 let the polyphase sums run
  int pulse_kind;
  float pulse_w0;
  float2* z;
};

constexpr int kFrontJ = 64;  // chips per CTA

template <bool BITS>
__device__ __forceinline__ float2 wipe(const FrontParams& p, int row, int n, double f) {
  float s;
  double ph_d;
  if (BITS) {
    const uint8_t byte = __ldg(p.src.bits + (size_t)row * p.src.row_bytes + (n >> 3));
    const double v = ((byte >> (7 - (n & 7))) & 1) ? 1.0 : -1.0;
    s = (float)(v - __ldg(p.src.mean + row));        // (v - mean) as f32
    ph_d = (p.src.pc * (double)n) * f;                // phasepoint * freq
  } else {
    s = __ldg(p.src.sig + (size_t)row * p.src.n_samples + n);
    ph_d = __ldg(p.src.pp + n) * f;
  }
  const float ph = __double2float_rn(ph_d);           // (p * freq) as f32
  float sn, cs;
  sincos_phase(ph, &sn, &cs);
  return make_float2(cs * s, sn * s);
}

template <bool BITS>
__global__ void __launch_bounds__(256) frontend_kernel(FrontParams p) {
  extern __shared__ float2 fsm[];
  const int S = p.S, P = p.P, Lc = p.Lc;
  const int ab = blockIdx.y;
  const int ant_slot = ab / p.nb, bin = ab - ant_slot * p.nb;
  const int row = p.src.ant[ant_slot];
  const double f = p.fc[bin];
  const int j0 = blockIdx.x * kFrontJ;
  const int nj = min(kFrontJ, Lc - j0);
  const int cnt = nj * S + S - 1;
  const int span = kFrontJ * S + S;
  float2* fsh = fsm;                         // padded: index i + i/S
  float2* gsh = fsm + span + span / S + 1;
  float2* tw = gsh + span + span / S + 1;    // twist per chip
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    int m = S * j0 + i;
    float sign = 1.f;
    if (m >= P) {  // wrap of the last chip: f is P-periodic, g antiperiodic
      m -= P;
      sign = -1.f;
    }
    const float2 x0 = wipe<BITS>(p, row, m, f);
    const float2 x1 = wipe<BITS>(p, row, m + P, f);
    const int pi = i + i / S;
    fsh[pi] = cadd(x0, x1);
    const float2 g = csub(x0, x1);
    gsh[pi] = make_float2(g.x * sign, g.y * sign);
  }
  for (int jj = threadIdx.x; jj < nj; jj += blockDim.x) {
    double sn, cs;
    sincospi((double)(j0 + jj) / (double)Lc, &sn, &cs);
    tw[jj] = make_float2((float)cs, (float)sn);
  }
  __syncthreads();
  const size_t seqA = ((size_t)ab * 2 + 0) * S, seqB = ((size_t)ab * 2 + 1) * S;
  if (p.pulse_kind != 0 && S >= 4) {
    // runs of L = S / 4 residues per thread: the first sum directly, each
    // next one from the previous (2 or 3 samples instead of S):
    //   constant w0:   z(rho + 1) = z(rho) + w0 (f[a + S] - f[a])
    //   w0 / -w0:      z(rho + 1) = z(rho) + w0 (2 f[a + S/2] - f[a] - f[a + S])
    // with a = jj S + rho; sample i sits at padded index i + i / S
    const int L = (S + 3) / 4;
    const float w0 = p.pulse_w0;
    const bool boc = p.pulse_kind == 2;
    const int H = S / 2;
    for (int o = threadIdx.x; o < 4 * nj; o += blockDim.x) {
      const int k = o / nj, jj = o - k * nj;
      const int rho0 = k * L, rho1 = min(rho0 + L, S);
      if (rho0 >= S) continue;
      float2 za = make_float2(0.f, 0.f), zb = make_float2(0.f, 0.f);
      const int base = jj * S + rho0 + jj;
      for (int s = 0; s < S; ++s) {
        const int pi = base + s + (rho0 + s >= S ? 1 : 0);
        const float w = p.pulse[s];
        za.x = fmaf(w, fsh[pi].x, za.x);
        za.y = fmaf(w, fsh[pi].y, za.y);
        zb.x = fmaf(w, gsh[pi].x, zb.x);
        zb.y = fmaf(w, gsh[pi].y, zb.y);
      }
      const int j = j0 + jj;
      p.z[(seqA + rho0) * Lc + j] = za;
      p.z[(seqB + rho0) * Lc + j] = cmul(zb, tw[jj]);
      for (int rho = rho0; rho + 1 < rho1; ++rho) {
        const int a = jj * S + rho;
        const int pa = a + jj, pe = a + S + jj + 1;
        if (boc) {
          const int pm = a + H + jj + (rho + H >= S ? 1 : 0);
          za.x += w0 * (2.f * fsh[pm].x - fsh[pa].x - fsh[pe].x);
          za.y += w0 * (2.f * fsh[pm].y - fsh[pa].y - fsh[pe].y);
          zb.x += w0 * (2.f * gsh[pm].x - gsh[pa].x - gsh[pe].x);
          zb.y += w0 * (2.f * gsh[pm].y - gsh[pa].y - gsh[pe].y);
        } else {
          za.x += w0 * (fsh[pe].x - fsh[pa].x);
          za.y += w0 * (fsh[pe].y - fsh[pa].y);
          zb.x += w0 * (gsh[pe].x - gsh[pa].x);
          zb.y += w0 * (gsh[pe].y - gsh[pa].y);
        }
        p.z[(seqA + rho + 1) * Lc + j] = za;
        p.z[(seqB + rho + 1) * Lc + j] = cmul(zb, tw[jj]);
      }
    }
    return;
  }
  for (int o = threadIdx.x; o < S * nj; o += blockDim.x) {
    const int rho = o / nj, jj = o - rho * nj;
    float2 za = make_float2(0.f, 0.f), zb = make_float2(0.f, 0.f);
    // tap s reads sample i = jj S + rho + s at padded index i + i / S, and
    // i / S = jj + (rho + s >= S) since rho + s < 2 S: no division per tap
    const int base = jj * S + rho + jj;
    for (int s = 0; s < S; ++s) {
      const int pi = base + s + (rho + s >= S ? 1 : 0);
      const float w = p.pulse[s];
      za.x = fmaf(w, fsh[pi].x, za.x);
      za.y = fmaf(w, fsh[pi].y, za.y);
      zb.x = fmaf(w, gsh[pi].x, zb.x);
      zb.y = fmaf(w, gsh[pi].y, zb.y);
    }
    const int j = j0 + jj;
    p.z[(seqA + rho) * Lc + j] = za;
    p.z[(seqB + rho) * Lc + j] = cmul(zb, tw[jj]);
  }
}

cudaError_t launch_frontend(const SampleSource& src, const SearchDims& dims, const PolyClass& pc,
                            float2* d_z, cudaStream_t st) {
  FrontParams p;
  p.src = src;
  p.fc = dims.fc;
  p.nb = dims.nb;
  p.P = pc.P;
  p.S = pc.S;
  p.Lc = pc.Lc;
  for (int i = 0; i < kMaxPulse; ++i) p.pulse[i] = pc.pulse[i];
  // the pulse's shape (see FrontParams)
  p.pulse_w0 = pc.pulse[0];
  bool constant = true, boc = pc.S % 2 == 0;
  for (int i = 0; i < pc.S; ++i) {
    constant = constant && pc.pulse[i] == pc.pulse[0];
    boc = boc && pc.pulse[i] == (i < pc.S / 2 ? pc.pulse[0] : -pc.pulse[0]);
  }
  p.pulse_kind = constant ? 1 : (boc ? 2 : 0);
  p.z = d_z;
  const int span = kFrontJ * pc.S + pc.S;
  const size_t smem = (size_t)(2 * (span + span / pc.S + 1) + kFrontJ) * sizeof(float2);
  dim3 grid((pc.Lc + kFrontJ - 1) / kFrontJ, dims.n_ant * dims.nb);
  if (src.bits) {
    cudaFuncSetAttribute(frontend_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    frontend_kernel<true><<<grid, 256, smem, st>>>(p);
  } else {
    cudaFuncSetAttribute(frontend_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    frontend_kernel<false><<<grid, 256, smem, st>>>(p);
  }
  return TGA_LAUNCHED();
}

// ---------------------------------------------------------------------------
// prime-factor transform engine
// ---------------------------------------------------------------------------
template <int M, int BC, int NT, int MINB, int MODE>
__global__ void __launch_bounds__(NT, MINB) pfa_kernel(PfaParams p) {
  using G = Geo<M>;
  constexpr int COLS = G::COLS, LC = G::LC, NC = G::NC;
  constexpr bool INV = (MODE == CORR || MODE == SECOND || MODE == CAND);
  constexpr bool ARGMAX = (MODE == CORR || MODE == CAND);
  extern __shared__ float2 buf[];
  __shared__ unsigned long long s_key;
  __shared__ unsigned int s_p2;
  // CAND with p2rows: for every residue of the row and every warp that
  // scanned it, its four largest |y|^2 as (value bits << 32) | lag, after
  // the transform buffer (TOP_WPS warps per residue)
  constexpr bool TOP = MODE == CAND;
  constexpr int TOP_WPS = NT / 32 / BC >= 1 ? NT / 32 / BC : 1;
  unsigned long long* s_res = reinterpret_cast<unsigned long long*>(buf + BC * LC);
  const bool keep_top = TOP && p.p2rows != nullptr;
  const int tid = threadIdx.x;
  const int S = p.S;
  const int groups = INV ? (S + BC - 1) / BC : 1;
  int n_work = INV ? p.n_items : (p.n_seq + BC - 1) / BC;
  if (MODE == CAND) n_work = min(n_work, *p.cand_count);

  for (int w = blockIdx.x; w < n_work; w += gridDim.x) {
    int ab_h = 0, prn = 0, tau_star = 0;
    if (MODE == CORR) {
      ab_h = w / p.n_prn;
      prn = w - ab_h * p.n_prn;
    } else if (MODE == SECOND) {
      const BestRow b = p.best[w];
      ab_h = b.ab * 2 + b.hyp;
      prn = w % p.n_prn;
      tau_star = b.tau;
    } else if (MODE == CAND) {
      const int2 c = p.cand[w];
      ab_h = c.x;
      prn = c.y;
    }
    // where the item's key goes: CORR's item w is the row ab_h * n_prn + prn
    const int key_at = MODE == CAND ? ab_h * p.n_prn + prn : w;
    const int hyp = ab_h & 1;
    // CORR: running maximum of |y|^2 and a compact code of its position
    // ((rho*31 + a)*33 + b)*16 + c; the lag is decoded only on ties and once
    // per item, which keeps the per-output epilogue to a compare and selects.
    float pmax = -1.f;
    int cmax = 0;
    auto lag_of = [&](int code) -> int {
      const int c = code & 15, q = code >> 4;
      const int b = q % 33, q2 = q / 33;
      const int a = q2 % 31, rho = q2 / 31;
      return rho + S * G::natural(a, b, c);
    };
    float pbest = 0.f;
    if (tid == 0) {
      s_key = 0ull;
      s_p2 = 0u;
    }

    for (int g = 0; g < groups; ++g) {
      // sequence of slot s in this group, or -1 when idle
      auto seq_of = [&](int s) -> int {
        if (INV) {
          const int rho = g * BC + s;
          return rho < S ? rho : -1;
        }
        const int q = w * BC + s;
        return q < p.n_seq ? q : -1;
      };
      // epilogue for output (s, a, b, c)
      auto epilogue = [&](int s, int a, int b, int c, float2 v) {
        if (MODE == FWD_Z) {
          p.z[(size_t)seq_of(s) * LC + G::offset(a, b, c)] = v;
          // the last stage reads and writes the same positions of its
          // thread: keep the output for the FP16 units below
          if (p.z16) buf[s * LC + G::offset(a, b, c)] = v;
        } else if (MODE == FWD_D) {
          p.Dout[(size_t)seq_of(s) * LC + G::offset(a, b, c)] = make_float2(v.x, -v.y);
        } else {
          const float pw = fmaf(v.x, v.x, v.y * v.y);
          if (ARGMAX) {
            const int code = ((seq_of(s) * 31 + a) * 33 + b) * 16 + c;
            if (pw == pmax) {
              // exact tie: the reference keeps the later lag (Iterator::max_by)
              if (lag_of(code) > lag_of(cmax)) cmax = code;
            }
            cmax = pw > pmax ? code : cmax;
            pmax = fmaxf(pw, pmax);
            // kept in place for the second peak: the stage read its inputs
            // from these positions into registers before any output
            if (keep_top) reinterpret_cast<float*>(buf)[2 * (s * LC + G::offset(a, b, c))] = pw;
          } else {
            const int tau = seq_of(s) + S * G::natural(a, b, c);
            int d = tau - tau_star;
            d = d < 0 ? -d : d;
            const int dist = min(d, p.P - d);
            if (dist > p.chip_width) pbest = fmaxf(pbest, pw);
          }
        }
      };

      // ---- stage 1: DFT-31 over digit a, input straight from global ----
      for (int u = tid; u < BC * COLS; u += NT) {
        const int s = u / COLS, col = u - s * COLS;
        const int q = seq_of(s);
        if (q < 0) continue;
        float2 x[31];
        if (INV) {
          const float2* zs = p.z + ((size_t)ab_h * S + q) * LC + col;
          const float2* ds = p.D + ((size_t)prn * 2 + hyp) * LC + col;
#pragma unroll
          // Z is read once per (row, rho): keep it out of L1 so the code
          // spectrum D, reused by every rho of the row, stays there.
          for (int a = 0; a < 31; ++a) x[a] = cmul(__ldcg(zs + a * COLS), __ldg(ds + a * COLS));
        } else if (MODE == FWD_Z) {
          const float2* zs = p.z + (size_t)q * LC;
          const int c = col / 33, b = col - c * 33;
#pragma unroll
          for (int a = 0; a < 31; ++a) x[a] = zs[G::natural(a, b, c)];
        } else {
          const int pr = q >> 1, hb = q & 1;
          const int8_t* ch = p.chips + (size_t)pr * LC;
          const int c = col / 33, b = col - c * 33;
#pragma unroll
          for (int a = 0; a < 31; ++a) {
            const int n = G::natural(a, b, c);
            const float v = (float)__ldg(ch + n);
            if (hb) {
              double sn, cs;
              sincospi((double)n / (double)LC, &sn, &cs);
              x[a] = make_float2(v * (float)cs, v * (float)sn);
            } else {
              x[a] = make_float2(v, 0.f);
            }
          }
        }
        float2* dst = buf + s * LC + col;
        dft_odd<31, INV>(x, [&](int ta, float2 v) { dst[ta * COLS] = v; });
      }
      __syncthreads();

      // ---- stage 2: DFT-33 over digit b ----
      for (int u = tid; u < BC * 31 * NC; u += NT) {
        const int s = u / (31 * NC), r = u - s * 31 * NC;
        const int a = r / NC, c = r - a * NC;
        if (seq_of(s) < 0) continue;
        float2* base = buf + s * LC + a * COLS + c * 33;
        float2 x[33];
#pragma unroll
        for (int b = 0; b < 33; ++b) x[b] = base[b];
        if constexpr (NC == 1) {
          dft33<INV>(x, [&](int tb, float2 v) { epilogue(s, a, tb, 0, v); });
        } else {
          dft33<INV>(x, [&](int tb, float2 v) { base[tb] = v; });
        }
      }

      // ---- stage 3: DFT-M over digit c ----
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
          dft_small<NC, INV>(x, [&](int tc, float2 v) { epilogue(s, a, b, tc, v); });
        }
      }
      __syncthreads();
      // CAND with p2rows: the four largest |y|^2 of every residue of the
      // group (kept in place in buf) with their lags.  TOP_WPS warps scan a
      // residue; each takes the fourth largest of its lanes' maxima as a
      // lower bound on its four largest values, keeps per lane the four
      // largest values at or above it, and stores the warp's four largest.
      if (TOP && keep_top) {
        const int warp = tid >> 5, lane = tid & 31;
        const int sl = warp / TOP_WPS, sub = warp - sl * TOP_WPS;
        if (sl < BC && seq_of(sl) >= 0) {  // uniform over the warp
          const float* pws = reinterpret_cast<const float*>(buf + sl * LC);
          unsigned mb = 0u;
          for (int i = sub * 32 + lane; i < LC; i += TOP_WPS * 32) mb = max(mb, __float_as_uint(pws[2 * i]));
          unsigned thr = 0u;
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            thr = __reduce_max_sync(0xffffffffu, mb);
            const unsigned h = __ballot_sync(0xffffffffu, mb == thr);
            if (lane == __ffs(h) - 1) mb = 0u;
          }
          Top4 t;
          for (int i = sub * 32 + lane; i < LC; i += TOP_WPS * 32) {
            const float x = pws[2 * i];
            if (__float_as_uint(x) >= thr) t.add(x, i);
          }
          const int rho = seq_of(sl);
          unsigned long long* dst = s_res + ((size_t)rho * TOP_WPS + sub) * 4;
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const unsigned vb = __float_as_uint(t.v[0]);
            const unsigned x = __reduce_max_sync(0xffffffffu, vb);
            const unsigned h = __ballot_sync(0xffffffffu, vb == x);
            const int src = __ffs(h) - 1;
            const int i = __shfl_sync(0xffffffffu, t.i[0], src);
            if (lane == src) t.pop();
            if (lane == r) {
              unsigned long long k = 0ull;
              if (x != 0u) {
                const int a = i / COLS, rem = i - a * COLS, c = rem / 33, b = rem - c * 33;
                k = ((unsigned long long)x << 32) | (unsigned)(rho + S * G::natural(a, b, c));
              }
              dst[r] = k;
            }
          }
        }
        // the next group's stage 1 overwrites the values scanned here
        __syncthreads();
      }
      // tensor-core operands: FP16 units straight from the transformed
      // sequences in shared memory (the work of tc_pack_kernel, without
      // reading the FP32 spectra back from memory)
      if (MODE == FWD_Z && p.z16) {
        using U = TcUnits<M>;
        for (int e = tid; e < BC * U::PER_SEQ; e += NT) {
          const int s = e / U::PER_SEQ, r = e - s * U::PER_SEQ;
          const int q = seq_of(s);
          if (q < 0) continue;
          const uint2 m = __ldg(p.z16_map + r);
          const unsigned off[4] = {m.x & 0xffffu, m.x >> 16, m.y & 0xffffu, m.y >> 16};
          float2 v[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            v[i] = make_float2(0.f, 0.f);
            if (off[i] != 0xffffu) {
              v[i] = buf[s * LC + (int)off[i]];
              v[i].x *= p.z16_scale;
              v[i].y *= p.z16_scale;
            }
          }
          p.z16[(size_t)q * U::PER_SEQ + r] = pack_unit(v);
        }
        __syncthreads();
      }
    }

    if (ARGMAX) {
      unsigned long long kbest =
          pmax < 0.f ? 0ull : (((unsigned long long)__float_as_uint(pmax) << 32) | (unsigned)lag_of(cmax));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, kbest, o);
        kbest = other > kbest ? other : kbest;
      }
      if ((tid & 31) == 0) atomicMax(&s_key, kbest);
      __syncthreads();
      if (tid == 0) p.keys[key_at] = s_key;
      // CAND with p2rows: the row's second peak against its own maximum,
      // the largest |y|^2 more than chip_width lags (circularly) from it.
      // At most ceil((2 chip_width + 1) / S) <= 3 lags of a residue lie that
      // close, so the four largest of each residue (among the lists of the
      // warps that scanned it) hold it.
      if (TOP && keep_top && tid < 32) {
        const unsigned long long kb = s_key;
        const int tau_star = (int)(unsigned)kb;
        float p2 = 0.f;
        if (kb != 0ull)
          for (int e = tid; e < S * TOP_WPS * 4; e += 32) {
            const unsigned long long k = s_res[e];
            int d = (int)(unsigned)k - tau_star;
            d = d < 0 ? -d : d;
            if (k != 0ull && min(d, p.P - d) > p.chip_width) p2 = fmaxf(p2, __uint_as_float((unsigned)(k >> 32)));
          }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p2 = fmaxf(p2, __shfl_xor_sync(0xffffffffu, p2, o));
        if (tid == 0) p.p2rows[key_at] = p2;
      }
    } else if (MODE == SECOND) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) pbest = fmaxf(pbest, __shfl_xor_sync(0xffffffffu, pbest, o));
      if ((tid & 31) == 0) atomicMax(&s_p2, __float_as_uint(pbest));
      __syncthreads();
      if (tid == 0) p.best[w].p2 = __uint_as_float(s_p2);
    }
    __syncthreads();
  }
}

// Launch configurations: (third digit M, slots per CTA, threads, min CTAs/SM).
// Variant 0 is the default; variant 1 doubles the polyphase branches (slots)
// and threads of a CTA at one CTA per SM, so more branches of one (row, PRN)
// item share the code spectrum in L1.  The correlation modes take the
// variant of the class (PolyClass::variant, set by tga_set_variant or
// tga_autotune); the forward transforms always run variant 0.
template <int M, int V>
struct PfaCfg;
template <>
struct PfaCfg<1, 0> {
  static constexpr int BC = 8, NT = 288, MINB = 2;  // 8 x 33 DFT-31 columns
};
template <>
struct PfaCfg<1, 1> {
  static constexpr int BC = 16, NT = 576, MINB = 1;
};
template <>
struct PfaCfg<4, 0> {
  static constexpr int BC = 2, NT = 288, MINB = 2;  // 2 x 132 columns
};
template <>
struct PfaCfg<4, 1> {
  static constexpr int BC = 4, NT = 576, MINB = 1;
};
template <>
struct PfaCfg<10, 0> {
  static constexpr int BC = 1, NT = 352, MINB = 2;  // 330 columns
};
template <>
struct PfaCfg<10, 1> {
  static constexpr int BC = 2, NT = 704, MINB = 1;  // two rho slots share D in L1
};

template <int M, int V, int MODE>
static cudaError_t run_pfa(const PfaParams& p, int n_work_slots, int num_sms, cudaStream_t st) {
  using C = PfaCfg<M, V>;
  constexpr int LC = Geo<M>::LC;
  size_t smem = (size_t)C::BC * LC * sizeof(float2);
  // CAND with p2rows: the four largest |y|^2 per residue and scanning warp
  if (MODE == CAND && p.p2rows) {
    constexpr int WPS = C::NT / 32 / C::BC >= 1 ? C::NT / 32 / C::BC : 1;
    smem += (size_t)p.S * WPS * 4 * sizeof(unsigned long long);
  }
  auto kern = pfa_kernel<M, C::BC, C::NT, C::MINB, MODE>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::NT, smem);
  if (per_sm < 1) per_sm = 1;
  // FWD modes: n_work_slots counts sequences, grouped BC per work unit
  const int n_work = (MODE == FWD_Z || MODE == FWD_D) ? (n_work_slots + C::BC - 1) / C::BC : n_work_slots;
  int grid = num_sms * per_sm;
  if (grid > n_work) grid = n_work;
  if (grid < 1) return cudaSuccess;
  kern<<<grid, C::NT, smem, st>>>(p);
  return TGA_LAUNCHED();
}

template <int MODE>
static cudaError_t dispatch_pfa(const PolyClass& pc, const PfaParams& p, int n_work_slots, int num_sms,
                                cudaStream_t st) {
  if constexpr (MODE == CORR || MODE == SECOND || MODE == CAND) {
    if (pc.variant == 1) {
      switch (pc.M) {
        case 1: return run_pfa<1, 1, MODE>(p, n_work_slots, num_sms, st);
        case 4: return run_pfa<4, 1, MODE>(p, n_work_slots, num_sms, st);
        case 10: return run_pfa<10, 1, MODE>(p, n_work_slots, num_sms, st);
      }
      return cudaErrorInvalidValue;
    }
  }
  switch (pc.M) {
    case 1: return run_pfa<1, 0, MODE>(p, n_work_slots, num_sms, st);
    case 4: return run_pfa<4, 0, MODE>(p, n_work_slots, num_sms, st);
    case 10: return run_pfa<10, 0, MODE>(p, n_work_slots, num_sms, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_forward_z(const PolyClass& pc, int n_ab, float2* d_z, int num_sms, cudaStream_t st) {
  PfaParams p = {};
  p.z = d_z;
  p.n_seq = n_ab * 2 * pc.S;
  p.S = pc.S;
  p.P = pc.P;
  return dispatch_pfa<FWD_Z>(pc, p, p.n_seq, num_sms, st);
}

std::vector<uint16_t> tc_unit_map(int M) {
  auto build = [](auto u) {
    using U = decltype(u);
    std::vector<uint16_t> t((size_t)U::PER_SEQ * 4);
    for (int r = 0; r < U::PER_SEQ; ++r) {
      const int j = r / U::ROWS1, row = r - j * U::ROWS1, kp = U::row_part(row);
      for (int i = 0; i < 4; ++i) {
        const int d1 = 4 * j + i;
        t[(size_t)r * 4 + i] = d1 < 31 ? (uint16_t)U::src_offset(d1, kp) : (uint16_t)0xffffu;
      }
    }
    return t;
  };
  switch (M) {
    case 1: return build(TcUnits<1>());
    case 4: return build(TcUnits<4>());
    case 10: return build(TcUnits<10>());
  }
  return {};
}

cudaError_t launch_forward_z_tc(const PolyClass& pc, int n_ab, float2* d_z, void* d_z16, const void* d_map,
                                float z16_scale, int num_sms, cudaStream_t st) {
  PfaParams p = {};
  p.z = d_z;
  p.z16 = static_cast<uint4*>(d_z16);
  p.z16_map = static_cast<const uint2*>(d_map);
  p.z16_scale = z16_scale;
  p.n_seq = n_ab * 2 * pc.S;
  p.S = pc.S;
  p.P = pc.P;
  return dispatch_pfa<FWD_Z>(pc, p, p.n_seq, num_sms, st);
}

cudaError_t launch_forward_seqs_tc(const PolyClass& pc, long long n_seq, float2* d_z, void* d_z16, const void* d_map,
                                   float z16_scale, int num_sms, cudaStream_t st) {
  if (n_seq > 0x7fffffffLL) return cudaErrorInvalidValue;
  PfaParams p = {};
  p.z = d_z;
  p.z16 = static_cast<uint4*>(d_z16);
  p.z16_map = static_cast<const uint2*>(d_map);
  p.z16_scale = z16_scale;
  p.n_seq = (int)n_seq;
  p.S = pc.S;
  p.P = pc.P;
  return dispatch_pfa<FWD_Z>(pc, p, p.n_seq, num_sms, st);
}

cudaError_t launch_forward_seqs(const PolyClass& pc, long long n_seq, float2* d_z, int num_sms, cudaStream_t st) {
  if (n_seq > 0x7fffffffLL) return cudaErrorInvalidValue;
  PfaParams p = {};
  p.z = d_z;
  p.n_seq = (int)n_seq;
  p.S = pc.S;
  p.P = pc.P;
  return dispatch_pfa<FWD_Z>(pc, p, p.n_seq, num_sms, st);
}

cudaError_t launch_code_spectra(const PolyClass& pc, const int8_t* d_chips, int n_prn, float2* d_D,
                                int num_sms, cudaStream_t st) {
  PfaParams p = {};
  p.chips = d_chips;
  p.Dout = d_D;
  p.n_seq = n_prn * 2;
  p.S = pc.S;
  p.P = pc.P;
  return dispatch_pfa<FWD_D>(pc, p, p.n_seq, num_sms, st);
}

cudaError_t launch_correlate(const PolyClass& pc, const SearchDims& dims, const float2* d_Z,
                             const float2* d_D, unsigned long long* d_keys, int num_sms,
                             cudaStream_t st) {
  PfaParams p = {};
  p.z = const_cast<float2*>(d_Z);
  p.D = d_D;
  p.keys = d_keys;
  p.n_prn = dims.n_prn;
  p.S = pc.S;
  p.P = pc.P;
  p.n_items = dims.n_ant * dims.nb * 2 * dims.n_prn;
  return dispatch_pfa<CORR>(pc, p, p.n_items, num_sms, st);
}

cudaError_t launch_second_peak(const PolyClass& pc, const SearchDims& dims, const float2* d_Z,
                               const float2* d_D, BestRow* d_best, int chip_width, int num_sms,
                               cudaStream_t st) {
  PfaParams p = {};
  p.z = const_cast<float2*>(d_Z);
  p.D = d_D;
  p.best = d_best;
  p.n_prn = dims.n_prn;
  p.S = pc.S;
  p.P = pc.P;
  p.chip_width = chip_width;
  p.n_items = dims.n_ant * dims.n_prn;
  return dispatch_pfa<SECOND>(pc, p, p.n_items, num_sms, st);
}

cudaError_t launch_correlate_listed(const PolyClass& pc, const SearchDims& dims, const float2* d_Z,
                                    const float2* d_D, const int2* d_cand, const int* d_count, int capacity,
                                    unsigned long long* d_keys, int num_sms, cudaStream_t st, float* d_p2rows,
                                    int chip_width) {
  PfaParams p = {};
  p.p2rows = d_p2rows;
  p.chip_width = chip_width;
  p.z = const_cast<float2*>(d_Z);
  p.D = d_D;
  p.keys = d_keys;
  p.cand = d_cand;
  p.cand_count = d_count;
  p.n_prn = dims.n_prn;
  p.S = pc.S;
  p.P = pc.P;
  p.n_items = capacity;
  return dispatch_pfa<CAND>(pc, p, p.n_items, num_sms, st);
}

// The second peak of each cell from the re-evaluated rows: the cell's
// chosen row is always one of them (its FP32 key is the cell's maximum; when
// every key is 0, every row was listed).
__global__ void second_from_rows_kernel(int n_cells, int n_hyp, int n_prn, const float* __restrict__ p2rows,
                                        BestRow* __restrict__ best) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_cells) return;
  const BestRow b = best[w];
  best[w].p2 = p2rows[(size_t)(b.ab * n_hyp + b.hyp) * n_prn + (w % n_prn)];
}

cudaError_t launch_second_from_rows(const SearchDims& dims, int n_hyp, const float* d_p2rows, BestRow* d_best,
                                    cudaStream_t st) {
  const int n = dims.n_ant * dims.n_prn;
  if (n <= 0) return cudaSuccess;
  second_from_rows_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, n_hyp, dims.n_prn, d_p2rows, d_best);
  return TGA_LAUNCHED();
}

// Rows of a reduced-precision search to re-evaluate in FP32.  Per (antenna,
// PRN), with K the largest reduced-precision key of its 2 nb rows, every row
// whose key is at least keep * K is listed (keep * K = 0 lists all rows).
// If every row's amplitude error is at most e and keep = (1 - 2 e / sqrt(K))^2
// or less, the row holding the FP32 maximum is always listed: its key is at
// least (sqrt(V) - e)^2 with V the FP32 maximum, and sqrt(K) <= sqrt(V) + e.
// Rows not listed hold FP32 values below V, so the FP32 keys of the listed
// rows alone give the FP32 search's choice under the same tie rules.
// Rows are [ant][bin][hyp] with n_hyp hypotheses (2 in the drop-in search,
// 1 in the non-coherent one); a listed row is (its row index, prn).
__global__ void tc_candidates_kernel(int n_ant, int n_rows, int n_prn, const unsigned long long* __restrict__ keys,
                                     float keep, int2* __restrict__ cand, int* __restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_ant * n_prn) return;
  const int ant = i / n_prn, prn = i - ant * n_prn;
  const size_t row0 = (size_t)ant * n_rows;
  float kmax = 0.f;
  for (int r = 0; r < n_rows; ++r)
    kmax = fmaxf(kmax, __uint_as_float((unsigned)(keys[(row0 + r) * n_prn + prn] >> 32)));
  const float t = kmax * keep;
  for (int r = 0; r < n_rows; ++r)
    if (__uint_as_float((unsigned)(keys[(row0 + r) * n_prn + prn] >> 32)) >= t)
      cand[atomicAdd(count, 1)] = make_int2((int)(row0 + r), prn);
}

cudaError_t launch_tc_candidates(const SearchDims& dims, int n_hyp, const unsigned long long* d_keys, float keep,
                                 int2* d_cand, int* d_count, cudaStream_t st) {
  const int n = dims.n_ant * dims.n_prn;
  if (n <= 0) return cudaSuccess;
  tc_candidates_kernel<<<(n + 127) / 128, 128, 0, st>>>(dims.n_ant, dims.nb * n_hyp, dims.n_prn, d_keys, keep,
                                                        d_cand, d_count);
  return TGA_LAUNCHED();
}

// ---------------------------------------------------------------------------
// reduction over hypotheses and Doppler bins (correlate.rs:125-154)
// ---------------------------------------------------------------------------
__global__ void reduce_bins_kernel(int n_ant, int nb, int n_prn, const unsigned long long* __restrict__ keys,
                                   BestRow* __restrict__ best) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_ant * n_prn) return;
  const int ant = i / n_prn, prn = i - ant * n_prn;
  float pb = -1.f;
  unsigned long long kb = 0ull;
  int hb = 0, bb = 0;
  for (int bin = 0; bin < nb; ++bin) {
    const size_t ab = (size_t)ant * nb + bin;
    const unsigned long long ka = keys[(ab * 2 + 0) * n_prn + prn];
    const unsigned long long kB = keys[(ab * 2 + 1) * n_prn + prn];
    const float pa = __uint_as_float((unsigned)(ka >> 32)), pB = __uint_as_float((unsigned)(kB >> 32));
    // hypotheses: [c,-c] replaces [c,c] only when strictly stronger
    const bool useB = pB > pa;
    const float pr = useB ? pB : pa;
    // bins: Iterator::max_by keeps the last maximum
    if (bin == 0 || pr >= pb) {
      pb = pr;
      kb = useB ? kB : ka;
      hb = useB ? 1 : 0;
      bb = bin;
    }
  }
  BestRow r;
  r.ab = ant * nb + bb;
  r.hyp = hb;
  r.tau = (int)(unsigned)(kb & 0xffffffffull);
  r.p = pb;
  r.p2 = 0.f;
  best[i] = r;
}

cudaError_t launch_reduce_bins(const SearchDims& dims, const unsigned long long* d_keys, BestRow* d_best,
                               cudaStream_t st) {
  const int n = dims.n_ant * dims.n_prn;
  if (n <= 0) return cudaSuccess;
  reduce_bins_kernel<<<(n + 127) / 128, 128, 0, st>>>(dims.n_ant, dims.nb, dims.n_prn, d_keys, d_best);
  return TGA_LAUNCHED();
}

// ---------------------------------------------------------------------------
// ACR C/N0 (acr.rs:49-84) and result finalisation (acquisition.rs:237-247)
// ---------------------------------------------------------------------------
__constant__ double kAcrGps[59][2];
__constant__ double kAcrGal[71][2];
__constant__ double kAcrBds[79][2];
__constant__ double kAcrL1c[79][2];
// The tables are uploaded once per device, on the first call that needs them
// (with that device current).  Host threads making their first calls at
// once are serialised by the mutex; later calls only read the flag.
constexpr int kAcrMaxDevices = 64;
static std::atomic<bool> g_acr_uploaded[kAcrMaxDevices];
static std::mutex g_acr_mutex;

static cudaError_t upload_acr_tables() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const bool cached = dev >= 0 && dev < kAcrMaxDevices;
  if (cached && g_acr_uploaded[dev].load(std::memory_order_acquire)) return cudaSuccess;
  std::lock_guard<std::mutex> lock(g_acr_mutex);
  if (cached && g_acr_uploaded[dev].load(std::memory_order_relaxed)) return cudaSuccess;
  e = cudaMemcpyToSymbol(kAcrGps, TGA_GPS_L1_CA_ACR_TABLE, sizeof(kAcrGps));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(kAcrGal, TGA_GALILEO_E1C_ACR_TABLE, sizeof(kAcrGal));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(kAcrBds, TGA_BEIDOU_B1C_ACR_TABLE, sizeof(kAcrBds));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(kAcrL1c, TGA_GPS_L1C_ACR_TABLE, sizeof(kAcrL1c));
  if (e == cudaSuccess && cached) g_acr_uploaded[dev].store(true, std::memory_order_release);
  return e;
}

__device__ bool estimate_cn0_dev(double r_a, int table, double* out) {
  const double(*t)[2];
  int n;
  switch (table) {
    case 0: t = kAcrGps; n = 59; break;
    case 1: t = kAcrGal; n = 71; break;
    case 2: t = kAcrBds; n = 79; break;
    default: t = kAcrL1c; n = 79; break;
  }
  if (!(r_a > 1.0) || !isfinite(r_a)) return false;
  if (r_a <= t[0][0]) { *out = t[0][1]; return true; }
  if (r_a >= t[n - 1][0]) { *out = t[n - 1][1]; return true; }
  int lo = 0, hi = n;  // first index with r >= r_a
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (t[mid][0] < r_a) lo = mid + 1; else hi = mid;
  }
  if (lo == 0) { *out = t[0][1]; return true; }
  if (lo >= n) { *out = t[n - 1][1]; return true; }
  const double la = log(t[lo - 1][0]), lb = log(t[lo][0]);
  const double tt = (log(r_a) - la) / (lb - la);
  double v = t[lo - 1][1] + tt * (t[lo][1] - t[lo - 1][1]);
  v = v < 20.0 ? 20.0 : (v > 70.0 ? 70.0 : v);
  *out = v;
  return true;
}

__global__ void finalize_kernel(int n_cells, int nb, int n_prn, int P, int Lc, const double* __restrict__ fc,
                                double center, const BestRow* __restrict__ best, const int8_t* __restrict__ tables,
                                int want_cn0, CellOut* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_cells) return;
  const BestRow b = best[i];
  const double scale = sqrt(2.0 * (double)P) / (double)Lc;
  const float vm = (float)(sqrt((double)b.p) * scale);
  float vs = (float)(sqrt((double)fmaxf(b.p2, 0.f)) * scale);
  if (vs <= 0.f) vs = 1e-6f;  // correlate.rs:173-175
  const int bin = b.ab % nb;
  CellOut o;
  o.strength = (double)vm;
  o.second = (double)vs;
  o.codephase_frac = (double)b.tau / (double)P;
  o.frequency = fc[bin] - center;
  o.bin = bin;
  o.tau = b.tau;
  o.hyp = b.hyp;
  o.cn0 = 0.0;
  o.cn0_valid = 0;
  if (want_cn0) {
    const double m = o.strength, s = o.second;
    if (s > 0.0 && m > s) {
      const double q = m / s;
      double c;
      if (estimate_cn0_dev(q * q, tables[i % n_prn], &c)) {
        o.cn0 = c;
        o.cn0_valid = 1;
      }
    }
  }
  out[i] = o;
}

cudaError_t launch_finalize(const PolyClass& pc, const SearchDims& dims, const BestRow* d_best,
                            double center_freq, const int8_t* d_tables, int want_cn0, CellOut* d_out,
                            cudaStream_t st) {
  cudaError_t e = upload_acr_tables();
  if (e != cudaSuccess) return e;
  const int n = dims.n_ant * dims.n_prn;
  if (n <= 0) return cudaSuccess;
  finalize_kernel<<<(n + 127) / 128, 128, 0, st>>>(n, dims.nb, dims.n_prn, pc.P, pc.Lc, dims.fc,
                                                   center_freq, d_best, d_tables, want_cn0, d_out);
  return TGA_LAUNCHED();
}

__global__ void acr_batch_kernel(const double* __restrict__ ra, int n, int table, double* __restrict__ cn0,
                                 uint8_t* __restrict__ valid) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double c = 0.0;
  const bool ok = estimate_cn0_dev(ra[i], table, &c);
  cn0[i] = ok ? c : 0.0;
  valid[i] = ok ? 1 : 0;
}

cudaError_t launch_acr_batch(const double* d_ra, int n, int table, double* d_cn0, uint8_t* d_valid,
                             cudaStream_t st) {
  cudaError_t e = upload_acr_tables();
  if (e != cudaSuccess) return e;
  if (n <= 0) return cudaSuccess;
  acr_batch_kernel<<<(n + 255) / 256, 256, 0, st>>>(d_ra, n, table, d_cn0, d_valid);
  return TGA_LAUNCHED();
}

// ---------------------------------------------------------------------------
// antenna cross-correlation counts (observation.rs:175-195):
// counts[i*n+j] = number of samples where antennas i and j agree
// ---------------------------------------------------------------------------
__global__ void xcorr_kernel(const uint8_t* __restrict__ bits, int n_ant, size_t row_bytes,
                             unsigned long long* __restrict__ counts) {
  const int i = blockIdx.y, j = blockIdx.x;
  if (j < i) return;
  const uint8_t* a = bits + (size_t)i * row_bytes;
  const uint8_t* b = bits + (size_t)j * row_bytes;
  unsigned long long diff = 0;
  const bool aligned = ((((uintptr_t)a) | ((uintptr_t)b)) & 15) == 0;
  size_t done = 0;
  if (aligned) {
    const size_t nv = row_bytes / 16;
    const uint4* av = reinterpret_cast<const uint4*>(a);
    const uint4* bv = reinterpret_cast<const uint4*>(b);
    for (size_t k = threadIdx.x; k < nv; k += blockDim.x) {
      const uint4 x = __ldg(av + k), y = __ldg(bv + k);
      diff += __popc(x.x ^ y.x) + __popc(x.y ^ y.y) + __popc(x.z ^ y.z) + __popc(x.w ^ y.w);
    }
    done = nv * 16;
  }
  for (size_t k = done + threadIdx.x; k < row_bytes; k += blockDim.x) diff += __popc((unsigned)(a[k] ^ b[k]));
  for (int o = 16; o > 0; o >>= 1) diff += __shfl_xor_sync(0xffffffffu, diff, o);
  __shared__ unsigned long long part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = diff;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
    const unsigned long long agree = (unsigned long long)row_bytes * 8ull - t;
    counts[(size_t)i * n_ant + j] = agree;
    counts[(size_t)j * n_ant + i] = agree;
  }
}

cudaError_t launch_xcorr_matrix(const uint8_t* d_bits, int n_ant, size_t row_bytes, unsigned long long* d_counts,
                                cudaStream_t st) {
  if (n_ant <= 0) return cudaSuccess;
  xcorr_kernel<<<dim3(n_ant, n_ant), 256, 0, st>>>(d_bits, n_ant, row_bytes, d_counts);
  return TGA_LAUNCHED();
}

}  // namespace tga
