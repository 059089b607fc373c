// Non-coherent search: coherent blocks of K code periods, |y|^2 summed over
// B blocks before the peak search (the weak-signal mode of the engine).
//
// The drop-in search (correlate.rs:91-183) correlates one two-period window.
// This mode extends it the usual way for weak signals: block b covers
// samples [start + b K P, start + (b+1) K P); its K periods are wiped off by
// the exact carrier phase from the block start (the sign convention of
// correlate.rs:110-115), folded into one period (a cyclic correlation with the periodic code), split
// into the S polyphase residues and transformed like the drop-in Z; the
// correlator multiplies by the code spectrum, inverts, and adds |y|^2 of
// every block into a shared-memory accumulator before it takes the maximum
// (last maximum in lag order) or, for the selected bin, the second peak at a
// circular distance of more than one chip.  Doppler bins are a centred grid
// center + (i - (nb - 1) / 2) step; the last maximum over bins wins.
#include <cuda_runtime.h>

#include <cstdint>

#include "dft.cuh"
#include "engine.h"
#include "pfa_common.cuh"

namespace tga {

namespace {

struct NcFrontParams {
  SampleSource src;
  const double* fc;
  int nb, P, S, Lc, K, B;
  long long start;
  float pulse[kMaxPulse];
  // pulse shape: 0 any, 1 constant w0, 2 w0 for the first S / 2 samples and
  // -w0 for the rest; 1 and 2 let the polyphase sums run
  int pulse_kind;
  float pulse_w0;
  float2* z;
};

constexpr int kNcJ = 256;  // chips per CTA: at S = 16, two groups of eight folded samples per thread

// bit n of the row (1 for a + sample)
__device__ __forceinline__ int sample_bit(const uint8_t* __restrict__ row_bits, long long n) {
  return (__ldg(row_bits + (n >> 3)) >> (7 - (int)(n & 7))) & 1;
}

// exp(+i 2 pi t) for a turn count t given in double precision: the turn is
// reduced to [-1/2, 1/2] in double, the phasor computed in f32
__device__ __forceinline__ float2 phasor_turns(double t) {
  float s, c;
  sincospif((float)(2.0 * (t - rint(t))), &s, &c);
  return make_float2(c, s);
}

// Block b of K periods starting at n0 is wiped off by exp(+i 2 pi f (n - n0)
// / fs) and folded into one period.  With the exact (linear) phase the fold
// factors: x(m) = exp(i phi(m)) sum_k s(n0 + k P + m) exp(i phi(k P)), so a
// folded sample costs K real-by-complex FMAs and one phasor.
__global__ void __launch_bounds__(256) nc_frontend_kernel(NcFrontParams p) {
  extern __shared__ float2 fsm[];
  const int S = p.S, P = p.P, Lc = p.Lc;
  const int ab = blockIdx.y / p.B, blk = blockIdx.y - ab * p.B;
  const int ant_slot = ab / p.nb, bin = ab - ant_slot * p.nb;
  const int row = p.src.ant[ant_slot];
  const double f = p.fc[bin];
  const double turns_per_sample = f * p.src.pc / 6.283185307179586;  // f / fs
  const long long n0 = p.start + (long long)blk * p.K * P;
  const int j0 = blockIdx.x * kNcJ;
  const int nj = min(kNcJ, Lc - j0);
  const int cnt = nj * S + S - 1;
  const int span = kNcJ * S + S;
  float2* rot = fsm + span + span / S + 1;  // exp(i phi(k P)), k < K
  float2* step = rot + p.K;                 // exp(i phi(j)), j < 8
  for (int k = threadIdx.x; k < p.K + 8; k += blockDim.x)
    rot[k] = k < p.K ? phasor_turns(turns_per_sample * (double)k * (double)P)
                     : phasor_turns(turns_per_sample * (double)(k - p.K));
  // the two sample values (+-1 - mean) as f32 (acquisition.rs:281-294)
  const double mean = __ldg(p.src.mean + row);
  const float s_one = (float)(1.0 - mean), s_zero = (float)(-1.0 - mean);
  const uint8_t* row_bits = p.src.bits + (size_t)row * p.src.row_bytes;
  const long long row_bits_n = (long long)p.src.row_bytes * 8;
  __syncthreads();
  // folded sample i (period position m = S j0 + i, mod P) at fsm[i + i / S]
  auto store = [&](int i, float2 v) { fsm[i + i / S] = v; };
  // eight consecutive folded samples per thread: one 16-bit window of each
  // period holds all eight bits
  for (int i0 = 8 * threadIdx.x; i0 < cnt; i0 += 8 * blockDim.x) {
    int m0 = S * j0 + i0;
    if (m0 >= P) m0 -= P;  // the folded block is P-periodic
    if (m0 + 7 < P) {
      float2 acc[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[j] = make_float2(0.f, 0.f);
#pragma unroll 5
      for (int k = 0; k < p.K; ++k) {
        const long long n = n0 + (long long)k * P + m0;
        const long long byte = n >> 3;
        unsigned w = (unsigned)__ldg(row_bits + byte) << 8;
        if (((byte + 1) << 3) < row_bits_n) w |= __ldg(row_bits + byte + 1);
        w <<= (int)(n & 7);  // sample n + j is bit 15 - j
        const float2 r = rot[k];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const float sv = (w >> (15 - j)) & 1u ? s_one : s_zero;
          acc[j].x = fmaf(sv, r.x, acc[j].x);
          acc[j].y = fmaf(sv, r.y, acc[j].y);
        }
      }
      const float2 ph0 = phasor_turns(turns_per_sample * (double)m0);
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (i0 + j < cnt) store(i0 + j, cmul(acc[j], cmul(ph0, step[j])));
    } else {
      // the group straddles the end of the period: one sample at a time
      for (int j = 0; j < 8 && i0 + j < cnt; ++j) {
        int m = m0 + j;
        if (m >= P) m -= P;
        float2 acc = make_float2(0.f, 0.f);
        for (int k = 0; k < p.K; ++k) {
          const float sv = sample_bit(row_bits, n0 + (long long)k * P + m) ? s_one : s_zero;
          acc.x = fmaf(sv, rot[k].x, acc.x);
          acc.y = fmaf(sv, rot[k].y, acc.y);
        }
        store(i0 + j, cmul(acc, phasor_turns(turns_per_sample * (double)m)));
      }
    }
  }
  __syncthreads();
  const size_t seq0 = ((size_t)ab * p.B + blk) * S;
  if (p.pulse_kind != 0 && S >= 4) {
    // runs of S / 4 residues per thread, each sum from the previous one
    // (the drop-in front end's rule): with a = jj S + rho,
    //   constant w0:   z(rho + 1) = z(rho) + w0 (f[a + S] - f[a])
    //   w0 / -w0:      z(rho + 1) = z(rho) + w0 (2 f[a + S/2] - f[a] - f[a + S])
    const int L = (S + 3) / 4, H = S / 2;
    const float w0 = p.pulse_w0;
    const bool boc = p.pulse_kind == 2;
    for (int o = threadIdx.x; o < 4 * nj; o += blockDim.x) {
      const int k = o / nj, jj = o - k * nj;
      const int rho0 = k * L, rho1 = min(rho0 + L, S);
      if (rho0 >= S) continue;
      float2 z = make_float2(0.f, 0.f);
      const int base = jj * S + rho0 + jj;
      for (int s = 0; s < S; ++s) {
        const float2 v = fsm[base + s + (rho0 + s >= S ? 1 : 0)];
        const float w = p.pulse[s];
        z.x = fmaf(w, v.x, z.x);
        z.y = fmaf(w, v.y, z.y);
      }
      p.z[(seq0 + rho0) * Lc + j0 + jj] = z;
      for (int rho = rho0; rho + 1 < rho1; ++rho) {
        const int a = jj * S + rho;
        const float2 fa = fsm[a + jj], fe = fsm[a + S + jj + 1];
        if (boc) {
          const float2 fm = fsm[a + H + jj + (rho + H >= S ? 1 : 0)];
          z.x += w0 * (2.f * fm.x - fa.x - fe.x);
          z.y += w0 * (2.f * fm.y - fa.y - fe.y);
        } else {
          z.x += w0 * (fe.x - fa.x);
          z.y += w0 * (fe.y - fa.y);
        }
        p.z[(seq0 + rho + 1) * Lc + j0 + jj] = z;
      }
    }
    return;
  }
  for (int o = threadIdx.x; o < S * nj; o += blockDim.x) {
    const int rho = o / nj, jj = o - rho * nj;
    float2 z = make_float2(0.f, 0.f);
    // tap s reads sample i = jj S + rho + s at padded index i + i / S, and
    // i / S = jj + (rho + s >= S) since rho + s < 2 S: no division per tap
    const int base = jj * S + rho + jj;
    for (int s = 0; s < S; ++s) {
      const float2 v = fsm[base + s + (rho + s >= S ? 1 : 0)];
      const float w = p.pulse[s];
      z.x = fmaf(w, v.x, z.x);
      z.y = fmaf(w, v.y, z.y);
    }
    p.z[(seq0 + rho) * Lc + j0 + jj] = z;
  }
}

// NC_CAND: NC_PEAK over a device-built list of (ab, prn) rows (the
// candidates of a reduced-precision search, re-evaluated in FP32): the list
// holds *cand_count rows, each row's key goes where NC_PEAK would write it.
enum NcMode { NC_PEAK = 0, NC_SECOND = 1, NC_CAND = 2 };

struct NcParams {
  const float2* z;  // [n_ab][B][S][Lc], digit layout
  const float2* D;  // [n_prn][2][Lc]; the cyclic spectrum (index 0) is used
  int n_items, n_prn, S, P, B, chip_width;
  unsigned long long* keys;  // NC_PEAK, NC_CAND: [n_ab][n_prn]
  BestRow* best;             // NC_SECOND: [n_ant][n_prn]
  const int2* cand;          // NC_CAND: the rows
  const int* cand_count;     // NC_CAND: their number (device)
  float* p2rows;             // NC_CAND (optional): each row's second peak
                             // against its own maximum, where its key goes
};

template <int M, int BC, int NT, int MODE>
__global__ void __launch_bounds__(NT, 1) nc_correlate_kernel(NcParams p) {
  using G = Geo<M>;
  constexpr int COLS = G::COLS, LC = G::LC, NC = G::NC;
  extern __shared__ float2 buf[];
  float* acc = reinterpret_cast<float*>(buf + BC * LC);
  __shared__ unsigned long long s_key;
  __shared__ unsigned int s_p2;
  // NC_CAND with p2rows: for every residue and every warp that scanned it,
  // its four largest summed |y|^2 as (value bits << 32) | lag, after acc
  constexpr int TOP_WPS = NT / 32 / BC >= 1 ? NT / 32 / BC : 1;
  const bool keep_top = MODE == NC_CAND && p.p2rows != nullptr;
  unsigned long long* s_res = reinterpret_cast<unsigned long long*>(acc + BC * LC);
  const int tid = threadIdx.x, S = p.S;
  const int groups = (S + BC - 1) / BC;
  const int n_work = MODE == NC_CAND ? min(p.n_items, *p.cand_count) : p.n_items;
  for (int w = blockIdx.x; w < n_work; w += gridDim.x) {
    constexpr bool ARGMAX = MODE == NC_PEAK || MODE == NC_CAND;
    int ab, prn, tau_star = 0;
    if (MODE == NC_PEAK) {
      ab = w / p.n_prn;
      prn = w - ab * p.n_prn;
    } else if (MODE == NC_CAND) {
      const int2 c = p.cand[w];
      ab = c.x;
      prn = c.y;
    } else {
      const BestRow b = p.best[w];
      ab = b.ab;
      prn = w % p.n_prn;
      tau_star = b.tau;
    }
    if (tid == 0) {
      s_key = 0ull;
      s_p2 = 0u;
    }
    unsigned long long kbest = 0ull;
    float pbest = 0.f;
    for (int g = 0; g < groups; ++g) {
      auto seq_of = [&](int s) -> int {
        const int rho = g * BC + s;
        return rho < S ? rho : -1;
      };
      for (int i = tid; i < BC * LC; i += NT) acc[i] = 0.f;
      __syncthreads();
      auto accumulate = [&](int s, int a, int b, int c, float2 v) {
        acc[s * LC + G::offset(a, b, c)] += fmaf(v.x, v.x, v.y * v.y);
      };
      for (int blk = 0; blk < p.B; ++blk) {
        // stage 1: products and DFT-31 over digit a
        for (int u = tid; u < BC * COLS; u += NT) {
          const int s = u / COLS, col = u - s * COLS;
          const int q = seq_of(s);
          if (q < 0) continue;
          const float2* zs = p.z + (((size_t)ab * p.B + blk) * S + q) * LC + col;
          const float2* ds = p.D + (size_t)prn * 2 * LC + col;
          float2 x[31];
#pragma unroll
          for (int a = 0; a < 31; ++a) x[a] = cmul(__ldcg(zs + a * COLS), __ldg(ds + a * COLS));
          float2* dst = buf + s * LC + col;
          dft_odd<31, true>(x, [&](int ta, float2 v) { dst[ta * COLS] = v; });
        }
        __syncthreads();
        // stage 2: DFT-33 over digit b
        for (int u = tid; u < BC * 31 * NC; u += NT) {
          const int s = u / (31 * NC), r = u - s * 31 * NC;
          const int a = r / NC, c = r - a * NC;
          if (seq_of(s) < 0) continue;
          float2* base = buf + s * LC + a * COLS + c * 33;
          float2 x[33];
#pragma unroll
          for (int b = 0; b < 33; ++b) x[b] = base[b];
          if constexpr (NC == 1) {
            dft33<true>(x, [&](int tb, float2 v) { accumulate(s, a, tb, 0, v); });
          } else {
            dft33<true>(x, [&](int tb, float2 v) { base[tb] = v; });
          }
        }
        // stage 3: DFT-M over digit c
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
            dft_small<NC, true>(x, [&](int tc, float2 v) { accumulate(s, a, b, tc, v); });
          }
        }
        __syncthreads();
      }
      // the accumulated powers of this group's residues
      for (int i = tid; i < BC * LC; i += NT) {
        const int s = i / LC, off = i - s * LC;
        const int q = seq_of(s);
        if (q < 0) continue;
        const int a = off / COLS, rem = off - a * COLS;
        const int c = rem / 33, b = rem - c * 33;
        const int lag = q + S * G::natural(a, b, c);
        const float pw = acc[i];
        if (ARGMAX) {
          const unsigned long long k = ((unsigned long long)__float_as_uint(pw) << 32) | (unsigned)lag;
          kbest = k > kbest ? k : kbest;  // ties: the later lag (Iterator::max_by)
        } else {
          int d = lag - tau_star;
          d = d < 0 ? -d : d;
          if (min(d, p.P - d) > p.chip_width) pbest = fmaxf(pbest, pw);
        }
      }
      // NC_CAND with p2rows: the four largest sums of every residue of the
      // group with their lags (as the drop-in search's re-evaluation does:
      // a warp's fourth largest lane maximum bounds its four largest from
      // below)
      if (keep_top) {
        const int warp = tid >> 5, lane = tid & 31;
        const int sl = warp / TOP_WPS, sub = warp - sl * TOP_WPS;
        if (sl < BC && seq_of(sl) >= 0) {  // uniform over the warp
          const float* pws = acc + sl * LC;
          unsigned mb = 0u;
          for (int i = sub * 32 + lane; i < LC; i += TOP_WPS * 32) mb = max(mb, __float_as_uint(pws[i]));
          unsigned thr = 0u;
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            thr = __reduce_max_sync(0xffffffffu, mb);
            const unsigned h = __ballot_sync(0xffffffffu, mb == thr);
            if (lane == __ffs(h) - 1) mb = 0u;
          }
          Top4 t;
          for (int i = sub * 32 + lane; i < LC; i += TOP_WPS * 32) {
            const float x = pws[i];
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
      }
      __syncthreads();
    }
    if (ARGMAX) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, kbest, o);
        kbest = other > kbest ? other : kbest;
      }
      if ((tid & 31) == 0) atomicMax(&s_key, kbest);
      __syncthreads();
      if (tid == 0) p.keys[(size_t)ab * p.n_prn + prn] = s_key;
      // NC_CAND with p2rows: the row's second peak against its own maximum
      // (at most three lags of a residue lie within chip_width of it)
      if (keep_top && tid < 32) {
        const unsigned long long kb = s_key;
        const int tau = (int)(unsigned)kb;
        float p2 = 0.f;
        if (kb != 0ull)
          for (int e = tid; e < S * TOP_WPS * 4; e += 32) {
            const unsigned long long k = s_res[e];
            int d = (int)(unsigned)k - tau;
            d = d < 0 ? -d : d;
            if (k != 0ull && min(d, p.P - d) > p.chip_width) p2 = fmaxf(p2, __uint_as_float((unsigned)(k >> 32)));
          }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p2 = fmaxf(p2, __shfl_xor_sync(0xffffffffu, p2, o));
        if (tid == 0) p.p2rows[(size_t)ab * p.n_prn + prn] = p2;
      }
    } else {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) pbest = fmaxf(pbest, __shfl_xor_sync(0xffffffffu, pbest, o));
      if ((tid & 31) == 0) atomicMax(&s_p2, __float_as_uint(pbest));
      __syncthreads();
      if (tid == 0) p.best[w].p2 = __uint_as_float(s_p2);
    }
    __syncthreads();
  }
}

template <int M>
struct NcCfg;
template <>
struct NcCfg<1> {
  static constexpr int BC = 8, NT = 288;
};
template <>
struct NcCfg<4> {
  static constexpr int BC = 2, NT = 288;
};
template <>
struct NcCfg<10> {
  static constexpr int BC = 1, NT = 352;
};

template <int M, int MODE>
cudaError_t run_nc(const NcParams& p, int num_sms, cudaStream_t st) {
  using C = NcCfg<M>;
  constexpr int LC = Geo<M>::LC;
  size_t smem = (size_t)C::BC * LC * (sizeof(float2) + sizeof(float));
  if (MODE == NC_CAND && p.p2rows) {
    constexpr int WPS = C::NT / 32 / C::BC >= 1 ? C::NT / 32 / C::BC : 1;
    smem += (size_t)p.S * WPS * 4 * sizeof(unsigned long long);
  }
  auto kern = nc_correlate_kernel<M, C::BC, C::NT, MODE>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::NT, smem);
  if (per_sm < 1) per_sm = 1;
  int grid = num_sms * per_sm;
  if (grid > p.n_items) grid = p.n_items;
  if (grid < 1) return cudaSuccess;
  kern<<<grid, C::NT, smem, st>>>(p);
  kernel_launch_add(1);
  return cudaGetLastError();
}

template <int MODE>
cudaError_t dispatch_nc(int M, const NcParams& p, int num_sms, cudaStream_t st) {
  switch (M) {
    case 1: return run_nc<1, MODE>(p, num_sms, st);
    case 4: return run_nc<4, MODE>(p, num_sms, st);
    case 10: return run_nc<10, MODE>(p, num_sms, st);
  }
  return cudaErrorInvalidValue;
}

// per (antenna, PRN): the last bin with the largest accumulated peak
__global__ void nc_reduce_kernel(int n_ant, int nb, int n_prn, const unsigned long long* __restrict__ keys,
                                 BestRow* __restrict__ best) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_ant * n_prn) return;
  const int ant = i / n_prn, prn = i - ant * n_prn;
  float pb = -1.f;
  unsigned long long kb = 0ull;
  int bb = 0;
  for (int bin = 0; bin < nb; ++bin) {
    const unsigned long long k = keys[((size_t)ant * nb + bin) * n_prn + prn];
    const float pr = __uint_as_float((unsigned)(k >> 32));
    if (bin == 0 || pr >= pb) {
      pb = pr;
      kb = k;
      bb = bin;
    }
  }
  BestRow r;
  r.ab = ant * nb + bb;
  r.hyp = 0;
  r.tau = (int)(unsigned)(kb & 0xffffffffull);
  r.p = pb;
  r.p2 = 0.f;
  best[i] = r;
}

}  // namespace

cudaError_t launch_nc_frontend(const SampleSource& src, const SearchDims& dims, const PolyClass& pc, int K, int B,
                               long long start, float2* d_z, cudaStream_t st) {
  NcFrontParams p;
  p.src = src;
  p.fc = dims.fc;
  p.nb = dims.nb;
  p.P = pc.P;
  p.S = pc.S;
  p.Lc = pc.Lc;
  p.K = K;
  p.B = B;
  p.start = start;
  for (int i = 0; i < kMaxPulse; ++i) p.pulse[i] = pc.pulse[i];
  // the pulse's shape (see NcFrontParams)
  p.pulse_w0 = pc.pulse[0];
  bool constant = true, boc = pc.S % 2 == 0;
  for (int i = 0; i < pc.S; ++i) {
    constant = constant && pc.pulse[i] == pc.pulse[0];
    boc = boc && pc.pulse[i] == (i < pc.S / 2 ? pc.pulse[0] : -pc.pulse[0]);
  }
  p.pulse_kind = constant ? 1 : (boc ? 2 : 0);
  p.z = d_z;
  const int span = kNcJ * pc.S + pc.S;
  const size_t smem = (size_t)(span + span / pc.S + 1 + K + 8) * sizeof(float2);
  const long long gy = (long long)dims.n_ant * dims.nb * B;
  if (gy > 65535) return cudaErrorInvalidValue;
  dim3 grid((pc.Lc + kNcJ - 1) / kNcJ, (unsigned)gy);
  cudaError_t e = cudaFuncSetAttribute(nc_frontend_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  nc_frontend_kernel<<<grid, 256, smem, st>>>(p);
  kernel_launch_add(1);
  return cudaGetLastError();
}

cudaError_t launch_nc_correlate(const PolyClass& pc, const SearchDims& dims, int B, const float2* d_z,
                                const float2* d_D, unsigned long long* d_keys, int num_sms, cudaStream_t st) {
  NcParams p = {};
  p.z = d_z;
  p.D = d_D;
  p.keys = d_keys;
  p.n_prn = dims.n_prn;
  p.S = pc.S;
  p.P = pc.P;
  p.B = B;
  p.n_items = dims.n_ant * dims.nb * dims.n_prn;
  return dispatch_nc<NC_PEAK>(pc.M, p, num_sms, st);
}

cudaError_t launch_nc_reduce(const SearchDims& dims, const unsigned long long* d_keys, BestRow* d_best,
                             cudaStream_t st) {
  const int n = dims.n_ant * dims.n_prn;
  if (n <= 0) return cudaSuccess;
  nc_reduce_kernel<<<(n + 127) / 128, 128, 0, st>>>(dims.n_ant, dims.nb, dims.n_prn, d_keys, d_best);
  kernel_launch_add(1);
  return cudaGetLastError();
}

cudaError_t launch_nc_second(const PolyClass& pc, const SearchDims& dims, int B, const float2* d_z,
                             const float2* d_D, BestRow* d_best, int chip_width, int num_sms, cudaStream_t st) {
  NcParams p = {};
  p.z = d_z;
  p.D = d_D;
  p.best = d_best;
  p.n_prn = dims.n_prn;
  p.S = pc.S;
  p.P = pc.P;
  p.B = B;
  p.chip_width = chip_width;
  p.n_items = dims.n_ant * dims.n_prn;
  return dispatch_nc<NC_SECOND>(pc.M, p, num_sms, st);
}

cudaError_t launch_nc_correlate_listed(const PolyClass& pc, const SearchDims& dims, int B, const float2* d_z,
                                       const float2* d_D, const int2* d_cand, const int* d_count, int capacity,
                                       unsigned long long* d_keys, int num_sms, cudaStream_t st, float* d_p2rows,
                                       int chip_width) {
  NcParams p = {};
  p.p2rows = d_p2rows;
  p.chip_width = chip_width;
  p.z = d_z;
  p.D = d_D;
  p.keys = d_keys;
  p.cand = d_cand;
  p.cand_count = d_count;
  p.n_prn = dims.n_prn;
  p.S = pc.S;
  p.P = pc.P;
  p.B = B;
  p.n_items = capacity;
  return dispatch_nc<NC_CAND>(pc.M, p, num_sms, st);
}

}  // namespace tga
