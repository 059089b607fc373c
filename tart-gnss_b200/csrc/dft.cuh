// Register-resident small DFTs used by the prime-factor transforms.
//
// All transforms are unnormalised:  forward X[k] = sum_n x[n] e^{-2 pi i nk/R},
// inverse uses e^{+2 pi i nk/R}.  Outputs are streamed to a store functor
// st(k, value) as soon as they are ready, so the inputs and the outputs of a
// DFT are never live in registers at the same time.
//
//  * odd prime R (3, 5, 11, 31): symmetric split into s_n = x_n + x_{R-n} and
//    d_n = x_n - x_{R-n}; each output pair (k, R-k) costs (R-1) real FMAs per
//    component, issued as packed FP32 pairs (re, im): 2*((R-1)/2)^2 + O(R)
//    instructions per R points.
//  * 33 = 3 x 11 and 10 = 2 x 5 as Good-Thomas prime-factor maps (no twiddles):
//    input digit map n = (N2*n1 + N1*n2) mod N, output map by the Chinese
//    remainder theorem.
//  * 4 as a radix-2 x 2 butterfly.
#pragma once
#include <cuda_runtime.h>

#include "dft_consts.cuh"

namespace tga {

// Complex adds use the packed FP32 instructions of sm_100 (one instruction
// for the real and imaginary parts; per component the same rounding as the
// scalar operation, so results are bit-identical to the scalar forms).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// sin and cos of the f32 carrier phase ph (the reference's `(p * f) as f32`,
// correlate.rs:110-115), rounded to f32 from double-precision values: ph / 2pi
// = n + t with 1/2pi as a two-term double (the product's rounding error
// recovered with an FMA), |t| <= 1/2, then sincospi(2 t) in double.  The
// reduced turn is exact to ~1e-20, so the f32 results are the correctly
// rounded sin / cos except within ~1e-16 of a rounding boundary, and the cost
// does not grow with |ph| (carrier phases reach ~5e5 rad over 20 ms).
__device__ __forceinline__ void sincos_phase(float ph, float* sn, float* cs) {
  constexpr double kInv2PiHi = 0x1.45f306dc9c883p-3;   // 1/2pi rounded to double
  constexpr double kInv2PiLo = -0x1.6b01ec5417056p-57;  // 1/2pi - kInv2PiHi
  const double x = (double)ph;
  const double th = x * kInv2PiHi;
  const double tl = fma(x, kInv2PiHi, -th) + x * kInv2PiLo;
  const double t = (th - rint(th)) + tl;
  double s, c;
  sincospi(2.0 * t, &s, &c);
  *sn = (float)s;
  *cs = (float)c;
}

template <int R> __device__ __forceinline__ float kcos(int m);
template <int R> __device__ __forceinline__ float ksin(int m);
template <> __device__ __forceinline__ float kcos<3>(int m) { return kCos3[m]; }
template <> __device__ __forceinline__ float ksin<3>(int m) { return kSin3[m]; }
template <> __device__ __forceinline__ float kcos<5>(int m) { return kCos5[m]; }
template <> __device__ __forceinline__ float ksin<5>(int m) { return kSin5[m]; }
template <> __device__ __forceinline__ float kcos<11>(int m) { return kCos11[m]; }
template <> __device__ __forceinline__ float ksin<11>(int m) { return kSin11[m]; }
template <> __device__ __forceinline__ float kcos<31>(int m) { return kCos31[m]; }
template <> __device__ __forceinline__ float ksin<31>(int m) { return kSin31[m]; }
// the same constants as (v, v) pairs
template <int R> __device__ __forceinline__ float2 kcos2(int m);
template <int R> __device__ __forceinline__ float2 ksin2(int m);
template <> __device__ __forceinline__ float2 kcos2<3>(int m) { return kCos3x2[m]; }
template <> __device__ __forceinline__ float2 ksin2<3>(int m) { return kSin3x2[m]; }
template <> __device__ __forceinline__ float2 kcos2<5>(int m) { return kCos5x2[m]; }
template <> __device__ __forceinline__ float2 ksin2<5>(int m) { return kSin5x2[m]; }
template <> __device__ __forceinline__ float2 kcos2<11>(int m) { return kCos11x2[m]; }
template <> __device__ __forceinline__ float2 ksin2<11>(int m) { return kSin11x2[m]; }
template <> __device__ __forceinline__ float2 kcos2<31>(int m) { return kCos31x2[m]; }
template <> __device__ __forceinline__ float2 ksin2<31>(int m) { return kSin31x2[m]; }

// DFT of odd prime length R; input x[0..R-1] (read only), outputs via st.
template <int R, bool INV, class St>
__device__ __forceinline__ void dft_odd(const float2 (&x)[R], St&& st) {
  constexpr int H = (R - 1) / 2;
  float2 s[H], d[H];
#pragma unroll
  for (int n = 1; n <= H; ++n) {
    s[n - 1] = cadd(x[n], x[R - n]);
    d[n - 1] = csub(x[n], x[R - n]);
  }
  const float2 x0 = x[0];
  float2 X0 = x0;
#pragma unroll
  for (int n = 0; n < H; ++n) X0 = cadd(X0, s[n]);
  st(0, X0);
#pragma unroll
  for (int k = 1; k <= H; ++k) {
    float2 A = x0;
    float2 B = make_float2(0.f, 0.f);
#pragma unroll
    for (int n = 1; n <= H; ++n) {
      const int m = (n * k) % R;
      const float c = kcos<R>(m), sn = ksin<R>(m);
      A.x = fmaf(s[n - 1].x, c, A.x);
      A.y = fmaf(s[n - 1].y, c, A.y);
      B.x = fmaf(d[n - 1].x, sn, B.x);
      B.y = fmaf(d[n - 1].y, sn, B.y);
    }
    // forward: X[k] = A - iB, X[R-k] = A + iB; inverse swaps them.
    const float2 lo = make_float2(A.x + B.y, A.y - B.x);
    const float2 hi = make_float2(A.x - B.y, A.y + B.x);
    if (!INV) {
      st(k, lo);
      st(R - k, hi);
    } else {
      st(k, hi);
      st(R - k, lo);
    }
  }
}

// 33 = 3 x 11.  Input digits: n = (11 n1 + 3 n2) mod 33; output k = (22 k1 + 12 k2) mod 33.
template <bool INV, class St>
__device__ __forceinline__ void dft33(const float2 (&x)[33], St&& st) {
  float2 u[3][11];
#pragma unroll
  for (int n2 = 0; n2 < 11; ++n2) {
    const float2 t[3] = {x[(3 * n2) % 33], x[(11 + 3 * n2) % 33], x[(22 + 3 * n2) % 33]};
    dft_odd<3, INV>(t, [&](int k1, float2 v) { u[k1][n2] = v; });
  }
#pragma unroll
  for (int k1 = 0; k1 < 3; ++k1) {
    dft_odd<11, INV>(u[k1], [&](int k2, float2 v) { st((22 * k1 + 12 * k2) % 33, v); });
  }
}

// 10 = 2 x 5.  Input digits: n = (5 n1 + 2 n2) mod 10; output k = (5 k1 + 6 k2) mod 10.
template <bool INV, class St>
__device__ __forceinline__ void dft10(const float2 (&x)[10], St&& st) {
  float2 u[2][5];
#pragma unroll
  for (int n2 = 0; n2 < 5; ++n2) {
    const float2 a = x[(2 * n2) % 10], b = x[(5 + 2 * n2) % 10];
    u[0][n2] = cadd(a, b);
    u[1][n2] = csub(a, b);
  }
#pragma unroll
  for (int k1 = 0; k1 < 2; ++k1) {
    dft_odd<5, INV>(u[k1], [&](int k2, float2 v) { st((5 * k1 + 6 * k2) % 10, v); });
  }
}

template <bool INV, class St>
__device__ __forceinline__ void dft4(const float2 (&x)[4], St&& st) {
  const float2 a = cadd(x[0], x[2]), b = csub(x[0], x[2]);
  const float2 c = cadd(x[1], x[3]), d = csub(x[1], x[3]);
  st(0, cadd(a, c));
  st(2, csub(a, c));
  // forward: X1 = b - i d, X3 = b + i d
  const float2 bmid = make_float2(b.x + d.y, b.y - d.x);
  const float2 bpid = make_float2(b.x - d.y, b.y + d.x);
  st(1, INV ? bpid : bmid);
  st(3, INV ? bmid : bpid);
}

template <bool INV, class St>
__device__ __forceinline__ void dft2(const float2 (&x)[2], St&& st) {
  st(0, cadd(x[0], x[1]));
  st(1, csub(x[0], x[1]));
}

// DFT of length M in {1, 2, 4, 10} (the third prime-factor digit).
template <int M, bool INV, class St>
__device__ __forceinline__ void dft_small(const float2 (&x)[M], St&& st) {
  if constexpr (M == 1) {
    st(0, x[0]);
  } else if constexpr (M == 2) {
    dft2<INV>(x, st);
  } else if constexpr (M == 4) {
    dft4<INV>(x, st);
  } else if constexpr (M == 10) {
    dft10<INV>(x, st);
  } else {
    static_assert(M == 1 || M == 2 || M == 4 || M == 10, "unsupported third digit");
  }
}

}  // namespace tga
