// Shared definitions of the prime-factor transform kernels (FP32 SIMT and
// tensor-core variants).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.h"

namespace tga {

constexpr int modinv_c(int a, int m) {
  a %= m;
  for (int x = 1; x < m; ++x)
    if ((a * x) % m == 1) return x;
  return 0;
}

// Geometry of the Lc = 31 * 33 * M prime-factor transform.
template <int M>
struct Geo {
  static constexpr int NC = M;
  static constexpr int COLS = 33 * M;  // columns of the DFT-31 stage
  static constexpr int LC = 31 * COLS;
  // natural index n = (a*EA + b*EB + c*EC) mod LC for digits (a, b, c)
  static constexpr int EA = (LC / 31) * modinv_c((LC / 31) % 31, 31);
  static constexpr int EB = (LC / 33) * modinv_c((LC / 33) % 33, 33);
  static constexpr int EC = (M == 1) ? 0 : (LC / M) * modinv_c((LC / M) % M, M);
  __device__ static __forceinline__ int natural(int a, int b, int c) {
    return (int)((unsigned)(a * EA + b * EB + c * EC) % (unsigned)LC);
  }
  // digit-layout offset of (a, b, c): [a][c][b]
  __device__ static __forceinline__ int offset(int a, int b, int c) { return a * COLS + c * 33 + b; }
};

// FP16 operands of the tensor-core search in its (31, R2, R3) frequency
// layout (Lc = 31 R2 R3; (R2, R3) = (33, 1), (12, 11), (30, 11) for M = 1,
// 4, 10).  Unit (seq, j, u), u = d3 R2 + d2, holds the spectrum at digits
// (d1, d2, d3), d1 = 4j .. 4j + 3 (zero for d1 >= 31), as 4 half2 (16
// bytes) split into real and imaginary parts: (re0, re1), (re2, re3),
// (im0, im1), (im2, im3) (pack_unit), so that the products of two units
// take four packed FP16 operations per pair of values and need no
// repacking; the stage-1 operand rows keep this order of their K entries
// and the stage-1 DFT matrix is built for it.  A frequency digit d of radix R stands for the natural
// frequencies k = d (LC / R) (mod R); src_offset is where the FP32 engine's
// digit layout [a][c][b] of the (31, 33, M) map holds the same frequency.
__device__ __forceinline__ uint4 pack_unit(const float2 (&v)[4]) {
  const __half2 a = __floats2half2_rn(v[0].x, v[1].x), b = __floats2half2_rn(v[2].x, v[3].x);
  const __half2 c = __floats2half2_rn(v[0].y, v[1].y), d = __floats2half2_rn(v[2].y, v[3].y);
  return make_uint4(*reinterpret_cast<const uint32_t*>(&a), *reinterpret_cast<const uint32_t*>(&b),
                    *reinterpret_cast<const uint32_t*>(&c), *reinterpret_cast<const uint32_t*>(&d));
}

template <int M>
struct TcUnits {
  static constexpr int R2 = M == 1 ? 33 : M == 4 ? 12 : 30, R3 = M == 1 ? 1 : 11;
  static constexpr int LC = 1023 * M, ROWS1 = R2 * R3, PER_SEQ = 8 * ROWS1;
  static constexpr int E1 = (LC / 31) * modinv_c((LC / 31) % 31, 31);
  static constexpr int E2 = (LC / R2) * modinv_c((LC / R2) % R2, R2);
  static constexpr int E3 = (LC / R3) * modinv_c((LC / R3) % R3, R3);
  static constexpr int UB = modinv_c((LC / 33) % 33, 33);
  static constexpr int UC = M == 1 ? 0 : modinv_c((LC / M) % M, M);
  __host__ __device__ static constexpr int freq_part(int d, int R, int E) { return ((d * (LC / R)) % R) * E; }
  // frequency contribution of the (d2, d3) digits of stage-1 row u
  __host__ __device__ static __forceinline__ int row_part(int u) {
    const int d3 = u / R2, d2 = u - d3 * R2;
    return freq_part(d2, R2, E2) + freq_part(d3, R3, E3);
  }
  // digit-layout offset [a][c][b] of slot d1 (< 31) of a row with row_part kp
  __host__ __device__ static __forceinline__ int src_offset(int d1, int kp) {
    const int k = (freq_part(d1, 31, E1) + kp) % LC;
    const int kb = (UB * k) % 33, kc = M == 1 ? 0 : (UC * k) % M;
    return d1 * 33 * M + kc * 33 + kb;
  }
};

// The four largest (value, index) pairs seen by a thread, largest first;
// values are non-negative |y|^2 (as bits they order like unsigned
// integers), an empty place holds 0.
struct Top4 {
  float v[4] = {0.f, 0.f, 0.f, 0.f};
  int i[4] = {0, 0, 0, 0};
  __device__ __forceinline__ void add(float x, int k) {
    if (!(x > v[3])) return;
    const bool g0 = x > v[0], g1 = x > v[1], g2 = x > v[2];
    v[3] = g2 ? v[2] : x;
    i[3] = g2 ? i[2] : k;
    v[2] = g1 ? v[1] : (g2 ? x : v[2]);
    i[2] = g1 ? i[1] : (g2 ? k : i[2]);
    v[1] = g0 ? v[0] : (g1 ? x : v[1]);
    i[1] = g0 ? i[0] : (g1 ? k : i[1]);
    v[0] = g0 ? x : v[0];
    i[0] = g0 ? k : i[0];
  }
  __device__ __forceinline__ void pop() {
    v[0] = v[1], i[0] = i[1];
    v[1] = v[2], i[1] = i[2];
    v[2] = v[3], i[2] = i[3];
    v[3] = 0.f;
  }
};

// CAND is CORR over a device-built list of rows (the candidates of a
// reduced-precision search, re-evaluated in FP32): row i of the list is
// (ab * 2 + hyp, prn), the list holds *cand_count rows, and each row's key
// goes where CORR would write it.
enum PfaMode { FWD_Z = 0, FWD_D = 1, CORR = 2, SECOND = 3, CAND = 4 };

struct PfaParams {
  float2* z;                  // FWD_Z: sequences, transformed in place; CORR/SECOND: Z
  const float2* D;            // CORR/SECOND: conjugated code spectra
  float2* Dout;               // FWD_D output
  const int8_t* chips;        // FWD_D input [n_prn][Lc]
  int n_seq;                  // FWD modes
  int n_items;                // CORR: n_ab*2*n_prn rows; SECOND: n_ant*n_prn; CAND: list capacity
  int n_prn, S, P, chip_width;
  unsigned long long* keys;   // CORR / CAND output, one per row ([ab * 2 + hyp][prn])
  BestRow* best;              // SECOND in/out
  const int2* cand;           // CAND: the rows to evaluate
  const int* cand_count;      // CAND: their number (device)
  float* p2rows;              // CAND (optional): each listed row's second peak
                              // against its own maximum, where its key goes
  uint4* z16;                 // FWD_Z (optional): the transformed sequences also as TcUnits, x z16_scale
  const uint2* z16_map;       // per unit: the 4 src_offset values as 16-bit fields (0xffff: zero)
  float z16_scale;
};

}  // namespace tga
