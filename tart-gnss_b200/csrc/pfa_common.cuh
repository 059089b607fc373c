// Shared definitions of the prime-factor transform kernels (FP32 SIMT and
// tensor-core variants).
#pragma once
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
  // position of output (a, b, c) in a row buffer of REFINE: the order in
  // which consecutive threads emit it ([b][a] for M = 1, whose last stage
  // runs per a; [a][c][b] otherwise)
  __device__ static __forceinline__ int row_pos(int a, int b, int c) { return M == 1 ? b * 31 + a : offset(a, b, c); }
};

// REFINE re-evaluates the selected row of each (antenna, PRN) in FP32 and
// rewrites its peak value and lag (used after a reduced-precision search).
enum PfaMode { FWD_Z = 0, FWD_D = 1, CORR = 2, SECOND = 3, REFINE = 4 };

struct PfaParams {
  float2* z;                  // FWD_Z: sequences, transformed in place; CORR/SECOND: Z
  const float2* D;            // CORR/SECOND: conjugated code spectra
  float2* Dout;               // FWD_D output
  const int8_t* chips;        // FWD_D input [n_prn][Lc]
  int n_seq;                  // FWD modes
  int n_items;                // CORR: n_ab*2*n_prn rows; SECOND: n_ant*n_prn
  int n_prn, S, P, chip_width;
  unsigned long long* keys;   // CORR output, one per row
  BestRow* best;              // SECOND in/out
  float* rowbuf;              // REFINE (optional): |y|^2 of each item's row, [item][rho][row_pos]
};

}  // namespace tga
