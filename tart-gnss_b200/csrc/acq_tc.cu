// Tensor-core correlator (sm_100a, tcgen05): reduced-precision search.
//
// The inverse transform of every product Z * conj(C) (length Lc = 31 R2 R3,
// (R2, R3) = (33, 1), (12, 11), (30, 11) for Lc = 1023, 4092, 10230) is a
// Good-Thomas prime-factor transform whose stages -- DFT-31, DFT-R2 and, for
// R3 > 1, DFT-R3 -- all run on the 5th-generation tensor cores as GEMMs:
//
//   stage i:  D_i[row][n] = sum_k A_i[row][k] * B_i[n][k]
//     A_i   = data, one row per transform column, K = 2 R_i halves
//             (R_i complex FP16 inputs as interleaved (re, im)), K-major
//     B_i   = the inverse DFT-R_i as a real 2R_i x 2R_i matrix, FP16
//     D_i   = FP32 accumulator in tensor memory (TMEM), one lane per row.
//
// Between stages the warps read D_i from TMEM (tcgen05.ld 32x32b), round it
// to FP16 and scatter it into the next stage's operand rows; this is the
// transposition of the prime-factor map.  The last stage's accumulator is
// read straight into the |y|^2 maximum, so no intermediate leaves the SM.
// The products are formed in FP16 (HMUL2/HFMA2) from FP16 copies of Z and
// conj(C) in a frequency layout matched to the (31, R2, R3) map
// (tc_pack_kernel), and a CTA keeps its Z in registers for all PRNs, so the
// search reads only the code spectra from L2.
//
// Scaling: Z and conj(C) are stored as Z 2^-kz and conj(C) 2^-kd with
// kz + kd = k and 4 S Lc^2 2^-k <= 32768.  Then |Z 2^-kz| <= 4 S Lc 2^-kz and
// |C 2^-kd| <= Lc 2^-kd stay inside FP16, every product is below 32768 and so
// is every correlation value; stage outputs are rounded with satfinite.
// Keys carry the row maximum of |y|^2 2^-2k (the lag bits are zero) and are
// only compared: every row of an (antenna, PRN) whose key lies within the
// FP16 error bound of its best is re-evaluated in FP32 afterwards
// (launch_tc_candidates, launch_correlate_listed), so the chosen row, and
// the reported peak, lag and second peak, are those of the FP32 search.
//
// One CTA per SM (all 512 TMEM columns) runs two PRN chains over the Z of a
// (row, group of BC code-phase residues) work item, so that the tensor cores
// work on one chain while the warps transpose the other; one dedicated warp
// per chain issues its MMAs.  Every wait is bounded (1 s): on expiry the kernel sets
// *err, drains (again bounded), frees its TMEM and returns.
//
// The same kernel (NCB) runs the non-coherent search: the two chains take
// consecutive coherent blocks of one PRN (BLKCH), the Z of each block is
// loaded into the registers in turn, and the |y|^2 of the blocks are summed
// in the free TMEM columns before the row maximum.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

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
// The same test with a suspend-time hint: a thread whose phase has not
// completed sleeps until it completes or `ns` nanoseconds pass, instead of
// returning at once to poll again, so waiting warps leave their
// sub-partition's issue slots to the warps that work.
__device__ __forceinline__ uint32_t mbar_try_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t ns) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity), "r"(ns)
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
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// bulk copy global -> this CTA's shared memory, completing `bytes` of the
// barrier's transaction count (both addresses 16-byte aligned, bytes % 16 == 0)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
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

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
}
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr)
               : "memory");
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
               "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
               : "memory");
}
__device__ __forceinline__ void tmem_st4(uint32_t taddr, const uint32_t (&r)[4]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(r[0]), "r"(r[1]),
               "r"(r[2]), "r"(r[3])
               : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
// Reads 16 N16 TMEM columns of this warp's 32 lanes starting at taddr and
// waits once.
template <int N16>
__device__ __forceinline__ void tmem_ld_cols(uint32_t taddr, uint32_t (&v)[16 * N16]) {
#pragma unroll
  for (int c = 0; c < N16; ++c) {
    uint32_t(&r)[16] = *reinterpret_cast<uint32_t(*)[16]>(&v[16 * c]);
    tmem_ld16(taddr + 16 * c, r);
  }
  tmem_wait_ld();
}

// K-major layouts of the DFT matrices with the 128-byte (KB = 128) or
// 64-byte (KB = 64) swizzle: rows of KB bytes, 8-row groups of 8 KB bytes;
// the 16-byte chunk j of row r is stored at chunk j ^ (r & 7) (128B) or
// j ^ ((r >> 1) & 3) (64B).
template <int KB>
struct Lay {
  static_assert(KB == 128 || KB == 64, "layout");
  __host__ __device__ static __forceinline__ uint32_t off(int r, int j) {
    if (KB == 128) return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((j ^ (r & 7)) << 4));
    return (uint32_t)((r >> 3) * 512 + (r & 7) * 64 + ((j ^ ((r >> 1) & 3)) << 4));
  }
  // shared-memory matrix descriptor (sm_100, version 1): start address,
  // stride between 8-row groups, swizzle mode 2 (128B) or 4 (64B)
  __device__ static __forceinline__ uint64_t desc(uint32_t addr) {
    const uint64_t mode = KB == 128 ? 2 : 4;
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)((8 * KB) >> 4) << 32) |
           ((uint64_t)1 << 46) | (mode << 61);
  }
};

// Data operands use the un-swizzled K-major layout with every row 16 bytes
// from the next inside a column of 8-half (16-byte) K chunks and chunk
// columns lbo = rows * 16 + 16 bytes apart: byte(r, chunk c) = r * 16 + c * lbo.
// Any store pattern is then affine in the row index, and the 16-byte pad
// puts chunk c of a row 4 banks after chunk c - 1, so a warp writing one
// row's K entries hits 32 different banks.
__device__ __forceinline__ uint64_t desc_kchunks(uint32_t addr, uint32_t lbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) | ((uint64_t)(128 >> 4) << 32) |
         ((uint64_t)1 << 46);
}

// instruction descriptor: kind::f16, A = B = FP16, D = FP32, K-major, M = 128
constexpr uint32_t idesc_f16(int n) { return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24); }
constexpr int pad16(int x) { return (x + 15) / 16 * 16; }
constexpr int cmax3(int a, int b, int c) { return a > b ? (a > c ? a : c) : (b > c ? b : c); }

constexpr int kSimtWarps = 12;  // a multiple of the 4 TMEM lane quadrants
constexpr int kSimtThreads = 32 * kSimtWarps;
// and the two warps that issue the tensor-core work (one per chain), and
// the warp that fetches the code blocks
constexpr int kTcThreads = kSimtThreads + 96;
constexpr int kTcTmemCols = 512;
constexpr long long kWaitPolls = 1LL << 22;
constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s per wait on the tensor cores
constexpr uint32_t kSuspendNs = 20000;                  // longest sleep of one test (20 us)

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// polls the mbarrier phase until it completes, at most kWaitPolls times and
// kWaitNs nanoseconds; after the first test each one may sleep up to
// kSuspendNs (woken when the phase completes), so the bound is on the timer
__device__ __forceinline__ uint32_t bounded_wait(uint64_t* bar, uint32_t phase) {
  uint32_t done = mbar_try_wait(bar, phase);
  if (done) return done;  // the common case reads no timer
  const unsigned long long t0 = globaltimer_ns();
  for (long long k = 0; k < kWaitPolls && !done; ++k) {
    done = mbar_try_wait_sleep(bar, phase, kSuspendNs);
    if (!done && (k & 7) == 7 && globaltimer_ns() - t0 > kWaitNs) break;
  }
  return done;
}

// factorisation Lc = 31 * R2 * R3 in NST stages (Lc = 1023 runs as the two
// stages 31 x 33, R3 = 1), the number of code-phase residues (transforms) a
// CTA runs together, the order of the stage-2 rows (S2O, see T3) and the
// padding of the K-chunk strides of stages 2 and 3 (16-byte units), chosen
// for the fewest shared-memory bank conflicts of the transposition stores
template <int M>
struct Tc3Cfg;
template <>
struct Tc3Cfg<1> {
  static constexpr int R2 = 33, R3 = 1, NST = 2, BC = 8, PAD2 = 1, PAD3 = 1;
  static constexpr bool S2O = false, PADR1 = false, T1F3 = false;
};
template <>
struct Tc3Cfg<4> {
  static constexpr int R2 = 12, R3 = 11, NST = 3, BC = 2, PAD2 = 3, PAD3 = 1;
  static constexpr bool S2O = true, PADR1 = false, T1F3 = true;
};
template <>
struct Tc3Cfg<10> {
  static constexpr int R2 = 30, R3 = 11, NST = 3, BC = 1, PAD2 = 1, PAD3 = 1;
  static constexpr bool S2O = true, PADR1 = true, T1F3 = false;
};

// NCB: the non-coherent search (Lc = 1023 only), with |y|^2 sums in shared
// memory
template <int M, bool NCB = false>
struct T3 {
  static constexpr int R2 = Tc3Cfg<M>::R2, R3 = Tc3Cfg<M>::R3, BC = Tc3Cfg<M>::BC;
  static constexpr int LC = 1023 * M, OCOLS = 33 * M;
  static constexpr int NST = Tc3Cfg<M>::NST;
  static_assert(31 * R2 * R3 == LC, "factorisation");
  static_assert(TcUnits<M>::R2 == R2 && TcUnits<M>::R3 == R3, "FP16 operand units of the forward transform");
  static_assert(NST == 2 ? R3 == 1 : R3 == 11, "the epilogue reads 22 TMEM columns per stage-3 transform");
  // With R2 even the stage-3 transforms (t1, 2j) and (t1, 2j + 1) share one
  // operand row: K entries [0, 2 R3) and [P3OFF, P3OFF + 2 R3), against a
  // block-diagonal DFT-R3 matrix whose outputs land in accumulator columns
  // [0, 2 R3) and [P3OFF, P3OFF + 2 R3).
  static constexpr bool PAIR3 = NST == 3 && R2 % 2 == 0;
  static constexpr int P3OFF = 24;
  static_assert(2 * R3 <= P3OFF, "paired stage-3 halves");
  // rows (transform columns) of each stage for one residue.  Stage-2 row
  // (t1, d3) is t1 R3 + d3, or with S2O ((d3 / 4) 32 + t1) 4 + d3 % 4 (384
  // rows, some of them padding): a warp then holds 8 consecutive t1 x 4
  // values of d3 % 4, whose stage-3 stores fall in 32 different banks
  static constexpr bool S2O = Tc3Cfg<M>::S2O;
  static_assert(!S2O || R3 <= 12, "S2O: three groups of four d3");
  static constexpr int ROWS1 = R2 * R3, ROWS2 = S2O ? 384 : 31 * R3, ROWS3 = 31 * R2;
  static constexpr int ROWS3P = NST == 2 ? 0 : PAIR3 ? ROWS3 / 2 : ROWS3;  // stage-3 operand rows
  // T1F3: the paired stage-3 row of (t1, j = t2 / 2) is j 31 + t1 instead of
  // t1 R2 / 2 + j (any order serves: the epilogue only takes the maximum
  // over the rows); with S2O a warp's 8 consecutive t1 then store to 8
  // consecutive rows
  static constexpr bool T1F3 = Tc3Cfg<M>::T1F3;
  static_assert(!T1F3 || PAIR3, "T1F3: paired stage 3");
  // stage-1 operand rows of one residue.  With PADR1 the row of (d2, d3) is
  // 32 d3 + d2 (rows 32 d3 + R2 .. 32 d3 + 31 are padding, never written nor
  // read back): a warp's TMEM lanes then hold one d3 and its R2 values of
  // d2, whose stage-2 stores (K entries d2, chunks LBO2 apart with LBO2 / 16
  // odd) fall in 32 different banks.  Otherwise the rows are d3 R2 + d2.
  static constexpr bool PADR1 = Tc3Cfg<M>::PADR1;
  static_assert(!PADR1 || R2 <= 32, "PADR1: one warp of lanes per d3");
  static constexpr int ROWS1P = PADR1 ? 32 * R3 : ROWS1;
  // NR1 counts the product rows (units), NR1P the stage-1 operand rows
  static constexpr int NR1 = BC * ROWS1, NR1P = BC * ROWS1P, NR2 = BC * ROWS2, NR3 = BC * ROWS3P;
  static constexpr int TILES1 = (NR1P + 127) / 128, TILES2 = (NR2 + 127) / 128, TILES3 = (NR3 + 127) / 128;
  // stage-1 operand row of product row r (residue r / ROWS1)
  __device__ static __forceinline__ int arow1(int r) {
    if constexpr (PADR1) {
      const int s = r / ROWS1, u = r - s * ROWS1;
      const int d3 = u / R2;
      return s * ROWS1P + 32 * d3 + (u - d3 * R2);
    } else {
      return r;
    }
  }
  static constexpr int K1 = 64, K2 = pad16(2 * R2), K3 = NST == 2 ? 0 : PAIR3 ? 2 * P3OFF : pad16(2 * R3);
  static_assert(K2 <= 128 && K3 <= 64, "matrix rows of at most two (stage 2) or one swizzle atoms");
  static constexpr int N1 = K1, N2 = K2, N3 = K3;
  static constexpr int KB1 = 128, KB2 = K2 > 32 ? 128 : 64, KB3 = K3 > 32 ? 128 : 64;
  // the stage-2 matrix in atoms of KB2 / 2 K entries; a K step (16 entries)
  // never straddles two atoms
  static constexpr int B2_ATOMS = (K2 + KB2 / 2 - 1) / (KB2 / 2), KS_PER_ATOM2 = KB2 / 32;
  // TMEM columns of one chain (its largest stage); two chains per CTA
  static constexpr int CHAIN_COLS = cmax3(TILES1 * N1, TILES2 * N2, TILES3 * N3);
  static_assert(CHAIN_COLS <= kTcTmemCols / 2, "two chains in the CTA's TMEM");
  // the stage the epilogue reads: its tiles, rows per residue and in all,
  // complex outputs per row
  static constexpr int LAST_TILES = NST == 3 ? TILES3 : TILES2;
  static constexpr int LAST_ROWS = NST == 3 ? ROWS3P : ROWS2, LAST_NR = NST == 3 ? NR3 : NR2;
  static constexpr int LAST_OUT = NST == 3 ? R3 : R2;
  // Non-coherent search (NCB): the two chains run consecutive blocks of ONE
  // PRN (chain x takes block 2 i + x; "block chains", BLKCH), so one code
  // block and one set of |y|^2 sums serve both.  The sums live in the TMEM
  // columns the two chains' accumulators leave free, [CHAIN_COLS, 256) of
  // each half: every last-stage row (a lane) has SLOTS slots of 11 outputs
  // (the 33 stage-2 outputs, or the 2 x 11 outputs of a paired stage-3
  // row), 12 columns per slot; tile t, slot c at sum_col(t, c).  Their
  // read-modify-write then uses the TMEM path instead of the shared memory
  // the MMAs read their operands from, and two sets of sums (66 to 96
  // columns each) would not fit the 128 free columns.
  static constexpr bool BLKCH = NCB;
  static_assert(!NCB || (NST == 2 && LAST_OUT == 33) || (NST == 3 && PAIR3 && LAST_OUT == 11),
                "non-coherent epilogue layouts");
  static constexpr int SLOTS = NST == 2 ? 3 : 2, TILE_COLS = 12 * SLOTS;
  static constexpr int PER_RANGE = (kTcTmemCols / 2 - CHAIN_COLS) / TILE_COLS;
  static_assert(!NCB || LAST_TILES <= 2 * PER_RANGE, "the sums fit the free TMEM columns");
  static constexpr int N_CODE = BLKCH ? 1 : 2;
  __device__ static __forceinline__ uint32_t sum_col(int t, int c) {
    return (uint32_t)((t / PER_RANGE) * (kTcTmemCols / 2) + CHAIN_COLS + (t % PER_RANGE) * TILE_COLS + 12 * c);
  }
  // data operand regions: rows padded to whole tiles, K chunks lbo apart
  static constexpr int LBO1 = TILES1 * 128 * 16 + 16, LBO2 = TILES2 * 128 * 16 + 16 * Tc3Cfg<M>::PAD2,
                       LBO3 = TILES3 * 128 * 16 + 16 * Tc3Cfg<M>::PAD3;
  static constexpr int A_RAW = cmax3(K1 / 8 * LBO1, K2 / 8 * LBO2, K3 / 8 * LBO3);
  static constexpr int A_BYTES = (A_RAW + 1023) / 1024 * 1024;
  static constexpr int B1_BYTES = N1 * KB1, B2_BYTES = B2_ATOMS * N2 * KB2, B3_BYTES = N3 * KB3;
  static_assert(B1_BYTES % 1024 == 0 && B2_BYTES % 1024 == 0 && B3_BYTES % 1024 == 0, "1024-byte aligned regions");
  // one (PRN, hypothesis) block of code units: 8 ROWS1 x 16 bytes
  static constexpr int CODE_BYTES = 8 * ROWS1 * 16;
  static constexpr int CODE_REGION = (CODE_BYTES + 1023) / 1024 * 1024;
  // product units: (row, 16-byte chunk of 4 complex inputs); U per SIMT thread
  static constexpr int UNITS = NR1 * 8;
  static constexpr int U = (UNITS + kSimtThreads - 1) / kSimtThreads;
  static_assert(8 * ROWS1 < 65536 && 8 * LBO1 < 65536, "packed unit offsets");
  static constexpr int SMEM_RAW =
      2 * A_BYTES + B1_BYTES + B2_BYTES + B3_BYTES + N_CODE * CODE_REGION + 1024;
  // more than half of the SM's shared memory: one CTA, and so one 512-column
  // TMEM allocation, per SM
  static constexpr int SMEM = SMEM_RAW > 120 * 1024 ? SMEM_RAW : 120 * 1024;
  static_assert(SMEM <= 227 * 1024, "shared memory");
  // CRT output map of the (31, R2, R3) transform: lag digits -> natural index
  static constexpr int E1 = (LC / 31) * modinv_c((LC / 31) % 31, 31);
  static constexpr int E2 = (LC / R2) * modinv_c((LC / R2) % R2, R2);
  static constexpr int E3 = (LC / R3) * modinv_c((LC / R3) % R3, R3);
  __device__ static __forceinline__ int natural(int t1, int t2, int t3) {
    return (int)((unsigned)(t1 * E1 + t2 * E2 + t3 * E3) % (unsigned)LC);
  }
  // frequency digits: digit d of radix R holds natural frequency k with
  // k = d (LC / R) (mod R); the (31, 33, M) layout of the FP32 engine follows
  // the same rule, so both hold X[k] under digits that differ only in R2/R3
  __device__ static __forceinline__ int freq_part(int d, int R, int E) { return ((d * (LC / R)) % R) * E; }
  static constexpr int UB = modinv_c((LC / 33) % 33, 33);
  static constexpr int UC = M == 1 ? 0 : modinv_c((LC / M) % M, M);
};

__device__ __forceinline__ uint32_t h2_bits(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }
__device__ __forceinline__ __half2 bits_h2(uint32_t u) { return *reinterpret_cast<__half2*>(&u); }
// round two FP32 values to FP16, clamping to +-65504 instead of overflowing
__device__ __forceinline__ uint32_t pack_h2_sat(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}
// The products of two split units (pack_unit): c z for each of the four
// values, as a split unit, per pair (re, im) = (cr zr - ci zi, cr zi + ci zr)
// with the products cr zr and cr zi rounded first.
__device__ __forceinline__ uint4 cmul_unit(uint4 z, uint4 c) {
  const __half2 zr0 = bits_h2(z.x), zr1 = bits_h2(z.y), zi0 = bits_h2(z.z), zi1 = bits_h2(z.w);
  const __half2 cr0 = bits_h2(c.x), cr1 = bits_h2(c.y), ci0 = bits_h2(c.z), ci1 = bits_h2(c.w);
  return make_uint4(h2_bits(__hfma2(ci0, __hneg2(zi0), __hmul2(cr0, zr0))),
                    h2_bits(__hfma2(ci1, __hneg2(zi1), __hmul2(cr1, zr1))),
                    h2_bits(__hfma2(ci0, zr0, __hmul2(cr0, zi0))), h2_bits(__hfma2(ci1, zr1, __hmul2(cr1, zi1))));
}
__device__ __forceinline__ void st_shared_u32(unsigned char* p, uint32_t v) { *reinterpret_cast<uint32_t*>(p) = v; }

// inverse DFT-R as a real N x K matrix in layout KB, built on the host in
// double precision and rounded once to FP16: row n = 2 t + (0 re | 1 im),
// column k = 2 d + (0 re | 1 im), entries of exp(+2 pi i t d / R); zero
// outside 2R x 2R.  PAIR repeats the block at row and column offset `off`.
// `atom` selects the K entries [atom KB / 2, (atom + 1) KB / 2) written here.
// SPLIT: the K entries in the order of split units (pack_unit), column
// k = 8 (d / 4) + 4 (0 re | 1 im) + d % 4.
template <int R, int N, int KB, bool PAIR, bool SPLIT = false>
void host_idft_matrix(unsigned char* dst, int off, int atom = 0) {
  const double kPi = 3.14159265358979323846;
  for (int n = 0; n < N; ++n)
    for (int k = 0; k < KB / 2; ++k) {
      int nn = n, kk = k + atom * (KB / 2);
      if (SPLIT) kk = 2 * (4 * (kk >> 3) + (kk & 3)) + ((kk >> 2) & 1);  // to the interleaved order
      bool in = nn < 2 * R && kk < 2 * R;
      if (!in && PAIR && nn >= off && nn < off + 2 * R && kk >= off && kk < off + 2 * R) {
        nn -= off;
        kk -= off;
        in = true;
      }
      double val = 0.0;
      if (in) {
        const int t = nn >> 1, u = nn & 1, d = kk >> 1, v = kk & 1;
        const double ang = 2.0 * kPi * (double)((t * d) % R) / (double)R;
        const double c = std::cos(ang), sn = std::sin(ang);
        val = (u == 0) ? (v == 0 ? c : -sn) : (v == 0 ? sn : c);
      }
      const __half h = __float2half_rn((float)val);
      std::memcpy(dst + Lay<KB>::off(n, k >> 3) + (k & 7) * 2, &h, 2);
    }
}

// ---------------------------------------------------------------------------
// FP16 operands in the (31, R2, R3) frequency layout.  Unit (seq, j, u) with
// u = d3 R2 + d2 holds inputs d1 = 4j .. 4j+3 of stage-1 row u as 4 half2
// (16 bytes), for Z and for the code spectra alike.
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(256) tc_pack_kernel(const float2* __restrict__ src, uint4* __restrict__ dst,
                                                      long long n_units, float scale) {
  using T = T3<M>;
  constexpr int PER_SEQ = 8 * T::ROWS1;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n_units;
       e += (long long)gridDim.x * blockDim.x) {
    const long long seq = e / PER_SEQ;
    const int rem = (int)(e - seq * PER_SEQ);
    const int j = rem / T::ROWS1, u = rem - j * T::ROWS1;
    const int d3 = u / T::R2, d2 = u - d3 * T::R2;
    const int kpart = T::freq_part(d2, T::R2, T::E2) + T::freq_part(d3, T::R3, T::E3);
    const float2* s = src + seq * T::LC;
    float2 v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int d1 = 4 * j + i;
      v[i] = make_float2(0.f, 0.f);
      if (d1 < 31) {
        // the 31-digit is the same in both layouts: (31, 33, M) digit a = d1
        const int k = (T::freq_part(d1, 31, T::E1) + kpart) % T::LC;
        const int kb = (T::UB * k) % 33, kc = M == 1 ? 0 : (T::UC * k) % M;
        v[i] = __ldg(s + d1 * T::OCOLS + kc * 33 + kb);
        v[i].x *= scale;
        v[i].y *= scale;
      }
    }
    dst[e] = pack_unit(v);
  }
}

struct Tc3Params {
  const uint4* bmat;  // the three DFT matrices in their shared-memory layouts
  const uint4* z16;   // [n_ab*2][S] sequences of 8*ROWS1 units
  const uint4* d16;   // [n_prn][2] sequences of 8*ROWS1 units
  unsigned long long* keys;
  int* err;
  int n_items;  // n_ab * groups: (row, residue group) work items
  int groups;   // ceil(S / BC)
  // work units: item u / split, its PRN pairs [r0, r1) of part u % split
  // (split > 1 only when the items are fewer than the SMs)
  int split;
  int n_prn, S;
  int B;        // coherent blocks summed non-coherently (1: the drop-in search)
  int skip_commit;  // test hook: see TGA_TEST_TC_SKIP_COMMIT
};

// PRN pairs [first, end) of work unit u, of n_rounds pairs per item, with
// `split` units per item
__device__ __forceinline__ int unit_round0(int split, int u, int n_rounds) { return (u % split) * n_rounds / split; }
__device__ __forceinline__ int unit_round1(int split, int u, int n_rounds) {
  return (u % split + 1) * n_rounds / split;
}

// Reads the 22 accumulator columns of stage-3 transform `half` of this warp's
// lane quadrant at column taddr into v[0..21] (v[22], v[23] are padding).
template <bool PAIR3>
__device__ __forceinline__ void tmem_ld_stage3(uint32_t taddr, int half, uint32_t (&v)[24]) {
  uint32_t(&lo)[16] = *reinterpret_cast<uint32_t(*)[16]>(&v[0]);
  uint32_t(&lo8)[8] = *reinterpret_cast<uint32_t(*)[8]>(&v[0]);
  uint32_t(&hi8)[8] = *reinterpret_cast<uint32_t(*)[8]>(&v[16]);
  uint32_t(&hi16)[16] = *reinterpret_cast<uint32_t(*)[16]>(&v[8]);
  if (!PAIR3 || half == 0) {
    tmem_ld16(taddr, lo);
    tmem_ld8(taddr + 16, hi8);
  } else {
    tmem_ld8(taddr + 24, lo8);
    tmem_ld16(taddr + 32, hi16);
  }
}

// One CTA per SM.  A work item is one (antenna, bin, hypothesis) row and one
// group of BC code-phase residues; its Z stays in registers while the CTA
// runs two chains through the PRNs in pairs: chain x takes PRN 2 i + x (the
// last PRN twice when their number is odd; the key update is idempotent).
// Each chain has its own code block in shared memory, fetched for its next
// PRN with one bulk copy as soon as the chain's products are formed, by a
// warp of its own (s_p1[x]: the 12 SIMT warps have read the block for the
// last time), so that the MMA warps do nothing but wait, issue and commit.
// Per PRN pair:
//   SIMT warps:  P1(a) P1(b) P2(a) P2(b) P3(a) P3(b) P4(a) P4(b)
//   MMA warps:         M1(a) M1(b) M2(a) M2(b) M3(a) M3(b)
// where Mi(x) runs while the SIMT warps work on the other chain.  Hand-offs:
// s_ready[x] (arrivals of the 12 SIMT warps: chain x's operands are in
// shared memory and its accumulator has been read), s_done[x]
// (tcgen05.commit) and s_code[x] (bulk copy).  A tcgen05.mma holds its
// thread until the tensor cores take it, so issuing has warps of its own,
// one per chain.  Every wait is bounded.
//
// NCB (non-coherent search, block chains): the row is an (antenna, bin), a
// round is one PRN, whose blocks 2 i and 2 i + 1 run on chains a and b; one
// code block and one set of |y|^2 sums (in TMEM) serve both chains, and each
// thread takes the row maximum of its sums after the last block.  The Z of
// chain a's next block is loaded into the registers while the current
// transforms run, chain b's after chain a has formed its products.
// The code warp's thread: after the 12 SIMT warps have formed chain x's
// products of a PRN's last block (s_p1[x]), bulk-copy the chain's next code
// block into its slot (s_code[x]).  Its own function, so that its registers
// are allocated apart from the SIMT warps'.  The parameters it needs come
// as scalars: a reference to the kernel's parameter block would make the
// kernel copy the block to local memory and read every field from there.
template <class T, bool NCB>
__device__ __noinline__ void code_warp(const uint4* d16, int groups, int split_nc, int n_items, int n_prn, int* err,
                                       uint64_t* s_p1, uint64_t* s_code, unsigned char* CODE0, int n_rounds) {
  // the PRN of chain x in round r: PRN pairs, or with BLKCH one PRN per round
  auto prn_of = [&](int r, int x) -> int {
    if (T::BLKCH) return r;
    return 2 * r + x < n_prn ? 2 * r + x : n_prn - 1;
  };
  // bit x for barrier / slot x, in registers (the loops over x are not
  // unrolled; arrays indexed by x would live in local memory): the phase of
  // s_p1[x], the parity of the copies issued into slot x and whether any was
  uint32_t ph_p1 = 0u, fetch_par = 0u, fetch_any = 0u;
  bool ok = true;
  // code block of chain x for round r of work item w, into slot `slot`
  auto fetch = [&](int slot, int x, int w, int r) {
    const int hyp = NCB ? 0 : (w / groups) & 1;
    const uint4* src = d16 + ((size_t)prn_of(r, x) * 2 + hyp) * 8 * T::ROWS1;
    mbar_arrive_expect_tx(&s_code[slot], (uint32_t)T::CODE_BYTES);
    bulk_g2s(smem_addr(CODE0 + slot * T::CODE_REGION), src, (uint32_t)T::CODE_BYTES, &s_code[slot]);
    fetch_par ^= 1u << slot;
    fetch_any |= 1u << slot;
  };
  const int split = NCB ? split_nc : 1;  // the drop-in search always has enough items
  const int n_units = n_items * split;
  constexpr int NSLOT = T::BLKCH ? 1 : 2;
  if ((int)blockIdx.x < n_units && n_rounds > 0)
    for (int x = 0; x < NSLOT; ++x) fetch(x, x, blockIdx.x / split, unit_round0(split, blockIdx.x, n_rounds));
#pragma unroll 1
  for (int u = blockIdx.x; u < n_units && ok; u += gridDim.x) {
    const int w = u / split, r1 = unit_round1(split, u, n_rounds), un = u + (int)gridDim.x;
#pragma unroll 1
    for (int r = unit_round0(split, u, n_rounds); r < r1 && ok; ++r) {
      // BLKCH: the one slot is refilled once both chains have formed the
      // products of the PRN's last blocks
      if constexpr (T::BLKCH) {
        for (int x = 0; x < 2 && ok; ++x) {
          ok = bounded_wait(&s_p1[x], (ph_p1 >> x) & 1u) != 0;
          ph_p1 ^= 1u << x;
        }
        if (!ok) break;
        if (r + 1 < r1)
          fetch(0, 0, w, r + 1);
        else if (un < n_units)
          fetch(0, 0, un / split, unit_round0(split, un, n_rounds));
      } else {
#pragma unroll 1
        for (int x = 0; x < 2 && ok; ++x) {
          if (!bounded_wait(&s_p1[x], (ph_p1 >> x) & 1u)) {
            ok = false;
            break;
          }
          ph_p1 ^= 1u << x;
          if (r + 1 < r1)
            fetch(x, x, w, r + 1);
          else if (un < n_units)
            fetch(x, x, un / split, unit_round0(split, un, n_rounds));
        }
      }
    }
  }
  // drain: the last bulk copy of each slot
  for (int x = 0; x < NSLOT; ++x)
    if ((fetch_any >> x) & 1u) bounded_wait(&s_code[x], ((fetch_par >> x) & 1u) ^ 1u);
  if (!ok) atomicExch(err, 1);
}

template <int M, bool NCB>
__global__ void __launch_bounds__(kTcThreads, 1) pfa_tc3_kernel(Tc3Params p) {
  using T = T3<M, NCB>;
  constexpr int NW = kSimtWarps, NTS = kSimtThreads, R2 = T::R2, R3 = T::R3, BC = T::BC, U = T::U;
  static_assert(NW % 4 == 0, "a warp task keeps its TMEM lane quadrant");
  // TMEM columns read by one warp task in the transposition phases
  constexpr int CS1 = T::N1 / 32, CS2 = T::N2 >= 32 ? T::N2 / 32 : 1;
  constexpr int W2 = T::N2 >= 32 ? 32 : T::N2;
  constexpr int HALVES3 = T::PAIR3 ? 2 : 1;
  constexpr int NT2 = T::TILES1 * 4 * CS1, NT3 = T::TILES2 * 4 * CS2, NT4 = T::LAST_TILES * 4 * HALVES3;
  constexpr int TPW2 = (NT2 + NW - 1) / NW, TPW3 = (NT3 + NW - 1) / NW, TPW4 = (NT4 + NW - 1) / NW;
  // P2 / P3: the 12 warps cover the 4 lane quadrants of 3 tiles at a time
  static_assert(NW == 12 && T::TILES1 % 3 == 0 && (T::NST == 2 || T::TILES2 % 3 == 0), "P2/P3 task map");
  // P4 reads TMEM in batches of LB4 tasks: all loads of a batch in flight,
  // one wait
  constexpr int LB4 = TPW4 < 2 ? TPW4 : 2;
  constexpr int kBatch = (U + 1) / 2;
  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t s_ready[2], s_done[2], s_code[2], s_p1[2];
  __shared__ uint32_t s_tmem;
  const uint32_t raw = smem_addr(smem_raw);
  unsigned char* A0 = smem_raw + ((1024 - (raw & 1023)) & 1023);
  unsigned char* B1 = A0 + 2 * T::A_BYTES;
  unsigned char* B2 = B1 + T::B1_BYTES;
  unsigned char* B3 = B2 + T::B2_BYTES;
  unsigned char* CODE0 = B3 + T::B3_BYTES;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, quad = warp & 3;
  // rounds: PRN pairs, or with BLKCH single PRNs; steps of a round: one per
  // coherent block, or with BLKCH one per pair of blocks (chain x takes
  // block 2 i + x; a block index >= B, when B is odd, stands for zero data)
  const int S = p.S, n_rounds = T::BLKCH ? p.n_prn : (p.n_prn + 1) / 2, B = NCB ? p.B : 1;
  const int NI = T::BLKCH ? (B + 1) / 2 : B;
  const int split = NCB ? p.split : 1;  // the drop-in search always has enough items

  if (warp == 0) {
    tmem_alloc(&s_tmem, kTcTmemCols);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int x = 0; x < 2; ++x) {
      mbar_init(&s_ready[x], NW);
      mbar_init(&s_done[x], 1);
      mbar_init(&s_code[x], 1);
      mbar_init(&s_p1[x], NW);
    }
  }
  // operand rows and K entries that no stage writes (padding) must hold
  // finite values: they meet zeros of the DFT matrices
  for (int i = tid; i < 2 * T::A_BYTES / 16; i += kTcThreads) reinterpret_cast<uint4*>(A0)[i] = make_uint4(0u, 0u, 0u, 0u);
  constexpr int B_CHUNKS = (T::B1_BYTES + T::B2_BYTES + T::B3_BYTES) / 16;
  for (int i = tid; i < B_CHUNKS; i += kTcThreads) reinterpret_cast<uint4*>(B1)[i] = __ldg(p.bmat + i);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = s_tmem;
  // PRN of chain x in round r
  auto prn_of = [&](int r, int x) -> int {
    if (T::BLKCH) return r;
    return 2 * r + x < p.n_prn ? 2 * r + x : p.n_prn - 1;
  };

  if (warp == NW || warp == NW + 1) {
    // ---------------- MMA warps: one thread each issues one chain's tensor-core work ----------------
    // A thread's barrier test queues behind its own MMAs still waiting for
    // the tensor cores, so with one issuing thread the tensor cores idled
    // between stages; with one per chain (on different SM sub-partitions)
    // the other chain's stage is issued meanwhile.
    const int x = warp - NW;
    if (lane == 0) {
      const uint32_t a_addr = smem_addr(A0);
      const uint64_t db1 = Lay<T::KB1>::desc(smem_addr(B1));
      const uint64_t db2 = Lay<T::KB2>::desc(smem_addr(B2));
      const uint64_t db3 = Lay<T::KB3>::desc(smem_addr(B3));
      uint32_t ph_ready = 0u;
      int commits = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < p.n_items * split && ok; u += gridDim.x) {
        const int r1 = unit_round1(split, u, n_rounds);
        for (int r = unit_round0(split, u, n_rounds); r < r1 && ok; ++r) {
#pragma unroll 1
         for (int b = 0; b < NI && ok; ++b) {
#pragma unroll 1
          for (int st = 0; st < T::NST && ok; ++st) {
            {
              if (!bounded_wait(&s_ready[x], ph_ready)) {
                ok = false;
                break;
              }
              ph_ready ^= 1u;
              tc_fence_after();
              const uint32_t tm = tmem_base + (uint32_t)(x * (kTcTmemCols / 2));
              const uint32_t ax = a_addr + (uint32_t)(x * T::A_BYTES);
              // test hook (TGA_TEST_TC_SKIP_COMMIT): issue nothing, so the
              // SIMT warps' first wait runs out with no tensor-core work in
              // flight
              if (!p.skip_commit) {
                // fully unrolled: descriptors are the stage's base plus
                // constants (start-address field in 16-byte units; a tile of
                // 128 rows is 2048 bytes, a K step two chunks)
                if (st == 0) {
                  const uint64_t da = desc_kchunks(ax, T::LBO1);
#pragma unroll
                  for (int t = 0; t < T::TILES1; ++t)
#pragma unroll
                    for (int ks = 0; ks < T::K1 / 16; ++ks)
                      mma_f16(tm + (uint32_t)(t * T::N1), da + (uint64_t)(t * 128 + 2 * ks * (T::LBO1 >> 4)),
                              db1 + 2 * ks, idesc_f16(T::N1), ks > 0 ? 1u : 0u);
                } else if (st == 1) {
                  const uint64_t da = desc_kchunks(ax, T::LBO2);
#pragma unroll
                  for (int t = 0; t < T::TILES2; ++t)
#pragma unroll
                    for (int ks = 0; ks < T::K2 / 16; ++ks)
                      mma_f16(tm + (uint32_t)(t * T::N2), da + (uint64_t)(t * 128 + 2 * ks * (T::LBO2 >> 4)),
                              db2 + (uint64_t)((ks / T::KS_PER_ATOM2) * (T::N2 * T::KB2 >> 4) + 2 * (ks % T::KS_PER_ATOM2)),
                              idesc_f16(T::N2), ks > 0 ? 1u : 0u);
                } else {
                  const uint64_t da = desc_kchunks(ax, T::LBO3);
#pragma unroll
                  for (int t = 0; t < T::TILES3; ++t)
#pragma unroll
                    for (int ks = 0; ks < T::K3 / 16; ++ks)
                      mma_f16(tm + (uint32_t)(t * T::N3), da + (uint64_t)(t * 128 + 2 * ks * (T::LBO3 >> 4)),
                              db3 + 2 * ks, idesc_f16(T::N3), ks > 0 ? 1u : 0u);
                }
                mma_commit(&s_done[x]);
                ++commits;
              }
            }
          }
         }
        }
      }
      // drain: the chain's last commit (after a timeout it may still be in
      // flight)
      if (commits > 0) bounded_wait(&s_done[x], (uint32_t)((commits - 1) & 1));
      if (!ok) atomicExch(p.err, 1);
    }
    __syncwarp();
  } else if (warp == NW + 2) {
    // ---------------- code warp: one thread fetches the code blocks ----------------
    if (lane == 0) code_warp<T, NCB>(p.d16, p.groups, p.split, p.n_items, p.n_prn, p.err, s_p1, s_code, CODE0, n_rounds);
    __syncwarp();
  } else {
    // ---------------- SIMT warps ----------------
    const uint32_t lane_off = (uint32_t)(quad * 32) << 16;
    // product units of this thread: unit e = tid + k NTS is (row r, chunk j);
    // packed (code unit index << 16) | operand byte offset
    uint32_t uoff[U];
    // and, with BC > 1, the residue slot s < BC of each unit, 4 bits per
    // unit (the unit's Z offset in its item is s * 8 ROWS1 + its code-unit
    // index)
    uint32_t uslot = 0u;
    static_assert(U <= 8 && BC <= 16, "packed unit slots");
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int e = tid + k * NTS;
      const int j = e / T::NR1, r = e - j * T::NR1;
      const int sl = r / T::ROWS1, u = r - sl * T::ROWS1;
      uoff[k] = e < T::UNITS ? ((uint32_t)(j * T::ROWS1 + u) << 16) | (uint32_t)(T::arow1(r) * 16 + j * T::LBO1)
                             : 0u;
      if (BC > 1 && e < T::UNITS) uslot |= (uint32_t)sl << (4 * k);
    }
    // mbarrier phases, bit x for chain (or code slot) x: in registers (the
    // chain loops are not unrolled; arrays indexed by x would live in local
    // memory, and every wait would first load its phase from there)
    uint32_t ph_done = 0u, ph_code = 0u;
    bool failed = false;

    // bounded wait of the whole warp: every lane tests the phase (one
    // instruction for the warp when it has completed, the common case); a
    // warp that must wait polls until all its lanes have seen it complete
    auto warp_wait = [&](uint64_t* bar, uint32_t ph) -> bool {
      if (__all_sync(0xffffffffu, mbar_try_wait(bar, ph))) return true;
      return __all_sync(0xffffffffu, bounded_wait(bar, ph)) != 0;
    };
    // chain x's operands are written and its accumulator read: hand over
    auto signal = [&](int x) {
      fence_async_smem();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&s_ready[x]);
    };
    // ---- P1: FP16 products Z conj(C) -> stage-1 operand rows of chain x ----
    auto p1 = [&](const uint4(&zr)[U], unsigned char* A, const unsigned char* code) {
      const uint4* cp = reinterpret_cast<const uint4*>(code);
#pragma unroll
      for (int k0 = 0; k0 < U; k0 += kBatch) {
        uint4 c[kBatch];
#pragma unroll
        for (int i = 0; i < kBatch; ++i) {
          const int k = k0 + i;
          if (k < U && (k < U - 1 || tid + k * NTS < T::UNITS)) c[i] = cp[uoff[k] >> 16];
        }
#pragma unroll
        for (int i = 0; i < kBatch; ++i) {
          const int k = k0 + i;
          if (k < U && (k < U - 1 || tid + k * NTS < T::UNITS)) {
            const uint4 cc = c[i], z = zr[k];
            *reinterpret_cast<uint4*>(A + (uoff[k] & 0xFFFFu)) = cmul_unit(z, cc);
          }
        }
      }
    };
    // P2 and P3 read the accumulators in chunks of 16 columns (8 complex
    // outputs).  At Lc = 10230 every chunk of the phase is loaded before one
    // wait (measured fastest there); otherwise through two register buffers,
    // the load of chunk q + 1 in flight while chunk q is rounded and stored.
    constexpr bool ONE_WAIT = M == 10;
    auto run_chunks = [&](auto nq, auto&& load, auto&& store) {
      constexpr int NQ = decltype(nq)::value;
      if constexpr (ONE_WAIT) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) load(q);
        tmem_wait_ld();
#pragma unroll
        for (int q = 0; q < NQ; ++q) store(q);
      } else {
        load(0);
        tmem_wait_ld();
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
          if (q + 1 < NQ) load(q + 1);
          store(q);
          if (q + 1 < NQ) tmem_wait_ld();
        }
      }
    };
    // ---- P2: stage-1 accumulators -> stage-2 rows (t1, d3), K = d2 ----
    auto p2 = [&](int x) {
      unsigned char* A = A0 + x * T::A_BYTES;
      const uint32_t tb = tmem_base + lane_off + (uint32_t)(x * (kTcTmemCols / 2));
      // warp w reads lane quadrant w % 4 of tiles w / 4 + 3 k, all CS1
      // column halves: task i is tile w / 4 + 3 (i / CS1), half i % CS1,
      // known at compile time but for the tile
      constexpr int NQ = TPW2 * 2;  // a task is 32 columns
      uint32_t buf[ONE_WAIT ? NQ : 2][16];
      auto load = [&](int q) {
        const int i = q >> 1, t = (warp >> 2) + 3 * (i / CS1), half = i % CS1;
        tmem_ld16(tb + (uint32_t)(t * T::N1 + 32 * half + 16 * (q & 1)), buf[ONE_WAIT ? q : q & 1]);
      };
      auto store = [&](int q) {
        const int i = q >> 1, t = (warp >> 2) + 3 * (i / CS1), half = i % CS1;
        const int r = t * 128 + quad * 32 + lane;
        int s, d3, d2;
        bool valid;
        if constexpr (T::PADR1) {
          s = r / T::ROWS1P;
          const int u = r - s * T::ROWS1P;
          d3 = u >> 5;
          d2 = u & 31;
          valid = s < BC && d2 < R2;
        } else {
          s = r / T::ROWS1;
          const int u = r - s * T::ROWS1;
          d3 = u / R2;
          d2 = u - d3 * R2;
          valid = r < T::NR1;
        }
        // stage-2 row (t1, d3), K entry d2
        constexpr int T1_STRIDE = T::S2O ? 4 * 16 : R3 * 16;
        unsigned char* dst = A + (s * T::ROWS2 + (T::S2O ? (d3 >> 2) * 128 + (d3 & 3) : d3)) * 16 +
                             (d2 >> 2) * T::LBO2 + (d2 & 3) * 4;
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          const int t1 = 16 * half + 8 * (q & 1) + h;
          if (valid && t1 < 31)
            st_shared_u32(dst + t1 * T1_STRIDE, pack_h2_sat(__uint_as_float(buf[ONE_WAIT ? q : q & 1][2 * h]),
                                                            __uint_as_float(buf[ONE_WAIT ? q : q & 1][2 * h + 1])));
        }
      };
      run_chunks(std::integral_constant<int, NQ>(), load, store);
    };
    // ---- P3: stage-2 accumulators -> stage-3 rows (t1, t2), K = d3 ----
    auto p3 = [&](int x) {
      unsigned char* A = A0 + x * T::A_BYTES;
      const uint32_t tb = tmem_base + lane_off + (uint32_t)(x * (kTcTmemCols / 2));
      // tasks as in P2: tile w / 4 + 3 (i / CS2), half i % CS2
      constexpr int CPT = W2 / 16;  // chunks per task
      constexpr int NQ = TPW3 * CPT;
      uint32_t buf[ONE_WAIT ? NQ : 2][16];
      auto load = [&](int q) {
        const int i = q / CPT, t = (warp >> 2) + 3 * (i / CS2), half = i % CS2;
        tmem_ld16(tb + (uint32_t)(t * T::N2 + W2 * half + 16 * (q % CPT)), buf[ONE_WAIT ? q : q & 1]);
      };
      auto store = [&](int q) {
        const int i = q / CPT, t = (warp >> 2) + 3 * (i / CS2), half = i % CS2;
        const int r = t * 128 + quad * 32 + lane;
        const int s = r / T::ROWS2, qq = r - s * T::ROWS2;
        const int t1 = T::S2O ? (qq & 127) >> 2 : qq / R3;
        const int d3 = T::S2O ? 4 * (qq >> 7) + (qq & 3) : qq - t1 * R3;
        const bool valid = r < T::NR2 && (!T::S2O || (d3 < R3 && t1 < 31));
        const uint32_t* v = buf[ONE_WAIT ? q : q & 1];
        if (T::PAIR3) {
          // paired stage-3 row (t1, t2 / 2) = s ROWS3P + t1 R2 / 2 + t2 / 2
          // (T1F3: s ROWS3P + (t2 / 2) 31 + t1), K entry d3 (t2 even) or
          // P3OFF / 2 + d3 (t2 odd)
          constexpr int JSTRIDE = T::T1F3 ? 31 * 16 : 16;  // bytes between rows j and j + 1
          unsigned char* dst0 = A + (s * T::ROWS3P + (T::T1F3 ? t1 : t1 * (R2 / 2))) * 16 + (d3 >> 2) * T::LBO3 +
                                (d3 & 3) * 4;
          unsigned char* dst1 = dst0 + (T::P3OFF / 8) * T::LBO3;
#pragma unroll
          for (int h = 0; h < 8; ++h) {
            const int t2 = (W2 / 2) * half + 8 * (q % CPT) + h;
            if (valid && t2 < R2)
              st_shared_u32(((t2 & 1) ? dst1 : dst0) + (t2 >> 1) * JSTRIDE,
                            pack_h2_sat(__uint_as_float(v[2 * h]), __uint_as_float(v[2 * h + 1])));
          }
        } else {
          // stage-3 row (t1, t2) = s ROWS3 + t1 R2 + t2, K entry d3
          unsigned char* dst = A + (s * T::ROWS3 + t1 * R2) * 16 + (d3 >> 2) * T::LBO3 + (d3 & 3) * 4;
#pragma unroll
          for (int h = 0; h < 8; ++h) {
            const int t2 = (W2 / 2) * half + 8 * (q % CPT) + h;
            if (valid && t2 < R2)
              st_shared_u32(dst + t2 * 16, pack_h2_sat(__uint_as_float(v[2 * h]), __uint_as_float(v[2 * h + 1])));
          }
        }
      };
      run_chunks(std::integral_constant<int, NQ>(), load, store);
    };
    // ---- P4: |y|^2 maximum over the stage-3 outputs of chain x ----
    // Only the row maximum is kept: rows near the best of their (antenna,
    // PRN) are searched again in FP32 (launch_correlate_listed), which finds
    // the lag with the reference's tie rule.  Padding rows and residues >= S are skipped.
    auto p4 = [&](int x, int g) -> float {
      const uint32_t tb = tmem_base + lane_off + (uint32_t)(x * (kTcTmemCols / 2));
      // accumulator words read per task: 24 for a stage-3 transform (22 used)
      constexpr int VW = 24;
      float best = 0.f;
      if constexpr (T::NST == 2) {
        // two-stage split: the stage-2 row (2 R2 words used) in pieces of 48
        // words, one task per warp at most
        static_assert(TPW4 == 1, "one epilogue task per warp");
        const int task = warp;
        if (task < NT4) {
          const int r = (task >> 2) * 128 + quad * 32 + lane;
          const bool valid = r < T::LAST_NR && g * BC + r / T::LAST_ROWS < S;
#pragma unroll
          for (int c0 = 0; c0 < 2 * T::LAST_OUT; c0 += 48) {
            uint32_t v[48];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              uint32_t(&a)[16] = *reinterpret_cast<uint32_t(*)[16]>(&v[16 * c]);
              if (c0 + 16 * c < 2 * T::LAST_OUT) tmem_ld16(tb + (uint32_t)((task >> 2) * T::N2 + c0 + 16 * c), a);
            }
            tmem_wait_ld();
            if (valid) {
#pragma unroll
              for (int h = 0; h < 24; ++h)
                if (c0 + 2 * h < 2 * T::LAST_OUT)
                  best = fmaxf(best, fmaf(__uint_as_float(v[2 * h]), __uint_as_float(v[2 * h]),
                                          __uint_as_float(v[2 * h + 1]) * __uint_as_float(v[2 * h + 1])));
            }
          }
        }
        return best;
      } else if constexpr (M == 4) {
        // Lc = 4092.  The stage-3 accumulator of a tile is 48 columns: the transforms
        // (t1, 2j) and (t1, 2j + 1) in columns [0, 22) and [24, 46), zeros
        // (zero rows of the DFT matrix) in the rest, so the maximum may take
        // whole 8-column chunks.  The LAST_TILES x 6 chunks of a lane
        // quadrant are split evenly over its 3 warps: chunk q = (w / 4) CPW
        // + i, tile q / 6, columns 8 (q % 6) .. + 8.
        static_assert(T::N3 == 48 && NW == 12 && (T::LAST_TILES * 6) % 3 == 0, "P4 chunk map");
        constexpr int CPW = T::LAST_TILES * 6 / 3, BATCH = CPW % 4 == 0 ? 4 : (CPW % 3 == 0 ? 3 : 2);
        static_assert(CPW % BATCH == 0, "P4 batches");
#pragma unroll
        for (int i0 = 0; i0 < CPW; i0 += BATCH) {
          uint32_t v[BATCH][8];
#pragma unroll
          for (int i = 0; i < BATCH; ++i) {
            const int q = (warp >> 2) * CPW + i0 + i;
            tmem_ld8(tb + (uint32_t)((q / 6) * T::N3 + 8 * (q % 6)), v[i]);
          }
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < BATCH; ++i) {
            const int q = (warp >> 2) * CPW + i0 + i;
            const int r = (q / 6) * 128 + quad * 32 + lane;
            if (r < T::LAST_NR && g * BC + r / T::LAST_ROWS < S) {
#pragma unroll
              for (int h = 0; h < 4; ++h)
                best = fmaxf(best, fmaf(__uint_as_float(v[i][2 * h]), __uint_as_float(v[i][2 * h]),
                                        __uint_as_float(v[i][2 * h + 1]) * __uint_as_float(v[i][2 * h + 1])));
            }
          }
        }
        return best;
      } else {
        // Lc = 10230 (where the chunks above measured slower): tasks in
        // batches of LB4, all loads of a batch in flight, one wait
#pragma unroll
        for (int i0 = 0; i0 < TPW4; i0 += LB4) {
          uint32_t v[LB4][VW];
#pragma unroll
          for (int i = 0; i < LB4; ++i) {
            const int task = warp + (i0 + i) * NW;
            if (i0 + i < TPW4 && task < NT4) {
              const int t = task / (4 * HALVES3), half = (task >> 2) % HALVES3;
              tmem_ld_stage3<T::PAIR3>(tb + (uint32_t)(t * T::N3), half, v[i]);
            }
          }
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < LB4; ++i) {
            const int task = warp + (i0 + i) * NW;
            if (i0 + i < TPW4 && task < NT4) {
              const int r = (task / (4 * HALVES3)) * 128 + quad * 32 + lane;
              if (r < T::LAST_NR && g * BC + r / T::LAST_ROWS < S) {
                // the task's powers, then their maximum as a pairwise tree
                // (a serial fmaxf chain left the warps waiting on latency)
                float pw[T::LAST_OUT];
#pragma unroll
                for (int h = 0; h < T::LAST_OUT; ++h)
                  pw[h] = fmaf(__uint_as_float(v[i][2 * h]), __uint_as_float(v[i][2 * h]),
                               __uint_as_float(v[i][2 * h + 1]) * __uint_as_float(v[i][2 * h + 1]));
#pragma unroll
                for (int w2 = 1; w2 < T::LAST_OUT; w2 *= 2)
#pragma unroll
                  for (int h = 0; h + w2 < T::LAST_OUT; h += 2 * w2) pw[h] = fmaxf(pw[h], pw[h + w2]);
                best = fmaxf(best, pw[0]);
              }
            }
          }
        }
        return best;
      }
    };

    // ---- P4 of the non-coherent search: add the block's |y|^2 to the sums
    // in TMEM (first: the sums start at it); after the last block (last),
    // the row maximum of the sums ----
    // Two-stage split: tasks are (stage-2 tile, lane quadrant, outputs
    // [11 c, 11 c + 11)).  Three-stage paired split: tasks are (stage-3
    // tile, lane quadrant, half c: the 11 outputs of accumulator columns
    // [24 c, 24 c + 22)).  task = warp + i NW keeps the warp's quadrant,
    // whose lanes hold the task's rows in the accumulator and in the sums.
    // One task at a time (unrolled, the tasks' registers spilled).
    auto p4_nc = [&](int x, int g, bool first, bool last) -> float {
      const uint32_t tb = tmem_base + lane_off + (uint32_t)(x * (kTcTmemCols / 2));
      float best = 0.f;
      // the 12 sum columns of slot c of tile t (11 used), issued before the
      // task's one wait on the TMEM loads
      auto load_sums = [&](int t, int c, uint32_t(&su)[12]) -> uint32_t {
        const uint32_t sa = tmem_base + lane_off + T::sum_col(t, c);
        if (!first) {
          tmem_ld8(sa, *reinterpret_cast<uint32_t(*)[8]>(&su[0]));
          tmem_ld4(sa + 8, *reinterpret_cast<uint32_t(*)[4]>(&su[8]));
        }
        return sa;
      };
      // adds the powers of 11 complex outputs (words v[2 h], v[2 h + 1]) to
      // the sums and stores them back, or after the last block takes their
      // maximum over the valid rows
      auto acc11 = [&](const uint32_t* v, uint32_t(&su)[12], uint32_t sa, bool valid) {
#pragma unroll
        for (int h = 0; h < 11; ++h) {
          const float re = __uint_as_float(v[2 * h]), im = __uint_as_float(v[2 * h + 1]);
          // two FMAs per output (these sums only rank rows for the FP32
          // re-evaluation, which recomputes the chosen values)
          su[h] = __float_as_uint(fmaf(re, re, fmaf(im, im, first ? 0.f : __uint_as_float(su[h]))));
        }
        if (!last) {
          su[11] = 0u;
          tmem_st8(sa, *reinterpret_cast<const uint32_t(*)[8]>(&su[0]));
          tmem_st4(sa + 8, *reinterpret_cast<const uint32_t(*)[4]>(&su[8]));
        } else if (valid) {
#pragma unroll
          for (int h = 0; h < 11; ++h) best = fmaxf(best, __uint_as_float(su[h]));
        }
      };
      if constexpr (T::NST == 2) {
        constexpr int NTN = T::LAST_TILES * 4 * 3, TPWN = (NTN + NW - 1) / NW;
#pragma unroll 1
        for (int i = 0; i < TPWN; ++i) {
          const int task = warp + i * NW;
          if (task >= NTN) break;
          const int t = task / 12, c = (task >> 2) % 3;
          const int s0 = c == 0 ? 0 : (c == 1 ? 16 : 40);  // 8-column aligned start covering [22 c, 22 c + 22)
          uint32_t v[32];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            uint32_t(&q)[8] = *reinterpret_cast<uint32_t(*)[8]>(&v[8 * k]);
            tmem_ld8(tb + (uint32_t)(t * T::N2 + s0 + 8 * k), q);
          }
          uint32_t su[12];
          const uint32_t sa = load_sums(t, c, su);
          tmem_wait_ld();
          const int r = t * 128 + quad * 32 + lane;
          const bool valid = r < T::LAST_NR && g * BC + r / T::LAST_ROWS < S;
          // the chunk starts 22 c - s0 = 0, 6 or 4 words into v (c is
          // uniform over the warp; constant offsets keep v in registers)
          if (c == 0)
            acc11(v, su, sa, valid);
          else if (c == 1)
            acc11(v + 6, su, sa, valid);
          else
            acc11(v + 4, su, sa, valid);
        }
      } else {
        constexpr int NTN = T::LAST_TILES * 4 * 2, TPWN = (NTN + NW - 1) / NW;
#pragma unroll 1
        for (int i = 0; i < TPWN; ++i) {
          const int task = warp + i * NW;
          if (task >= NTN) break;
          const int t = task / 8, half = (task >> 2) & 1;
          uint32_t v[24];
          tmem_ld_stage3<T::PAIR3>(tb + (uint32_t)(t * T::N3), half, v);
          uint32_t su[12];
          const uint32_t sa = load_sums(t, half, su);
          tmem_wait_ld();
          const int r = t * 128 + quad * 32 + lane;
          const bool valid = r < T::LAST_NR && g * BC + r / T::LAST_ROWS < S;
          acc11(v, su, sa, valid);
        }
      }
      // the sums' stores land before this thread reads them again
      tmem_wait_st();
      return best;
    };

    for (int u = blockIdx.x; u < p.n_items * split && !failed; u += gridDim.x) {
      const int w = u / split, ab_h = w / p.groups, g = w - ab_h * p.groups;
      const int r0 = unit_round0(split, u, n_rounds), r1 = unit_round1(split, u, n_rounds);
      // this item's Z units of block blk, in registers
      uint4 zr[U];
      auto load_z = [&](int blk) {
        // the drop-in search reads its Z once (evict first); the
        // non-coherent search reads each block again for every PRN,
        // so it keeps the blocks in L2.  blk >= B (BLKCH, B odd) stands for
        // zero data, which adds nothing to the sums.
        const uint4* seq = p.z16 + (((size_t)ab_h * B + blk) * S + (size_t)g * BC) * 8 * T::ROWS1;
        const int live = blk < B ? S - g * BC : 0;  // residue slots with data
#pragma unroll
        for (int k = 0; k < U; ++k) {
          zr[k] = make_uint4(0u, 0u, 0u, 0u);
          const int sl = BC == 1 ? 0 : (int)((uslot >> (4 * k)) & 15u);
          if (sl < live && (k < U - 1 || tid + k * NTS < T::UNITS)) {
            const uint4* src = seq + (uint32_t)sl * (8u * T::ROWS1) + (uoff[k] >> 16);
            zr[k] = NCB ? __ldcg(src) : __ldcs(src);
          }
        }
      };
      // the code slot of chain x (BLKCH: one slot for both)
      auto slot = [](int x) -> int { return T::BLKCH ? 0 : x; };
      // chain x: wait for its code block when a new PRN starts (the blocks of
      // one PRN share it), form the products, hand over
      // code_ready: this lane's earlier test of the block (issued before the
      // epilogue, so its latency overlaps that work); the warp waits only if
      // a lane saw it incomplete
      auto products = [&](int x, bool new_code, uint32_t code_ready = 0u) -> bool {
        const int c = slot(x);
        if (new_code) {
          if (!__all_sync(0xffffffffu, code_ready) && !warp_wait(&s_code[c], (ph_code >> c) & 1u)) return false;
          ph_code ^= 1u << c;
        }
        p1(zr, A0 + x * T::A_BYTES, CODE0 + c * T::CODE_REGION);
        signal(x);
        return true;
      };
      // after the products of a PRN's last block the code warp may refill
      // the chain's code block
      auto released = [&](int x) {
        if (lane == 0) mbar_arrive(&s_p1[x]);
      };
      // the first step of the unit's first round
      if (T::BLKCH) {
        load_z(0);
        failed = !products(0, true);
        if (!failed) {
          load_z(1);
          failed = !products(1, false);
        }
        if (!failed && NI == 1) {
          released(0);
          released(1);
        }
      } else {
        load_z(0);
        for (int x = 0; x < 2 && !failed; ++x) {
          failed = !products(x, true);
          if (!failed && NI == 1) released(x);
        }
      }
      for (int r = r0; r < r1 && !failed; ++r)
       for (int b = 0; b < NI && !failed; ++b) {
        const bool more = b + 1 < NI || r + 1 < r1;  // a next step of this unit follows
        const int bn = b + 1 < NI ? b + 1 : 0;        // its index
        // both chains have formed this step's products: bring the next
        // step's Z (BLKCH: that of chain a's next block) into the registers
        // while the transforms run
        if (NCB && more) load_z(T::BLKCH ? 2 * bn : bn);
        // P2, P3 for chain a then chain b, each after its own MMA stage
#pragma unroll 1
        for (int st = 0; st < T::NST - 1 && !failed; ++st) {
#pragma unroll 1
          for (int x = 0; x < 2; ++x) {
            if (!warp_wait(&s_done[x], (ph_done >> x) & 1u)) {
              failed = true;
              break;
            }
            ph_done ^= 1u << x;
            tc_fence_after();
            if (st == 0)
              p2(x);
            else
              p3(x);
            signal(x);
          }
        }
        // P4 of this step, then at once the products of the chain's next
        // step, so that the tensor cores are not left idle across rounds
#pragma unroll 1
        for (int x = 0; x < 2 && !failed; ++x) {
          if (!warp_wait(&s_done[x], (ph_done >> x) & 1u)) {
            failed = true;
            break;
          }
          ph_done ^= 1u << x;
          tc_fence_after();
          // a new PRN starts with the next step (BLKCH: chain a waits for
          // the shared slot, chain b follows it); test its code block now,
          // use the answer after P4
          const bool new_code = more && b + 1 == NI && (!T::BLKCH || x == 0);
          const uint32_t code_ready = new_code ? mbar_try_wait(&s_code[slot(x)], (ph_code >> slot(x)) & 1u) : 0u;
          // non-negative floats order like their bit patterns
          float pmax;
          if constexpr (NCB) {
            // BLKCH: chain a's block 0 starts the sums, chain b's last block
            // ends them
            const bool first = T::BLKCH ? (b == 0 && x == 0) : b == 0;
            const bool last = T::BLKCH ? (b + 1 == NI && x == 1) : b + 1 == NI;
            pmax = p4_nc(x, g, first, last);
          } else {
            pmax = p4(x, g);
          }
          const unsigned bits = __reduce_max_sync(0xffffffffu, __float_as_uint(pmax));
          if (lane == 0 && bits != 0u)
            atomicMax(p.keys + (size_t)ab_h * p.n_prn + prn_of(r, x), (unsigned long long)bits << 32);
          // the next products are those of step b + 1, or of the next
          // round's step 0
          if (more) {
            failed = !products(x, new_code, code_ready);
            // BLKCH: the Z of chain b's next block, for its products after
            // its P4
            if (!failed && T::BLKCH && x == 0) load_z(2 * bn + 1);
            if (!failed && (NCB ? bn == NI - 1 : true)) released(x);
          }
        }
       }
    }
    if (failed && lane == 0) atomicExch(p.err, 1);
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, kTcTmemCols);
}

template <int M, bool NCB>
cudaError_t run_tc3(const PolyClass& pc, const SearchDims& dims, int B, const void* d_bmat, const void* d_z16,
                    const void* d_d16, unsigned long long* d_keys, int* d_err, int test_flags, int num_sms,
                    cudaStream_t st) {
  using T = T3<M, NCB>;
  Tc3Params p = {};
  p.skip_commit = test_flags & 1;
  p.bmat = static_cast<const uint4*>(d_bmat);
  p.z16 = static_cast<const uint4*>(d_z16);
  p.d16 = static_cast<const uint4*>(d_d16);
  p.keys = d_keys;
  p.err = d_err;
  p.n_prn = dims.n_prn;
  p.S = pc.S;
  p.groups = (pc.S + T::BC - 1) / T::BC;
  p.B = NCB ? B : 1;
  p.n_items = dims.n_ant * dims.nb * (NCB ? 1 : 2) * p.groups;
  // too few items to fill the SMs (the non-coherent search on a few rows):
  // split each item's rounds (PRN pairs, or PRNs with BLKCH) over CTAs
  const int n_rounds = T::BLKCH ? dims.n_prn : (dims.n_prn + 1) / 2;
  p.split = 1;
  if (NCB && p.n_items > 0 && p.n_items < num_sms && n_rounds > 1) {
    p.split = (num_sms + p.n_items - 1) / p.n_items;
    if (p.split > n_rounds) p.split = n_rounds;
  }
  auto kern = pfa_tc3_kernel<M, NCB>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, T::SMEM);
  if (e != cudaSuccess) return e;
  // one CTA per SM: T::SMEM is above half of the SM's shared memory, so the
  // 512-column TMEM allocation never meets another one
  int grid = num_sms;
  if (grid > p.n_items * p.split) grid = p.n_items * p.split;
  if (grid < 1) return cudaSuccess;
  kern<<<grid, kTcThreads, T::SMEM, st>>>(p);
  kernel_launch_add(1);
  return cudaGetLastError();
}

// FP16 scale exponents (kz, kd) of Z and the code spectra, kz + kd = k with
// 4 S Lc^2 2^-k <= 32768
void tc_scales(const PolyClass& pc, int* kz, int* kd) {
  const double bound = 4.0 * pc.S * (double)pc.Lc * (double)pc.Lc;
  int k = 0;
  while (bound / (double)(1ull << k) > 32768.0 && k < 60) ++k;
  *kz = (k + 1) / 2;
  *kd = k - *kz;
}

template <int M>
cudaError_t run_pack(const float2* src, long long n_seq, void* dst, float scale, int num_sms, cudaStream_t st) {
  const long long n_units = n_seq * 8 * T3<M>::ROWS1;
  if (n_units == 0) return cudaSuccess;
  long long blocks = (n_units + 255) / 256;
  if (blocks > (long long)num_sms * 16) blocks = (long long)num_sms * 16;
  tc_pack_kernel<M><<<(int)blocks, 256, 0, st>>>(src, static_cast<uint4*>(dst), n_units, scale);
  kernel_launch_add(1);
  return cudaGetLastError();
}

template <int M>
std::vector<unsigned char> build_matrices() {
  using T = T3<M>;
  std::vector<unsigned char> b((size_t)(T::B1_BYTES + T::B2_BYTES + T::B3_BYTES), 0);
  host_idft_matrix<31, T::N1, T::KB1, false, true>(b.data(), 0);
  for (int a = 0; a < T::B2_ATOMS; ++a)
    host_idft_matrix<T::R2, T::N2, T::KB2, false>(b.data() + T::B1_BYTES + a * T::N2 * T::KB2, 0, a);
  if (T::NST == 3)
    host_idft_matrix<T::R3, T::N3, T::KB3, T::PAIR3>(b.data() + T::B1_BYTES + T::B2_BYTES, T::P3OFF);
  return b;
}

}  // namespace

size_t tc_operand_bytes(const PolyClass& pc, long long n_seq, bool code) {
  const int rows1 = pc.Lc / 31;  // R2 * R3
  (void)code;
  return (size_t)n_seq * 8 * rows1 * 16;
}

std::vector<unsigned char> tc_dft_matrices(int M) {
  switch (M) {
    case 1: return build_matrices<1>();
    case 4: return build_matrices<4>();
    case 10: return build_matrices<10>();
  }
  return {};
}

double tc_key_amplitude(const PolyClass& pc) {
  int kz = 0, kd = 0;
  tc_scales(pc, &kz, &kd);
  return (double)(1ull << (kz + kd));
}

float tc_z_scale(const PolyClass& pc) {
  int kz = 0, kd = 0;
  tc_scales(pc, &kz, &kd);
  return (float)(1.0 / (double)(1ull << kz));
}

cudaError_t launch_tc_pack(const PolyClass& pc, const float2* d_src, long long n_seq, bool code, void* d_dst,
                           int num_sms, cudaStream_t st) {
  int kz = 0, kd = 0;
  tc_scales(pc, &kz, &kd);
  const float scale = (float)(1.0 / (double)(1ull << (code ? kd : kz)));
  switch (pc.M) {
    case 1: return run_pack<1>(d_src, n_seq, d_dst, scale, num_sms, st);
    case 4: return run_pack<4>(d_src, n_seq, d_dst, scale, num_sms, st);
    case 10: return run_pack<10>(d_src, n_seq, d_dst, scale, num_sms, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_correlate_tc(const PolyClass& pc, const SearchDims& dims, const void* d_bmat, const void* d_z16,
                                const void* d_d16, unsigned long long* d_keys, int* d_err, int test_flags,
                                int num_sms, cudaStream_t st) {
  switch (pc.M) {
    case 1: return run_tc3<1, false>(pc, dims, 1, d_bmat, d_z16, d_d16, d_keys, d_err, test_flags, num_sms, st);
    case 4: return run_tc3<4, false>(pc, dims, 1, d_bmat, d_z16, d_d16, d_keys, d_err, test_flags, num_sms, st);
    case 10: return run_tc3<10, false>(pc, dims, 1, d_bmat, d_z16, d_d16, d_keys, d_err, test_flags, num_sms, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_correlate_tc_nc(const PolyClass& pc, const SearchDims& dims, int B, const void* d_bmat,
                                   const void* d_z16, const void* d_d16, unsigned long long* d_keys, int* d_err,
                                   int test_flags, int num_sms, cudaStream_t st) {
  if (B < 1) return cudaErrorInvalidValue;
  switch (pc.M) {
    case 1: return run_tc3<1, true>(pc, dims, B, d_bmat, d_z16, d_d16, d_keys, d_err, test_flags, num_sms, st);
    case 4: return run_tc3<4, true>(pc, dims, B, d_bmat, d_z16, d_d16, d_keys, d_err, test_flags, num_sms, st);
    case 10: return run_tc3<10, true>(pc, dims, B, d_bmat, d_z16, d_d16, d_keys, d_err, test_flags, num_sms, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace tga
