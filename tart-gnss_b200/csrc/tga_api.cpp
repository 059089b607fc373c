// Host side of libtga.so: context, planning and the C ABI of include/tga.h.
//
// Planning.  For each constellation the drivers of the reference search a
// window of two code periods (acquisition.rs:274-275, galileo.rs:230-232,
// beidou.rs:182-184, l1c.rs:191-193).  When the resampled code over that
// window is exactly chip((n / S) mod Lc) * pulse(n % S) for the constellation's
// chip count Lc (1023, 4092 or 10230) -- true at every integer number of
// samples per chip, e.g. 16.368 MHz -- the fused polyphase kernels run.
// Constellations that share the period, the Doppler grid and the pulse
// (GPS/SBAS/QZSS; BeiDou/L1C) share one front end.  Anything else runs the
// generic GPU path (the reference algorithm with Bluestein FFTs).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tga.h"
#include "codes.h"
#include "engine.h"
#include "gnss_tables.h"

using namespace tga;

namespace {

constexpr double kTau = 6.283185307179586;  // std::f64::consts::TAU

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

}  // namespace

struct tga_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  // tga_acquire_all_stream: the stream of the host-to-device copies and the
  // event of each of its two bits buffers (created on first use)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copied[2] = {nullptr, nullptr};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  std::map<std::string, DevBuf> bufs;
  // cached fused-path code spectra: key -> (device D, n_prn)
  double last_cells = 0.0;
  int last_launches = 0;
  double last_ms = 0.0;
  uint64_t h2d = 0, d2h = 0;
  int precision = 0;  // TGA_PRECISION_*
  // FP32 correlation launch shape per precision for Lc = 1023, 4092, 10230
  int variant[2][3] = {{0, 0, 0}, {0, 0, 0}};
  // per-kernel event timing
  bool profiling = false;
  struct Pending {
    std::string name;
    int ev;
    double flops;
  };
  std::vector<cudaEvent_t> evpool;
  std::vector<Pending> pending;
  int ev_used = 0;
  struct KTime {
    double ms = 0.0, flops = 0.0;
    int launches = 0;
  };
  std::vector<std::pair<std::string, KTime>> ktimes;
  int* tc_err_pending = nullptr;  // device flag of the last tensor-core launch
  int test_flags = 0;             // TGA_TEST_* hooks (tga_set_test_flags)
  // planning caches: verified polyphase classes, host chips, uploaded chips
  struct ClassCache {
    bool structure_ok = false;
    PolyClass pc;
    std::map<int, bool> prn_ok;
  };
  std::map<std::string, ClassCache> class_cache;
  std::map<std::pair<int, int>, std::vector<int8_t>> chip_cache;
  std::map<std::string, std::vector<std::pair<int, int>>> uploaded;  // device chips buffer -> PRN list
  // CUDA graphs of the --all pipeline, one per plan (key: everything the
  // launches capture by value).  A plan runs eagerly on its first call, is
  // captured on its second and replayed after that.  `gen` counts buffer
  // (re)allocations: a graph captured under another generation holds stale
  // pointers and is rebuilt.
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    size_t gen = 0;
    bool seen = false, failed = false;
    int launches = 0;
    double cells = 0.0;
    uint64_t d2h = 0;
    int* tc_err = nullptr;
  };
  bool graphs_enabled = true;
  size_t gen = 0;
  std::map<std::string, GraphEntry> graphs;
  int last_graph = TGA_GRAPH_NONE;
  // the fused class groups of the last --all call (tga_last_row_peaks)
  struct LastGroup {
    int Lc = 0, P = 0, n_ant = 0, nb = 0, n_prn = 0;
    bool tc = false;
    double amp = 1.0;  // |y| = sqrt(key power) x amp
    const unsigned long long* keys = nullptr;
    const int* count = nullptr;
    int n_chunks = 1;             // counts in `count`
    double nc_power_scale = 0.0;  // > 0: a non-coherent search (one hypothesis, power units)
  };
  std::vector<LastGroup> last_groups;
  // pinned host staging for results
  void* pinned = nullptr;
  size_t pinned_cap = 0;
  void* host_pinned(size_t bytes) {
    if (pinned_cap >= bytes && pinned) return pinned;
    ++gen;
    if (pinned) cudaFreeHost(pinned);
    pinned = nullptr;
    pinned_cap = 0;
    if (cudaMallocHost(&pinned, bytes) != cudaSuccess) {
      cudaGetLastError();
      throw std::runtime_error("cudaMallocHost failed");
    }
    pinned_cap = bytes;
    return pinned;
  }

  int next_event() {
    if (ev_used >= (int)evpool.size()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) throw std::runtime_error("cudaEventCreate failed");
      evpool.push_back(e);
    }
    return ev_used++;
  }

  void* buf(const std::string& name, size_t bytes) {
    DevBuf& b = bufs[name];
    if (b.cap >= bytes && b.p) return b.p;
    ++gen;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    size_t want = bytes < 256 ? 256 : bytes;
    if (cudaMalloc(&b.p, want) != cudaSuccess) {
      cudaGetLastError();
      throw std::runtime_error("cudaMalloc failed for " + name + " (" + std::to_string(want) + " bytes)");
    }
    b.cap = want;
    return b.p;
  }
};

namespace {

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_));                \
  } while (0)

struct TimeoutError : std::runtime_error {
  explicit TimeoutError(const std::string& s) : std::runtime_error(s) {}
};

struct InvalidArg : std::invalid_argument {
  explicit InvalidArg(const std::string& s) : std::invalid_argument(s) {}
};

template <class F>
int guarded(tga_ctx* ctx, F&& f) {
  if (!ctx) return TGA_ERR_INVALID_ARG;
  try {
    CK(cudaSetDevice(ctx->device));
    ctx->err.clear();
    return f();
  } catch (const CudaError& e) {
    ctx->err = e.what();
    return TGA_ERR_CUDA;
  } catch (const TimeoutError& e) {
    ctx->err = e.what();
    return TGA_ERR_TIMEOUT;
  } catch (const std::invalid_argument& e) {
    ctx->err = e.what();
    return TGA_ERR_INVALID_ARG;
  } catch (const std::bad_alloc& e) {
    ctx->err = "host allocation failed";
    return TGA_ERR_OUT_OF_MEMORY;
  } catch (const std::runtime_error& e) {
    ctx->err = e.what();
    return std::string(e.what()).find("cudaMalloc") != std::string::npos ? TGA_ERR_OUT_OF_MEMORY
                                                                          : TGA_ERR_CUDA;
  }
}

// acquisition.rs:188-198: n = round(2B/300) + 1 bins centred on center_freq.
std::vector<double> freq_grid(double center, double band) {
  const double x = 2.0 * band / 300.0;
  double r = std::round(x);  // f64::round: half away from zero
  size_t n = (r > 0.0) ? (size_t)r : 0;  // `as usize` saturates (NaN -> 0)
  n += 1;
  if (n > (size_t)kMaxBins) throw InvalidArg("search band gives too many Doppler bins");
  std::vector<double> fc(n);
  if (n == 1) {
    fc[0] = center;
  } else {
    for (size_t i = 0; i < n; ++i) fc[i] = (center - band) + ((double)i * (2.0 * band)) / ((double)n - 1.0);
  }
  return fc;
}

int chip_width_of(double fs) {
  double w = std::ceil(fs / 1.023e6);  // correlate.rs:157
  return w > 0 ? (int)w : 0;
}

// Begin a new call: reset counters and per-kernel timing.
void begin_call(tga_ctx* ctx) {
  kernel_launch_count_reset();
  ctx->last_cells = 0.0;
  ctx->h2d = ctx->d2h = 0;
  ctx->pending.clear();
  ctx->ev_used = 0;
  ctx->ktimes.clear();
}

// Launch through `fn` (returns cudaError_t), bracketed by events when profiling.
template <class F>
void timed(tga_ctx* ctx, const char* name, double flops, F&& fn) {
  if (!ctx->profiling) {
    CK(fn());
    return;
  }
  const int a = ctx->next_event();
  CK(cudaEventRecord(ctx->evpool[a], ctx->stream));
  CK(fn());
  const int b = ctx->next_event();
  CK(cudaEventRecord(ctx->evpool[b], ctx->stream));
  ctx->pending.push_back({name, a, flops});
}

// After the stream is idle: fold event pairs into per-kernel totals.
void collect_times(tga_ctx* ctx) {
  for (const auto& pd : ctx->pending) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->evpool[pd.ev], ctx->evpool[pd.ev + 1]));
    auto it = ctx->ktimes.begin();
    for (; it != ctx->ktimes.end(); ++it)
      if (it->first == pd.name) break;
    if (it == ctx->ktimes.end()) {
      ctx->ktimes.push_back({pd.name, tga_ctx::KTime()});
      it = ctx->ktimes.end() - 1;
    }
    it->second.ms += ms;
    it->second.flops += pd.flops;
    it->second.launches += 1;
  }
  ctx->pending.clear();
}

// After the stream is idle: did a tensor-core wait expire?
void check_tc_error(tga_ctx* ctx) {
  if (!ctx->tc_err_pending) return;
  int flag = 0;
  CK(cudaMemcpy(&flag, ctx->tc_err_pending, sizeof(int), cudaMemcpyDeviceToHost));
  ctx->tc_err_pending = nullptr;
  if (flag) throw TimeoutError("tensor-core correlator: a bounded wait on the MMA pipeline expired");
}

// Runs `enqueue` (launches and stream-ordered copies only) for the plan
// `key`: eagerly on the plan's first call, captured into a CUDA graph and
// launched on its second, replayed from the graph after that.  A replay
// restores what the enqueue would have recorded (launch count, cells, bytes
// read back, the tensor-core error flag).  A capture that fails for any
// reason leaves the plan eager.
template <class F>
void run_planned(tga_ctx* ctx, const std::string& key, F&& enqueue) {
  ctx->last_graph = TGA_GRAPH_NONE;
  if (!ctx->graphs_enabled || ctx->profiling) {
    enqueue();
    return;
  }
  if (ctx->graphs.size() >= 64 && !ctx->graphs.count(key)) {
    for (auto& kv : ctx->graphs)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    ctx->graphs.clear();
  }
  tga_ctx::GraphEntry& ge = ctx->graphs[key];
  if (ge.exec && ge.gen != ctx->gen) {
    cudaGraphExecDestroy(ge.exec);
    ge.exec = nullptr;
  }
  if (ge.exec) {
    CK(cudaGraphLaunch(ge.exec, ctx->stream));
    kernel_launch_add(ge.launches);
    ctx->last_cells += ge.cells;
    ctx->d2h += ge.d2h;
    ctx->tc_err_pending = ge.tc_err;
    ctx->last_graph = TGA_GRAPH_REPLAYED;
    return;
  }
  if (!ge.seen || ge.failed) {
    enqueue();
    ge.seen = true;
    return;
  }
  const int l0 = kernel_launch_count();
  const double c0 = ctx->last_cells;
  const uint64_t d0 = ctx->d2h;
  const size_t gen0 = ctx->gen;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ex = nullptr;
  bool ok = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed) == cudaSuccess;
  if (ok) {
    try {
      enqueue();
    } catch (const std::exception&) {
      ok = false;
    }
    ok = (cudaStreamEndCapture(ctx->stream, &g) == cudaSuccess) && ok && g && ctx->gen == gen0;
    if (ok) ok = cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
  }
  if (!ok) {
    cudaGetLastError();
    if (ex) cudaGraphExecDestroy(ex);
    ge.failed = true;
    kernel_launch_count_reset();
    kernel_launch_add(l0);
    ctx->last_cells = c0;
    ctx->d2h = d0;
    enqueue();
    return;
  }
  ge.exec = ex;
  ge.gen = ctx->gen;
  ge.launches = kernel_launch_count() - l0;
  ge.cells = ctx->last_cells - c0;
  ge.d2h = ctx->d2h - d0;
  ge.tc_err = ctx->tc_err_pending;
  CK(cudaGraphLaunch(ex, ctx->stream));
  ctx->last_graph = TGA_GRAPH_CAPTURED;
}

// Algorithmic FLOPs reported per kernel (tga_kernel_times) and used by the
// roofline: 5 N log2 N per complex FFT of N points, 6 per complex product,
// 3 per |y|^2 and 10 per sample of carrier wipe-off, whatever a kernel
// executes (the prime-factor transforms execute more per point, the
// tensor-core stages far more).  One correlation row of P lags is a
// product, an inverse transform and the power of every lag.
double fft_flops(double n) { return n > 1.0 ? 5.0 * n * std::log2(n) : 0.0; }
double corr_row_flops(int P) { return fft_flops((double)P) + 9.0 * (double)P; }

// Tensor-core search: rows whose FP16 key is at least kTcKeyKeep x the best
// key of their (antenna, PRN) are re-evaluated in FP32.  kTcKeyKeep =
// (1 - 2 d)^2 with d = 2^-8 a bound on the FP16 transform's amplitude error
// at any lag, relative to the largest row amplitude of the (antenna, PRN):
// the FP16 stages round 5 to 7 times at a unit roundoff of 2^-11, and the
// largest error measured over the test and benchmark workloads (every code
// length, drop-in and non-coherent, noise-only cells) is 5.6e-4, 7x below d
// (tga_last_row_peaks reports the keys for that measurement).
constexpr float kTcKeyKeep = (1.0f - 2.0f / 256.0f) * (1.0f - 2.0f / 256.0f);

// Device bytes the non-coherent search's Z may take at once (FP32, plus the
// FP16 operands in tensor-core mode); more antennas than fit run in chunks.
constexpr double kNcZBudget = 24e9;

const std::vector<int8_t>& cached_chips(tga_ctx* ctx, int c, int prn) {
  auto key = std::make_pair(c, prn);
  auto it = ctx->chip_cache.find(key);
  if (it != ctx->chip_cache.end()) return it->second;
  return ctx->chip_cache[key] = primary_chips(c, prn);
}

// Try to express the reference's resampled code over 2P samples as
// chip((n/S) mod Lc) * pulse(n % S).  Returns false if it is not exact or the
// chip count has no fused kernel.  The check is exact (every sample of every
// PRN is compared with the reference's resampling rule) and cached per
// context, since it depends only on (constellation, rate, period, PRN).
int variant_slot(int M) { return M == 1 ? 0 : M == 4 ? 1 : 2; }

bool poly_class_for(tga_ctx* ctx, int c, double samples_per_code, size_t P, size_t N,
                    const std::vector<int>& prns, PolyClass* out) {
  const ConstellationInfo& ci = info(c);
  const int Lc = ci.primary_chips;
  if (N != 2 * P || P == 0 || P % (size_t)Lc != 0) return false;
  const size_t S = P / (size_t)Lc;
  if (S < 1 || S > (size_t)kMaxPulse) return false;
  if (Lc != 1023 && Lc != 4092 && Lc != 10230) return false;
  char keybuf[96];
  uint64_t spc_bits;
  std::memcpy(&spc_bits, &samples_per_code, 8);
  std::snprintf(keybuf, sizeof keybuf, "%d/%zu/%zu/%llx", c, P, N, (unsigned long long)spc_bits);
  tga_ctx::ClassCache& cc = ctx->class_cache[keybuf];
  for (int prn : prns) {
    auto hit = cc.prn_ok.find(prn);
    if (hit != cc.prn_ok.end()) {
      if (!hit->second) return false;
      continue;
    }
    const std::vector<int8_t>& chips = cached_chips(ctx, c, prn);
    std::vector<int8_t> code = resampled_code(c, prn, samples_per_code, N);
    PolyClass pc;
    pc.P = (int)P;
    pc.S = (int)S;
    pc.Lc = Lc;
    pc.M = Lc / 1023;
    for (size_t s2 = 0; s2 < S; ++s2) pc.pulse[s2] = (float)(code[s2] * chips[0]);
    bool ok = true;
    for (size_t n = 0; n < N && ok; ++n)
      ok = chips[(n / S) % (size_t)Lc] * (int)pc.pulse[n % S] == code[n];
    if (ok && cc.structure_ok) {
      for (size_t s2 = 0; s2 < S; ++s2) ok = ok && pc.pulse[s2] == cc.pc.pulse[s2];
    }
    cc.prn_ok[prn] = ok;
    if (!ok) return false;
    if (!cc.structure_ok) {
      cc.pc = pc;
      cc.structure_ok = true;
    }
  }
  if (!cc.structure_ok) return false;
  *out = cc.pc;
  out->variant = ctx->variant[ctx->precision][variant_slot(out->M)];
  return true;
}

bool same_class(const PolyClass& a, const PolyClass& b) {
  if (a.P != b.P || a.S != b.S || a.Lc != b.Lc) return false;
  for (int s = 0; s < a.S; ++s)
    if (a.pulse[s] != b.pulse[s]) return false;
  return true;
}

// One group of constellations sharing a fused front end.
struct ClassGroup {
  PolyClass pc;
  std::vector<int> consts;               // constellation ids in the group
  std::vector<std::pair<int, int>> prns; // (constellation, prn) in search order
};

struct SearchOut {
  std::vector<CellOut> cells;  // [n_ant][n_prn] of the group
};

// The offset table of the FP16 Z units (tc_unit_map), uploaded once per context.
void* tc_unit_map_buf(tga_ctx* ctx, int M) {
  const std::string map_name = "tcmap." + std::to_string(M);
  if (ctx->uploaded.count(map_name)) return ctx->buf(map_name, 0);
  const std::vector<uint16_t> map = tc_unit_map(M);
  void* d = ctx->buf(map_name, map.size() * sizeof(uint16_t));
  CK(cudaMemcpy(d, map.data(), map.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
  ctx->uploaded[map_name] = {};
  return d;
}

// Device buffers of one class group, allocated (and the code chips and DFT
// matrices uploaded) by prepare_group before anything is launched, so that
// enqueue_group is launches and stream-ordered copies only and can be
// captured into a CUDA graph.
struct GroupBufs {
  int8_t* chips = nullptr;
  const int8_t* tables = nullptr;
  float2* z = nullptr;
  float2* D = nullptr;
  unsigned long long* keys = nullptr;
  BestRow* best = nullptr;
  CellOut* cells = nullptr;
  int* err = nullptr;
  void* z16 = nullptr;
  void* d16 = nullptr;
  void* bmat = nullptr;
  void* zmap = nullptr;   // tensor-core mode: FP16 unit offsets (tc_unit_map)
  // tensor-core mode: FP32 keys of the rows re-evaluated, the list of those
  // rows and its length
  unsigned long long* keys32 = nullptr;
  int2* cand = nullptr;
  int* count = nullptr;
  // and each re-evaluated row's second peak against its own maximum
  float* p2rows = nullptr;
};

GroupBufs prepare_group(tga_ctx* ctx, const ClassGroup& grp, int n_ant, int nb, const std::string& tag) {
  const PolyClass& pc = grp.pc;
  const int n_prn = (int)grp.prns.size();
  const int n_ab = n_ant * nb;
  cudaStream_t st = ctx->stream;
  GroupBufs b;
  // code chips and ACR table ids -> device (re-uploaded only when the PRN list changes)
  const size_t chip_bytes = (size_t)n_prn * pc.Lc;
  b.chips = (int8_t*)ctx->buf(tag + ".chips", chip_bytes + (size_t)n_prn);
  auto up = ctx->uploaded.find(tag + ".chips");
  if (up == ctx->uploaded.end() || up->second != grp.prns) {
    std::vector<int8_t> chips(chip_bytes + (size_t)n_prn);
    for (int i = 0; i < n_prn; ++i) {
      const std::vector<int8_t>& ch = cached_chips(ctx, grp.prns[i].first, grp.prns[i].second);
      std::memcpy(&chips[(size_t)i * pc.Lc], ch.data(), (size_t)pc.Lc);
      chips[chip_bytes + i] = (int8_t)info(grp.prns[i].first).acr_table;
    }
    CK(cudaMemcpyAsync(b.chips, chips.data(), chips.size(), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));  // chips is a host temporary
    ctx->h2d += chips.size();
    ctx->uploaded[tag + ".chips"] = grp.prns;
  }
  b.tables = b.chips + chip_bytes;
  b.z = (float2*)ctx->buf(tag + ".z", (size_t)n_ab * 2 * pc.S * pc.Lc * sizeof(float2));
  b.D = (float2*)ctx->buf(tag + ".D", (size_t)n_prn * 2 * pc.Lc * sizeof(float2));
  b.keys = (unsigned long long*)ctx->buf(tag + ".keys", (size_t)n_ab * 2 * n_prn * sizeof(unsigned long long));
  b.best = (BestRow*)ctx->buf(tag + ".best", (size_t)n_ant * n_prn * sizeof(BestRow));
  b.cells = (CellOut*)ctx->buf(tag + ".cells", (size_t)n_ant * n_prn * sizeof(CellOut));
  if (ctx->precision == TGA_PRECISION_FP16_TC) {
    b.err = (int*)ctx->buf("tc.err", sizeof(int));
    const long long n_zseq = (long long)n_ab * 2 * pc.S;
    b.z16 = ctx->buf(tag + ".z16", tc_operand_bytes(pc, n_zseq, false));
    b.d16 = ctx->buf(tag + ".d16", tc_operand_bytes(pc, (long long)n_prn * 2, true));
    b.keys32 = (unsigned long long*)ctx->buf(tag + ".keys32", (size_t)n_ab * 2 * n_prn * sizeof(unsigned long long));
    b.p2rows = (float*)ctx->buf(tag + ".p2rows", (size_t)n_ab * 2 * n_prn * sizeof(float));
    b.cand = (int2*)ctx->buf(tag + ".cand", (size_t)n_ab * 2 * n_prn * sizeof(int2));
    b.count = (int*)ctx->buf(tag + ".count", sizeof(int));
    // DFT matrices of the class (they depend on Lc only), uploaded once per context
    const std::string mat_name = "tcmat." + std::to_string(pc.M);
    if (!ctx->uploaded.count(mat_name)) {
      const std::vector<unsigned char> mats = tc_dft_matrices(pc.M);
      b.bmat = ctx->buf(mat_name, mats.size());
      CK(cudaMemcpy(b.bmat, mats.data(), mats.size(), cudaMemcpyHostToDevice));
      ctx->uploaded[mat_name] = {};
    } else {
      b.bmat = ctx->buf(mat_name, 0);
    }
    b.zmap = tc_unit_map_buf(ctx, pc.M);
  }
  return b;
}

// Enqueues the fused pipeline of one class group on the context stream
// (launches, memsets and the copy of the finalised cells into host_out,
// pinned memory of n_ant * n_prn CellOut).
void enqueue_group(tga_ctx* ctx, const ClassGroup& grp, const GroupBufs& b, const SampleSource& src,
                   const double* d_fc, int nb, double center, int want_cn0, int chip_width, CellOut* host_out) {
  const PolyClass& pc = grp.pc;
  const int n_ant = src.n_ant;
  const int n_prn = (int)grp.prns.size();
  const int n_ab = n_ant * nb;
  cudaStream_t st = ctx->stream;

  SearchDims dims;
  dims.n_ant = n_ant;
  dims.nb = nb;
  dims.n_prn = n_prn;
  dims.fc = d_fc;

  const double row = corr_row_flops(pc.P);
  const std::string cls = "[Lc=" + std::to_string(pc.Lc) + "]";
  // tensor-core mode takes the second peaks from the FP32 re-evaluation,
  // which keeps the four largest |y|^2 of every residue of a row: enough
  // while at most three lags of a residue lie within chip_width of the peak
  // (chip_width = S samples at every fused rate)
  const bool rows_p2 = ctx->precision == TGA_PRECISION_FP16_TC && (2 * chip_width + pc.S) / pc.S <= 3;
  timed(ctx, ("code_spectra" + cls).c_str(), (double)n_prn * 2 * fft_flops(pc.Lc),
        [&] { return launch_code_spectra(pc, b.chips, n_prn, b.D, ctx->num_sms, st); });
  timed(ctx, ("frontend" + cls).c_str(), (double)n_ab * 10.0 * pc.P,
        [&] { return launch_frontend(src, dims, pc, b.z, st); });
  if (ctx->precision == TGA_PRECISION_FP16_TC) {
    // the forward transform also writes Z's FP16 operands; the code spectra
    // are packed apart
    timed(ctx, ("forward_z" + cls).c_str(), (double)n_ab * 2 * fft_flops(pc.P), [&] {
      return launch_forward_z_tc(pc, n_ab, b.z, b.z16, b.zmap, tc_z_scale(pc), ctx->num_sms, st);
    });
    timed(ctx, ("tc_pack" + cls).c_str(), 0.0,
          [&] { return launch_tc_pack(pc, b.D, (long long)n_prn * 2, true, b.d16, ctx->num_sms, st); });
    CK(cudaMemsetAsync(b.err, 0, sizeof(int), st));
    CK(cudaMemsetAsync(b.keys, 0, (size_t)n_ab * 2 * n_prn * sizeof(unsigned long long), st));
    timed(ctx, ("correlate_tc" + cls).c_str(), (double)n_ab * 2 * n_prn * row, [&] {
      return launch_correlate_tc(pc, dims, b.bmat, b.z16, b.d16, b.keys, b.err, ctx->test_flags, ctx->num_sms, st);
    });
    ctx->tc_err_pending = b.err;
    // every row within the FP16 key error of its (antenna, PRN)'s best,
    // re-evaluated in FP32; the bins are then reduced over the FP32 keys as
    // in the FP32 search (rows not listed keep key 0)
    CK(cudaMemsetAsync(b.count, 0, sizeof(int), st));
    CK(cudaMemsetAsync(b.keys32, 0, (size_t)n_ab * 2 * n_prn * sizeof(unsigned long long), st));
    if (rows_p2) CK(cudaMemsetAsync(b.p2rows, 0, (size_t)n_ab * 2 * n_prn * sizeof(float), st));
    timed(ctx, ("candidates" + cls).c_str(), 0.0,
          [&] { return launch_tc_candidates(dims, 2, b.keys, kTcKeyKeep, b.cand, b.count, st); });
    // the re-evaluation also keeps each row's second peak, so the chosen
    // rows need no second transform
    timed(ctx, ("refine" + cls).c_str(), 0.0, [&] {
      return launch_correlate_listed(pc, dims, b.z, b.D, b.cand, b.count, n_ab * 2 * n_prn, b.keys32, ctx->num_sms,
                                     st, rows_p2 ? b.p2rows : nullptr, chip_width);
    });
  } else {
    timed(ctx, ("forward_z" + cls).c_str(), (double)n_ab * 2 * fft_flops(pc.P),
          [&] { return launch_forward_z(pc, n_ab, b.z, ctx->num_sms, st); });
    timed(ctx, ("correlate" + cls).c_str(), (double)n_ab * 2 * n_prn * row,
          [&] { return launch_correlate(pc, dims, b.z, b.D, b.keys, ctx->num_sms, st); });
  }
  const unsigned long long* keys32 = ctx->precision == TGA_PRECISION_FP16_TC ? b.keys32 : b.keys;
  timed(ctx, ("reduce_bins" + cls).c_str(), 0.0, [&] { return launch_reduce_bins(dims, keys32, b.best, st); });
  if (rows_p2)
    timed(ctx, ("second_peak" + cls).c_str(), 0.0,
          [&] { return launch_second_from_rows(dims, 2, b.p2rows, b.best, st); });
  else
    timed(ctx, ("second_peak" + cls).c_str(), (double)n_ant * n_prn * row,
          [&] { return launch_second_peak(pc, dims, b.z, b.D, b.best, chip_width, ctx->num_sms, st); });
  timed(ctx, ("finalize" + cls).c_str(), 0.0,
        [&] { return launch_finalize(pc, dims, b.best, center, b.tables, want_cn0, b.cells, st); });
  CK(cudaMemcpyAsync(host_out, b.cells, (size_t)n_ant * n_prn * sizeof(CellOut), cudaMemcpyDeviceToHost, st));
  ctx->d2h += (size_t)n_ant * n_prn * sizeof(CellOut);
  ctx->last_cells += (double)n_ant * nb * n_prn * (double)pc.P;
}

void validate_prn(int c, int prn) {
  const ConstellationInfo& ci = info(c);
  if (prn < ci.prn_first || prn > ci.prn_last)
    throw InvalidArg(std::string(ci.sv_prefix) + " PRN out of range: " + std::to_string(prn));
}

std::vector<int> prn_list(int c, const tga_all_options* opt) {
  std::vector<int> v;
  if (opt->prn_filter) {
    for (size_t i = 0; i < opt->n_prn_filter; ++i) {
      validate_prn(c, opt->prn_filter[i]);
      v.push_back(opt->prn_filter[i]);
    }
  } else {
    const ConstellationInfo& ci = info(c);
    for (int p = ci.prn_first; p <= ci.prn_last; ++p) v.push_back(p);
  }
  return v;
}

tga_result generic_one(tga_ctx* ctx, int c, const float* d_sig, const double* d_pp, size_t n, double fs,
                       const double* d_fc, const std::vector<double>& fc, double center, int prn, size_t period);

// acr.rs:49-84 on the host, for cells of the generic path (the fused path
// evaluates the same rule in its finalize kernel).
bool estimate_cn0_host(double r_a, int table, double* out);

int acquire_all_impl(tga_ctx* ctx, const uint8_t* d_bits, size_t n_ant_total, size_t row_bytes, double fs,
                     const tga_all_options* opt, tga_cell* out, size_t cap, size_t* n_out) {
  if (!opt || !n_out) throw InvalidArg("null options or n_out");
  if (!(fs > 0.0)) throw InvalidArg("sampling frequency must be positive");
  if (n_ant_total == 0 || row_bytes == 0) throw InvalidArg("empty observation");
  std::vector<int32_t> ants;
  if (opt->ant_filter) {
    for (size_t i = 0; i < opt->n_ant_filter; ++i) {
      if (opt->ant_filter[i] < 0 || (size_t)opt->ant_filter[i] >= n_ant_total)
        throw InvalidArg("antenna index " + std::to_string(opt->ant_filter[i]) + " out of range (have " +
                         std::to_string(n_ant_total) + ")");
      ants.push_back(opt->ant_filter[i]);
    }
  } else {
    for (size_t i = 0; i < n_ant_total; ++i) ants.push_back((int32_t)i);
  }
  if (ants.empty()) throw InvalidArg("no antennas selected");
  size_t total = 0;
  std::vector<int> consts;
  std::map<int, std::vector<int>> prns;
  for (int c = 0; c < N_CONST; ++c) {
    if (!(opt->constellation_mask & (1u << c))) continue;
    consts.push_back(c);
    prns[c] = prn_list(c, opt);
    total += prns[c].size() * ants.size();
  }
  *n_out = total;
  if (total > cap || (!out && total)) return TGA_ERR_CAPACITY;
  if (total == 0) return TGA_OK;

  std::vector<double> fc = freq_grid(opt->center_freq, opt->search_band);
  const int nb = (int)fc.size();
  const size_t n_rec = row_bytes * 8;

  // plan class groups; constellations the fused kernels cannot express go
  // to the generic path
  std::vector<ClassGroup> groups;
  std::vector<int> generic_consts;
  ctx->last_groups.clear();
  for (int c : consts) {
    const size_t P = period_samples(c, fs);
    if (P == 0) throw InvalidArg("sampling frequency too low for " + std::string(info(c).json_key));
    const size_t N = std::min(2 * P, n_rec);
    PolyClass pc;
    if (!poly_class_for(ctx, c, (double)P, P, N, prns[c], &pc)) {
      generic_consts.push_back(c);
      continue;
    }
    bool placed = false;
    for (auto& g : groups) {
      if (same_class(g.pc, pc)) {
        g.consts.push_back(c);
        for (int p : prns[c]) g.prns.push_back({c, p});
        placed = true;
        break;
      }
    }
    if (!placed) {
      ClassGroup g;
      g.pc = pc;
      g.consts.push_back(c);
      for (int p : prns[c]) g.prns.push_back({c, p});
      groups.push_back(g);
    }
  }

  cudaStream_t st = ctx->stream;
  // buffers and uploads first (host side, outside any graph)
  double* d_mean = (double*)ctx->buf("mean", n_ant_total * sizeof(double));
  int32_t* d_ants = (int32_t*)ctx->buf("ants", ants.size() * sizeof(int32_t));
  double* d_fc = (double*)ctx->buf("fc", fc.size() * sizeof(double));
  std::vector<GroupBufs> gbufs;
  for (const auto& g : groups)
    gbufs.push_back(prepare_group(ctx, g, (int)ants.size(), nb,
                                  "g" + std::to_string(g.pc.P) + "_" + std::to_string(g.pc.Lc)));
  size_t n_group_cells = 0;
  for (const auto& g : groups) n_group_cells += ants.size() * g.prns.size();
  CellOut* pinned = (CellOut*)ctx->host_pinned((n_group_cells ? n_group_cells : 1) * sizeof(CellOut));
  std::vector<CellOut*> gout(groups.size());
  {
    size_t off = 0;
    for (size_t gi = 0; gi < groups.size(); ++gi) {
      gout[gi] = pinned + off;
      off += ants.size() * groups[gi].prns.size();
    }
  }
  // the call's antenna list and Doppler grid
  CK(cudaMemcpyAsync(d_ants, ants.data(), ants.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_fc, fc.data(), fc.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  ctx->h2d += ants.size() * sizeof(int32_t) + fc.size() * sizeof(double);

  SampleSource src;
  src.bits = d_bits;
  src.row_bytes = row_bytes;
  src.mean = d_mean;
  src.ant = d_ants;
  src.n_ant = (int)ants.size();
  src.pc = kTau / fs;

  auto enqueue = [&] {
    // antenna means over the whole rows
    timed(ctx, "antenna_means", 0.0,
          [&] { return launch_antenna_means(d_bits, (int)n_ant_total, row_bytes, d_mean, st); });
    for (size_t gi = 0; gi < groups.size(); ++gi)
      enqueue_group(ctx, groups[gi], gbufs[gi], src, d_fc, nb, opt->center_freq, opt->cn0, chip_width_of(fs),
                    gout[gi]);
  };
  CK(cudaEventRecord(ctx->ev0, st));
  if (generic_consts.empty()) {
    // the plan: everything the launches take by value or by address
    std::string key;
    char kb[512];
    const int kn = std::snprintf(kb, sizeof kb, "%p/%zu/%zu/%a/%a/%d/%d/%d/%d/%d%d%d/%d|", (const void*)d_bits,
                                 n_ant_total, row_bytes, fs, opt->center_freq, nb, opt->cn0, ctx->precision,
                                 ctx->test_flags, ctx->variant[ctx->precision][0],
                                 ctx->variant[ctx->precision][1], ctx->variant[ctx->precision][2],
                                 chip_width_of(fs));
    if (kn < 0 || kn >= (int)sizeof kb) throw std::runtime_error("search plan key does not fit");
    key = kb;
    for (int32_t a : ants) key += std::to_string(a) + ",";
    key += "|";
    for (const auto& g : groups)
      for (const auto& cp : g.prns) key += std::to_string(cp.first) + ":" + std::to_string(cp.second) + ",";
    for (double f : fc) {
      std::snprintf(kb, sizeof kb, "%a,", f);
      key += kb;
    }
    run_planned(ctx, key, enqueue);
  } else {
    ctx->last_graph = TGA_GRAPH_NONE;
    enqueue();
  }
  // generic path: per (constellation, antenna, PRN), reference algorithm on the GPU
  std::map<int, std::vector<CellOut>> gen_out;  // constellation -> [prn][ant]
  for (int c : generic_consts) {
    const size_t P = period_samples(c, fs);
    const size_t N = std::min(2 * P, n_rec);
    float* d_sig = (float*)ctx->buf("gen.sig", N * sizeof(float));
    double* d_pp = (double*)ctx->buf("gen.pp", N * sizeof(double));
    std::vector<CellOut>& v = gen_out[c];
    v.resize(prns[c].size() * ants.size());
    for (size_t a = 0; a < ants.size(); ++a) {
      timed(ctx, "bits_to_signal", 0.0, [&] {
        return launch_bits_to_signal(d_bits, row_bytes, ants[a], d_mean, (int)N, kTau / fs, d_sig, d_pp, st);
      });
      for (size_t i = 0; i < prns[c].size(); ++i) {
        tga_result r = generic_one(ctx, c, d_sig, d_pp, N, fs, d_fc, fc, opt->center_freq, prns[c][i], P);
        CellOut o{};
        o.strength = r.signal_strength;
        o.second = r.second_peak;
        o.codephase_frac = r.codephase_frac;
        o.frequency = r.frequency;
        o.bin = r.best_freq_idx;
        o.tau = (int32_t)r.best_codephase;
        o.hyp = r.hypothesis;
        o.cn0_valid = 0;
        if (opt->cn0 && o.second > 0.0 && o.strength > o.second) {
          const double q = o.strength / o.second;
          double cn0 = 0.0;
          if (estimate_cn0_host(q * q, info(c).acr_table, &cn0)) {
            o.cn0 = cn0;
            o.cn0_valid = 1;
          }
        }
        v[i * ants.size() + a] = o;
      }
    }
  }
  CK(cudaEventRecord(ctx->ev1, st));
  CK(cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->last_ms = ms;
  ctx->last_launches = kernel_launch_count();
  collect_times(ctx);
  check_tc_error(ctx);
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    tga_ctx::LastGroup lg;
    lg.Lc = groups[gi].pc.Lc;
    lg.P = groups[gi].pc.P;
    lg.n_ant = (int)ants.size();
    lg.nb = nb;
    lg.n_prn = (int)groups[gi].prns.size();
    lg.tc = ctx->precision == TGA_PRECISION_FP16_TC;
    lg.amp = lg.tc ? tc_key_amplitude(groups[gi].pc) : 1.0;
    lg.keys = gbufs[gi].keys;
    lg.count = gbufs[gi].count;
    ctx->last_groups.push_back(lg);
  }

  // assemble in (constellation, prn order, antenna) order
  size_t k = 0;
  for (int c : consts) {
    for (int prn : prns[c]) {
      if (gen_out.count(c)) {
        const size_t i = std::find(prns[c].begin(), prns[c].end(), prn) - prns[c].begin();
        for (size_t a = 0; a < ants.size(); ++a) {
          const CellOut& o = gen_out[c][i * ants.size() + a];
          tga_cell& t = out[k++];
          t.constellation = c;
          t.prn = prn;
          t.antenna = ants[a];
          t.best_freq_idx = o.bin;
          t.best_codephase = o.tau;
          t.signal_strength = o.strength;
          t.second_peak = o.second;
          t.codephase_frac = o.codephase_frac;
          t.frequency = o.frequency;
          t.cn0_acr = o.cn0;
          t.cn0_valid = o.cn0_valid;
          t.hypothesis = o.hyp;
        }
        continue;
      }
      // locate group / index
      const ClassGroup* g = nullptr;
      size_t gidx = 0, pidx = 0;
      for (size_t gi = 0; gi < groups.size() && !g; ++gi)
        for (size_t i = 0; i < groups[gi].prns.size(); ++i)
          if (groups[gi].prns[i].first == c && groups[gi].prns[i].second == prn) {
            g = &groups[gi];
            gidx = gi;
            pidx = i;
            break;
          }
      const int n_prn_g = (int)g->prns.size();
      for (size_t a = 0; a < ants.size(); ++a) {
        const CellOut o = gout[gidx][a * n_prn_g + pidx];
        tga_cell& t = out[k++];
        t.constellation = c;
        t.prn = prn;
        t.antenna = ants[a];
        t.best_freq_idx = o.bin;
        t.best_codephase = o.tau;
        t.signal_strength = o.strength;
        t.second_peak = o.second;
        t.codephase_frac = o.codephase_frac;
        t.frequency = o.frequency;
        t.cn0_acr = o.cn0;
        t.cn0_valid = o.cn0_valid;
        t.hypothesis = o.hyp;
      }
    }
  }
  return TGA_OK;
}

// Generic path for one (signal, PRN): the reference algorithm on the GPU.
// d_sig/d_pp are device arrays of n samples; d_fc the Doppler grid.
tga_result generic_one(tga_ctx* ctx, int c, const float* d_sig, const double* d_pp, size_t n, double fs,
                       const double* d_fc, const std::vector<double>& fc, double center, int prn, size_t period) {
  if (n > (size_t)(1 << 26)) throw InvalidArg("signal too long for the generic path");
  cudaStream_t st = ctx->stream;
  const int nb = (int)fc.size();
  // code replicas [c..] and [c, -c] split at min(period, n) (correlate.rs:47-58)
  std::vector<int8_t> code = resampled_code(c, prn, (double)period, n);
  std::vector<float> ca(n), cb(n);
  const size_t split = std::min(period, n);
  for (size_t i = 0; i < n; ++i) {
    ca[i] = (float)code[i];
    cb[i] = i < split ? ca[i] : -ca[i];
  }
  float* d_ca = (float*)ctx->buf("gen.ca", n * sizeof(float));
  float* d_cb = (float*)ctx->buf("gen.cb", n * sizeof(float));
  CK(cudaMemcpyAsync(d_ca, ca.data(), n * sizeof(float), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_cb, cb.data(), n * sizeof(float), cudaMemcpyHostToDevice, st));
  ctx->h2d += 2 * n * sizeof(float);
  GenericPlan gp;
  gp.N = (int)n;
  gp.Mpow2 = 1;
  gp.log2M = 0;
  while (gp.Mpow2 < 2 * gp.N - 1) {
    gp.Mpow2 <<= 1;
    gp.log2M++;
  }
  if (gp.Mpow2 < 2) {
    gp.Mpow2 = 2;
    gp.log2M = 1;
  }
  const size_t welems = generic_work_elems(gp, nb);
  float2* d_work = (float2*)ctx->buf("gen.work", welems * sizeof(float2));
  float* d_corr = (float*)ctx->buf("gen.corr", (size_t)2 * nb * n * sizeof(float));
  int* d_ri = (int*)ctx->buf("gen.ri", 4 * sizeof(int));
  float* d_rf = (float*)ctx->buf("gen.rf", 4 * sizeof(float));
  timed(ctx, "generic", 0.0, [&] {
    return launch_generic(gp, d_sig, d_pp, d_fc, nb, d_ca, d_cb, (int)period, fs, d_work, welems, d_corr, d_ri,
                          d_rf, st);
  });
  int ri[4];
  float rf[4];
  CK(cudaMemcpyAsync(ri, d_ri, sizeof ri, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(rf, d_rf, sizeof rf, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  ctx->d2h += sizeof ri + sizeof rf;
  tga_result r;
  r.prn = prn;
  r.best_freq_idx = ri[0];
  const size_t cp = (size_t)ri[1] % period;
  r.best_codephase = (int64_t)cp;
  r.signal_strength = (double)rf[0];
  r.second_peak = (double)rf[1];
  r.codephase_frac = (double)cp / (double)period;
  r.frequency = fc[ri[0]] - center;
  r.hypothesis = ri[2];
  r.path = 1;
  ctx->last_cells += (double)nb * (double)period;
  return r;
}

int acquire_single_impl(tga_ctx* ctx, int c, const float* h_sig, const double* h_pp, size_t n, double fs,
                        double center, double band, int prn, size_t period, tga_result* out) {
  if (!h_sig || !h_pp || !out) throw InvalidArg("null pointer");
  if (n == 0) throw InvalidArg("empty signal");
  if (period == 0) throw InvalidArg("zero code period");
  validate_prn(c, prn);
  std::vector<double> fc = freq_grid(center, band);
  const int nb = (int)fc.size();
  PolyClass pc;
  const bool fused = poly_class_for(ctx, c, (double)period, period, n, {prn}, &pc);
  begin_call(ctx);
  cudaStream_t st = ctx->stream;
  float* d_sig = (float*)ctx->buf("single.sig", n * sizeof(float));
  double* d_pp = (double*)ctx->buf("single.pp", n * sizeof(double));
  CK(cudaMemcpyAsync(d_sig, h_sig, n * sizeof(float), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_pp, h_pp, n * sizeof(double), cudaMemcpyHostToDevice, st));
  int32_t zero = 0;
  int32_t* d_ant = (int32_t*)ctx->buf("single.ant", sizeof(int32_t));
  CK(cudaMemcpyAsync(d_ant, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, st));
  double* d_fc = (double*)ctx->buf("single.fc", fc.size() * sizeof(double));
  CK(cudaMemcpyAsync(d_fc, fc.data(), fc.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  if (!fused) {
    ctx->h2d += n * (sizeof(float) + sizeof(double));
    *out = generic_one(ctx, c, d_sig, d_pp, n, fs, d_fc, fc, center, prn, period);
    ctx->last_launches = kernel_launch_count();
    collect_times(ctx);
    return TGA_OK;
  }
  SampleSource src;
  src.sig = d_sig;
  src.pp = d_pp;
  src.n_samples = n;
  src.ant = d_ant;
  src.n_ant = 1;
  ClassGroup g;
  g.pc = pc;
  g.consts.push_back(c);
  g.prns.push_back({c, prn});
  ctx->h2d += n * (sizeof(float) + sizeof(double));
  const GroupBufs gb = prepare_group(ctx, g, 1, nb, "single");
  CellOut* cell = (CellOut*)ctx->host_pinned(sizeof(CellOut));
  enqueue_group(ctx, g, gb, src, d_fc, nb, center, 0, chip_width_of(fs), cell);
  CK(cudaStreamSynchronize(st));
  ctx->last_launches = kernel_launch_count();
  collect_times(ctx);
  check_tc_error(ctx);
  const CellOut o = *cell;
  out->prn = prn;
  out->best_freq_idx = o.bin;
  out->best_codephase = o.tau;
  out->signal_strength = o.strength;
  out->second_peak = o.second;
  out->codephase_frac = o.codephase_frac;
  out->frequency = o.frequency;
  out->hypothesis = o.hyp;
  out->path = 0;
  return TGA_OK;
}

bool estimate_cn0_host(double r_a, int table, double* out) {
  const double(*t)[2];
  int n;
  switch (table) {
    case TGA_ACR_GPS_L1_CA: t = TGA_GPS_L1_CA_ACR_TABLE; n = 59; break;
    case TGA_ACR_GALILEO_E1C: t = TGA_GALILEO_E1C_ACR_TABLE; n = 71; break;
    case TGA_ACR_BEIDOU_B1C: t = TGA_BEIDOU_B1C_ACR_TABLE; n = 79; break;
    default: t = TGA_GPS_L1C_ACR_TABLE; n = 79; break;
  }
  if (!(r_a > 1.0) || !std::isfinite(r_a)) return false;
  if (r_a <= t[0][0]) { *out = t[0][1]; return true; }
  if (r_a >= t[n - 1][0]) { *out = t[n - 1][1]; return true; }
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if (t[mid][0] < r_a) lo = mid + 1; else hi = mid;
  }
  if (lo == 0) { *out = t[0][1]; return true; }
  if (lo >= n) { *out = t[n - 1][1]; return true; }
  const double la = std::log(t[lo - 1][0]), lb = std::log(t[lo][0]);
  const double tt = (std::log(r_a) - la) / (lb - la);
  double v = t[lo - 1][1] + tt * (t[lo][1] - t[lo - 1][1]);
  *out = std::min(70.0, std::max(20.0, v));
  return true;
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

const char* tga_version(void) { return "tga 0.1.0 (sm_100a)"; }

int tga_create(int device, tga_ctx** out) {
  if (!out) return TGA_ERR_INVALID_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) {
    cudaGetLastError();
    return TGA_ERR_NO_DEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return TGA_ERR_NO_DEVICE;
  if (prop.major != 10) return TGA_ERR_NO_DEVICE;  // built for sm_100a only
  tga_ctx* ctx = new (std::nothrow) tga_ctx();
  if (!ctx) return TGA_ERR_OUT_OF_MEMORY;
  ctx->device = device;
  ctx->num_sms = prop.multiProcessorCount;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) {
    delete ctx;
    return TGA_ERR_CUDA;
  }
  *out = ctx;
  return TGA_OK;
}

int tga_destroy(tga_ctx* ctx) {
  if (!ctx) return TGA_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  for (auto& kv : ctx->bufs)
    if (kv.second.p) cudaFree(kv.second.p);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  for (cudaEvent_t& e : ctx->copied)
    if (e) cudaEventDestroy(e);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  for (cudaEvent_t e : ctx->evpool) cudaEventDestroy(e);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return TGA_OK;
}

const char* tga_last_error(const tga_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int tga_acquire_single(tga_ctx* ctx, int constellation, const float* h_signal_f32, const double* h_phasepoints,
                       size_t num_samples, double sampling_freq, double center_freq, double search_band, int prn,
                       size_t samples_per_chunk, tga_result* out) {
  return guarded(ctx, [&] {
    if (constellation < 0 || constellation >= N_CONST) throw InvalidArg("unknown constellation");
    return acquire_single_impl(ctx, constellation, h_signal_f32, h_phasepoints, num_samples, sampling_freq,
                               center_freq, search_band, prn, samples_per_chunk, out);
  });
}

#define TGA_SINGLE_WRAPPER(name, cid)                                                                  \
  int name(tga_ctx* ctx, const float* s, const double* pp, size_t n, double fs, double fc, double band, \
           int prn, size_t per, tga_result* out) {                                                      \
    return tga_acquire_single(ctx, cid, s, pp, n, fs, fc, band, prn, per, out);                         \
  }
TGA_SINGLE_WRAPPER(tga_acquire_full, TGA_GPS)
TGA_SINGLE_WRAPPER(tga_acquire_sbas, TGA_SBAS)
TGA_SINGLE_WRAPPER(tga_acquire_qzss, TGA_QZSS)
TGA_SINGLE_WRAPPER(tga_acquire_galileo_single, TGA_GALILEO)
TGA_SINGLE_WRAPPER(tga_acquire_beidou_single, TGA_BEIDOU)
TGA_SINGLE_WRAPPER(tga_acquire_l1c_single, TGA_L1C)

int tga_acquire_all_device(tga_ctx* ctx, const uint8_t* d_packed_bits, size_t n_ant, size_t row_bytes,
                           double sampling_freq, const tga_all_options* opt, tga_cell* out, size_t out_capacity,
                           size_t* n_out) {
  return guarded(ctx, [&] {
    if (!d_packed_bits) throw InvalidArg("null bits");
    begin_call(ctx);
    return acquire_all_impl(ctx, d_packed_bits, n_ant, row_bytes, sampling_freq, opt, out, out_capacity, n_out);
  });
}

int tga_acquire_all(tga_ctx* ctx, const uint8_t* h_packed_bits, size_t n_ant, size_t row_bytes,
                    double sampling_freq, const tga_all_options* opt, tga_cell* out, size_t out_capacity,
                    size_t* n_out) {
  return guarded(ctx, [&] {
    if (!h_packed_bits) throw InvalidArg("null bits");
    const size_t bytes = n_ant * row_bytes;
    begin_call(ctx);
    uint8_t* d_bits = (uint8_t*)ctx->buf("bits", bytes);
    CK(cudaMemcpyAsync(d_bits, h_packed_bits, bytes, cudaMemcpyHostToDevice, ctx->stream));
    ctx->h2d += bytes;
    return acquire_all_impl(ctx, d_bits, n_ant, row_bytes, sampling_freq, opt, out, out_capacity, n_out);
  });
}

int tga_acquire_all_stream(tga_ctx* ctx, const uint8_t* const* h_packed_bits, size_t n_obs, size_t n_ant,
                           size_t row_bytes, double sampling_freq, const tga_all_options* opt, tga_cell* out,
                           size_t out_capacity, size_t* n_out) {
  return guarded(ctx, [&] {
    if (!h_packed_bits || !opt || !n_out) throw InvalidArg("null argument");
    for (size_t i = 0; i < n_obs; ++i)
      if (!h_packed_bits[i]) throw InvalidArg("null bits of observation " + std::to_string(i));
    size_t per = 0;
    int rc = tga_all_cell_count(n_ant, opt, &per);
    if (rc != TGA_OK) return rc;
    *n_out = per * n_obs;
    if (!out) return TGA_OK;
    if (out_capacity < per * n_obs) return TGA_ERR_CAPACITY;
    if (n_obs == 0) return TGA_OK;
    if (!ctx->copy_stream) {
      CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
      for (cudaEvent_t& e : ctx->copied) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    const size_t bytes = n_ant * row_bytes;
    begin_call(ctx);
    // both buffers before the first search, so that neither is reallocated
    // (and the searches' cached graphs stay valid) in the middle of the run
    uint8_t* buf[2] = {(uint8_t*)ctx->buf("bits", bytes), (uint8_t*)ctx->buf("bits.2", bytes)};
    auto copy = [&](size_t i) {
      CK(cudaMemcpyAsync(buf[i & 1], h_packed_bits[i], bytes, cudaMemcpyHostToDevice, ctx->copy_stream));
      CK(cudaEventRecord(ctx->copied[i & 1], ctx->copy_stream));
      ctx->h2d += bytes;
    };
    // the copy of observation i + 1 is queued before the search of i, which
    // returns only when it has finished (so buffer (i + 1) & 1, read by
    // search i - 1, is free)
    copy(0);
    double total_ms = 0.0;
    size_t n_i = 0;
    for (size_t i = 0; i < n_obs; ++i) {
      CK(cudaStreamWaitEvent(ctx->stream, ctx->copied[i & 1], 0));
      if (i + 1 < n_obs) copy(i + 1);
      rc = acquire_all_impl(ctx, buf[i & 1], n_ant, row_bytes, sampling_freq, opt, out + i * per, per, &n_i);
      if (rc != TGA_OK) return rc;
      total_ms += ctx->last_ms;
    }
    ctx->last_ms = total_ms;
    return TGA_OK;
  });
}

int tga_benchmark(tga_ctx* ctx, const uint8_t* h_packed_bits, size_t n_ant, size_t row_bytes, double fs,
                  tga_bench_entry out[6]) {
  return guarded(ctx, [&] {
    if (!h_packed_bits || !out || n_ant == 0 || row_bytes == 0) throw InvalidArg("empty observation or null output");
    if (!(fs > 0.0)) throw InvalidArg("sampling frequency must be positive");
    // main.rs:518-595: samples per period as `usize` truncations of f64 products
    const size_t per_ms = (size_t)(fs / 1000.0);
    const size_t per_gal = (size_t)(fs * (4092.0 / 1.023e6));
    const size_t per_10ms = (size_t)(fs * (10230.0 / 1.023e6));
    struct E {
      int c, prn;
      size_t per;
    };
    const E es[6] = {{TGA_GPS, 1, per_ms},    {TGA_GALILEO, 1, per_gal}, {TGA_BEIDOU, 1, per_10ms},
                     {TGA_SBAS, 120, per_ms}, {TGA_QZSS, 184, per_ms},   {TGA_L1C, 1, per_10ms}};
    const size_t n_rec = row_bytes * 8;
    const double pc = kTau / fs;
    for (int e = 0; e < 6; ++e) {
      const auto t0 = std::chrono::steady_clock::now();
      // setup: every antenna's window, as extract_ant_data (main.rs:497-517)
      const size_t n = std::min(2 * es[e].per, n_rec);
      std::vector<std::vector<float>> sig(n_ant, std::vector<float>(n));
      std::vector<double> pp(n);
      for (size_t k = 0; k < n; ++k) pp[k] = pc * (double)k;
      for (size_t a = 0; a < n_ant; ++a) {
        const uint8_t* row = h_packed_bits + a * row_bytes;
        long long ones = 0;
        for (size_t k = 0; k < row_bytes; ++k) ones += __builtin_popcount(row[k]);
        const double mean = (2.0 * (double)ones - (double)n_rec) / (double)n_rec;
        for (size_t k = 0; k < n; ++k) sig[a][k] = (float)((((row[k >> 3] >> (7 - (k & 7))) & 1) ? 1.0 : -1.0) - mean);
      }
      const auto t1 = std::chrono::steady_clock::now();
      // every entry uses IF 4.092 MHz and a 6 kHz band (acquisition.rs:72-75,
      // sbas.rs:24-27, qzss.rs:24-27, l1c.rs:27-30, main.rs:525-590)
      tga_result r;
      const int rc =
          acquire_single_impl(ctx, es[e].c, sig[0].data(), pp.data(), n, fs, 4.092e6, 6000.0, es[e].prn, es[e].per, &r);
      if (rc != TGA_OK) return rc;
      const auto t2 = std::chrono::steady_clock::now();
      out[e].constellation = es[e].c;
      out[e].prn = es[e].prn;
      out[e].setup_s = std::chrono::duration<double>(t1 - t0).count();
      out[e].search_s = std::chrono::duration<double>(t2 - t1).count();
      out[e].result = r;
    }
    return TGA_OK;
  });
}

int tga_all_cell_count(size_t n_ant, const tga_all_options* opt, size_t* n_cells) {
  if (!opt || !n_cells) return TGA_ERR_INVALID_ARG;
  try {
    size_t na = opt->ant_filter ? opt->n_ant_filter : n_ant, t = 0;
    for (int c = 0; c < N_CONST; ++c)
      if (opt->constellation_mask & (1u << c)) t += prn_list(c, opt).size() * na;
    *n_cells = t;
    return TGA_OK;
  } catch (...) {
    return TGA_ERR_INVALID_ARG;
  }
}

int tga_last_search_stats(const tga_ctx* ctx, double* cells, int32_t* launches, double* device_ms) {
  if (!ctx) return TGA_ERR_INVALID_ARG;
  if (cells) *cells = ctx->last_cells;
  if (launches) *launches = ctx->last_launches;
  if (device_ms) *device_ms = ctx->last_ms;
  return TGA_OK;
}

int tga_last_transfer_bytes(const tga_ctx* ctx, uint64_t* h2d, uint64_t* d2h) {
  if (!ctx) return TGA_ERR_INVALID_ARG;
  if (h2d) *h2d = ctx->h2d;
  if (d2h) *d2h = ctx->d2h;
  return TGA_OK;
}

void* tga_stream(tga_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int tga_set_test_flags(tga_ctx* ctx, int flags) {
  if (!ctx || (flags & ~TGA_TEST_TC_SKIP_COMMIT)) return TGA_ERR_INVALID_ARG;
  ctx->test_flags = flags;
  return TGA_OK;
}

int tga_set_precision(tga_ctx* ctx, int precision) {
  if (!ctx || (precision != TGA_PRECISION_FP32 && precision != TGA_PRECISION_FP16_TC)) return TGA_ERR_INVALID_ARG;
  ctx->precision = precision;
  return TGA_OK;
}

int tga_set_variant(tga_ctx* ctx, int lc, int variant) {
  if (!ctx || (lc != 1023 && lc != 4092 && lc != 10230) || variant < 0 || variant > 1) return TGA_ERR_INVALID_ARG;
  ctx->variant[ctx->precision][variant_slot(lc / 1023)] = variant;
  return TGA_OK;
}

int tga_autotune(tga_ctx* ctx, const uint8_t* d_packed_bits, size_t n_ant, size_t row_bytes, double fs,
                 const tga_all_options* opt, int reps, tga_tune_entry out[3], size_t* n_out) {
  return guarded(ctx, [&] {
    if (!d_packed_bits || !opt || !out || !n_out) throw InvalidArg("null argument");
    if (reps < 1 || reps > 100) throw InvalidArg("reps must be 1-100");
    size_t n_cells = 0;
    if (tga_all_cell_count(n_ant, opt, &n_cells) != TGA_OK) throw InvalidArg("invalid options");
    bool has[3] = {false, false, false};
    for (int c = 0; c < N_CONST; ++c)
      if (opt->constellation_mask & (1u << c)) has[variant_slot(info(c).primary_chips / 1023)] = true;
    // every candidate runs eagerly, so no graph is kept for a rejected one
    struct GraphsOff {
      tga_ctx* c;
      bool was;
      ~GraphsOff() { c->graphs_enabled = was; }
    } graphs_off{ctx, ctx->graphs_enabled};
    ctx->graphs_enabled = false;
    int* var = ctx->variant[ctx->precision];
    std::vector<tga_cell> ref(n_cells), cur(n_cells);
    // one untimed run, then the median device time of `reps` runs
    auto measure = [&](std::vector<tga_cell>& cells, double* ms) -> int {
      std::vector<double> t;
      for (int r = 0; r <= reps; ++r) {
        size_t n = 0;
        begin_call(ctx);
        const int rc = acquire_all_impl(ctx, d_packed_bits, n_ant, row_bytes, fs, opt, cells.data(),
                                        cells.size(), &n);
        if (rc != TGA_OK) return rc;
        if (r > 0) t.push_back(ctx->last_ms);
      }
      std::sort(t.begin(), t.end());
      *ms = t[t.size() / 2];
      return TGA_OK;
    };
    auto same = [](const std::vector<tga_cell>& a, const std::vector<tga_cell>& b) {
      return a.size() == b.size() && std::memcmp(a.data(), b.data(), a.size() * sizeof(tga_cell)) == 0;
    };
    static const int kLc[3] = {1023, 4092, 10230};
    size_t k = 0;
    for (int slot = 0; slot < 3; ++slot) {
      if (!has[slot]) continue;
      tga_tune_entry& e = out[k++];
      e.lc = kLc[slot];
      int best = 0;
      for (int v = 0; v < 2; ++v) {
        var[slot] = v;
        const int rc = measure(v == 0 ? ref : cur, &e.ms[v]);
        if (rc != TGA_OK) {
          var[slot] = 0;
          return rc;
        }
        e.same_results[v] = v == 0 ? 1 : same(ref, cur);
        if (e.same_results[v] && e.ms[v] < e.ms[best]) best = v;
      }
      var[slot] = best;
      e.variant = best;
    }
    *n_out = k;
    return TGA_OK;
  });
}

int tga_last_row_peaks(tga_ctx* ctx, int chips, double* out, size_t cap, size_t* n_out, int64_t* n_rows_refined) {
  return guarded(ctx, [&] {
    if (!n_out) throw InvalidArg("null n_out");
    const tga_ctx::LastGroup* g = nullptr;
    for (const auto& lg : ctx->last_groups)
      if (lg.Lc == chips) g = &lg;
    if (!g) throw InvalidArg("the last search had no fused group of " + std::to_string(chips) + " chips");
    const bool nc = g->nc_power_scale > 0.0;
    const size_t n = (size_t)g->n_ant * g->nb * (nc ? 1 : 2) * g->n_prn;
    *n_out = n;
    if (n_rows_refined) {
      std::vector<int> cnt((size_t)g->n_chunks, 0);
      if (g->tc) CK(cudaMemcpy(cnt.data(), g->count, cnt.size() * sizeof(int), cudaMemcpyDeviceToHost));
      int64_t sum = 0;
      for (int c : cnt) sum += c;
      *n_rows_refined = sum;
    }
    if (!out) return TGA_OK;
    if (cap < n) return TGA_ERR_CAPACITY;
    std::vector<unsigned long long> keys(n);
    CK(cudaMemcpy(keys.data(), g->keys, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    // the reference's |IFFT_2P| / sqrt(2P) is |y| sqrt(2P) / Lc; the
    // non-coherent power is |y|^2 nc_power_scale
    const double scale = g->amp * std::sqrt(2.0 * (double)g->P) / (double)g->Lc;
    for (size_t i = 0; i < n; ++i) {
      const uint32_t bits = (uint32_t)(keys[i] >> 32);
      float pw;
      std::memcpy(&pw, &bits, sizeof pw);
      out[i] = nc ? (double)pw * g->amp * g->amp * g->nc_power_scale : std::sqrt((double)pw) * scale;
    }
    return TGA_OK;
  });
}

int tga_set_graphs(tga_ctx* ctx, int enable) {
  if (!ctx) return TGA_ERR_INVALID_ARG;
  ctx->graphs_enabled = enable != 0;
  return TGA_OK;
}

int tga_last_graph(const tga_ctx* ctx, int* state) {
  if (!ctx || !state) return TGA_ERR_INVALID_ARG;
  *state = ctx->last_graph;
  return TGA_OK;
}

int tga_set_profiling(tga_ctx* ctx, int enable) {
  if (!ctx) return TGA_ERR_INVALID_ARG;
  ctx->profiling = enable != 0;
  return TGA_OK;
}

int tga_kernel_times(const tga_ctx* ctx, int cap, const char** names, double* ms, int32_t* launches,
                     double* flops, int* n) {
  if (!ctx || !n) return TGA_ERR_INVALID_ARG;
  *n = (int)ctx->ktimes.size();
  for (int i = 0; i < *n && i < cap; ++i) {
    if (names) names[i] = ctx->ktimes[i].first.c_str();
    if (ms) ms[i] = ctx->ktimes[i].second.ms;
    if (launches) launches[i] = ctx->ktimes[i].second.launches;
    if (flops) flops[i] = ctx->ktimes[i].second.flops;
  }
  return *n > cap ? TGA_ERR_CAPACITY : TGA_OK;
}

int tga_acr_cn0(tga_ctx* ctx, const double* h_r_a, size_t n, int table, double* h_cn0, uint8_t* h_valid) {
  return guarded(ctx, [&] {
    if (table < 0 || table > 3) throw InvalidArg("unknown ACR table");
    if (n == 0) return TGA_OK;
    if (!h_r_a || !h_cn0 || !h_valid) throw InvalidArg("null pointer");
    double* d_ra = (double*)ctx->buf("acr.ra", n * sizeof(double));
    double* d_c = (double*)ctx->buf("acr.cn0", n * sizeof(double));
    uint8_t* d_v = (uint8_t*)ctx->buf("acr.valid", n);
    CK(cudaMemcpyAsync(d_ra, h_r_a, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_acr_batch(d_ra, (int)n, table, d_c, d_v, ctx->stream));
    CK(cudaMemcpyAsync(h_cn0, d_c, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(h_valid, d_v, n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TGA_OK;
  });
}

int tga_antenna_xcorr_matrix(tga_ctx* ctx, const uint8_t* h_bits, size_t n_ant, size_t row_bytes, double* out) {
  return guarded(ctx, [&] {
    if (!h_bits || !out || n_ant == 0 || row_bytes == 0) throw InvalidArg("bad arguments");
    uint8_t* d_bits = (uint8_t*)ctx->buf("xc.bits", n_ant * row_bytes);
    unsigned long long* d_cnt = (unsigned long long*)ctx->buf("xc.cnt", n_ant * n_ant * 8);
    CK(cudaMemcpyAsync(d_bits, h_bits, n_ant * row_bytes, cudaMemcpyHostToDevice, ctx->stream));
    CK(launch_xcorr_matrix(d_bits, (int)n_ant, row_bytes, d_cnt, ctx->stream));
    std::vector<unsigned long long> cnt(n_ant * n_ant);
    CK(cudaMemcpyAsync(cnt.data(), d_cnt, cnt.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const double n = (double)(row_bytes * 8);
    // sum of +-1 products = agree - disagree = 2*agree - n (exact), / n
    for (size_t i = 0; i < cnt.size(); ++i) out[i] = (2.0 * (double)cnt[i] - n) / n;
    return TGA_OK;
  });
}

int tga_antenna_xcorr(tga_ctx* ctx, const uint8_t* h_bits, size_t n_ant, size_t row_bytes, int i, int j,
                      double* out) {
  return guarded(ctx, [&] {
    if (!h_bits || !out || row_bytes == 0) throw InvalidArg("bad arguments");
    if (i < 0 || (size_t)i >= n_ant) throw InvalidArg("antenna index " + std::to_string(i) + " out of range");
    if (j < 0 || (size_t)j >= n_ant) throw InvalidArg("antenna index " + std::to_string(j) + " out of range");
    uint8_t* d_bits = (uint8_t*)ctx->buf("xc.pair", 2 * row_bytes);
    CK(cudaMemcpyAsync(d_bits, h_bits + (size_t)i * row_bytes, row_bytes, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_bits + row_bytes, h_bits + (size_t)j * row_bytes, row_bytes, cudaMemcpyHostToDevice,
                       ctx->stream));
    unsigned long long* d_cnt = (unsigned long long*)ctx->buf("xc.cnt2", 4 * 8);
    CK(launch_xcorr_matrix(d_bits, 2, row_bytes, d_cnt, ctx->stream));
    unsigned long long cnt[4];
    CK(cudaMemcpyAsync(cnt, d_cnt, sizeof cnt, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const double n = (double)(row_bytes * 8);
    *out = (2.0 * (double)cnt[1] - n) / n;
    return TGA_OK;
  });
}

// ---------------------------------------------------------------------------
// fine acquisition (tga_fine_eval, tga_fine_acquire)
// ---------------------------------------------------------------------------
namespace {

using cplx = std::complex<double>;

struct FineOpts {
  double sigma_chips = 0.1, scan_hw = 0.0, tol_tau = 1e-4, tol_f = 1e-3;
  int max_iter = 20;
};

FineOpts fine_opts(const tga_fine_options* o) {
  FineOpts r;
  if (!o) return r;
  if (o->edge_sigma_chips > 0) r.sigma_chips = o->edge_sigma_chips;
  r.scan_hw = o->scan_half_width_hz;
  if (o->max_iter > 0) r.max_iter = o->max_iter;
  if (o->tol_code_phase > 0) r.tol_tau = o->tol_code_phase;
  if (o->tol_frequency > 0) r.tol_f = o->tol_frequency;
  return r;
}

// replica model of one satellite: its (sub)chip sequence on the device, T
// samples per (sub)chip, edge smoothing sigma in samples
struct FineJob {
  tga_fine_task t;
  const int8_t* d_seq = nullptr;
  int L = 0;
  double T = 0, sigma = 0;
};

FineJob fine_job(tga_ctx* ctx, double fs, const tga_fine_task& t, double sigma_chips, size_t total_samples) {
  if (t.constellation < 0 || t.constellation >= N_CONST) throw InvalidArg("bad constellation");
  validate_prn(t.constellation, t.prn);
  if (t.length <= 0 || t.start < 0 || (size_t)(t.start + t.length) > total_samples)
    throw InvalidArg("fine-acquisition window outside the recording");
  if (!std::isfinite(t.code_phase) || !std::isfinite(t.frequency)) throw InvalidArg("non-finite start point");
  const ConstellationInfo& ci = info(t.constellation);
  FineJob j;
  j.t = t;
  const std::string name = "fine.seq." + std::to_string(t.constellation) + "." + std::to_string(t.prn);
  const std::vector<int8_t> seq = resample_sequence(t.constellation, t.prn);
  j.L = (int)seq.size();
  j.d_seq = (const int8_t*)ctx->buf(name, seq.size());
  if (!ctx->uploaded.count(name)) {
    CK(cudaMemcpy((void*)j.d_seq, seq.data(), seq.size(), cudaMemcpyHostToDevice));
    ctx->uploaded[name] = {};
  }
  j.T = fs * ci.code_period_s / (double)j.L;
  j.sigma = sigma_chips * fs * ci.code_period_s / (double)ci.primary_chips;
  return j;
}

FineTask fine_task(const FineJob& j, double fs, double tau, double f, int slot) {
  FineTask k;
  k.seq = j.d_seq;
  k.seq_len = j.L;
  k.slot = slot;
  k.T = j.T;
  k.tau = tau;
  k.f_over_fs = f / fs;
  k.two_pi_over_fs = 2.0 * M_PI / fs;
  k.start = j.t.start;
  k.length = j.t.length;
  k.n0 = (double)j.t.start + 0.5 * (double)j.t.length;
  k.sigma = j.sigma;
  return k;
}

// device bits and the antenna means (over the whole row, as the search)
void fine_upload(tga_ctx* ctx, const uint8_t* h_bits, size_t A, size_t row_bytes, const uint8_t** d_bits,
                 const double** d_mean) {
  uint8_t* b = (uint8_t*)ctx->buf("fine.bits", A * row_bytes);
  CK(cudaMemcpyAsync(b, h_bits, A * row_bytes, cudaMemcpyHostToDevice, ctx->stream));
  ctx->h2d += A * row_bytes;
  double* m = (double*)ctx->buf("fine.mean", A * sizeof(double));
  CK(launch_antenna_means(b, (int)A, row_bytes, m, ctx->stream));
  *d_bits = b;
  *d_mean = m;
}

// sums of a batch of evaluations, normalised by the window length:
// out[task][antenna][R, dR/dtau, dR/df, d2R/dtau2, d2R/df2, d2R/dtau df]
void fine_sums(tga_ctx* ctx, const uint8_t* d_bits, size_t A, size_t row_bytes, const double* d_mean,
               const std::vector<FineTask>& tasks, std::vector<cplx>& out) {
  const size_t n = tasks.size();
  FineTask* d_tasks = (FineTask*)ctx->buf("fine.tasks", n * sizeof(FineTask));
  double* d_out = (double*)ctx->buf("fine.sums", n * A * 12 * sizeof(double));
  CK(cudaMemcpyAsync(d_tasks, tasks.data(), n * sizeof(FineTask), cudaMemcpyHostToDevice, ctx->stream));
  long long max_len = 0;
  for (const FineTask& t : tasks) max_len = std::max(max_len, t.length);
  CK(launch_fine_sums(d_bits, (int)A, row_bytes, d_mean, d_tasks, (int)n, max_len, d_out, ctx->stream));
  std::vector<double> h(n * A * 12);
  CK(cudaMemcpyAsync(h.data(), d_out, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  out.resize(n * A * 6);
  for (size_t i = 0; i < n; ++i) {
    const double inv = 1.0 / (double)tasks[i].length;
    for (size_t k = 0; k < A * 6; ++k)
      out[i * A * 6 + k] = cplx(h[i * A * 12 + 2 * k], h[i * A * 12 + 2 * k + 1]) * inv;
  }
}

// P = |sum_a exp(-i phi_a) R_a|^2 with its gradient and Hessian in the order
// (tau, f, phi_0 .. phi_{A-1}); g and H may be null
void fine_assemble(const cplx* R, int A, const double* phi, double* P, double* g, double* H) {
  cplx S, St, Sf, Stt, Sff, Stf;
  std::vector<cplx> u(A);
  for (int a = 0; a < A; ++a) {
    u[a] = std::polar(1.0, -phi[a]);
    const cplx* r = R + (size_t)a * 6;
    S += u[a] * r[0];
    St += u[a] * r[1];
    Sf += u[a] * r[2];
    Stt += u[a] * r[3];
    Sff += u[a] * r[4];
    Stf += u[a] * r[5];
  }
  const cplx cS = std::conj(S);
  *P = std::norm(S);
  const int D = 2 + A;
  const cplx mi(0.0, -1.0);
  if (g) {
    g[0] = 2.0 * (cS * St).real();
    g[1] = 2.0 * (cS * Sf).real();
    for (int a = 0; a < A; ++a) g[2 + a] = 2.0 * (cS * (mi * u[a] * R[(size_t)a * 6])).real();
  }
  if (H) {
    H[0] = 2.0 * (std::conj(St) * St + cS * Stt).real();
    H[D + 1] = 2.0 * (std::conj(Sf) * Sf + cS * Sff).real();
    H[1] = H[D] = 2.0 * (std::conj(St) * Sf + cS * Stf).real();
    for (int a = 0; a < A; ++a) {
      const cplx* r = R + (size_t)a * 6;
      const cplx Q = mi * u[a] * r[0], Qt = mi * u[a] * r[1], Qf = mi * u[a] * r[2];
      H[2 + a] = H[(size_t)(2 + a) * D] = 2.0 * (std::conj(St) * Q + cS * Qt).real();
      H[D + 2 + a] = H[(size_t)(2 + a) * D + 1] = 2.0 * (std::conj(Sf) * Q + cS * Qf).real();
      for (int b = 0; b < A; ++b) {
        const cplx Qb = mi * u[b] * R[(size_t)b * 6];
        double v = 2.0 * (std::conj(Q) * Qb).real();
        if (a == b) v += 2.0 * (cS * (-u[a] * r[0])).real();
        H[(size_t)(2 + a) * D + 2 + b] = v;
      }
    }
  }
}

// solves M x = b for symmetric positive definite M (n x n, overwritten);
// false when M is not positive definite
bool cholesky_solve(std::vector<double>& M, std::vector<double>& b, int n) {
  for (int j = 0; j < n; ++j) {
    double d = M[(size_t)j * n + j];
    for (int k = 0; k < j; ++k) d -= M[(size_t)j * n + k] * M[(size_t)j * n + k];
    if (!(d > 0.0)) return false;
    d = std::sqrt(d);
    M[(size_t)j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double v = M[(size_t)i * n + j];
      for (int k = 0; k < j; ++k) v -= M[(size_t)i * n + k] * M[(size_t)j * n + k];
      M[(size_t)i * n + j] = v / d;
    }
  }
  for (int i = 0; i < n; ++i) {
    double v = b[i];
    for (int k = 0; k < i; ++k) v -= M[(size_t)i * n + k] * b[k];
    b[i] = v / M[(size_t)i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    double v = b[i];
    for (int k = i + 1; k < n; ++k) v -= M[(size_t)k * n + i] * b[k];
    b[i] = v / M[(size_t)i * n + i];
  }
  return true;
}

}  // namespace

int tga_fine_eval(tga_ctx* ctx, const uint8_t* h_bits, size_t n_ant, size_t row_bytes, double fs,
                  const tga_fine_task* task, const double* phases, double edge_sigma_chips, double* power,
                  double* grad, double* hess) {
  return guarded(ctx, [&] {
    if (!h_bits || !task || !power || n_ant == 0 || row_bytes == 0 || !(fs > 0)) throw InvalidArg("bad arguments");
    const FineJob j = fine_job(ctx, fs, *task, edge_sigma_chips > 0 ? edge_sigma_chips : 0.1, row_bytes * 8);
    const uint8_t* d_bits;
    const double* d_mean;
    fine_upload(ctx, h_bits, n_ant, row_bytes, &d_bits, &d_mean);
    std::vector<cplx> R;
    fine_sums(ctx, d_bits, n_ant, row_bytes, d_mean, {fine_task(j, fs, task->code_phase, task->frequency, 0)}, R);
    std::vector<double> phi(n_ant);
    for (size_t a = 0; a < n_ant; ++a) phi[a] = phases ? phases[a] : std::arg(R[a * 6]);
    fine_assemble(R.data(), (int)n_ant, phi.data(), power, grad, hess);
    return TGA_OK;
  });
}

int tga_fine_acquire(tga_ctx* ctx, const uint8_t* h_bits, size_t n_ant, size_t row_bytes, double fs,
                     const tga_fine_task* tasks, size_t n_tasks, const tga_fine_options* opt,
                     tga_fine_result* out, double* phases) {
  return guarded(ctx, [&] {
    if (!h_bits || (!tasks && n_tasks) || (!out && n_tasks) || n_ant == 0 || row_bytes == 0 || !(fs > 0))
      throw InvalidArg("bad arguments");
    if (n_tasks == 0) return TGA_OK;
    const FineOpts o = fine_opts(opt);
    const int A = (int)n_ant;
    std::vector<FineJob> jobs;
    for (size_t i = 0; i < n_tasks; ++i) jobs.push_back(fine_job(ctx, fs, tasks[i], o.sigma_chips, row_bytes * 8));
    const uint8_t* d_bits;
    const double* d_mean;
    fine_upload(ctx, h_bits, n_ant, row_bytes, &d_bits, &d_mean);

    struct St {
      double tau, f, P = 0, lambda = 0;
      std::vector<double> phi;
      std::vector<cplx> R;  // sums at (tau, f)
      bool done = false, conv = false;
      int iters = 0;
    };
    std::vector<St> st(n_tasks);
    std::vector<cplx> R;
    auto aligned = [&](const cplx* r, std::vector<double>& phi) {
      double s = 0;
      phi.resize(A);
      for (int a = 0; a < A; ++a) {
        phi[a] = std::arg(r[(size_t)a * 6]);
        s += std::abs(r[(size_t)a * 6]);
      }
      return s * s;  // P with every antenna phase-aligned
    };

    // 1. frequency pre-scan: the grid's Doppler bins are coarser than the
    //    main lobe of a long window, so the start may sit on a side lobe
    std::vector<int> nscan(n_tasks, 0);
    std::vector<FineTask> batch;
    for (size_t i = 0; i < n_tasks; ++i) {
      const double win = (double)tasks[i].length / fs;
      const double df = 0.25 / win;
      const double hw = o.scan_hw == 0.0 ? 150.0 + 1.0 / win : o.scan_hw;
      const int K = hw < 0 ? 0 : (int)std::ceil(hw / df);
      nscan[i] = K;
      for (int k = -K; k <= K; ++k)
        batch.push_back(fine_task(jobs[i], fs, tasks[i].code_phase, tasks[i].frequency + k * df, (int)batch.size()));
    }
    fine_sums(ctx, d_bits, n_ant, row_bytes, d_mean, batch, R);
    size_t pos = 0;
    for (size_t i = 0; i < n_tasks; ++i) {
      const double df = 0.25 * fs / (double)tasks[i].length;
      const int K = nscan[i];
      double best = -1;
      int kb = 0;
      std::vector<double> tmp;
      for (int k = -K; k <= K; ++k, ++pos) {
        const double p = aligned(&R[pos * n_ant * 6], tmp);
        if (k == 0) out[i].power_start = p;
        if (p > best) {
          best = p;
          kb = k;
        }
      }
      st[i].tau = tasks[i].code_phase;
      st[i].f = tasks[i].frequency + kb * df;
    }
    // 2. phase-aligned start at the scan maximum
    batch.clear();
    for (size_t i = 0; i < n_tasks; ++i) batch.push_back(fine_task(jobs[i], fs, st[i].tau, st[i].f, (int)i));
    fine_sums(ctx, d_bits, n_ant, row_bytes, d_mean, batch, R);
    for (size_t i = 0; i < n_tasks; ++i) {
      st[i].R.assign(R.begin() + i * n_ant * 6, R.begin() + (i + 1) * n_ant * 6);
      st[i].P = aligned(st[i].R.data(), st[i].phi);
    }

    // 3. damped Newton (Levenberg-Marquardt) on (tau, f, phi_1 .. phi_{A-1});
    //    phi_0 stays fixed because P does not change with a common phase
    const int D = 2 + A, Dr = 1 + A;
    std::vector<double> g(D), H((size_t)D * D), M((size_t)Dr * Dr), b(Dr);
    for (int it = 0; it < o.max_iter; ++it) {
      batch.clear();
      std::vector<int> who;
      std::vector<std::vector<double>> trial_phi;
      std::vector<double> trial_dtau, trial_df;
      for (size_t i = 0; i < n_tasks; ++i) {
        St& s = st[i];
        if (s.done) continue;
        double P;
        fine_assemble(s.R.data(), A, s.phi.data(), &P, g.data(), H.data());
        // reduced system (drop phi_0 = index 2)
        auto red = [&](int r) { return r < 2 ? r : r + 1; };
        double dmax = 0;
        for (int r = 0; r < Dr; ++r) dmax = std::max(dmax, std::abs(H[(size_t)red(r) * D + red(r)]));
        bool ok = false;
        for (int tries = 0; tries < 12 && !ok; ++tries) {
          for (int r = 0; r < Dr; ++r) {
            b[r] = g[red(r)];
            for (int c = 0; c < Dr; ++c) M[(size_t)r * Dr + c] = -H[(size_t)red(r) * D + red(c)];
            M[(size_t)r * Dr + r] += s.lambda * std::max(std::abs(H[(size_t)red(r) * D + red(r)]), 1e-12 * dmax);
          }
          ok = cholesky_solve(M, b, Dr);
          if (!ok) s.lambda = s.lambda == 0 ? 1e-3 : s.lambda * 10;
        }
        if (!ok) {
          s.done = true;
          continue;
        }
        // stay inside the smooth peak: at most 2 samples and half a main lobe per step
        const double win = (double)tasks[i].length / fs;
        double scale = 1.0;
        if (std::abs(b[0]) > 2.0) scale = 2.0 / std::abs(b[0]);
        if (std::abs(b[1]) > 0.5 / win) scale = std::min(scale, 0.5 / win / std::abs(b[1]));
        std::vector<double> phi = s.phi;
        for (int a = 1; a < A; ++a) phi[a] += scale * b[1 + a];
        who.push_back((int)i);
        trial_phi.push_back(phi);
        trial_dtau.push_back(scale * b[0]);
        trial_df.push_back(scale * b[1]);
        batch.push_back(fine_task(jobs[i], fs, s.tau + scale * b[0], s.f + scale * b[1], (int)batch.size()));
      }
      if (batch.empty()) break;
      fine_sums(ctx, d_bits, n_ant, row_bytes, d_mean, batch, R);
      for (size_t k = 0; k < who.size(); ++k) {
        St& s = st[who[k]];
        ++s.iters;
        double Pn;
        fine_assemble(&R[k * n_ant * 6], A, trial_phi[k].data(), &Pn, nullptr, nullptr);
        if (Pn >= s.P) {
          s.tau += trial_dtau[k];
          s.f += trial_df[k];
          s.phi = trial_phi[k];
          s.R.assign(R.begin() + k * n_ant * 6, R.begin() + (k + 1) * n_ant * 6);
          s.P = Pn;
          s.lambda = s.lambda < 1e-6 ? 0.0 : s.lambda * 0.1;
          if (std::abs(trial_dtau[k]) < o.tol_tau && std::abs(trial_df[k]) < o.tol_f) {
            s.conv = true;
            s.done = true;
          }
        } else {
          s.lambda = s.lambda == 0 ? 1e-3 : s.lambda * 10;
          if (s.lambda > 1e12) s.done = true;
        }
      }
    }
    for (size_t i = 0; i < n_tasks; ++i) {
      out[i].code_phase = st[i].tau;
      out[i].frequency = st[i].f;
      out[i].power = st[i].P;
      out[i].iterations = st[i].iters;
      out[i].converged = st[i].conv ? 1 : 0;
      if (phases)
        for (int a = 0; a < A; ++a) phases[i * n_ant + a] = st[i].phi[a];
    }
    return TGA_OK;
  });
}

// ---------------------------------------------------------------------------
// narrowband RFI scan (tga_rfi_scan), rfi.rs:91-168
// ---------------------------------------------------------------------------
int tga_rfi_scan(tga_ctx* ctx, const uint8_t* h_bits, size_t n_ant, size_t row_bytes, double fs,
                 tga_rfi_channel* out) {
  return guarded(ctx, [&] {
    if (!h_bits || !out || n_ant == 0 || row_bytes == 0 || !(fs > 0)) throw InvalidArg("bad arguments");
    const size_t A = n_ant;
    const long long n = (long long)row_bytes * 8, half = n / 2;
    if (n > 0x7fffffffLL) throw InvalidArg("record longer than 2^31 samples");
    constexpr int kCap = 1 << 16;  // candidate lines per antenna
    cudaStream_t st = ctx->stream;
    uint8_t* d_bits = (uint8_t*)ctx->buf("rfi.bits", A * row_bytes);
    CK(cudaMemcpyAsync(d_bits, h_bits, A * row_bytes, cudaMemcpyHostToDevice, st));
    ctx->h2d += A * row_bytes;
    double* d_mean = (double*)ctx->buf("rfi.mean", A * sizeof(double));
    CK(launch_antenna_means(d_bits, (int)A, row_bytes, d_mean, st));
    double* d_z = (double*)ctx->buf("rfi.z", A * (size_t)n * sizeof(double));
    void* d_X = ctx->buf("rfi.X", A * (size_t)(n / 2 + 1) * 16);
    void* d_work = ctx->buf("rfi.work", fft64_workspace_bytes(n, (int)A));
    double* d_p = (double*)ctx->buf("rfi.p", A * (size_t)half * sizeof(double));
    unsigned* d_hist = (unsigned*)ctx->buf("rfi.hist", A * 256 * sizeof(unsigned));
    unsigned long long* d_prefix = (unsigned long long*)ctx->buf("rfi.prefix", A * 8);
    unsigned long long* d_rank = (unsigned long long*)ctx->buf("rfi.rank", A * 8);
    unsigned* d_count = (unsigned*)ctx->buf("rfi.count", A * sizeof(unsigned));
    long long* d_bins = (long long*)ctx->buf("rfi.bins", A * kCap * sizeof(long long));
    double* d_excess = (double*)ctx->buf("rfi.excess", A * kCap * sizeof(double));
    unsigned long long* d_acf = (unsigned long long*)ctx->buf("rfi.acf", A * 9 * 8);
    std::string why;
    const cudaError_t e = rfi_scan_device(d_bits, (int)A, row_bytes, d_mean, d_z, d_X, d_work, d_p, d_hist, d_prefix,
                                          d_rank, kCap, d_count, d_bins, d_excess, d_acf, ctx->num_sms, st, &why);
    if (!why.empty()) throw std::runtime_error(why);
    CK(e);
    std::vector<double> mean(A);
    std::vector<unsigned> count(A);
    std::vector<unsigned long long> acf(A * 9);
    CK(cudaMemcpyAsync(mean.data(), d_mean, A * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(count.data(), d_count, A * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(acf.data(), d_acf, A * 9 * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (size_t a = 0; a < A; ++a)
      if (count[a] > (unsigned)kCap) throw std::runtime_error("more than 65536 candidate RFI lines on one antenna");
    const int lags[3] = {1, 3, 16};
    for (size_t a = 0; a < A; ++a) {
      tga_rfi_channel& ch = out[a];
      std::memset(&ch, 0, sizeof ch);
      ch.antenna = (int32_t)a;
      const double m = mean[a];
      // variance of z = s - m over the row (rfi.rs:148): ones (1-m)^2 + zeros (1+m)^2
      const double ones = 0.5 * (m + 1.0) * (double)n;
      const double var = (ones * (1.0 - m) * (1.0 - m) + ((double)n - ones) * (1.0 + m) * (1.0 + m)) / (double)n;
      const double nan = std::nan("");
      ch.acf_lag1 = ch.acf_lag3 = ch.acf_lag16 = ch.period_samples = nan;
      if (var < 1e-9 || n < 8) {
        ch.dead = var < 1e-9 ? 1 : 0;
        continue;
      }
      double* acfs[3] = {&ch.acf_lag1, &ch.acf_lag3, &ch.acf_lag16};
      for (int l = 0; l < 3; ++l) {
        const double cnt = (double)(n - lags[l]);
        const double diff = (double)acf[a * 9 + 3 * l], oh = (double)acf[a * 9 + 3 * l + 1],
                     ot = (double)acf[a * 9 + 3 * l + 2];
        const double sss = cnt - 2.0 * diff, sh = 2.0 * oh - cnt, stl = 2.0 * ot - cnt;
        *acfs[l] = (sss - m * (sh + stl) + cnt * m * m) / cnt;
      }
      // candidate lines: strongest first, ties in bin order (a stable sort of
      // the bin-ordered list, rfi.rs:126), then 10 kHz clustering
      const unsigned c = count[a];
      std::vector<long long> bins(c);
      std::vector<double> ex(c);
      if (c) {
        CK(cudaMemcpy(bins.data(), d_bins + a * kCap, c * sizeof(long long), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(ex.data(), d_excess + a * kCap, c * sizeof(double), cudaMemcpyDeviceToHost));
      }
      std::vector<size_t> idx(c);
      for (size_t i = 0; i < c; ++i) idx[i] = i;
      std::sort(idx.begin(), idx.end(), [&](size_t x, size_t y) {
        if (ex[x] != ex[y]) return ex[x] > ex[y];
        return bins[x] < bins[y];
      });
      const double bin_hz = fs / (double)n;
      for (size_t i : idx) {
        const double f = (double)bins[i] * bin_hz;
        bool far = true;
        for (int k = 0; k < ch.n_lines; ++k)
          if (!(std::abs(ch.lines[k].frequency - f) > 10000.0)) far = false;
        if (!far) continue;
        ch.lines[ch.n_lines].frequency = f;
        ch.lines[ch.n_lines].excess_db = ex[i];
        if (++ch.n_lines == 3) break;
      }
      if (ch.n_lines) ch.period_samples = fs / ch.lines[0].frequency;
    }
    return TGA_OK;
  });
}

// ---------------------------------------------------------------------------
// non-coherent search (tga_search_noncoherent, tga_search_noncoherent_multi)
// ---------------------------------------------------------------------------
namespace {

// One constellation's search of a multi call, validated.
struct NcMember {
  const tga_nc_options* opt = nullptr;
  int c = 0;
  std::vector<int32_t> ants, prns;
  PolyClass pc;
  size_t out_off = 0;  // first cell of this member in the caller's output
};

NcMember nc_member(tga_ctx* ctx, const tga_nc_options* opt, size_t n_ant_total, size_t row_bytes, double fs) {
  NcMember m;
  m.opt = opt;
  const int c = opt->constellation;
  if (c < 0 || c >= N_CONST) throw InvalidArg("bad constellation");
  m.c = c;
  if (opt->n_bins < 1 || opt->coherent_periods < 1 || opt->blocks < 1 || opt->start < 0 || !(opt->bin_step_hz >= 0))
    throw InvalidArg("bad search geometry");
  if (opt->ant_filter) {
    for (size_t i = 0; i < opt->n_ant_filter; ++i) {
      if (opt->ant_filter[i] < 0 || (size_t)opt->ant_filter[i] >= n_ant_total)
        throw InvalidArg("antenna index out of range");
      m.ants.push_back(opt->ant_filter[i]);
    }
  } else {
    for (size_t i = 0; i < n_ant_total; ++i) m.ants.push_back((int32_t)i);
  }
  if (m.ants.empty()) throw InvalidArg("no antennas selected");
  const ConstellationInfo& ci = info(c);
  if (opt->prn_filter) {
    for (size_t i = 0; i < opt->n_prn_filter; ++i) {
      validate_prn(c, opt->prn_filter[i]);
      m.prns.push_back(opt->prn_filter[i]);
    }
  } else {
    for (int q = ci.prn_first; q <= ci.prn_last; ++q) m.prns.push_back(q);
  }
  const size_t P = period_samples(c, fs);
  if (P == 0) throw InvalidArg("sampling frequency too low for " + std::string(ci.json_key));
  const long long need = opt->start + (long long)opt->blocks * opt->coherent_periods * (long long)P;
  if (need > (long long)row_bytes * 8) throw InvalidArg("the blocks run past the end of the recording");
  std::vector<int> prns_i(m.prns.begin(), m.prns.end());
  if (!poly_class_for(ctx, c, (double)P, P, 2 * P, prns_i, &m.pc)) {
    ctx->err = "non-coherent search needs an integer number of samples per chip";
    throw std::domain_error(ctx->err);
  }
  return m;
}

// Members that can share one front end: the same polyphase class and the
// same blocks, Doppler grid and antennas.
bool nc_same_group(const NcMember& a, const NcMember& b) {
  const tga_nc_options *x = a.opt, *y = b.opt;
  return same_class(a.pc, b.pc) && x->center_freq == y->center_freq && x->bin_step_hz == y->bin_step_hz &&
         x->n_bins == y->n_bins && x->coherent_periods == y->coherent_periods && x->blocks == y->blocks &&
         x->start == y->start && a.ants == b.ants;
}

// The search of one group on the device bits (means already computed):
// front end and forward transform once, then every member's PRNs together.
// Writes each member's cells at its out_off.  gi names the group's key
// buffers, which stay alive for tga_last_row_peaks.
void nc_run_group(tga_ctx* ctx, const uint8_t* d_bits, size_t row_bytes, const double* d_mean, double fs,
                  const std::vector<NcMember*>& mem, int gi, tga_nc_cell* out) {
  const NcMember& m0 = *mem[0];
  const tga_nc_options* opt = m0.opt;
  const PolyClass& pc = m0.pc;
  const size_t P = pc.P;
  cudaStream_t st = ctx->stream;
  const std::vector<int32_t>& ants = m0.ants;
  std::vector<std::pair<int, int>> prns;  // (constellation, prn) in member order
  for (const NcMember* m : mem)
    for (int q : m->prns) prns.push_back({m->c, q});
  const int n_ant = (int)ants.size(), n_prn = (int)prns.size(), nb = opt->n_bins, B = opt->blocks;
  const std::string tag = "nc" + std::to_string(gi);
  int32_t* d_ant = (int32_t*)ctx->buf(tag + ".ant", ants.size() * sizeof(int32_t));
  CK(cudaMemcpyAsync(d_ant, ants.data(), ants.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  std::vector<double> fc(nb);
  for (int i = 0; i < nb; ++i) fc[i] = opt->center_freq + (double)(i - (nb - 1) / 2) * opt->bin_step_hz;
  double* d_fc = (double*)ctx->buf(tag + ".fc", fc.size() * sizeof(double));
  CK(cudaMemcpyAsync(d_fc, fc.data(), fc.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  std::vector<int8_t> chips((size_t)n_prn * pc.Lc);
  for (int i = 0; i < n_prn; ++i) {
    const std::vector<int8_t>& ch = cached_chips(ctx, prns[i].first, prns[i].second);
    std::memcpy(&chips[(size_t)i * pc.Lc], ch.data(), (size_t)pc.Lc);
  }
  int8_t* d_chips = (int8_t*)ctx->buf(tag + ".chips", chips.size());
  CK(cudaMemcpyAsync(d_chips, chips.data(), chips.size(), cudaMemcpyHostToDevice, st));
  ctx->h2d += ants.size() * sizeof(int32_t) + fc.size() * sizeof(double) + chips.size();
  SampleSource src;
  src.bits = d_bits;
  src.row_bytes = row_bytes;
  src.mean = d_mean;
  src.ant = d_ant;
  src.n_ant = n_ant;
  src.pc = 6.283185307179586 / fs;
  SearchDims dims;
  dims.n_ant = n_ant;
  dims.nb = nb;
  dims.n_prn = n_prn;
  dims.fc = d_fc;
  // Antennas run in chunks, so that Z (FP32, and in tensor-core mode its
  // FP16 operands) stays within kNcZBudget bytes; keys and results are
  // [antenna]-major, so each chunk owns a contiguous part of them.
  const bool tc = ctx->precision == TGA_PRECISION_FP16_TC;
  const long long seq_per_ant = (long long)nb * B * pc.S;
  const double z_per_ant = (double)seq_per_ant * pc.Lc * (sizeof(float2) + (tc ? 4.0 : 0.0));
  long long chunk = (long long)std::floor(kNcZBudget / z_per_ant);
  chunk = std::min<long long>(std::max<long long>(chunk, 1), n_ant);
  chunk = std::min<long long>(chunk, 65535 / ((long long)nb * B));  // front-end grid rows
  if (chunk < 1) throw InvalidArg("too many bins x blocks for one front-end launch");
  const int n_chunks = (int)((n_ant + chunk - 1) / chunk);
  const long long n_seq = chunk * seq_per_ant;
  const size_t n_rows = (size_t)n_ant * nb * n_prn;
  float2* d_z = (float2*)ctx->buf("nc.z", (size_t)n_seq * pc.Lc * sizeof(float2));
  float2* d_D = (float2*)ctx->buf(tag + ".D", (size_t)n_prn * 2 * pc.Lc * sizeof(float2));
  unsigned long long* d_keys = (unsigned long long*)ctx->buf(tag + ".keys", n_rows * sizeof(unsigned long long));
  BestRow* d_best = (BestRow*)ctx->buf(tag + ".best", (size_t)n_ant * n_prn * sizeof(BestRow));
  const double row = corr_row_flops(pc.P);
  const std::string cls = "[Lc=" + std::to_string(pc.Lc) + "]";
  timed(ctx, ("nc_code_spectra" + cls).c_str(), (double)n_prn * 2 * fft_flops(pc.Lc),
        [&] { return launch_code_spectra(pc, d_chips, n_prn, d_D, ctx->num_sms, st); });
  // tensor-core mode: FP16 operands, DFT matrices, and the FP32
  // re-evaluation's keys, row list and per-chunk counts
  void *d_z16 = nullptr, *d_zmap = nullptr, *d_d16 = nullptr, *d_bmat = nullptr;
  int *d_err = nullptr, *d_count = nullptr;
  unsigned long long* d_keys32 = nullptr;
  int2* d_cand = nullptr;
  // tensor-core mode takes the second peaks from the FP32 re-evaluation
  // (the four largest sums per residue; exact while at most three lags of a
  // residue lie within chip_width of the peak)
  float* d_p2rows = nullptr;
  const int cw = chip_width_of(fs);
  const bool rows_p2 = tc && (2 * cw + pc.S) / pc.S <= 3;
  if (tc) {
    d_z16 = ctx->buf("nc.z16", tc_operand_bytes(pc, n_seq, false));
    d_zmap = tc_unit_map_buf(ctx, pc.M);
    d_err = (int*)ctx->buf("tc.err", sizeof(int));
    d_d16 = ctx->buf(tag + ".d16", tc_operand_bytes(pc, (long long)n_prn * 2, true));
    const std::string mat_name = "tcmat." + std::to_string(pc.M);
    if (!ctx->uploaded.count(mat_name)) {
      const std::vector<unsigned char> mats = tc_dft_matrices(pc.M);
      d_bmat = ctx->buf(mat_name, mats.size());
      CK(cudaMemcpy(d_bmat, mats.data(), mats.size(), cudaMemcpyHostToDevice));
      ctx->uploaded[mat_name] = {};
    } else {
      d_bmat = ctx->buf(mat_name, 0);
    }
    d_keys32 = (unsigned long long*)ctx->buf(tag + ".keys32", n_rows * sizeof(unsigned long long));
    if (rows_p2) d_p2rows = (float*)ctx->buf(tag + ".p2rows", n_rows * sizeof(float));
    d_cand = (int2*)ctx->buf(tag + ".cand", n_rows * sizeof(int2));
    d_count = (int*)ctx->buf(tag + ".count", (size_t)n_chunks * sizeof(int));
    timed(ctx, ("nc_tc_pack" + cls).c_str(), 0.0,
          [&] { return launch_tc_pack(pc, d_D, (long long)n_prn * 2, true, d_d16, ctx->num_sms, st); });
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    CK(cudaMemsetAsync(d_count, 0, (size_t)n_chunks * sizeof(int), st));
    CK(cudaMemsetAsync(d_keys, 0, n_rows * sizeof(unsigned long long), st));
    CK(cudaMemsetAsync(d_keys32, 0, n_rows * sizeof(unsigned long long), st));
    if (rows_p2) CK(cudaMemsetAsync(d_p2rows, 0, n_rows * sizeof(float), st));
    ctx->tc_err_pending = d_err;
  }
  for (int ch = 0; ch < n_chunks; ++ch) {
    const int a0 = (int)(ch * chunk), na = (int)std::min<long long>(chunk, n_ant - a0);
    const size_t r0 = (size_t)a0 * nb * n_prn;
    SampleSource cs = src;
    cs.ant = d_ant + a0;
    cs.n_ant = na;
    SearchDims cd = dims;
    cd.n_ant = na;
    const long long cseq = (long long)na * seq_per_ant;
    BestRow* cbest = d_best + (size_t)a0 * n_prn;
    timed(ctx, ("nc_frontend" + cls).c_str(), (double)na * nb * B * 10.0 * pc.P * opt->coherent_periods,
          [&] { return launch_nc_frontend(cs, cd, pc, opt->coherent_periods, B, opt->start, d_z, st); });
    // in tensor-core mode the forward transform also writes Z's FP16 operands
    timed(ctx, ("nc_forward_z" + cls).c_str(), (double)na * nb * B * fft_flops(pc.P), [&] {
      return tc ? launch_forward_seqs_tc(pc, cseq, d_z, d_z16, d_zmap, tc_z_scale(pc), ctx->num_sms, st)
                : launch_forward_seqs(pc, cseq, d_z, ctx->num_sms, st);
    });
    if (tc) {
      timed(ctx, ("nc_correlate_tc" + cls).c_str(), (double)na * nb * n_prn * B * row, [&] {
        return launch_correlate_tc_nc(pc, cd, B, d_bmat, d_z16, d_d16, d_keys + r0, d_err, ctx->test_flags,
                                      ctx->num_sms, st);
      });
      // rows within the FP16 key error of their (antenna, PRN)'s best,
      // re-evaluated in FP32; the bins are then reduced over the FP32 keys
      timed(ctx, ("nc_candidates" + cls).c_str(), 0.0, [&] {
        return launch_tc_candidates(cd, 1, d_keys + r0, kTcKeyKeep, d_cand + r0, d_count + ch, st);
      });
      timed(ctx, ("nc_refine" + cls).c_str(), 0.0, [&] {
        return launch_nc_correlate_listed(pc, cd, B, d_z, d_D, d_cand + r0, d_count + ch, na * nb * n_prn,
                                          d_keys32 + r0, ctx->num_sms, st, rows_p2 ? d_p2rows + r0 : nullptr, cw);
      });
    } else {
      timed(ctx, ("nc_correlate" + cls).c_str(), (double)na * nb * n_prn * B * row,
            [&] { return launch_nc_correlate(pc, cd, B, d_z, d_D, d_keys + r0, ctx->num_sms, st); });
    }
    timed(ctx, ("nc_reduce" + cls).c_str(), 0.0, [&] { return launch_nc_reduce(cd, (tc ? d_keys32 : d_keys) + r0, cbest, st); });
    if (rows_p2)
      timed(ctx, ("nc_second" + cls).c_str(), 0.0,
            [&] { return launch_second_from_rows(cd, 1, d_p2rows + r0, cbest, st); });
    else
      timed(ctx, ("nc_second" + cls).c_str(), (double)na * n_prn * B * row,
            [&] { return launch_nc_second(pc, cd, B, d_z, d_D, cbest, cw, ctx->num_sms, st); });
  }
  std::vector<BestRow> best((size_t)n_ant * n_prn);
  CK(cudaMemcpyAsync(best.data(), d_best, best.size() * sizeof(BestRow), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  ctx->d2h += best.size() * sizeof(BestRow);
  check_tc_error(ctx);
  ctx->last_cells += (double)n_ant * nb * n_prn * (double)P * B;
  // |y| of the polyphase correlator is Lc |r|; report (|r| sqrt(N))^2 per block
  const double scale = (double)opt->coherent_periods * (double)P / ((double)pc.Lc * (double)pc.Lc);
  tga_ctx::LastGroup lg;
  lg.Lc = pc.Lc;
  lg.P = pc.P;
  lg.n_ant = n_ant;
  lg.nb = nb;
  lg.n_prn = n_prn;
  lg.tc = tc;
  lg.amp = tc ? tc_key_amplitude(pc) : 1.0;
  lg.keys = d_keys;
  lg.count = d_count;
  lg.n_chunks = n_chunks;
  lg.nc_power_scale = scale;
  ctx->last_groups.push_back(lg);
  // each member's cells in (PRN, antenna) order
  int q0 = 0;
  for (const NcMember* m : mem) {
    size_t k = m->out_off;
    for (size_t qi = 0; qi < m->prns.size(); ++qi)
      for (int a = 0; a < n_ant; ++a, ++k) {
        const BestRow& r = best[(size_t)a * n_prn + q0 + qi];
        tga_nc_cell& o = out[k];
        std::memset(&o, 0, sizeof o);
        o.prn = m->prns[qi];
        o.antenna = ants[a];
        o.best_freq_idx = r.ab % nb;  // r.ab counts antennas within the chunk
        o.best_codephase = r.tau;
        o.power = (double)r.p * scale;
        o.second_power = (double)r.p2 * scale;
        o.frequency = fc[o.best_freq_idx] - opt->center_freq;
      }
    q0 += (int)m->prns.size();
  }
}

int nc_search(tga_ctx* ctx, const uint8_t* h_bits, size_t n_ant_total, size_t row_bytes, double fs,
              const tga_nc_options* opts, size_t n_opts, tga_nc_cell* out, size_t cap, size_t* n_out) {
  if (!h_bits || !opts || !n_out || n_opts == 0 || n_ant_total == 0 || row_bytes == 0 || !(fs > 0))
    throw InvalidArg("bad arguments");
  std::vector<NcMember> mem;
  size_t n_cells = 0;
  for (size_t i = 0; i < n_opts; ++i) {
    try {
      mem.push_back(nc_member(ctx, &opts[i], n_ant_total, row_bytes, fs));
    } catch (const std::domain_error&) {
      return TGA_ERR_UNSUPPORTED;
    }
    mem.back().out_off = n_cells;
    n_cells += mem.back().ants.size() * mem.back().prns.size();
  }
  *n_out = n_cells;
  if (!out) return TGA_OK;
  if (cap < n_cells) return TGA_ERR_CAPACITY;
  begin_call(ctx);
  ctx->last_groups.clear();
  cudaStream_t st = ctx->stream;
  uint8_t* d_bits = (uint8_t*)ctx->buf("nc.bits", n_ant_total * row_bytes);
  CK(cudaMemcpyAsync(d_bits, h_bits, n_ant_total * row_bytes, cudaMemcpyHostToDevice, st));
  ctx->h2d += n_ant_total * row_bytes;
  double* d_mean = (double*)ctx->buf("nc.mean", n_ant_total * sizeof(double));
  CK(launch_antenna_means(d_bits, (int)n_ant_total, row_bytes, d_mean, st));
  // members sharing a front end run together, in the order of their first member
  std::vector<bool> done(mem.size(), false);
  int gi = 0;
  for (size_t i = 0; i < mem.size(); ++i) {
    if (done[i]) continue;
    std::vector<NcMember*> grp{&mem[i]};
    done[i] = true;
    for (size_t j = i + 1; j < mem.size(); ++j)
      if (!done[j] && nc_same_group(mem[i], mem[j])) {
        grp.push_back(&mem[j]);
        done[j] = true;
      }
    nc_run_group(ctx, d_bits, row_bytes, d_mean, fs, grp, gi++, out);
  }
  collect_times(ctx);
  return TGA_OK;
}

}  // namespace

int tga_search_noncoherent(tga_ctx* ctx, const uint8_t* h_bits, size_t n_ant_total, size_t row_bytes, double fs,
                           const tga_nc_options* opt, tga_nc_cell* out, size_t cap, size_t* n_out) {
  return guarded(ctx, [&] { return nc_search(ctx, h_bits, n_ant_total, row_bytes, fs, opt, 1, out, cap, n_out); });
}

int tga_search_noncoherent_multi(tga_ctx* ctx, const uint8_t* h_bits, size_t n_ant_total, size_t row_bytes,
                                 double fs, const tga_nc_options* opts, size_t n_opts, tga_nc_cell* out, size_t cap,
                                 size_t* n_out) {
  return guarded(ctx, [&] { return nc_search(ctx, h_bits, n_ant_total, row_bytes, fs, opts, n_opts, out, cap, n_out); });
}

// ---------------------------------------------------------------------------
// ACR table Monte Carlo (tga_acr_table), examples/gen_acr_tables.rs:134-173
// ---------------------------------------------------------------------------
int tga_acr_table(tga_ctx* ctx, int constellation, int prn, double fs, double cn0_lo, double cn0_hi,
                  double cn0_step, int trials, double* out, size_t cap, size_t* n_out) {
  return guarded(ctx, [&] {
    if (constellation < 0 || constellation >= N_CONST) throw InvalidArg("bad constellation");
    validate_prn(constellation, prn);
    if (trials < 1 || !(cn0_step > 0) || !(cn0_hi >= cn0_lo) || !(fs > 0) || !n_out)
      throw InvalidArg("bad arguments");
    const int points = (int)std::floor((cn0_hi - cn0_lo) / cn0_step + 1e-9) + 1;
    *n_out = (size_t)points;
    if (!out) return TGA_OK;
    if (cap < (size_t)points) return TGA_ERR_CAPACITY;
    const size_t period = period_samples(constellation, fs);
    if ((2 * period) % 8) throw InvalidArg("two code periods are not a whole number of bytes");
    const size_t row_bytes = 2 * period / 8;
    const std::vector<int8_t> code = resampled_code(constellation, prn, (double)period, 2 * period);
    int8_t* d_code = (int8_t*)ctx->buf("acr.code", code.size());
    CK(cudaMemcpyAsync(d_code, code.data(), code.size(), cudaMemcpyHostToDevice, ctx->stream));
    uint8_t* d_bits = (uint8_t*)ctx->buf("acr.bits", (size_t)points * trials * row_bytes);
    CK(launch_acr_synth(d_code, (int)period, trials, cn0_lo, cn0_step, points, fs, 100e3, d_bits, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));  // code is a host temporary
    int32_t prns[1] = {prn};
    tga_all_options o;
    std::memset(&o, 0, sizeof o);
    o.constellation_mask = 1u << constellation;
    o.prn_filter = prns;
    o.n_prn_filter = 1;
    o.center_freq = 100e3;  // gen_acr_tables.rs:38 F_CARRIER, search band 0: one bin
    o.search_band = 0.0;
    std::vector<tga_cell> cells((size_t)trials);
    double prev = 0.0;
    for (int j = 0; j < points; ++j) {
      size_t nc = 0;
      const int rc = tga_acquire_all_device(ctx, d_bits + (size_t)j * trials * row_bytes, (size_t)trials, row_bytes,
                                            fs, &o, cells.data(), cells.size(), &nc);
      if (rc != TGA_OK) return rc;
      double p2 = 0, s2 = 0;
      for (size_t k = 0; k < nc; ++k) {
        p2 += cells[k].signal_strength * cells[k].signal_strength;
        s2 += cells[k].second_peak * cells[k].second_peak;
      }
      double r_a = p2 / s2;
      if (r_a <= prev) r_a = prev + 0.001;  // strictly increasing (gen_acr_tables.rs:148-152)
      prev = r_a;
      out[2 * j] = r_a;
      out[2 * j + 1] = cn0_lo + (double)j * cn0_step;
    }
    return TGA_OK;
  });
}

int tga_code_chips(int constellation, int prn, int8_t* out, size_t capacity, size_t* n) {
  try {
    std::vector<int8_t> s = resample_sequence(constellation, prn);
    if (n) *n = s.size();
    if (!out) return TGA_OK;
    if (capacity < s.size()) return TGA_ERR_CAPACITY;
    std::memcpy(out, s.data(), s.size());
    return TGA_OK;
  } catch (...) {
    return TGA_ERR_INVALID_ARG;
  }
}

int tga_code_resampled(int constellation, int prn, double samples_per_code, size_t num_samples, float* out) {
  try {
    if (!out && num_samples) return TGA_ERR_INVALID_ARG;
    std::vector<int8_t> s = resampled_code(constellation, prn, samples_per_code, num_samples);
    for (size_t i = 0; i < num_samples; ++i) out[i] = (float)s[i];
    return TGA_OK;
  } catch (...) {
    return TGA_ERR_INVALID_ARG;
  }
}

}  // extern "C"
