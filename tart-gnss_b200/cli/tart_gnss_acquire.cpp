// tart-gnss-acquire: command-line front end of the B200 acquisition engine.
//
// Mirrors the reference CLI (main.rs): the same flags (parse_args
// main.rs:61-167), implications (apply_mode_implications main.rs:172-210),
// acquisition mode (main.rs:696-904, JSON CombinedOutput on stdout or
// --output), correlation mode --i/--j (main.rs:907-928) and --benchmark
// (main.rs:482-694) and the RFI report --rfi (main.rs:439-478, rfi.rs).
// Modes outside these (--simulate, --test-antennas) are reported as
// unsupported.  Errors exit with status 1 like the reference.
//
// Flags of this engine beyond the reference's, each off by default so the
// default run is the reference's search:
//   --precision fp32|fp16tc   arithmetic of the search transforms (fp32);
//   --coherent-periods K, --noncoh B
//                             non-coherent search: B coherent blocks of K code
//                             periods summed in power (default: the
//                             reference's single two-period window);
//   --bin-hz H                Doppler bin width of the non-coherent search
//                             (default 1 / (2 K T), T the code period);
//   --refine                  fine acquisition of every detected satellite
//                             (joint Newton refinement of delay, Doppler and
//                             per-antenna phase), added as "refined".
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/tga.h"

namespace {

struct Args {
  std::string file, output;
  bool has_i = false, has_j = false;
  long i = 0, j = 0;
  bool gps = false, galileo = false, beidou = false, sbas = false, l1c = false, qzss = false, all = false;
  bool has_ant = false, has_prn = false;
  std::vector<int> ant, prn;
  double fpm = NAN, ffm = NAN;
  bool debug = false, cn0 = false, benchmark = false, test_antennas = false, version = false, rfi = false,
       simulate = false;
  bool has_min_cn0 = false;
  double min_cn0 = 44.0;
  // extensions (see the header comment)
  int precision = TGA_PRECISION_FP32;
  bool nc = false, refine = false;
  long coherent_periods = 1, blocks = 1;
  double bin_hz = NAN;
};

[[noreturn]] void die(const std::string& msg, const char* prog, bool usage) {
  std::fprintf(stderr, "%s\n", msg.c_str());
  if (usage)
    std::fprintf(stderr,
                 "usage: %s --file <observation.hdf> [--i <i> --j <j>] [--all] [--gps] [--galileo] [--beidou] "
                 "[--sbas] [--l1c] [--qzss] [--cn0] [--test-antennas] [--test-min-cn0 <x>] [--rfi] [--prn <a,b,...>] "
                 "[--ant <a,b,...>] [--filter-phase-mad <x>] [--filter-freq-mad <x>] [--output <path>] [--debug] "
                 "[--benchmark] [--precision <fp32|fp16tc>] [--coherent-periods <K>] [--noncoh <B>] [--bin-hz <H>] "
                 "[--refine]\n",
                 prog);
  std::exit(1);
}

bool parse_int(const std::string& s, long* v) {
  std::string t = s;
  while (!t.empty() && t.front() == ' ') t.erase(t.begin());
  while (!t.empty() && t.back() == ' ') t.pop_back();
  if (t.empty()) return false;
  for (char c : t)
    if (c < '0' || c > '9') return false;
  *v = std::strtol(t.c_str(), nullptr, 10);
  return true;
}

bool parse_f64(const std::string& s, double* v) {
  char* e = nullptr;
  *v = std::strtod(s.c_str(), &e);
  return e && *e == '\0' && !s.empty();
}

std::vector<int> parse_list(const std::string& v, const char* flag, const char* prog) {
  std::vector<int> out;
  size_t p = 0;
  while (true) {
    size_t q = v.find(',', p);
    std::string item = v.substr(p, q == std::string::npos ? std::string::npos : q - p);
    long x;
    if (!parse_int(item, &x)) die(std::string("invalid integer in ") + flag + ": " + item, prog, true);
    out.push_back((int)x);
    if (q == std::string::npos) break;
    p = q + 1;
  }
  return out;
}

Args parse_args(int argc, char** argv) {
  Args a;
  const char* prog = argv[0];
  auto val = [&](int& k, const char* flag) -> std::string {
    if (k + 1 >= argc) die(std::string("missing value for ") + flag, prog, true);
    return argv[++k];
  };
  for (int k = 1; k < argc; ++k) {
    const std::string s = argv[k];
    if (s == "--file") a.file = val(k, "--file");
    else if (s == "--i") { std::string v = val(k, "--i"); if (!parse_int(v, &a.i)) die("invalid integer for --i: " + v, prog, true); a.has_i = true; }
    else if (s == "--j") { std::string v = val(k, "--j"); if (!parse_int(v, &a.j)) die("invalid integer for --j: " + v, prog, true); a.has_j = true; }
    else if (s == "--gps") a.gps = true;
    else if (s == "--galileo") a.galileo = true;
    else if (s == "--beidou") a.beidou = true;
    else if (s == "--sbas") a.sbas = true;
    else if (s == "--l1c") a.l1c = true;
    else if (s == "--qzss") a.qzss = true;
    else if (s == "--all") a.all = true;
    else if (s == "--ant") { a.ant = parse_list(val(k, "--ant"), "--ant", prog); a.has_ant = true; }
    else if (s == "--prn") { a.prn = parse_list(val(k, "--prn"), "--prn", prog); a.has_prn = true; }
    else if (s == "--filter-phase-mad") { std::string v = val(k, s.c_str()); if (!parse_f64(v, &a.fpm)) die("invalid float for --filter-phase-mad: " + v, prog, true); }
    else if (s == "--filter-freq-mad") { std::string v = val(k, s.c_str()); if (!parse_f64(v, &a.ffm)) die("invalid float for --filter-freq-mad: " + v, prog, true); }
    else if (s == "--output") a.output = val(k, "--output");
    else if (s == "--debug") a.debug = true;
    else if (s == "--cn0") a.cn0 = true;
    else if (s == "--benchmark") a.benchmark = true;
    else if (s == "--test-antennas") a.test_antennas = true;
    else if (s == "--test-min-cn0") { std::string v = val(k, s.c_str()); if (!parse_f64(v, &a.min_cn0)) die("invalid float for --test-min-cn0: " + v, prog, true); a.has_min_cn0 = true; }
    else if (s == "--version") a.version = true;
    else if (s == "--rfi") a.rfi = true;
    else if (s == "--simulate") a.simulate = true;
    else if (s == "--precision") {
      const std::string v = val(k, "--precision");
      if (v == "fp32") a.precision = TGA_PRECISION_FP32;
      else if (v == "fp16tc") a.precision = TGA_PRECISION_FP16_TC;
      else die("invalid value for --precision: " + v + " (fp32 or fp16tc)", prog, true);
    }
    else if (s == "--coherent-periods") { std::string v = val(k, s.c_str()); if (!parse_int(v, &a.coherent_periods) || a.coherent_periods < 1) die("invalid positive integer for --coherent-periods: " + v, prog, true); a.nc = true; }
    else if (s == "--noncoh") { std::string v = val(k, s.c_str()); if (!parse_int(v, &a.blocks) || a.blocks < 1) die("invalid positive integer for --noncoh: " + v, prog, true); a.nc = true; }
    else if (s == "--bin-hz") { std::string v = val(k, s.c_str()); if (!parse_f64(v, &a.bin_hz) || !(a.bin_hz > 0)) die("invalid positive float for --bin-hz: " + v, prog, true); }
    else if (s == "--refine") a.refine = true;
    else if (s == "--sources" || s == "--positions" || s == "--N" || s == "--diameter" || s == "--seed" ||
             s == "--sample-rate" || s == "--center-freq" || s == "--band" || s == "--snr") (void)val(k, s.c_str());
    else die("unknown argument: " + s, prog, true);
  }
  // main.rs:172-210
  if (a.all) a.gps = a.galileo = a.beidou = a.sbas = a.l1c = a.qzss = true;
  if (a.test_antennas) {
    a.cn0 = true;
    if (a.benchmark) die("--test-antennas cannot be combined with --benchmark", prog, true);
    if (!(a.gps || a.galileo || a.beidou || a.sbas || a.l1c || a.qzss))
      a.gps = a.galileo = a.beidou = a.sbas = a.l1c = a.qzss = true;
  }
  if (!std::isnan(a.bin_hz) && !a.nc)
    die("--bin-hz sets the non-coherent search's grid: give --noncoh or --coherent-periods (the reference's "
        "two-period search keeps its 300 Hz grid)", prog, true);
  if (a.nc && (a.benchmark || a.rfi || a.test_antennas))
    die("--noncoh / --coherent-periods apply to the acquisition search only", prog, true);
  if (a.refine && (a.benchmark || a.rfi || a.test_antennas))
    die("--refine applies to the acquisition search only", prog, true);
  if (a.rfi) {
    if (a.benchmark) die("--rfi cannot be combined with --benchmark", prog, true);
    if (a.test_antennas) die("--rfi cannot be combined with --test-antennas", prog, true);
    if (a.has_i || a.has_j) die("--rfi cannot be combined with --i/--j", prog, true);
    if (a.simulate) die("--rfi cannot be combined with --simulate", prog, true);
  }
  return a;
}

void write_out(const std::string& json, const std::string& path, const char* what) {
  if (path.empty()) {
    std::printf("%s\n", json.c_str());
    return;
  }
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f || std::fwrite(json.data(), 1, json.size(), f) != json.size()) {
    std::fprintf(stderr, "error writing output file %s\n", path.c_str());
    std::exit(1);
  }
  std::fclose(f);
  std::fprintf(stderr, "Wrote %s to %s\n", what, path.c_str());
}

const char* kNames[6] = {"GPS L1 C/A", "Galileo E1-C", "BeiDou B1C", "SBAS L1 C/A", "GPS L1C", "QZSS L1 C/A"};
const int kNumPrns[6] = {38, 50, 63, 39, 63, 23};
const int kFirstPrn[6] = {1, 1, 1, 120, 1, 184};
// CombinedOutput field order (lib.rs:32-45) and sv labels (acquisition.rs:351 and twins)
const int kJsonOrder[6] = {TGA_GPS, TGA_GALILEO, TGA_BEIDOU, TGA_SBAS, TGA_L1C, TGA_QZSS};
const char* kJsonKey[6] = {"gps", "galileo", "beidou", "sbas", "l1c", "qzss"};
const double kPeriodS[6] = {0.001, 0.004, 0.010, 0.001, 0.010, 0.001};

std::string sv_label(int c, int prn) {
  char b[32];
  switch (c) {
    case TGA_GPS: std::snprintf(b, sizeof b, "GPS%02d", prn); break;
    case TGA_GALILEO: std::snprintf(b, sizeof b, "GSAT%02d", prn); break;
    case TGA_BEIDOU: std::snprintf(b, sizeof b, "BEIDOU%02d", prn); break;
    case TGA_SBAS: std::snprintf(b, sizeof b, "SBAS%03d", prn); break;
    case TGA_L1C: std::snprintf(b, sizeof b, "GPSL1C%02d", prn); break;
    default: std::snprintf(b, sizeof b, "QZSS%03d", prn); break;
  }
  return b;
}

// samples per code period (the library's rule: fs / 1000 for the 1 ms codes)
size_t period_of(int c, double fs) {
  const double v = kPeriodS[c] == 0.001 ? fs / 1000.0 : fs * kPeriodS[c];
  return v > 0 ? (size_t)v : 0;
}

std::string num(double v) {
  char b[64];
  tga_format_f64(v, b, sizeof b);
  return b;
}

void arr(std::string& s, const std::vector<double>& v, int lvl) {
  if (v.empty()) {
    s += "[]";
    return;
  }
  s += "[\n";
  for (size_t i = 0; i < v.size(); ++i)
    s += std::string(2 * (lvl + 1), ' ') + num(v[i]) + (i + 1 < v.size() ? ",\n" : "\n");
  s += std::string(2 * lvl, ' ') + "]";
}

// One satellite to refine: the grid estimate of its strongest antenna.
struct Detected {
  int c, prn;
  double code_phase, frequency;  // samples; Hz relative to the centre
  size_t period;
  int64_t length;
};

// The "refined" list: tga_fine_acquire on every detected satellite, in the
// serde pretty layout of the rest of the output.
std::string refined_json(tga_ctx* ctx, const tga_observation& obs, const std::vector<Detected>& det) {
  std::vector<tga_fine_task> tasks;
  for (const Detected& d : det) {
    tga_fine_task t;
    t.constellation = d.c;
    t.prn = d.prn;
    t.code_phase = d.code_phase;
    t.frequency = 4.092e6 + d.frequency;
    t.start = 0;
    t.length = d.length;
    tasks.push_back(t);
  }
  std::vector<tga_fine_result> res(tasks.size());
  if (!tasks.empty() &&
      tga_fine_acquire(ctx, obs.data, obs.num_antenna, obs.row_bytes, obs.sampling_frequency, tasks.data(),
                       tasks.size(), nullptr, res.data(), nullptr) != TGA_OK) {
    std::fprintf(stderr, "fine acquisition failed: %s\n", tga_last_error(ctx));
    std::exit(1);
  }
  std::string s = "[";
  for (size_t i = 0; i < det.size(); ++i) {
    const tga_fine_result& r = res[i];
    s += std::string(i ? ",\n" : "\n") + "    {\n      \"sv\": \"" + sv_label(det[i].c, det[i].prn) +
         "\",\n      \"code_phase_samples\": " + num(r.code_phase) + ",\n      \"codephase_frac\": " +
         num(r.code_phase / (double)det[i].period) + ",\n      \"frequency\": " + num(r.frequency - 4.092e6) +
         ",\n      \"power\": " + num(r.power) + ",\n      \"power_start\": " + num(r.power_start) +
         ",\n      \"iterations\": " + std::to_string(r.iterations) + ",\n      \"converged\": " +
         (r.converged ? "true" : "false") + "\n    }";
  }
  s += det.empty() ? "]" : "\n  ]";
  return s;
}

// Appends a top-level field to a pretty-printed JSON object.
void append_field(std::string& json, const std::string& key, const std::string& value) {
  const size_t end = json.rfind('}');
  size_t body = end;
  while (body > 0 && (json[body - 1] == '\n' || json[body - 1] == ' ')) --body;
  const bool empty = json[body - 1] == '{';
  json = json.substr(0, body) + (empty ? "\n" : ",\n") + "  \"" + key + "\": " + value + "\n}";
}

}  // namespace

int main(int argc, char** argv) {
  Args a = parse_args(argc, argv);
  if (a.version) {
    std::printf("tart-gnss-acquire v0.4.0 (%s)\n", tga_version());
    return 0;
  }
  if (a.simulate) die("--simulate is not part of this engine (acquisition search only)", argv[0], false);

  tga_observation obs;
  std::memset(&obs, 0, sizeof obs);
  if (!a.file.empty()) {
    if (tga_observation_read_hdf5(a.file.c_str(), &obs) != TGA_OK) {
      std::fprintf(stderr, "error loading HDF5 file: %s\n", obs.error);
      return 1;
    }
  } else if (a.benchmark) {
    // main.rs:425-430: 2 antennas of random 0/1 data, 16 MHz, 500k samples
    std::fprintf(stderr, "--benchmark without --file: using random data\n");
    obs.num_antenna = 2;
    obs.sampling_frequency = 16e6;
    obs.row_bytes = 500000 / 8;
    obs.data = (uint8_t*)std::malloc(2 * obs.row_bytes);
    std::mt19937_64 rng((uint64_t)std::chrono::steady_clock::now().time_since_epoch().count());
    for (size_t k = 0; k < 2 * obs.row_bytes; ++k) obs.data[k] = (uint8_t)rng();
    std::snprintf(obs.timestamp, sizeof obs.timestamp, "now");
  } else {
    die("missing --file (or use --benchmark)", argv[0], true);
  }
  const size_t n_ant = obs.num_antenna;
  const double fs = obs.sampling_frequency;
  std::fprintf(stderr, "timestamp:   %s\nantennas:    %zu\nsample rate: %.1f Hz\n", obs.timestamp, n_ant, fs);

  tga_ctx* ctx = nullptr;
  int rc = tga_create(0, &ctx);
  if (rc != TGA_OK) {
    std::fprintf(stderr, "no usable B200 (sm_100) GPU: status %d\n", rc);
    return 1;
  }

  if (a.rfi) {
    // main.rs:439-478: the RFI report of every antenna, then exit
    std::vector<tga_rfi_channel> ch(n_ant);
    rc = tga_rfi_scan(ctx, obs.data, n_ant, obs.row_bytes, fs, ch.data());
    if (rc != TGA_OK) {
      std::fprintf(stderr, "RFI scan failed: %s\n", tga_last_error(ctx));
      return 1;
    }
    char* json = nullptr;
    if (tga_rfi_json(ch.data(), ch.size(), &json) != TGA_OK) return 1;
    write_out(json, a.output, "RFI JSON");
    tga_free(json);
    tga_destroy(ctx);
    tga_observation_free(&obs);
    return 0;
  }

  if (a.benchmark) {
    // main.rs:482-694: one PRN per constellation on antenna 0; setup = antenna
    // extraction, search = the single-PRN acquisition (tga_benchmark).
    const char* names[6] = {"GPS", "Galileo", "BeiDou", "SBAS", "QZSS", "L1C"};
    std::fprintf(stderr, "Running benchmark (one PRN per constellation, setup timed separately)...\n");
    tga_bench_entry be[6];
    rc = tga_benchmark(ctx, obs.data, n_ant, obs.row_bytes, fs, be);
    if (rc != TGA_OK) {
      std::fprintf(stderr, "%s\n", tga_last_error(ctx));
      return 1;
    }
    std::string json = "[";
    double tot_setup = 0, tot_search = 0;
    for (int e = 0; e < 6; ++e) {
      const double setup = be[e].setup_s, search = be[e].search_s;
      std::fprintf(stderr, "  %s (PRN %d)...\n", names[e], be[e].prn);
      tot_setup += setup;
      tot_search += search;
      std::fprintf(stderr, "    %s: setup=%.4fs  search=%.4fs  total=%.4fs\n", names[e], setup, search, setup + search);
      char b1[64], b2[64], b3[64];
      tga_format_f64(setup, b1, sizeof b1);
      tga_format_f64(search, b2, sizeof b2);
      tga_format_f64(setup + search, b3, sizeof b3);
      json += std::string(e ? ",\n" : "\n") + "  {\n    \"constellation\": \"" + names[e] + "\",\n    \"prns\": 1,\n" +
              "    \"setup_s\": " + b1 + ",\n    \"search_s\": " + b2 + ",\n    \"duration_s\": " + b3 + "\n  }";
    }
    json += "\n]";
    std::fprintf(stderr, "  Combined: startup=%.4fs  search=%.4fs  total=%.4fs  acq/s=%.1f\n", tot_setup, tot_search,
                 tot_setup + tot_search, 6.0 / tot_search);
    write_out(json, a.output, "benchmark JSON");
    tga_destroy(ctx);
    tga_observation_free(&obs);
    return 0;
  }

  const bool any = a.gps || a.galileo || a.beidou || a.sbas || a.l1c || a.qzss;
  if (any) {
    if (a.test_antennas)
      die("--test-antennas (antenna ranking report) is not part of this engine", argv[0], false);
    if (a.has_ant)
      for (int x : a.ant)
        if (x < 0 || (size_t)x >= n_ant) {
          std::fprintf(stderr, "antenna index %d out of range (have %zu)\n", x, n_ant);
          return 1;
        }
    uint32_t mask = 0;
    const bool flags[6] = {a.gps, a.galileo, a.beidou, a.sbas, a.l1c, a.qzss};
    for (int c = 0; c < 6; ++c)
      if (flags[c]) {
        mask |= 1u << c;
        std::fprintf(stderr, "Running %s search (%zu PRNs)...\n", kNames[c],
                     a.has_prn ? a.prn.size() : (size_t)kNumPrns[c]);
      }
    if (tga_set_precision(ctx, a.precision) != TGA_OK) {
      std::fprintf(stderr, "%s\n", tga_last_error(ctx));
      return 1;
    }
    std::vector<int32_t> ants;
    if (a.has_ant) ants.assign(a.ant.begin(), a.ant.end());
    else for (size_t k = 0; k < n_ant; ++k) ants.push_back((int32_t)k);
    if (a.nc) {
      // non-coherent search of every selected constellation in one call
      std::vector<tga_nc_options> opts;
      std::vector<int> consts;
      std::vector<double> steps;
      for (int c = 0; c < 6; ++c) {
        if (!flags[c]) continue;
        tga_nc_options q;
        std::memset(&q, 0, sizeof q);
        q.constellation = c;
        q.prn_filter = a.has_prn ? a.prn.data() : nullptr;
        q.n_prn_filter = a.prn.size();
        q.ant_filter = ants.data();
        q.n_ant_filter = ants.size();
        q.center_freq = 4.092e6;
        const double step = std::isnan(a.bin_hz) ? 1.0 / (2.0 * a.coherent_periods * kPeriodS[c]) : a.bin_hz;
        q.bin_step_hz = step;
        q.n_bins = 2 * (int)std::floor(6000.0 / step + 1e-9) + 1;  // the reference's +-6 kHz band
        q.coherent_periods = (int32_t)a.coherent_periods;
        q.blocks = (int32_t)a.blocks;
        opts.push_back(q);
        consts.push_back(c);
        steps.push_back(step);
      }
      size_t n_cells = 0;
      rc = tga_search_noncoherent_multi(ctx, obs.data, n_ant, obs.row_bytes, fs, opts.data(), opts.size(), nullptr,
                                        0, &n_cells);
      std::vector<tga_nc_cell> nc(n_cells);
      if (rc == TGA_OK)
        rc = tga_search_noncoherent_multi(ctx, obs.data, n_ant, obs.row_bytes, fs, opts.data(), opts.size(),
                                          nc.data(), nc.size(), &n_cells);
      if (rc != TGA_OK) {
        std::fprintf(stderr, "non-coherent search failed: %s\n", tga_last_error(ctx));
        return 1;
      }
      // {key: {antenna_numbers, coherent_periods, blocks, bin_hz, results: [{sv, powers,
      // second_powers, phases, freqs}]}} in CombinedOutput order, results sorted by sv
      std::string json = "{";
      std::vector<Detected> det;
      bool first = true;
      for (int jc : kJsonOrder) {
        size_t oi = 0, off = 0;
        for (; oi < consts.size() && consts[oi] != jc; ++oi)
          off += ants.size() * (a.has_prn ? a.prn.size() : (size_t)kNumPrns[consts[oi]]);
        if (oi == consts.size()) continue;
        const size_t n_prn = a.has_prn ? a.prn.size() : (size_t)kNumPrns[jc];
        const size_t P = period_of(jc, fs);
        std::vector<std::pair<std::string, size_t>> order;  // (sv, prn index)
        for (size_t qi = 0; qi < n_prn; ++qi)
          order.push_back({sv_label(jc, a.has_prn ? a.prn[qi] : kFirstPrn[jc] + (int)qi), qi});
        std::sort(order.begin(), order.end());
        json += std::string(first ? "\n" : ",\n") + "  \"" + kJsonKey[jc] + "\": {\n    \"antenna_numbers\": ";
        first = false;
        if (ants.empty()) {
          json += "[]";
        } else {
          json += "[\n";
          for (size_t k = 0; k < ants.size(); ++k)
            json += "      " + std::to_string(ants[k]) + (k + 1 < ants.size() ? ",\n" : "\n");
          json += "    ]";
        }
        json += ",\n    \"coherent_periods\": " + std::to_string(a.coherent_periods) + ",\n    \"blocks\": " +
                std::to_string(a.blocks) + ",\n    \"bin_hz\": " + num(steps[oi]) + ",\n    \"results\": [";
        for (size_t r = 0; r < order.size(); ++r) {
          const tga_nc_cell* row = &nc[off + order[r].second * ants.size()];
          std::vector<double> pw, sp, ph, fr;
          size_t best = 0;
          for (size_t k = 0; k < ants.size(); ++k) {
            pw.push_back(row[k].power);
            sp.push_back(row[k].second_power);
            ph.push_back((double)row[k].best_codephase / (double)P);
            fr.push_back(row[k].frequency);
            if (row[k].power > row[best].power) best = k;
          }
          json += std::string(r ? ",\n" : "\n") + "      {\n        \"sv\": \"" + order[r].first +
                  "\",\n        \"powers\": ";
          arr(json, pw, 4);
          json += ",\n        \"second_powers\": ";
          arr(json, sp, 4);
          json += ",\n        \"phases\": ";
          arr(json, ph, 4);
          json += ",\n        \"freqs\": ";
          arr(json, fr, 4);
          json += "\n      }";
          // detected: summed peak power at least 4 x the second peak (2 x in amplitude)
          if (!ants.empty() && row[best].power >= 4.0 * row[best].second_power)
            det.push_back({jc, row[best].prn, (double)row[best].best_codephase, row[best].frequency, P,
                           (int64_t)(a.coherent_periods * P)});
        }
        json += order.empty() ? "]" : "\n    ]";
        json += "\n  }";
      }
      json += first ? "}" : "\n}";
      if (a.refine) append_field(json, "refined", refined_json(ctx, obs, det));
      write_out(json, a.output, "JSON output");
      tga_destroy(ctx);
      tga_observation_free(&obs);
      return 0;
    }
    tga_all_options o;
    std::memset(&o, 0, sizeof o);
    o.constellation_mask = mask;
    o.ant_filter = a.has_ant ? a.ant.data() : nullptr;
    o.n_ant_filter = a.ant.size();
    o.prn_filter = a.has_prn ? a.prn.data() : nullptr;
    o.n_prn_filter = a.prn.size();
    o.center_freq = 4.092e6;
    o.search_band = 6000.0;
    o.cn0 = a.cn0;
    o.debug = a.debug;
    size_t n_cells = 0;
    if (tga_all_cell_count(n_ant, &o, &n_cells) != TGA_OK) {
      std::fprintf(stderr, "invalid PRN list for the selected constellations\n");
      return 1;
    }
    std::vector<tga_cell> cells(n_cells);
    rc = tga_acquire_all(ctx, obs.data, n_ant, obs.row_bytes, fs, &o, cells.data(), cells.size(), &n_cells);
    if (rc != TGA_OK) {
      std::fprintf(stderr, "acquisition failed: %s\n", tga_last_error(ctx));
      return 1;
    }
    if (a.debug)
      for (const tga_cell& t : cells)
        std::fprintf(stderr, "  %d PRN %3d ant %2d: strength=%.3f  phase=%.6f  freq=%.1f Hz\n", t.constellation,
                     t.prn, t.antenna, t.signal_strength, t.codephase_frac, t.frequency);
    char* json = nullptr;
    size_t nf = 0;
    rc = tga_results_json(cells.data(), n_cells, ants.data(), ants.size(), mask, a.cn0, a.fpm, a.ffm, &json, &nf);
    if (rc != TGA_OK) {
      std::fprintf(stderr, "JSON serialization failed\n");
      return 1;
    }
    if (nf > 0) std::fprintf(stderr, "Filtered out %zu results (MAD thresholds)\n", nf);
    std::string text = json;
    tga_free(json);
    if (a.refine) {
      // every (constellation, PRN) detected on some antenna (strength at least
      // twice the second peak), from its strongest antenna's grid estimate over
      // the search window of two periods
      std::vector<Detected> det;
      for (size_t k = 0; k < cells.size();) {
        size_t e = k, best = k;
        while (e < cells.size() && cells[e].constellation == cells[k].constellation && cells[e].prn == cells[k].prn) {
          if (cells[e].signal_strength > cells[best].signal_strength) best = e;
          ++e;
        }
        const tga_cell& b = cells[best];
        const size_t P = period_of(b.constellation, fs);
        if (b.signal_strength >= 2.0 * b.second_peak)
          det.push_back({b.constellation, b.prn, (double)b.best_codephase, b.frequency, P, (int64_t)(2 * P)});
        k = e;
      }
      append_field(text, "refined", refined_json(ctx, obs, det));
    }
    write_out(text, a.output, "JSON output");
    tga_destroy(ctx);
    tga_observation_free(&obs);
    return 0;
  }

  // correlation mode (main.rs:907-928)
  if (!a.has_i) die("missing --i <antenna_i> (or use --gps, --galileo, --beidou, --sbas, --l1c, --qzss, or --all)",
                    argv[0], false);
  if (!a.has_j) die("missing --j <antenna_j>", argv[0], false);
  if (a.i < 0 || (size_t)a.i >= n_ant) {
    std::fprintf(stderr, "antenna index %ld out of range (have %zu)\n", a.i, n_ant);
    return 1;
  }
  if (a.j < 0 || (size_t)a.j >= n_ant) {
    std::fprintf(stderr, "antenna index %ld out of range (have %zu)\n", a.j, n_ant);
    return 1;
  }
  double corr = 0.0;
  rc = tga_antenna_xcorr(ctx, obs.data, n_ant, obs.row_bytes, (int)a.i, (int)a.j, &corr);
  if (rc != TGA_OK) {
    std::fprintf(stderr, "%s\n", tga_last_error(ctx));
    return 1;
  }
  std::printf("antenna_i:   %ld\nantenna_j:   %ld\ncorrelation: %.6f\n", a.i, a.j, corr);
  tga_destroy(ctx);
  tga_observation_free(&obs);
  return 0;
}
