// tart-gnss-acquire: command-line front end of the B200 acquisition engine.
//
// Mirrors the reference CLI (main.rs): the same flags (parse_args
// main.rs:61-167), implications (apply_mode_implications main.rs:172-210),
// acquisition mode (main.rs:696-904, JSON CombinedOutput on stdout or
// --output), correlation mode --i/--j (main.rs:907-928) and --benchmark
// (main.rs:482-694) and the RFI report --rfi (main.rs:439-478, rfi.rs).
// Modes outside these (--simulate, --test-antennas) are reported as
// unsupported.  Errors exit with status 1 like the reference.
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
};

[[noreturn]] void die(const std::string& msg, const char* prog, bool usage) {
  std::fprintf(stderr, "%s\n", msg.c_str());
  if (usage)
    std::fprintf(stderr,
                 "usage: %s --file <observation.hdf> [--i <i> --j <j>] [--all] [--gps] [--galileo] [--beidou] "
                 "[--sbas] [--l1c] [--qzss] [--cn0] [--test-antennas] [--test-min-cn0 <x>] [--rfi] [--prn <a,b,...>] "
                 "[--ant <a,b,...>] [--filter-phase-mad <x>] [--filter-freq-mad <x>] [--output <path>] [--debug] "
                 "[--benchmark]\n",
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
    std::vector<int32_t> ants;
    if (a.has_ant) ants.assign(a.ant.begin(), a.ant.end());
    else for (size_t k = 0; k < n_ant; ++k) ants.push_back((int32_t)k);
    char* json = nullptr;
    size_t nf = 0;
    rc = tga_results_json(cells.data(), n_cells, ants.data(), ants.size(), mask, a.cn0, a.fpm, a.ffm, &json, &nf);
    if (rc != TGA_OK) {
      std::fprintf(stderr, "JSON serialization failed\n");
      return 1;
    }
    if (nf > 0) std::fprintf(stderr, "Filtered out %zu results (MAD thresholds)\n", nf);
    write_out(json, a.output, "JSON output");
    tga_free(json);
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
