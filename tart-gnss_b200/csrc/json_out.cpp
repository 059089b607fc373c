// Result aggregation and JSON output of an all-PRN search.
//
// Builds CombinedOutput (lib.rs:32-45): per selected constellation
// {antenna_numbers, results[]} with each PRN's sv label, per-antenna
// strengths / phases / freqs, optional cn0_acr (null entries where the
// estimate failed; omitted when every entry failed, acquisition.rs:341-357),
// and median / MAD of phase and frequency when more than one antenna was
// searched (acquisition.rs:365-377, stats.rs:10-30).  Results are sorted by
// sv string (acquisition.rs:393).  The optional MAD filters of the CLI
// (main.rs:242-256) drop results whose MAD exceeds the threshold.
//
// Layout follows serde_json's pretty printer: two-space indentation,
// "key": value, one array element per line, `[]` for empty arrays; floats
// use the shortest decimal that round-trips, printed with a ".0" suffix for
// integral values and in exponent form outside 1e-5 <= |x| < 1e16.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/tga.h"
#include "codes.h"

namespace {

// Shortest round-trip decimal digits of a finite non-zero double:
// digits d1..dn and exponent e with value = 0.d1..dn * 10^e.
void shortest_digits(double v, std::string* digits, int* e) {
  char buf[64];
  for (int prec = 1; prec <= 17; ++prec) {
    std::snprintf(buf, sizeof buf, "%.*e", prec - 1, v);
    if (std::strtod(buf, nullptr) == v) break;
  }
  // buf = "d.ddddde[+-]xx"
  std::string s(buf);
  const size_t epos = s.find('e');
  std::string mant = s.substr(0, epos);
  const int exp10 = std::atoi(s.c_str() + epos + 1);
  std::string d;
  for (char ch : mant)
    if (ch >= '0' && ch <= '9') d.push_back(ch);
  while (d.size() > 1 && d.back() == '0') d.pop_back();
  *digits = d;
  *e = exp10 + 1;
}

std::string fmt_f64(double v) {
  if (std::isnan(v) || std::isinf(v)) return "null";  // serde_json writes non-finite floats as null
  if (v == 0.0) return std::signbit(v) ? "-0.0" : "0.0";
  std::string out = v < 0 ? "-" : "";
  std::string d;
  int kk;
  shortest_digits(std::fabs(v), &d, &kk);
  const int n = (int)d.size();
  const int k = kk - n;  // value = digits * 10^k
  if (k >= 0 && kk <= 16) {
    out += d + std::string(k, '0') + ".0";
  } else if (kk > 0 && kk <= 16) {
    out += d.substr(0, kk) + "." + d.substr(kk);
  } else if (kk > -5 && kk <= 0) {
    out += "0." + std::string(-kk, '0') + d;
  } else if (n == 1) {
    out += d + "e" + std::to_string(kk - 1);
  } else {
    out += d.substr(0, 1) + "." + d.substr(1) + "e" + std::to_string(kk - 1);
  }
  return out;
}

double median(std::vector<double> x) {
  std::sort(x.begin(), x.end());
  const size_t m = x.size() / 2;
  return x.size() % 2 == 0 ? (x[m - 1] + x[m]) / 2.0 : x[m];
}

double mad(const std::vector<double>& x, double med) {
  std::vector<double> d;
  for (double v : x) d.push_back(std::fabs(v - med));
  return median(d);
}

struct W {
  std::string s;
  void ind(int n) { s.append(2 * n, ' '); }
  void arr_f64(const std::vector<double>& v, int lvl) {
    if (v.empty()) {
      s += "[]";
      return;
    }
    s += "[\n";
    for (size_t i = 0; i < v.size(); ++i) {
      ind(lvl + 1);
      s += fmt_f64(v[i]);
      s += i + 1 < v.size() ? ",\n" : "\n";
    }
    ind(lvl);
    s += "]";
  }
};

struct PrnRes {
  std::string sv;
  std::vector<double> strengths, phases, freqs, cn0;
  std::vector<int> cn0_ok;
  bool has_cn0 = false;
  bool multi = false;
  double pm = 0, pmad = 0, fm = 0, fmad = 0;
};

}  // namespace

extern "C" int tga_results_json(const tga_cell* cells, size_t n_cells, const int32_t* ant_numbers, size_t n_ant,
                                uint32_t mask, int cn0, double filter_phase_mad, double filter_freq_mad,
                                char** json, size_t* n_filtered) {
  if (!json || (!cells && n_cells) || (!ant_numbers && n_ant)) return TGA_ERR_INVALID_ARG;
  try {
    W w;
    size_t filtered = 0;
    w.s = "{";
    bool first_const = true;
    for (int c = 0; c < tga::N_CONST; ++c) {
      if (!(mask & (1u << c))) continue;
      // group cells of this constellation by PRN in their given order
      std::vector<PrnRes> res;
      for (size_t i = 0; i < n_cells; ++i) {
        const tga_cell& t = cells[i];
        if (t.constellation != c) continue;
        const std::string sv = tga::sv_label(c, t.prn);
        if (res.empty() || res.back().sv != sv) {
          res.push_back(PrnRes());
          res.back().sv = sv;
        }
        PrnRes& r = res.back();
        r.strengths.push_back(t.signal_strength);
        r.phases.push_back(t.codephase_frac);
        r.freqs.push_back(t.frequency);
        r.cn0.push_back(t.cn0_acr);
        r.cn0_ok.push_back(t.cn0_valid);
      }
      std::vector<PrnRes> keep;
      for (PrnRes& r : res) {
        if (cn0) r.has_cn0 = std::any_of(r.cn0_ok.begin(), r.cn0_ok.end(), [](int v) { return v != 0; });
        r.multi = r.phases.size() > 1;
        if (r.multi) {
          r.pm = median(r.phases);
          r.pmad = mad(r.phases, r.pm);
          r.fm = median(r.freqs);
          r.fmad = mad(r.freqs, r.fm);
        }
        const bool drop = r.multi && ((!std::isnan(filter_phase_mad) && !(r.pmad <= filter_phase_mad)) ||
                                      (!std::isnan(filter_freq_mad) && !(r.fmad <= filter_freq_mad)));
        if (drop) ++filtered;
        else keep.push_back(r);
      }
      std::stable_sort(keep.begin(), keep.end(), [](const PrnRes& a, const PrnRes& b) { return a.sv < b.sv; });

      w.s += first_const ? "\n" : ",\n";
      first_const = false;
      w.ind(1);
      w.s += "\"" + std::string(tga::info(c).json_key) + "\": {\n";
      w.ind(2);
      w.s += "\"antenna_numbers\": ";
      if (n_ant == 0) {
        w.s += "[]";
      } else {
        w.s += "[\n";
        for (size_t a = 0; a < n_ant; ++a) {
          w.ind(3);
          w.s += std::to_string(ant_numbers[a]) + (a + 1 < n_ant ? ",\n" : "\n");
        }
        w.ind(2);
        w.s += "]";
      }
      w.s += ",\n";
      w.ind(2);
      w.s += "\"results\": ";
      if (keep.empty()) {
        w.s += "[]\n";
      } else {
        w.s += "[\n";
        for (size_t i = 0; i < keep.size(); ++i) {
          const PrnRes& r = keep[i];
          w.ind(3);
          w.s += "{\n";
          w.ind(4);
          w.s += "\"sv\": \"" + r.sv + "\",\n";
          w.ind(4);
          w.s += "\"strengths\": ";
          w.arr_f64(r.strengths, 4);
          w.s += ",\n";
          w.ind(4);
          w.s += "\"phases\": ";
          w.arr_f64(r.phases, 4);
          w.s += ",\n";
          w.ind(4);
          w.s += "\"freqs\": ";
          w.arr_f64(r.freqs, 4);
          if (r.has_cn0) {
            w.s += ",\n";
            w.ind(4);
            w.s += "\"cn0_acr\": [\n";
            for (size_t k = 0; k < r.cn0.size(); ++k) {
              w.ind(5);
              w.s += r.cn0_ok[k] ? fmt_f64(r.cn0[k]) : "null";
              w.s += k + 1 < r.cn0.size() ? ",\n" : "\n";
            }
            w.ind(4);
            w.s += "]";
          }
          if (r.multi) {
            const char* names[4] = {"phase_median", "phase_mad", "freq_median", "freq_mad"};
            const double vals[4] = {r.pm, r.pmad, r.fm, r.fmad};
            for (int k = 0; k < 4; ++k) {
              w.s += ",\n";
              w.ind(4);
              w.s += "\"" + std::string(names[k]) + "\": " + fmt_f64(vals[k]);
            }
          }
          w.s += "\n";
          w.ind(3);
          w.s += i + 1 < keep.size() ? "},\n" : "}\n";
        }
        w.ind(2);
        w.s += "]\n";
      }
      w.ind(1);
      w.s += "}";
    }
    w.s += first_const ? "}" : "\n}";
    *json = (char*)std::malloc(w.s.size() + 1);
    if (!*json) return TGA_ERR_OUT_OF_MEMORY;
    std::memcpy(*json, w.s.c_str(), w.s.size() + 1);
    if (n_filtered) *n_filtered = filtered;
    return TGA_OK;
  } catch (...) {
    return TGA_ERR_INVALID_ARG;
  }
}

// RfiReport (rfi.rs:76-81) in serde_json's pretty layout: Option::None is
// written as null, empty line lists as [].
extern "C" int tga_rfi_json(const tga_rfi_channel* ch, size_t n, char** json) {
  if (!json || (!ch && n)) return TGA_ERR_INVALID_ARG;
  auto opt = [](double v) { return std::isnan(v) ? std::string("null") : fmt_f64(v); };
  std::string s = "{\n  \"antenna_numbers\": [";
  if (n == 0) {
    s += "]";
  } else {
    for (size_t i = 0; i < n; ++i) s += (i ? ",\n    " : "\n    ") + std::to_string(ch[i].antenna);
    s += "\n  ]";
  }
  s += ",\n  \"channels\": [";
  if (n == 0) s += "]";
  for (size_t i = 0; i < n; ++i) {
    const tga_rfi_channel& c = ch[i];
    s += i ? ",\n    {\n" : "\n    {\n";
    s += "      \"antenna\": " + std::to_string(c.antenna) + ",\n";
    s += std::string("      \"dead\": ") + (c.dead ? "true" : "false") + ",\n";
    s += "      \"acf_lag1\": " + opt(c.acf_lag1) + ",\n";
    s += "      \"acf_lag3\": " + opt(c.acf_lag3) + ",\n";
    s += "      \"acf_lag16\": " + opt(c.acf_lag16) + ",\n";
    s += "      \"period_samples\": " + opt(c.period_samples) + ",\n";
    s += "      \"lines\": [";
    if (c.n_lines == 0) {
      s += "]";
    } else {
      for (int k = 0; k < c.n_lines; ++k) {
        s += k ? ",\n        {\n" : "\n        {\n";
        s += "          \"frequency\": " + fmt_f64(c.lines[k].frequency) + ",\n";
        s += "          \"excess_db\": " + fmt_f64(c.lines[k].excess_db) + "\n        }";
      }
      s += "\n      ]";
    }
    s += "\n    }";
    if (i + 1 == n) s += "\n  ]";
  }
  s += "\n}";
  char* out = (char*)std::malloc(s.size() + 1);
  if (!out) return TGA_ERR_OUT_OF_MEMORY;
  std::memcpy(out, s.c_str(), s.size() + 1);
  *json = out;
  return TGA_OK;
}

extern "C" int tga_format_f64(double v, char* out, size_t cap) {
  const std::string s = fmt_f64(v);
  if (!out || cap < s.size() + 1) return TGA_ERR_CAPACITY;
  std::memcpy(out, s.c_str(), s.size() + 1);
  return TGA_OK;
}

extern "C" void tga_free(void* p) { std::free(p); }
