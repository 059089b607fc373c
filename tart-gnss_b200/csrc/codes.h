// Host-side GNSS code generation for the acquisition engine.
//
// Primary code chips (+1/-1) and the reference's resampling rule, for the six
// constellations searched by tart-gnss-acquire.  Every function names the
// reference function whose output it reproduces exactly.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace tga {

enum Constellation { GPS = 0, GALILEO = 1, BEIDOU = 2, SBAS = 3, L1C = 4, QZSS = 5, N_CONST = 6 };

struct ConstellationInfo {
  const char* json_key;    // CombinedOutput field (lib.rs:32-45)
  const char* sv_prefix;   // sv label prefix, e.g. "GPS" -> "GPS03"
  int prn_first, prn_last; // valid PRN range (inclusive)
  int primary_chips;       // chips per primary period (1023, 4092, 10230)
  int seq_len;             // resampling sequence length (BOC doubles it)
  double code_period_s;    // seconds per primary period
  int acr_table;           // TGA_ACR_* table id
  bool boc;                // BOC(1,1) half-chip sequence
  bool one_ms_chunk;       // period derived as (fs/1000) as usize (C/A drivers)
};

const ConstellationInfo& info(int c);

// +-1 primary chips for one PRN (BOC constellations: the 10230 Weil chips
// before BOC modulation).  Throws std::invalid_argument on a bad PRN.
std::vector<int8_t> primary_chips(int c, int prn);

// The sequence the reference resamples from: primary chips, or for BeiDou
// B1C / GPS L1C the BOC(1,1) half-chip sequence [+c0,-c0,+c1,-c1,...]
// (beidou_codes.rs:145-157, l1c_codes.rs:175-189).
std::vector<int8_t> resample_sequence(int c, int prn);

// Code resampled to exactly num_samples samples with the reference rule
// idx = floor(n / (samples_per_code / seq_len)) % seq_len, evaluated in f64
// (acquisition.rs:146-159, galileo.rs:112-122, beidou_codes.rs:166-177,
// l1c_codes.rs:197-208).
std::vector<int8_t> resampled_code(int c, int prn, double samples_per_code, size_t num_samples);

// Samples per code period as the all-PRN drivers compute it:
// C/A: (fs / 1000.0) as usize (acquisition.rs:272-273);
// others: (fs * period_seconds) as usize (galileo.rs:230).
size_t period_samples(int c, double fs);

// sv label, e.g. "GPS03", "GSAT07", "BEIDOU12", "SBAS120", "L1C05", "QZSS184".
std::string sv_label(int c, int prn);

}  // namespace tga
