// Host-side GNSS primary-code generation (see codes.h).
#include "codes.h"

#include <cmath>
#include <cstdio>
#include <stdexcept>

#include "../../include/tga.h"
#include "gnss_tables.h"

namespace tga {

namespace {

// Constellation properties.  PRN ranges: acquisition.rs:69, galileo_codes.rs:10,
// beidou_codes.rs:15, sbas.rs:21+30, l1c_codes.rs:14, qzss.rs:21+30.
const ConstellationInfo kInfo[N_CONST] = {
    {"gps", "GPS", 1, 38, 1023, 1023, 0.001, TGA_ACR_GPS_L1_CA, false, true},
    {"galileo", "GSAT", 1, 50, 4092, 4092, 0.004, TGA_ACR_GALILEO_E1C, false, false},
    {"beidou", "BEIDOU", 1, 63, 10230, 20460, 0.010, TGA_ACR_BEIDOU_B1C, true, false},
    {"sbas", "SBAS", 120, 158, 1023, 1023, 0.001, TGA_ACR_GPS_L1_CA, false, true},
    {"l1c", "GPSL1C", 1, 63, 10230, 20460, 0.010, TGA_ACR_GPS_L1C, true, false},
    {"qzss", "QZSS", 184, 206, 1023, 1023, 0.001, TGA_ACR_GPS_L1_CA, false, true},
};

void check_prn(int c, int prn) {
  const ConstellationInfo& ci = info(c);
  if (prn < ci.prn_first || prn > ci.prn_last) {
    char msg[128];
    std::snprintf(msg, sizeof msg, "%s PRN must be in %d..=%d, got %d", ci.sv_prefix,
                  ci.prn_first, ci.prn_last, prn);
    throw std::invalid_argument(msg);
  }
}

// C/A Gold code from the two 10-stage maximal-length registers of IS-GPS-200:
// G1 feedback from stages 3 and 10, G2 from stages 2,3,6,8,9,10, both seeded
// with all ones, output taken from stage 10.  G2 is delayed by `g2delay`
// chips.  The reference represents register bits as bipolar values with
// bit 1 <-> -1 and emits -(g1*g2) (acquisition.rs:96-125), i.e. the chip is
// +1 exactly when the two output bits differ.
std::vector<int8_t> ca_from_g2_delay(int g2delay) {
  uint8_t g1[1023], g2[1023];
  unsigned r1 = 0x3FF, r2 = 0x3FF;  // bit i = stage i+1
  auto bit = [](unsigned r, int stage) { return (r >> (stage - 1)) & 1u; };
  for (int i = 0; i < 1023; ++i) {
    g1[i] = (uint8_t)bit(r1, 10);
    g2[i] = (uint8_t)bit(r2, 10);
    unsigned f1 = bit(r1, 3) ^ bit(r1, 10);
    unsigned f2 = bit(r2, 2) ^ bit(r2, 3) ^ bit(r2, 6) ^ bit(r2, 8) ^ bit(r2, 9) ^ bit(r2, 10);
    r1 = ((r1 << 1) | f1) & 0x3FF;
    r2 = ((r2 << 1) | f2) & 0x3FF;
  }
  std::vector<int8_t> ca(1023);
  for (int i = 0; i < 1023; ++i) {
    int j = ((i - g2delay) % 1023 + 1023) % 1023;  // G2 rotated right by g2delay
    ca[i] = (g1[i] ^ g2[j]) ? int8_t(1) : int8_t(-1);
  }
  return ca;
}

// Legendre sequence of prime length n: L[i] = 1 iff i is a non-zero
// quadratic residue mod n (beidou_codes.rs:74-86, l1c_codes.rs:76-88).
std::vector<uint8_t> legendre(int n) {
  std::vector<uint8_t> qr(n, 0);
  for (long x = 1; x < n; ++x) qr[(x * x) % n] = 1;
  qr[0] = 0;
  return qr;
}

// Weil chips W[k] = L[k] ^ L[(k + w) mod n].
std::vector<uint8_t> weil(const std::vector<uint8_t>& L, int w) {
  int n = (int)L.size();
  std::vector<uint8_t> out(n);
  for (int k = 0; k < n; ++k) out[k] = L[k] ^ L[(k + w) % n];
  return out;
}

// BeiDou B1C pilot: 10230 chips of the Weil code of length 10243 read from
// offset p-1 (beidou_codes.rs:113-126); chip bit 0 -> +1, 1 -> -1 (:131-138).
std::vector<int8_t> b1c_chips(int prn) {
  static const std::vector<uint8_t> L = legendre(10243);
  int w = TGA_B1CP_WP[prn - 1][0], p = TGA_B1CP_WP[prn - 1][1];
  std::vector<uint8_t> W = weil(L, w);
  std::vector<int8_t> out(10230);
  for (int i = 0; i < 10230; ++i) out[i] = W[(i + p - 1) % 10243] ? int8_t(-1) : int8_t(1);
  return out;
}

// GPS L1C pilot: Weil code of length 10223 with the 7-chip expansion
// 0110100 inserted before Weil index p-1 (IS-GPS-800, l1c_codes.rs:118-157).
std::vector<int8_t> l1c_chips(int prn) {
  static const std::vector<uint8_t> L = legendre(10223);
  static const uint8_t kExpansion[7] = {0, 1, 1, 0, 1, 0, 0};
  int w = TGA_L1CP_WP[prn - 1][0], p = TGA_L1CP_WP[prn - 1][1];
  std::vector<uint8_t> W = weil(L, w);
  std::vector<int8_t> out;
  out.reserve(10230);
  auto push = [&](uint8_t b) { out.push_back(b ? int8_t(-1) : int8_t(1)); };
  for (int i = 0; i < p - 1; ++i) push(W[i]);
  for (uint8_t b : kExpansion) push(b);
  for (int i = p - 1; i < 10223; ++i) push(W[i]);
  return out;
}

// Galileo E1-C memory code: 1023 hex digits, 4 chips each MSB-first,
// bit 1 -> +1, bit 0 -> -1 (galileo.rs:82-94).
std::vector<int8_t> e1c_chips(int prn) {
  const char* hex = TGA_GALILEO_E1C_HEX[prn - 1];
  std::vector<int8_t> out(4092);
  for (int i = 0; i < 1023; ++i) {
    char ch = hex[i];
    int v = (ch >= '0' && ch <= '9') ? ch - '0' : (ch >= 'A' && ch <= 'F') ? ch - 'A' + 10 : ch - 'a' + 10;
    for (int b = 0; b < 4; ++b) out[4 * i + b] = ((v >> (3 - b)) & 1) ? int8_t(1) : int8_t(-1);
  }
  return out;
}

}  // namespace

const ConstellationInfo& info(int c) {
  if (c < 0 || c >= N_CONST) throw std::invalid_argument("unknown constellation");
  return kInfo[c];
}

std::vector<int8_t> primary_chips(int c, int prn) {
  check_prn(c, prn);
  switch (c) {
    case GPS: return ca_from_g2_delay(TGA_GPS_G2_DELAY[prn - 1]);
    case SBAS: return ca_from_g2_delay(TGA_SBAS_G2_DELAY[prn - 120]);
    case QZSS: return ca_from_g2_delay(TGA_QZSS_G2_DELAY[prn - 184]);
    case GALILEO: return e1c_chips(prn);
    case BEIDOU: return b1c_chips(prn);
    case L1C: return l1c_chips(prn);
  }
  throw std::invalid_argument("unknown constellation");
}

std::vector<int8_t> resample_sequence(int c, int prn) {
  std::vector<int8_t> chips = primary_chips(c, prn);
  if (!info(c).boc) return chips;
  std::vector<int8_t> boc(2 * chips.size());
  for (size_t i = 0; i < chips.size(); ++i) {
    boc[2 * i] = chips[i];
    boc[2 * i + 1] = (int8_t)-chips[i];
  }
  return boc;
}

std::vector<int8_t> resampled_code(int c, int prn, double samples_per_code, size_t num_samples) {
  std::vector<int8_t> seq = resample_sequence(c, prn);
  const double spc = samples_per_code / (double)seq.size();
  std::vector<int8_t> out(num_samples);
  for (size_t n = 0; n < num_samples; ++n) {
    double q = std::floor((double)n / spc);
    // Rust `as usize` saturates: negative/NaN -> 0, huge -> usize::MAX.
    size_t idx = (q > 0.0) ? (q >= 1.8446744073709552e19 ? SIZE_MAX : (size_t)q) : 0;
    out[n] = seq[idx % seq.size()];
  }
  return out;
}

size_t period_samples(int c, double fs) {
  const ConstellationInfo& ci = info(c);
  double v = ci.one_ms_chunk ? fs / 1000.0 : fs * ci.code_period_s;
  if (!(v > 0.0)) return 0;
  return (size_t)v;
}

std::string sv_label(int c, int prn) {
  char buf[32];
  const ConstellationInfo& ci = info(c);
  if (c == SBAS || c == QZSS)
    std::snprintf(buf, sizeof buf, "%s%03d", ci.sv_prefix, prn);
  else
    std::snprintf(buf, sizeof buf, "%s%02d", ci.sv_prefix, prn);
  return buf;
}

}  // namespace tga
