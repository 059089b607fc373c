/*
 * codes_oracle.c -- CPU ORACLE (test infrastructure, not product code).
 *
 * A plain-C restatement of the integer / table parts of tart-gnss-acquire
 * v0.4.0, used only by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline to check the B200 engine.  Nothing in the product links it.
 *
 * Pinned by the reference's own known-answer tests (tests/test_oracle_*.py):
 * octal chip KATs of beidou_codes.rs:225-279, l1c_codes.rs:256-315,
 * sbas.rs:436-455, qzss.rs:437-454; ACR table points of acr.rs:103-169;
 * stats.rs:36-60; observation.rs:246-289.
 *
 * Written in the reference's own bipolar formulation (values +-1 multiplied
 * together) on purpose, so that it is independent of the product's bitwise
 * LFSR code in tart-gnss_b200/csrc/codes.cpp.  Its data tables (G2 delays,
 * Weil parameters, Galileo hex codes, ACR tables) are its own copy, read
 * from the reference sources into tests/golden/tables.json and handed over
 * by acq_oracle.py through the oracle_set_* calls below before any use; the
 * product's generated header is not included.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---- tables (set once by the loader) -------------------------------------- */
static int g_gps_g2[38], g_sbas_g2[39], g_qzss_g2[23];
static int g_b1cp_wp[63][2], g_l1cp_wp[63][2];
static char g_e1c_hex[50][1024];
static double g_acr[4][128][2];
static int g_acr_n[4];

void oracle_set_ca_delays(const int* gps /*38*/, const int* sbas /*39*/, const int* qzss /*23*/) {
  memcpy(g_gps_g2, gps, sizeof g_gps_g2);
  memcpy(g_sbas_g2, sbas, sizeof g_sbas_g2);
  memcpy(g_qzss_g2, qzss, sizeof g_qzss_g2);
}
void oracle_set_weil(const int* b1cp /*63 x 2*/, const int* l1cp /*63 x 2*/) {
  memcpy(g_b1cp_wp, b1cp, sizeof g_b1cp_wp);
  memcpy(g_l1cp_wp, l1cp, sizeof g_l1cp_wp);
}
void oracle_set_e1c_hex(int prn, const char* hex /*1023 digits*/) {
  memcpy(g_e1c_hex[prn - 1], hex, 1023);
  g_e1c_hex[prn - 1][1023] = 0;
}
/* Returns 0 when the table does not fit. */
int oracle_set_acr(int id, const double* rows /*n x 2*/, int n) {
  if (id < 0 || id > 3 || n < 1 || n > 128) return 0;
  memcpy(g_acr[id], rows, (size_t)n * 2 * sizeof(double));
  g_acr_n[id] = n;
  return 1;
}

/* ---- C/A Gold codes: acquisition.rs:96-125 ------------------------------- */
void oracle_ca_from_delay(int g2shift, double* out /*1023*/) {
  double g1[1023], g2[1023], lfsr[10];
  int i, k;
  for (k = 0; k < 10; ++k) lfsr[k] = -1.0;
  for (i = 0; i < 1023; ++i) {
    double save;
    g1[i] = lfsr[9];
    save = lfsr[2] * lfsr[9];
    for (k = 9; k >= 1; --k) lfsr[k] = lfsr[k - 1];
    lfsr[0] = save;
  }
  for (k = 0; k < 10; ++k) lfsr[k] = -1.0;
  for (i = 0; i < 1023; ++i) {
    double save;
    g2[i] = lfsr[9];
    save = lfsr[1] * lfsr[2] * lfsr[5] * lfsr[7] * lfsr[8] * lfsr[9];
    for (k = 9; k >= 1; --k) lfsr[k] = lfsr[k - 1];
    lfsr[0] = save;
  }
  for (i = 0; i < 1023; ++i) {
    int src = ((i - g2shift) % 1023 + 1023) % 1023; /* rotate_right */
    out[i] = -(g1[i] * g2[src]);
  }
}

/* ---- Legendre / Weil: beidou_codes.rs:74-126, l1c_codes.rs:76-157 -------- */
static void legendre(int n, unsigned char* seq) {
  int x;
  memset(seq, 0, (size_t)n);
  for (x = 1; x < n; ++x) seq[(long)x * x % n] = 1;
  seq[0] = 0;
}

void oracle_b1cp_bits(int prn, unsigned char* out /*10230*/) {
  static unsigned char L[10243];
  int n, w = g_b1cp_wp[prn - 1][0], p = g_b1cp_wp[prn - 1][1];
  legendre(10243, L);
  for (n = 0; n < 10230; ++n) {
    int k = (n + p - 1) % 10243;
    out[n] = L[k] ^ L[(k + w) % 10243];
  }
}

void oracle_l1cp_bits(int prn, unsigned char* out /*10230*/) {
  static unsigned char L[10223], W[10223];
  static const unsigned char ex[7] = {0, 1, 1, 0, 1, 0, 0};
  int k, o = 0, w = g_l1cp_wp[prn - 1][0], p = g_l1cp_wp[prn - 1][1];
  legendre(10223, L);
  for (k = 0; k < 10223; ++k) W[k] = L[k] ^ L[(k + w) % 10223];
  for (k = 0; k < p - 1; ++k) out[o++] = W[k];
  for (k = 0; k < 7; ++k) out[o++] = ex[k];
  for (k = p - 1; k < 10223; ++k) out[o++] = W[k];
}

/* ---- Galileo hex decode: galileo.rs:82-94 -------------------------------- */
void oracle_e1c_chips(int prn, double* out /*4092*/) {
  const char* hex = g_e1c_hex[prn - 1];
  int i, bit;
  for (i = 0; i < 1023; ++i) {
    char c = hex[i];
    int v = (c <= '9') ? c - '0' : (c | 0x20) - 'a' + 10;
    for (bit = 0; bit < 4; ++bit) out[i * 4 + bit] = ((v >> (3 - bit)) & 1) ? 1.0 : -1.0;
  }
}

/*
 * Base sequence the reference resamples from, as +-1 doubles.
 * constellation ids follow include/tga.h (0 GPS, 1 Galileo, 2 BeiDou,
 * 3 SBAS, 4 L1C, 5 QZSS).  Returns the length, or 0 for a bad PRN.
 */
int oracle_base_sequence(int constellation, int prn, double* out /*>=20460*/) {
  int i;
  unsigned char bits[10230];
  switch (constellation) {
    case 0:
      if (prn < 1 || prn > 38) return 0;
      oracle_ca_from_delay(g_gps_g2[prn - 1], out);
      return 1023;
    case 3:
      if (prn < 120 || prn > 158) return 0;
      oracle_ca_from_delay(g_sbas_g2[prn - 120], out);
      return 1023;
    case 5:
      if (prn < 184 || prn > 206) return 0;
      oracle_ca_from_delay(g_qzss_g2[prn - 184], out);
      return 1023;
    case 1:
      if (prn < 1 || prn > 50) return 0;
      oracle_e1c_chips(prn, out);
      return 4092;
    case 2:
    case 4:
      if (prn < 1 || prn > 63) return 0;
      if (constellation == 2) oracle_b1cp_bits(prn, bits); else oracle_l1cp_bits(prn, bits);
      for (i = 0; i < 10230; ++i) { /* 1 - 2x, then BOC(1,1) [+c, -c] */
        double c = 1.0 - 2.0 * bits[i];
        out[2 * i] = c;
        out[2 * i + 1] = -c;
      }
      return 20460;
  }
  return 0;
}

/* gold_code_from_ca / e1c_code_resampled / b1c_code_resampled rule. */
int oracle_resampled(int constellation, int prn, double samples_per_code, size_t num_samples,
                     double* out) {
  static double seq[20460];
  size_t n;
  int len = oracle_base_sequence(constellation, prn, seq);
  double spc;
  if (!len) return 0;
  spc = samples_per_code / (double)len;
  for (n = 0; n < num_samples; ++n) {
    double q = floor((double)n / spc);
    size_t idx = q > 0.0 ? (size_t)q : 0;
    out[n] = seq[idx % (size_t)len];
  }
  return len;
}

/* ---- ACR: acr.rs:49-84 ---------------------------------------------------- */
static const double (*acr_table(int id, int* n))[2] {
  if (id < 0 || id > 3 || g_acr_n[id] == 0) {
    *n = 0;
    return 0;
  }
  *n = g_acr_n[id];
  return (const double(*)[2])g_acr[id];
}

int oracle_acr_table(int id, double* out, int cap) {
  int n, i;
  const double(*t)[2] = acr_table(id, &n);
  for (i = 0; i < n && i < cap; ++i) { out[2 * i] = t[i][0]; out[2 * i + 1] = t[i][1]; }
  return n;
}

/* Returns 1 and writes *cn0 for Some(v), 0 for None. */
int oracle_estimate_cn0(double r_a, int id, double* cn0) {
  int n, lo = 0, hi;
  const double(*t)[2] = acr_table(id, &n);
  double l, a, b, tt, v;
  if (!t || !(r_a > 1.0) || !isfinite(r_a)) return 0;
  if (r_a <= t[0][0]) { *cn0 = t[0][1]; return 1; }
  if (r_a >= t[n - 1][0]) { *cn0 = t[n - 1][1]; return 1; }
  hi = n; /* partition_point(r < r_a): first index with r >= r_a */
  while (lo < hi) { int mid = (lo + hi) / 2; if (t[mid][0] < r_a) lo = mid + 1; else hi = mid; }
  if (lo == 0) { *cn0 = t[0][1]; return 1; }
  if (lo >= n) { *cn0 = t[n - 1][1]; return 1; }
  l = log(r_a); a = log(t[lo - 1][0]); b = log(t[lo][0]);
  tt = (l - a) / (b - a);
  v = t[lo - 1][1] + tt * (t[lo][1] - t[lo - 1][1]);
  if (v < 20.0) v = 20.0;
  if (v > 70.0) v = 70.0;
  *cn0 = v;
  return 1;
}

/* ---- stats.rs:10-30 --------------------------------------------------------- */
static int cmp_d(const void* a, const void* b) {
  double x = *(const double*)a, y = *(const double*)b;
  return (x > y) - (x < y);
}
double oracle_median(const double* x, size_t n) {
  double* c = (double*)malloc(n * sizeof(double)), r;
  memcpy(c, x, n * sizeof(double));
  qsort(c, n, sizeof(double), cmp_d);
  r = (n % 2 == 0) ? (c[n / 2 - 1] + c[n / 2]) / 2.0 : c[n / 2];
  free(c);
  return r;
}
double oracle_mad(const double* x, size_t n, double med) {
  double* d = (double*)malloc(n * sizeof(double)), r;
  size_t i;
  for (i = 0; i < n; ++i) d[i] = fabs(x[i] - med);
  r = oracle_median(d, n);
  free(d);
  return r;
}

/* ---- observation.rs:232-240 and :175-195 ------------------------------------ */
void oracle_unpack_bits(const uint8_t* packed, size_t nbytes, uint8_t* out) {
  size_t i;
  int b;
  for (i = 0; i < nbytes; ++i)
    for (b = 7; b >= 0; --b) out[i * 8 + (7 - b)] = (packed[i] >> b) & 1;
}

double oracle_correlate(const uint8_t* a_bits, const uint8_t* b_bits, size_t n) {
  double sum = 0.0;
  size_t i;
  for (i = 0; i < n; ++i) sum += (a_bits[i] ? 1.0 : -1.0) * (b_bits[i] ? 1.0 : -1.0);
  return sum / (double)n;
}

/* Antenna mean of the bipolar samples, summed in order as acquisition.rs:285. */
double oracle_bipolar_mean(const uint8_t* bits, size_t n) {
  double s = 0.0;
  size_t i;
  for (i = 0; i < n; ++i) s += bits[i] ? 1.0 : -1.0;
  return s / (double)n;
}

/* ---- testutil.rs:84-100: xorshift64 uniform and Box-Muller normal ----------- */
static double xs_next(uint64_t* s) {
  uint64_t x = *s;
  x ^= x << 13;
  x ^= x >> 7;
  x ^= x << 17;
  *s = x;
  return (double)(x >> 11) / (double)(1ull << 53);
}
void oracle_xorshift_uniform(uint64_t seed, size_t n, double* out) {
  size_t i;
  for (i = 0; i < n; ++i) out[i] = xs_next(&seed);
}
void oracle_xorshift_gaussian(uint64_t seed, size_t n, double* out) {
  size_t i;
  const double tau = 6.283185307179586;
  for (i = 0; i < n; ++i) {
    double u1 = xs_next(&seed), u2;
    if (u1 < 1e-12) u1 = 1e-12;
    u2 = xs_next(&seed);
    out[i] = sqrt(-2.0 * log(u1)) * cos(tau * u2);
  }
}
