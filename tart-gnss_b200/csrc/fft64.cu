// Double-precision FFT of any length for the RFI scan (rfi.rs:91-106 takes
// the f64 spectrum of a whole record per antenna).
//
// Mixed-radix Stockham autosort passes (the formulation of Govindaraju et
// al., SC'08, generalised from radix 2 to any radix R): with the
// sub-transforms of length Ns done, one pass writes
//
//   out[q Ns R + r Ns + k] = sum_{s < R} in[q Ns + k + s L / R] W_L^{s (k + r Ns) L / (Ns R)}
//
// (k < Ns, r < R, W_L = exp(-2 pi i / L)), so after the passes of all
// factors of L the result is in natural order.  Powers of two run as
// radix-16/8/4/2 butterflies, one per thread; other prime factors (up to
// kMaxRadix) as one output per thread, an R-term sum.  Twiddles come from one
// table W_L^m, m < L, built in double precision with sincospi.  A length
// with a prime factor above kMaxRadix is transformed by Bluestein's chirp-z
// identity over a power-of-two convolution.
//
// The real record of n samples is transformed as n/2 complex points z[m] =
// x[2m] + i x[2m+1] (the layout the record already has as doubles), then
//   X[k] = (Z[k] + conj(Z[L-k])) / 2 - i W_n^k (Z[k] - conj(Z[L-k])) / 2,
// L = n/2, of which the scan keeps |X[k]|^2 for k < n/2.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "engine.h"

namespace tga {

namespace {

constexpr int kMaxRadix = 1024;

__device__ __forceinline__ double2 cmul64(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// tw[m] = exp(-2 pi i m / L), m < L
__global__ void twiddle64_kernel(double2* __restrict__ tw, long long L) {
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < L; m += (long long)gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)m / (double)L, &s, &c);
    tw[m] = make_double2(c, -s);
  }
}

// One pass of power-of-two radix R, one butterfly (R outputs) per thread.
template <int R>
__global__ void __launch_bounds__(256) pass_pow2_kernel(const double2* __restrict__ in, double2* __restrict__ out,
                                                        const double2* __restrict__ tw, long long L, long long Ns,
                                                        long long total_j) {
  const long long LR = L / R, NsR = Ns * R, step = L / NsR;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total_j;
       t += (long long)gridDim.x * blockDim.x) {
    const long long a = t / LR, j = t - a * LR;
    const long long k = j % Ns, q = j / Ns;
    const double2* x = in + a * L + j;
    double2 v[R];
#pragma unroll
    for (int s = 0; s < R; ++s) {
      const double2 u = x[s * LR];
      v[s] = s == 0 ? u : cmul64(u, __ldg(tw + (s * k * step) % L));
    }
    // DFT-R of v: W_R^{r s} = tw[(r s mod R) L / R]
    double2* y = out + a * L + q * NsR + k;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      double2 acc = v[0];
#pragma unroll
      for (int s = 1; s < R; ++s) {
        const double2 w = __ldg(tw + ((r * s) % R) * LR);
        acc.x += v[s].x * w.x - v[s].y * w.y;
        acc.y += v[s].x * w.y + v[s].y * w.x;
      }
      y[r * Ns] = acc;
    }
  }
}

// One pass of any radix R, one output per thread (an R-term sum).
__global__ void __launch_bounds__(256) pass_any_kernel(const double2* __restrict__ in, double2* __restrict__ out,
                                                       const double2* __restrict__ tw, long long L, int R,
                                                       long long Ns, long long total) {
  const long long LR = L / R, NsR = Ns * R, step = L / NsR;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long a = i / L, o = i - a * L;
    const long long q = o / NsR, rem = o - q * NsR, r = rem / Ns, k = rem - r * Ns;
    const double2* x = in + a * L + q * Ns + k;
    const long long base = (k + r * Ns) * step;  // < L
    double2 acc = make_double2(0.0, 0.0);
    long long m = 0;
    for (int s = 0; s < R; ++s) {
      const double2 u = x[s * LR], w = __ldg(tw + m);
      acc.x += u.x * w.x - u.y * w.y;
      acc.y += u.x * w.y + u.y * w.x;
      m += base;
      if (m >= L) m -= L;
    }
    out[i] = acc;
  }
}

// factors of L in pass order: 16, 8, 4, 2 for the power of two, then the
// odd primes ascending; false when a prime factor exceeds kMaxRadix
bool factorise(long long L, std::vector<int>* radices) {
  radices->clear();
  long long m = L;
  int twos = 0;
  while (m % 2 == 0) {
    m /= 2;
    ++twos;
  }
  while (twos >= 4) {
    radices->push_back(16);
    twos -= 4;
  }
  if (twos == 3) radices->push_back(8);
  if (twos == 2) radices->push_back(4);
  if (twos == 1) radices->push_back(2);
  for (long long p = 3; p * p <= m || m > 1; p += 2) {
    if (p * p > m) p = m;  // m is prime
    while (m % p == 0) {
      if (p > kMaxRadix) return false;
      radices->push_back((int)p);
      m /= p;
    }
    if (m == 1) break;
  }
  return true;
}

int grid_for(long long work, int num_sms) {
  long long g = (work + 255) / 256;
  const long long cap = (long long)num_sms * 32;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

// Stockham passes over `batch` sequences of length L in a (ping-pong with
// b); returns the buffer holding the result.
double2* stockham(double2* a, double2* b, const double2* tw, long long L, int batch, const std::vector<int>& radices,
                  int num_sms, cudaStream_t st, cudaError_t* err) {
  long long Ns = 1;
  double2* x = a;
  double2* y = b;
  for (int R : radices) {
    const long long total = L * batch, total_j = total / R;
    switch (R) {
      case 16: pass_pow2_kernel<16><<<grid_for(total_j, num_sms), 256, 0, st>>>(x, y, tw, L, Ns, total_j); break;
      case 8: pass_pow2_kernel<8><<<grid_for(total_j, num_sms), 256, 0, st>>>(x, y, tw, L, Ns, total_j); break;
      case 4: pass_pow2_kernel<4><<<grid_for(total_j, num_sms), 256, 0, st>>>(x, y, tw, L, Ns, total_j); break;
      case 2: pass_pow2_kernel<2><<<grid_for(total_j, num_sms), 256, 0, st>>>(x, y, tw, L, Ns, total_j); break;
      default: pass_any_kernel<<<grid_for(total, num_sms), 256, 0, st>>>(x, y, tw, L, R, Ns, total); break;
    }
    kernel_launch_add(1);
    if ((*err = cudaGetLastError()) != cudaSuccess) return x;
    Ns *= R;
    double2* t = x;
    x = y;
    y = t;
  }
  return x;
}

// ---- Bluestein: X[k] = c[k] sum_m (x[m] c[m]) conj(c[k - m]), c[m] = W_{2L}^{m^2}
__global__ void chirp64_kernel(double2* __restrict__ c, long long L) {
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < L; m += (long long)gridDim.x * blockDim.x) {
    const unsigned long long r = ((unsigned long long)m * (unsigned long long)m) % (2ull * (unsigned long long)L);
    double s, co;
    sincospi((double)r / (double)L, &s, &co);
    c[m] = make_double2(co, -s);
  }
}
// h = conj(c) wrapped circularly into length M (index M - m for m > 0), zero elsewhere
__global__ void chirp_filter64_kernel(const double2* __restrict__ c, long long L, long long M, double2* __restrict__ h) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (long long)gridDim.x * blockDim.x) {
    long long m = -1;
    if (i < L) m = i;
    else if (i > M - L) m = M - i;
    h[i] = m >= 0 ? make_double2(c[m].x, -c[m].y) : make_double2(0.0, 0.0);
  }
}
__global__ void premul64_kernel(const double2* __restrict__ x, const double2* __restrict__ c, long long L, long long M,
                                double2* __restrict__ y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (long long)gridDim.x * blockDim.x)
    y[i] = i < L ? cmul64(x[i], c[i]) : make_double2(0.0, 0.0);
}
// conj(a * b): the inverse transform of the product runs as a forward one
__global__ void conjmul64_kernel(double2* __restrict__ a, const double2* __restrict__ b, long long M) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (long long)gridDim.x * blockDim.x) {
    const double2 v = cmul64(a[i], b[i]);
    a[i] = make_double2(v.x, -v.y);
  }
}
__global__ void postmul64_kernel(const double2* __restrict__ y, const double2* __restrict__ c, long long L, long long M,
                                 double2* __restrict__ out) {
  const double inv = 1.0 / (double)M;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < L; k += (long long)gridDim.x * blockDim.x) {
    const double2 v = make_double2(y[k].x * inv, -y[k].y * inv);  // conj of the forward transform, / M
    out[k] = cmul64(v, c[k]);
  }
}

// |X[k]|^2 for k < L of the real record whose n = 2 L point spectrum is
// recovered from Z = FFT_L(z), z[m] = x[2m] + i x[2m+1]
__global__ void real_power_kernel(const double2* __restrict__ Z, long long L, int batch, double* __restrict__ p) {
  const long long total = L * batch;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long a = i / L, k = i - a * L;
    const double2 zk = Z[a * L + k], zc = Z[a * L + (k == 0 ? 0 : L - k)];
    const double2 e = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y - zc.y));  // (Z[k] + conj Z[L-k]) / 2
    const double2 o = make_double2(0.5 * (zk.x - zc.x), 0.5 * (zk.y + zc.y));  // (Z[k] - conj Z[L-k]) / 2
    double s, c;
    sincospi((double)k / (double)L, &s, &c);  // W_n^k = exp(-i pi k / L) = (c, -s)
    // X = e - i W o
    const double2 wo = make_double2(c * o.x + s * o.y, c * o.y - s * o.x);
    const double xr = e.x + wo.y, xi = e.y - wo.x;
    p[i] = xr * xr + xi * xi;
  }
}

long long next_pow2(long long v) {
  long long m = 1;
  while (m < v) m <<= 1;
  return m;
}

}  // namespace

size_t fft64_workspace_bytes(long long n, int batch) {
  const long long L = n / 2;
  std::vector<int> r;
  if (factorise(L, &r)) return (size_t)L * 16;  // the twiddle table
  const long long M = next_pow2(2 * L - 1);
  return (size_t)(M + L + 3 * M) * 16;  // table of M, chirp, filter spectrum, two work buffers
}

cudaError_t real_power_spectrum(double* d_x, void* d_buf, void* d_work, long long n, int batch, double* d_p,
                                int num_sms, cudaStream_t st, std::string* why) {
  if (n % 2 != 0 || n < 4) {
    *why = "the RFI spectrum needs an even record of at least 4 samples";
    return cudaErrorInvalidValue;
  }
  const long long L = n / 2;
  double2* z = reinterpret_cast<double2*>(d_x);  // the record as L complex points
  double2* buf = static_cast<double2*>(d_buf);
  double2* work = static_cast<double2*>(d_work);
  cudaError_t e = cudaSuccess;
  std::vector<int> radices;
  double2* Z = nullptr;
  if (factorise(L, &radices)) {
    twiddle64_kernel<<<grid_for(L, num_sms), 256, 0, st>>>(work, L);
    kernel_launch_add(1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    Z = stockham(z, buf, work, L, batch, radices, num_sms, st, &e);
    if (e != cudaSuccess) return e;
  } else {
    // Bluestein per sequence: convolution length M = 2^m >= 2L - 1
    const long long M = next_pow2(2 * L - 1);
    factorise(M, &radices);
    double2* tw = work;
    double2* chirp = tw + M;
    double2* H = chirp + L;
    double2* u = H + M;
    double2* v = u + M;
    twiddle64_kernel<<<grid_for(M, num_sms), 256, 0, st>>>(tw, M);
    chirp64_kernel<<<grid_for(L, num_sms), 256, 0, st>>>(chirp, L);
    chirp_filter64_kernel<<<grid_for(M, num_sms), 256, 0, st>>>(chirp, L, M, u);
    kernel_launch_add(3);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    double2* h = stockham(u, v, tw, M, 1, radices, num_sms, st, &e);
    if (e != cudaSuccess) return e;
    if (h != H) e = cudaMemcpyAsync(H, h, (size_t)M * 16, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    for (int a = 0; a < batch; ++a) {
      premul64_kernel<<<grid_for(M, num_sms), 256, 0, st>>>(z + a * L, chirp, L, M, u);
      kernel_launch_add(1);
      double2* y = stockham(u, v, tw, M, 1, radices, num_sms, st, &e);
      if (e != cudaSuccess) return e;
      conjmul64_kernel<<<grid_for(M, num_sms), 256, 0, st>>>(y, H, M);
      kernel_launch_add(1);
      double2* w = stockham(y, y == u ? v : u, tw, M, 1, radices, num_sms, st, &e);
      if (e != cudaSuccess) return e;
      postmul64_kernel<<<grid_for(L, num_sms), 256, 0, st>>>(w, chirp, L, M, buf + a * L);
      kernel_launch_add(1);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    Z = buf;
  }
  real_power_kernel<<<grid_for(L * batch, num_sms), 256, 0, st>>>(Z, L, batch, d_p);
  kernel_launch_add(1);
  return cudaGetLastError();
}

}  // namespace tga
