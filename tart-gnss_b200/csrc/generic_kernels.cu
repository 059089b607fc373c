// Generic acquisition path: the reference algorithm (correlate.rs:91-183) for
// any signal length N, on the GPU.
//
// Used when the fused polyphase kernels do not apply: windows that are not
// exactly two code periods, or codes that are not a whole number of samples
// per chip (e.g. 16 MHz sampling).  Per Doppler bin: carrier wipe-off,
// forward FFT of length N, for both hypotheses ([c,c] and [c,-c]) the product
// with the conjugated code spectrum, inverse FFT, |.|/sqrt(N), last-max
// argmax; then the hypothesis / bin reduction and the second peak.
//
// FFTs of arbitrary length use Bluestein's chirp-z identity
//   X[k] = w[k] * sum_n (x[n] w[n]) conj(w[k-n]),  w[n] = exp(i s pi n^2 / N)
// evaluated as a circular convolution of length M = 2^m >= 2N-1 with a radix-2
// Stockham FFT (Govindaraju et al., SC'08 formulation).
#include <cuda_runtime.h>

#include <cstdint>

#include "dft.cuh"
#include "engine.h"

namespace tga {

#define TGA_GLAUNCHED() (kernel_launch_add(1), cudaGetLastError())

namespace {

struct Ws {  // workspace views (float2 units unless noted)
  float2 *w, *Hf, *Hi, *tw, *C, *X, *Y, *buf, *tmp;
};

Ws carve(float2* base, int N, int M, int nb) {
  Ws v;
  float2* p = base;
  v.w = p; p += N;
  v.Hf = p; p += M;
  v.Hi = p; p += M;
  v.tw = p; p += M / 2;
  v.C = p; p += 2 * (size_t)N;
  v.X = p; p += (size_t)nb * N;
  v.Y = p; p += (size_t)2 * nb * N;
  const int batch = 2 * nb > 2 ? 2 * nb : 2;
  v.buf = p; p += (size_t)batch * M;
  v.tmp = p; p += (size_t)batch * M;
  return v;
}

__global__ void chirp_kernel(int N, int M, float2* w, float2* tw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) {
    // exp(-i pi n^2 / N) with n^2 reduced mod 2N exactly in integers
    const long long r = ((long long)i * i) % (2LL * N);
    double s, c;
    sincospi((double)r / (double)N, &s, &c);
    w[i] = make_float2((float)c, (float)-s);
  }
  if (i < M / 2) {
    double s, c;
    sincospi(2.0 * (double)i / (double)M, &s, &c);
    tw[i] = make_float2((float)c, (float)-s);  // exp(-2 pi i j / M)
  }
}

// h[m] = conj(w_sigma[m]) wrapped onto the length-M circle; sigma<0 forward.
__global__ void chirp_filter_kernel(int N, int M, const float2* w, int inverse, float2* h) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  int n = -1;
  if (m < N) n = m;
  else if (m > M - N) n = M - m;
  float2 v = make_float2(0.f, 0.f);
  if (n >= 0) {
    const float2 ws = inverse ? make_float2(w[n].x, -w[n].y) : w[n];  // w_sigma
    v = make_float2(ws.x, -ws.y);                                   // conj
  }
  h[m] = v;
}

__global__ void stockham_r2(const float2* __restrict__ x, float2* __restrict__ y, int M, int Ns, long long total,
                            const float2* __restrict__ tw, int inverse) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= total) return;
  const int half = M >> 1;
  const long long s = j / half;
  const int jj = (int)(j - s * half);
  const int k = jj & (Ns - 1);
  float2 t = tw[(long long)k * (M / (2 * Ns))];
  if (inverse) t.y = -t.y;
  const float2* xs = x + s * M;
  float2* ys = y + s * M;
  const float2 a = xs[jj];
  const float2 b = cmul(xs[jj + half], t);
  const int idx = (jj - k) * 2 + k;
  ys[idx] = cadd(a, b);
  ys[idx + Ns] = csub(a, b);
}

// returns pointer holding the result (x or y)
float2* fft_pow2(float2* x, float2* y, int M, int log2M, int nseq, const float2* tw, int inverse, cudaStream_t st,
                 cudaError_t* err) {
  const long long total = (long long)nseq * (M / 2);
  const int threads = 256;
  const unsigned blocks = (unsigned)((total + threads - 1) / threads);
  for (int p = 0, Ns = 1; p < log2M; ++p, Ns <<= 1) {
    stockham_r2<<<blocks, threads, 0, st>>>(x, y, M, Ns, total, tw, inverse);
    kernel_launch_add(1);
    float2* t = x;
    x = y;
    y = t;
  }
  *err = cudaGetLastError();
  return x;
}

__global__ void premul_kernel(const float2* __restrict__ in, int N, int M, long long total, const float2* __restrict__ w,
                              int inverse, float2* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const long long s = i / M;
  const int m = (int)(i - s * M);
  float2 v = make_float2(0.f, 0.f);
  if (m < N) {
    const float2 ws = inverse ? make_float2(w[m].x, -w[m].y) : w[m];
    v = cmul(in[s * N + m], ws);
  }
  out[i] = v;
}

__global__ void pointwise_kernel(float2* __restrict__ a, const float2* __restrict__ h, int M, long long total) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  a[i] = cmul(a[i], h[i % M]);
}

__global__ void postmul_kernel(const float2* __restrict__ c, int N, int M, long long total, const float2* __restrict__ w,
                               int inverse, float2* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const long long s = i / N;
  const int k = (int)(i - s * N);
  const float2 ws = inverse ? make_float2(w[k].x, -w[k].y) : w[k];
  const float2 v = cmul(c[s * M + k], ws);
  const float inv = 1.0f / (float)M;  // M is a power of two: exact
  out[i] = make_float2(v.x * inv, v.y * inv);
}

unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// Unnormalised DFT of nseq sequences of length N (in -> out), forward or inverse.
cudaError_t bluestein(const GenericPlan& gp, const Ws& v, const float2* in, float2* out, int nseq, int inverse,
                      cudaStream_t st) {
  const int N = gp.N, M = gp.Mpow2;
  const long long tot = (long long)nseq * M;
  premul_kernel<<<nblk(tot, 256), 256, 0, st>>>(in, N, M, tot, v.w, inverse, v.buf);
  kernel_launch_add(1);
  cudaError_t e;
  float2* r = fft_pow2(v.buf, v.tmp, M, gp.log2M, nseq, v.tw, 0, st, &e);
  if (e != cudaSuccess) return e;
  pointwise_kernel<<<nblk(tot, 256), 256, 0, st>>>(r, inverse ? v.Hi : v.Hf, M, tot);
  kernel_launch_add(1);
  float2* other = (r == v.buf) ? v.tmp : v.buf;
  float2* r2 = fft_pow2(r, other, M, gp.log2M, nseq, v.tw, 1, st, &e);
  if (e != cudaSuccess) return e;
  const long long totN = (long long)nseq * N;
  postmul_kernel<<<nblk(totN, 256), 256, 0, st>>>(r2, N, M, totN, v.w, inverse, out);
  return TGA_GLAUNCHED();
}

__global__ void code_in_kernel(const float* __restrict__ a, const float* __restrict__ b, int N, float2* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  out[i] = make_float2(a[i], 0.f);
  out[N + i] = make_float2(b[i], 0.f);
}

__global__ void conj_kernel(float2* a, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i].y = -a[i].y;
}

// correlate.rs:110-115 (carrier wipe-off, f32 phase)
__global__ void wipe_kernel(const float* __restrict__ sig, const double* __restrict__ pp, const double* __restrict__ fc,
                            int N, int nb, float2* __restrict__ X) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nb * N) return;
  const int b = (int)(i / N), n = (int)(i - (long long)b * N);
  const float ph = __double2float_rn(pp[n] * fc[b]);
  float sn, cs;
  sincos_phase(ph, &sn, &cs);
  const float s = sig[n];
  X[i] = make_float2(cs * s, sn * s);
}

__global__ void hyp_product_kernel(const float2* __restrict__ X, const float2* __restrict__ C, int N, int nb,
                                   float2* __restrict__ Y) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)2 * nb * N) return;
  const long long q = i / N;  // q = b*2 + h
  const int n = (int)(i - q * N);
  const int b = (int)(q >> 1), h = (int)(q & 1);
  Y[i] = cmul(X[(long long)b * N + n], C[(long long)h * N + n]);
}

// |.| * 1/sqrt(N) and last-max argmax per (bin, hypothesis) row.
__global__ void norm_argmax_kernel(const float2* __restrict__ Y, int N, float* __restrict__ corr,
                                   unsigned long long* __restrict__ keys) {
  const long long q = blockIdx.x;
  const float scale = 1.0f / sqrtf((float)N);
  unsigned long long best = 0ull;
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    const float2 v = Y[q * N + n];
    const float c = hypotf(v.x, v.y) * scale;  // Complex::norm() * scale
    corr[q * N + n] = c;
    const unsigned long long k = ((unsigned long long)__float_as_uint(c) << 32) | (unsigned)n;
    best = k > best ? k : best;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
    best = t > best ? t : best;
  }
  __shared__ unsigned long long part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) best = part[w] > best ? part[w] : best;
    best = part[0] > best ? part[0] : best;
    keys[q] = best;
  }
}

// second peak over the winning row (correlate.rs:156-175); one block.
__global__ void select_second_kernel(const float* __restrict__ corr, const unsigned long long* __restrict__ keys, int N,
                                     int nb, int period, int chip_width, int* __restrict__ res_i,
                                     float* __restrict__ res_f) {
  __shared__ int s_q, s_idx;
  __shared__ float s_peak;
  if (threadIdx.x == 0) {
    float pb = 0.f;
    int qb = 0, ib = 0;
    for (int b = 0; b < nb; ++b) {
      const unsigned long long ka = keys[2 * b], kb = keys[2 * b + 1];
      const float pa = __uint_as_float((unsigned)(ka >> 32)), pB = __uint_as_float((unsigned)(kb >> 32));
      const bool useB = pB > pa;  // strict: [c,c] wins ties
      const float pr = useB ? pB : pa;
      if (b == 0 || pr >= pb) {  // last maximum over bins
        pb = pr;
        qb = 2 * b + (useB ? 1 : 0);
        ib = (int)(unsigned)((useB ? kb : ka) & 0xffffffffu);
      }
    }
    s_q = qb;
    s_idx = ib;
    s_peak = pb;
  }
  __syncthreads();
  const int main_cp = s_idx % period;
  float m = -1.f;  // below every |.|
  const float* row = corr + (long long)s_q * N;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int cp = i % period;
    const int dist = cp >= main_cp ? min(cp - main_cp, period - cp + main_cp) : min(main_cp - cp, period - main_cp + cp);
    if (dist > chip_width) m = fmaxf(m, row[i]);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ float part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, part[w]);
    float second = m;
    if (!(second > 0.f)) second = 1e-6f;  // also covers "no candidate"
    res_i[0] = s_q >> 1;
    res_i[1] = s_idx;
    res_i[2] = s_q & 1;
    res_f[0] = s_peak;
    res_f[1] = second;
  }
}

// acquisition.rs:281-294 on the GPU: +-1 samples minus the row mean, first n
// as f32, and phase points TAU/fs * i in f64.
__global__ void bits_to_signal_kernel(const uint8_t* __restrict__ bits, size_t row_bytes, int row,
                                      const double* __restrict__ mean, int n, double pc, float* __restrict__ sig,
                                      double* __restrict__ pp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t byte = bits[(size_t)row * row_bytes + (i >> 3)];
  const double v = ((byte >> (7 - (i & 7))) & 1) ? 1.0 : -1.0;
  sig[i] = (float)(v - mean[row]);
  pp[i] = pc * (double)i;
}

}  // namespace

cudaError_t launch_bits_to_signal(const uint8_t* d_bits, size_t row_bytes, int row, const double* d_mean, int n,
                                  double pc, float* d_sig, double* d_pp, cudaStream_t st) {
  bits_to_signal_kernel<<<nblk(n, 256), 256, 0, st>>>(d_bits, row_bytes, row, d_mean, n, pc, d_sig, d_pp);
  return TGA_GLAUNCHED();
}

size_t generic_work_elems(const GenericPlan& gp, int nb) {
  const size_t N = gp.N, M = gp.Mpow2, batch = 2 * nb > 2 ? 2 * nb : 2;
  return N + 2 * M + M / 2 + 2 * N + nb * N + 2 * nb * N + 2 * batch * M;
}

cudaError_t launch_generic(const GenericPlan& gp, const float* d_sig, const double* d_pp, const double* d_fc, int nb,
                           const float* d_code_a, const float* d_code_b, int period, double fs, float2* d_work,
                           size_t work_elems, float* d_corr, int* d_res_i, float* d_res_f, cudaStream_t st) {
  if (work_elems < generic_work_elems(gp, nb)) return cudaErrorInvalidValue;
  const int N = gp.N, M = gp.Mpow2;
  Ws v = carve(d_work, N, M, nb);
  const int mx = N > M / 2 ? N : M / 2;
  chirp_kernel<<<nblk(mx, 256), 256, 0, st>>>(N, M, v.w, v.tw);
  kernel_launch_add(1);
  chirp_filter_kernel<<<nblk(M, 256), 256, 0, st>>>(N, M, v.w, 0, v.Hf);
  kernel_launch_add(1);
  chirp_filter_kernel<<<nblk(M, 256), 256, 0, st>>>(N, M, v.w, 1, v.Hi);
  cudaError_t e;
  float2* r = fft_pow2(v.Hf, v.buf, M, gp.log2M, 1, v.tw, 0, st, &e);
  if (e != cudaSuccess) return e;
  if (r != v.Hf) cudaMemcpyAsync(v.Hf, r, (size_t)M * sizeof(float2), cudaMemcpyDeviceToDevice, st);
  r = fft_pow2(v.Hi, v.buf, M, gp.log2M, 1, v.tw, 0, st, &e);
  if (e != cudaSuccess) return e;
  if (r != v.Hi) cudaMemcpyAsync(v.Hi, r, (size_t)M * sizeof(float2), cudaMemcpyDeviceToDevice, st);
  // code spectra (correlate.rs:47-68): conj(FFT(code)), conj(FFT(alt))
  code_in_kernel<<<nblk(N, 256), 256, 0, st>>>(d_code_a, d_code_b, N, v.X);
  kernel_launch_add(1);
  if ((e = bluestein(gp, v, v.X, v.C, 2, 0, st)) != cudaSuccess) return e;
  conj_kernel<<<nblk(2LL * N, 256), 256, 0, st>>>(v.C, 2LL * N);
  kernel_launch_add(1);
  // wipe-off and forward FFT per bin
  wipe_kernel<<<nblk((long long)nb * N, 256), 256, 0, st>>>(d_sig, d_pp, d_fc, N, nb, v.X);
  kernel_launch_add(1);
  if ((e = bluestein(gp, v, v.X, v.X, nb, 0, st)) != cudaSuccess) return e;
  hyp_product_kernel<<<nblk(2LL * nb * N, 256), 256, 0, st>>>(v.X, v.C, N, nb, v.Y);
  kernel_launch_add(1);
  if ((e = bluestein(gp, v, v.Y, v.Y, 2 * nb, 1, st)) != cudaSuccess) return e;
  // reuse tmp as keys storage (2*nb u64)
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(v.tmp);
  norm_argmax_kernel<<<2 * nb, 512, 0, st>>>(v.Y, N, d_corr, keys);
  kernel_launch_add(1);
  select_second_kernel<<<1, 1024, 0, st>>>(d_corr, keys, N, nb, period, (int)ceil(fs / 1.023e6), d_res_i, d_res_f);
  (void)fs;
  return TGA_GLAUNCHED();
}

}  // namespace tga
