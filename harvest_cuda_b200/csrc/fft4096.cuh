// 4096-point complex FP64 FFT in shared memory for one CTA of 256 threads:
// three Stockham radix-16 passes, each thread holding one 16-point group in
// registers. The buffer is padded by one element per 16 so the strided
// stores of the first pass spread over the banks.
//
// Conventions: kSign = -1 computes X[k] = sum_m x[m] e^{-2 pi i m k / N};
// kSign = +1 the unnormalised inverse. Twiddles come from a table
// tw[t] = e^{-2 pi i t / 8192}, t in [0, 8192), shared with the real-FFT
// packing of 8192-point real blocks.
#pragma once
#include <cuda_runtime.h>

namespace hv {

constexpr int kFftN = 4096;          // complex points
constexpr int kFftThreads = 256;
constexpr int kRealN = 2 * kFftN;    // real block length
constexpr int kFftPadded = kFftN + kFftN / 16;

__device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }

// e^{kSign 2 pi i t / 8192} from the table (which stores the minus sign).
template <int kSign>
__device__ __forceinline__ double2 twiddle(const double2* __restrict__ tw, int t) {
  double2 w = tw[t & (kRealN - 1)];
  return kSign < 0 ? w : conj2(w);
}

// Multiplication by kSign * i.
template <int kSign>
__device__ __forceinline__ double2 rot90(double2 a) {
  return kSign < 0 ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
}

template <int kSign>
__device__ __forceinline__ void dft4(double2& a, double2& b, double2& c, double2& d) {
  double2 t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = rot90<kSign>(csub(b, d));
  a = cadd(t0, t2);
  c = csub(t0, t2);
  b = cadd(t1, t3);
  d = csub(t1, t3);
}

// In-register 16-point DFT, x[n] -> X[k], as 4 x 4 with internal twiddles.
template <int kSign>
__device__ __forceinline__ void dft16(double2 (&x)[16]) {
  const double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173;  // cos, sin pi/8
  const double r2 = 0.70710678118654752440;
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) dft4<kSign>(x[n2], x[n2 + 4], x[n2 + 8], x[n2 + 12]);
  // x[n2 + 4 k1] now holds A[n2][k1]; twiddle by e^{kSign 2 pi i n2 k1 / 16}.
  const double2 w1 = make_double2(c1, kSign * s1), w2 = make_double2(r2, kSign * r2),
                w3 = make_double2(s1, kSign * c1), w6 = make_double2(-r2, kSign * r2),
                w9 = make_double2(-c1, -kSign * s1);
  x[5] = cmul(x[5], w1);
  x[6] = cmul(x[6], w2);
  x[7] = cmul(x[7], w3);
  x[9] = cmul(x[9], w2);
  x[10] = rot90<kSign>(x[10]);
  x[11] = cmul(x[11], w6);
  x[13] = cmul(x[13], w3);
  x[14] = cmul(x[14], w6);
  x[15] = cmul(x[15], w9);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) dft4<kSign>(x[4 * k1], x[4 * k1 + 1], x[4 * k1 + 2], x[4 * k1 + 3]);
  // X[k1 + 4 k2] sits at x[4 k1 + k2]: transpose the 4 x 4 index.
  double2 t[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) t[i] = x[i];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) x[k1 + 4 * k2] = t[4 * k1 + k2];
}

// One Stockham pass with sub-transform length ls (1, 16, 256).
template <int kSign>
__device__ __forceinline__ void stockham_pass(double2* buf, const double2* __restrict__ tw, int ls) {
  const int j = threadIdx.x;
  const int k = j & (ls - 1);
  double2 x[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) x[m] = buf[fpad(j + m * (kFftN / 16))];
  if (ls > 1) {
    // w = e^{kSign 2 pi i k / (16 ls)}; x[m] *= w^m.
    const double2 w = twiddle<kSign>(tw, k * (kRealN / (16 * ls)));
    double2 wm = w;
#pragma unroll
    for (int m = 1; m < 16; ++m) {
      x[m] = cmul(x[m], wm);
      wm = cmul(wm, w);
    }
  }
  dft16<kSign>(x);
  __syncthreads();
  const int out0 = (j - k) * 16 + k;
#pragma unroll
  for (int m = 0; m < 16; ++m) buf[fpad(out0 + m * ls)] = x[m];
  __syncthreads();
}

// Exact quotient q / d for 0 <= q < 2^24 without an integer division: a
// float reciprocal estimate corrected by one step either way.
struct RunDivider {
  int d;
  float inv;
  __device__ __forceinline__ int operator()(int q) const {
    int r = static_cast<int>(static_cast<float>(q) * inv);
    if (r * d > q) --r;
    else if ((r + 1) * d <= q) ++r;
    return r;
  }
};

// WORLD's final-bin term for the samples of one block: sample q (absolute
// index origin + q of the unnormalised output) gets
// (-1)^(origin + q) (c0 + 2 (c1r cos phi + c1i sin phi)), phi = 2 pi (origin + q) / n,
// for q < limit; n is a power of two.
struct FinalBinTerm {
  double c0, c1r, c1i;
  long long origin;
  int n, limit;
  double step1_c, step1_s;      // e^{2 pi i / n}
  double step512_c, step512_s;  // e^{2 pi i 512 / n}
};

// Last pass of an inverse transform whose result is read as 8192 real
// samples x[2m] = Re z[m], x[2m+1] = Im z[m]: instead of storing z in natural
// order it stores samples p >= first into lin[(p - first) + (p - first) / run],
// one pad slot per `run` samples, the layout the event scan reads, with the
// final-bin term added on the way.
__device__ __forceinline__ void inverse_last_pass_to_runs(double2* buf, const double2* __restrict__ tw,
                                                          int first, RunDivider run, const FinalBinTerm& fb) {
  const int j = threadIdx.x;
  const int ls = 256;
  const int k = j & (ls - 1);
  double2 x[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) x[m] = buf[fpad(j + m * (kFftN / 16))];
  const double2 w = twiddle<+1>(tw, k * (2 * kFftN / (16 * ls)));
  double2 wm = w;
#pragma unroll
  for (int m = 1; m < 16; ++m) {
    x[m] = cmul(x[m], wm);
    wm = cmul(wm, w);
  }
  dft16<+1>(x);
  const int out0 = (j - k) * 16 + k;
  // Phasor of this thread's first (even) sample; its samples advance by 512.
  double pc, ps;
  {
    const long long r = (fb.origin + 2 * out0 - first) & (fb.n - 1);
    sincospi(2.0 * static_cast<double>(r) / fb.n, &ps, &pc);
  }
  const bool odd = (fb.origin - first) & 1;   // parity of origin + p for even p (first is even)
  // z = (c1r + i c1i) e^{-i phi} turns by e^{-i 2 pi / n} per sample; corr = c0 + 2 Re z.
  double zr = fb.c1r * pc + fb.c1i * ps, zi = fb.c1i * pc - fb.c1r * ps;
  __syncthreads();
  double* lin = reinterpret_cast<double*>(buf);
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    const int p = 2 * (out0 + m * ls) - first;
    const double zr1 = fma(fb.step1_c, zr, fb.step1_s * zi);
    if (p >= 0) {
      double v = x[m].x;
      if (p < fb.limit) {
        const double corr = fma(2.0, zr, fb.c0);
        v += odd ? -corr : corr;
      }
      lin[p + run(p)] = v;
    }
    if (p + 1 >= 0) {
      double v = x[m].y;
      if (p + 1 < fb.limit) {
        const double corr = fma(2.0, zr1, fb.c0);
        v += odd ? corr : -corr;
      }
      lin[p + 1 + run(p + 1)] = v;
    }
    const double nr = fma(fb.step512_c, zr, fb.step512_s * zi);
    zi = fma(fb.step512_c, zi, -fb.step512_s * zr);
    zr = nr;
  }
  __syncthreads();
}

// Full transform of buf (natural order in and out). Callers synchronise
// before the first pass; the last pass ends with a barrier.
template <int kSign>
__device__ __forceinline__ void fft4096(double2* buf, const double2* __restrict__ tw) {
  stockham_pass<kSign>(buf, tw, 1);
  stockham_pass<kSign>(buf, tw, 16);
  stockham_pass<kSign>(buf, tw, 256);
}

}  // namespace hv
