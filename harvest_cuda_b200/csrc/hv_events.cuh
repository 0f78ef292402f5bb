// Device helpers shared by both band-bank kernels (direct FIR and FFT):
// WORLD's final-bin correction terms, the sub-sample event positions, and
// the interpolation of the four interval tracks onto the 1 ms frames.
#pragma once
#include "hv_stages.cuh"

namespace hv {

// WORLD multiplies spectra in place while mirroring each product into bin
// n-i-1, so bins n/2-1 and n/2 both end up holding H[n/2-1] Y[n/2-1] Y[n/2]
// (harvest.cpp:116-133). Relative to the plain convolution this adds, at
// output index q of the unnormalised inverse transform,
//   (-1)^q [c0 + 2 (Re c1 cos(2 pi q / n) + Im c1 sin(2 pi q / n))]
// with P = H[n/2-1] Y[n/2-1], Q = Y[n/2] P, c0 = Re Q - H[n/2] Y[n/2],
// c1 = Q - P. Returns c0, Re c1, Im c1 multiplied by `scale`, reduced over
// the whole block (every thread receives the result). `taps` are the
// reversed taps of one band (taps[j] = h[2 half - j]); `red` is shared
// scratch of 3 x (blockDim.x / 32) doubles.
__device__ inline void final_bin_terms(const double* __restrict__ taps, int half, int n,
                                       const double* __restrict__ edge_bins, double scale,
                                       double* red, double& c0, double& c1r, double& c1i) {
  const int tid = threadIdx.x, warps = blockDim.x >> 5;
  double hn = 0.0, hr = 0.0, hi = 0.0;
  for (int m = tid; m <= 2 * half; m += blockDim.x) {
    const double h = taps[2 * half - m];
    const double sg = (m & 1) ? -h : h;
    double s, co;
    sincospi(2.0 * m / n, &s, &co);
    hn += sg;
    hr += sg * co;
    hi += sg * s;
  }
  for (int o = 16; o; o >>= 1) {
    hn += __shfl_down_sync(0xffffffffu, hn, o);
    hr += __shfl_down_sync(0xffffffffu, hr, o);
    hi += __shfl_down_sync(0xffffffffu, hi, o);
  }
  __syncthreads();
  if ((tid & 31) == 0) {
    red[tid >> 5] = hn;
    red[warps + (tid >> 5)] = hr;
    red[2 * warps + (tid >> 5)] = hi;
  }
  __syncthreads();
  hn = hr = hi = 0.0;
  for (int w = 0; w < warps; ++w) {
    hn += red[w];
    hr += red[warps + w];
    hi += red[2 * warps + w];
  }
  const double yn = edge_bins[0], yr = edge_bins[1], yi = edge_bins[2];
  // P = Y[n/2-1] H[n/2-1] and Q = Y[n/2] P in the reference's order.
  const double pr = yr * hr - yi * hi, pi = yr * hi + yi * hr;
  const double qr = yn * pr, qi = yn * pi;
  c0 = (qr - hn * yn) * scale;
  c1r = (qr - pr) * scale;
  c1i = (qi - pi) * scale;
}

// Exclusive scan over the block of four 16-bit counters packed in 64 bits;
// `scratch` holds blockDim.x / 32 words. Every thread receives the total.
__device__ inline unsigned long long block_scan_packed(unsigned long long v, unsigned long long* scratch,
                                                       unsigned long long& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  unsigned long long inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long n = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += n;
  }
  __syncthreads();
  if (lane == 31) scratch[warp] = inc;
  __syncthreads();
  unsigned long long before = 0, all = 0;
  for (int w = 0; w < warps; ++w) {
    if (w < warp) before += scratch[w];
    all += scratch[w];
  }
  total = all;
  return before + inc - v;
}

// Sub-sample position of a negative-going crossing between s0 > 0 and
// s1 <= 0 at integer edge e (harvest.cpp:184-186).
__device__ __forceinline__ double fine_edge(int64_t e, double s0, double s1) {
  return static_cast<double>(e) - s0 / (s1 - s0);
}

// interp1 with histc clamping (matlabfunctions.cpp:136-176) of the
// interval tracks derived from the fine edges (harvest.cpp:188-191):
// locations (e_j + e_{j+1}) / 2 / fs, values fs / (e_{j+1} - e_j), and
// GetF0CandidateContour(Sub) (harvest.cpp:240-293): the mean of the four
// interpolated tracks at t = frame / 1000, limited to [0.9, 1.1] x centre and
// [floor, ceil]; all zero unless every track has more than two intervals.

// band_contour for one CTA, each thread walking a contiguous run of frames.
// The histc segment of a time t is the number of interval locations <= t,
// clamped to [1, intervals - 1]. A binary search finds it for the run's
// first frame; frame times only increase, so for every later frame it is
// found by stepping forward while the next interval location is <= t. The four
// tracks step in lockstep (one iteration advances every track that needs it)
// so that their loads and divisions overlap; each track keeps the two edges
// of its current right interval and the edge after them, loaded one step
// ahead. The reference's expressions are evaluated with fewer divisions,
// each within a few roundings of its value: locations (e_j + e_{j+1}) (0.5 / fs),
// and on a step, with the edges em < ea < eb of the two intervals and
// r = 1 / ((eb - ea)(eb - em)), the value fs / (eb - ea) = fs (eb - em) r and
// interp1's slope divisor 1 / (x1 - x0) = 2 fs / (eb - em) = 2 fs (eb - ea) r.
// interp1 is continuous across intervals, so a location a rounding away
// moves a frame's value by no more than that.
__device__ inline void band_contour_walk(const BatchView& B, double* const ev[4], const int count[4],
                                         double centre, double* out, int frames) {
  const int nt = blockDim.x, tid = threadIdx.x;
  const int per = (frames + nt - 1) / nt;
  const int fa = imin(tid * per, frames), fb = imin(fa + per, frames);
  const bool usable = count[0] - 1 > 2 && count[1] - 1 > 2 && count[2] - 1 > 2 && count[3] - 1 > 2;
  if (!usable) {
    for (int f = fa; f < fb; ++f) out[f] = 0.0;
    return;
  }
  if (fa >= fb) return;
  const double fs = B.fs_r;
  const double half_rfs = 0.5 / fs, two_fs = 2.0 * fs;
  const double upper = centre * 1.1, lower = centre * 0.9;
  // val > upper || val > ceil is val > min(upper, ceil); likewise below.
  const double val_hi = fmin(upper, B.f0_ceil), val_lo = fmax(lower, B.f0_floor);
  int seg[4], last[4];
  double x0[4], x1[4], y0[4], y1[4], ea[4], eb[4];   // ea, eb: edges seg, seg + 1
  double inv[4];                                      // 1 / (x1 - x0)
  const double t0 = frame_seconds(fa);
  // The first frame's segment of the four tracks, by binary searches
  // interleaved so that their dependent loads overlap.
  int lo[4], hi[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    last[k] = count[k] - 2;                       // intervals - 1
    lo[k] = 0;
    hi[k] = count[k] - 1;
  }
  for (bool more = true; more;) {
    more = false;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (lo[k] >= hi[k]) continue;
      const int mid = (lo[k] + hi[k]) >> 1;
      if ((ev[k][mid] + ev[k][mid + 1]) * half_rfs <= t0) lo[k] = mid + 1; else hi[k] = mid;
      more |= lo[k] < hi[k];
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double* e = ev[k];
    seg[k] = imin(imax(lo[k], 1), last[k]);
    const int j = seg[k];
    const double em = e[j - 1];
    ea[k] = e[j];
    eb[k] = e[j + 1];
    x0[k] = (em + ea[k]) * half_rfs;
    x1[k] = (ea[k] + eb[k]) * half_rfs;
    y0[k] = fs / (ea[k] - em);
    y1[k] = fs / (eb[k] - ea[k]);
    inv[k] = two_fs / (eb[k] - em);
  }
  double nxt[4];   // the edge after eb
#pragma unroll
  for (int k = 0; k < 4; ++k) nxt[k] = ev[k][imin(seg[k] + 2, count[k] - 1)];
  for (int f = fa; f < fb; ++f) {
    const double t = frame_seconds(f);
    for (;;) {
      bool step[4], any = false;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        step[k] = seg[k] < last[k] && x1[k] <= t;
        any |= step[k];
      }
      if (!any) break;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (!step[k]) continue;
        ++seg[k];
        x0[k] = x1[k];
        y0[k] = y1[k];
        const double em = ea[k];
        ea[k] = eb[k];
        eb[k] = nxt[k];
        nxt[k] = ev[k][imin(seg[k] + 2, count[k] - 1)];
        x1[k] = (ea[k] + eb[k]) * half_rfs;
        const double dl = eb[k] - ea[k], dw = eb[k] - em;
        const double r = 1.0 / (dl * dw);
        y1[k] = fs * dw * r;
        inv[k] = two_fs * dl * r;
      }
    }
    double track[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double s = (t - x0[k]) * inv[k];
      track[k] = y0[k] + s * (y1[k] - y0[k]);
    }
    double val = (track[0] + track[1] + track[2] + track[3]) / 4.0;
    if (val > val_hi || val < val_lo) val = 0.0;
    out[f] = val;
  }
}

}  // namespace hv
