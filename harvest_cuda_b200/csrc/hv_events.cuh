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
// interval track derived from `count` fine edges (harvest.cpp:188-191):
// locations (e_j + e_{j+1}) / 2 / fs, values fs / (e_{j+1} - e_j).
__device__ inline double interval_at(const double* edges, int count, double fs, double t) {
  const int intervals = count - 1;
  int lo = 0, hi = intervals;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const double loc = (edges[mid] + edges[mid + 1]) / 2.0 / fs;
    if (loc <= t) lo = mid + 1; else hi = mid;
  }
  const int seg = imin(imax(lo, 1), intervals - 1);
  const double x0 = (edges[seg - 1] + edges[seg]) / 2.0 / fs;
  const double x1 = (edges[seg] + edges[seg + 1]) / 2.0 / fs;
  const double y0 = fs / (edges[seg] - edges[seg - 1]);
  const double y1 = fs / (edges[seg + 1] - edges[seg]);
  const double s = (t - x0) / (x1 - x0);
  return y0 + s * (y1 - y0);
}

// GetF0CandidateContour(Sub) (harvest.cpp:240-293) for one band of one
// clip: the mean of the four interpolated tracks at t = frame / 1000,
// limited to [0.9, 1.1] x centre and [floor, ceil]; all zero unless every
// track has more than two intervals.
__device__ inline void band_contour(const BatchView& B, double* const ev[4], const int count[4],
                                    double centre, double* out, int frames) {
  const bool usable = count[0] - 1 > 2 && count[1] - 1 > 2 && count[2] - 1 > 2 && count[3] - 1 > 2;
  const double upper = centre * 1.1, lower = centre * 0.9;
  for (int f = threadIdx.x; f < frames; f += blockDim.x) {
    double val = 0.0;
    if (usable) {
      const double t = f * 1 / 1000.0;
      const double i0 = interval_at(ev[0], count[0], B.fs_r, t);
      const double i1 = interval_at(ev[1], count[1], B.fs_r, t);
      const double i2 = interval_at(ev[2], count[2], B.fs_r, t);
      const double i3 = interval_at(ev[3], count[3], B.fs_r, t);
      val = (i0 + i1 + i2 + i3) / 4.0;
      if (val > upper || val < lower || val > B.f0_ceil || val < B.f0_floor) val = 0.0;
    }
    out[f] = val;
  }
}

// Interval segment used at time t (histc clamping): the number of interval
// locations <= t, clamped to [1, intervals - 1]; by binary search over the
// fine edges in global memory.
__device__ inline int segment_at(const double* edges, int count, double fs, double t) {
  const int intervals = count - 1;
  int lo = 0, hi = intervals;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if ((edges[mid] + edges[mid + 1]) / 2.0 / fs <= t) lo = mid + 1; else hi = mid;
  }
  return imin(imax(lo, 1), intervals - 1);
}

// band_contour for one CTA, with the event lists staged through shared
// memory: frames go in chunks of blockDim.x; the segments a chunk can use
// lie between the segments of its first and last frame, so that slice of
// every list is copied to `stage` (coalesced) and searched there. Chunk
// bounds are found for up to blockDim.x chunks at once, one thread each.
// `bounds` holds 8 * blockDim.x ints; `stage` holds `capacity` doubles.
// A chunk whose slices do not fit falls back to searches in global memory.
__device__ inline void band_contour_staged(const BatchView& B, double* const ev[4], const int count[4],
                                           double centre, double* out, int frames, int* bounds,
                                           double* stage, int capacity) {
  const int nt = blockDim.x, tid = threadIdx.x;
  const bool usable = count[0] - 1 > 2 && count[1] - 1 > 2 && count[2] - 1 > 2 && count[3] - 1 > 2;
  if (!usable) {
    for (int f = tid; f < frames; f += nt) out[f] = 0.0;
    return;
  }
  const double fs = B.fs_r;
  const double upper = centre * 1.1, lower = centre * 0.9;
  const int chunks = (frames + nt - 1) / nt;
  for (int g0 = 0; g0 < chunks; g0 += nt) {
    const int group = imin(nt, chunks - g0);
    __syncthreads();
    // 8 searches per chunk (first and last frame, four tracks), one per
    // thread, so their dependent loads overlap instead of queueing.
    for (int w = tid; w < 8 * group; w += nt) {
      const int ci = w >> 3, which = w & 7, k = which >> 1;
      const int first = (g0 + ci) * nt;
      const int frame = (which & 1) ? imin(first + nt, frames) - 1 : first;
      bounds[which * nt + ci] = segment_at(ev[k], count[k], fs, frame * 1 / 1000.0);
    }
    __syncthreads();
    for (int ci = 0; ci < group; ++ci) {
      // Intervals lo-1 .. hi of each track: their locations and values,
      // computed once per chunk exactly as the reference writes them
      // (harvest.cpp:188-191).
      int lo[4], hi[4], base[4], total = 0;
      for (int k = 0; k < 4; ++k) {
        lo[k] = bounds[(2 * k) * nt + ci];
        hi[k] = bounds[(2 * k + 1) * nt + ci];
        base[k] = total;
        total += 2 * (hi[k] - lo[k] + 2);
      }
      const bool staged = total <= capacity;
      __syncthreads();
      if (staged)
        for (int k = 0; k < 4; ++k) {
          const int n_int = hi[k] - lo[k] + 2;
          double* loc = stage + base[k];
          double* val = loc + n_int;
          for (int i = tid; i < n_int; i += nt) {
            const double a = ev[k][lo[k] - 1 + i], b = ev[k][lo[k] + i];
            loc[i] = (a + b) / 2.0 / fs;
            val[i] = fs / (b - a);
          }
        }
      __syncthreads();
      const int f = (g0 + ci) * nt + tid;
      if (f >= frames) continue;
      const double t = f * 1 / 1000.0;
      double track[4];
      if (staged) {
        // The four searches are independent; unrolled they overlap.
        int a[4], b[4];
        const double* loc[4];
        const double* val[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int n_int = hi[k] - lo[k] + 2;
          loc[k] = stage + base[k] - (lo[k] - 1);   // loc[j], j in [lo-1, hi]
          val[k] = loc[k] + n_int;
          a[k] = lo[k];
          b[k] = hi[k];
        }
        // seg = lo + #{j in [lo, hi) : loc[j] <= t}
        bool more = true;
        while (more) {
          more = false;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            if (a[k] < b[k]) {
              const int mid = (a[k] + b[k]) >> 1;
              if (loc[k][mid] <= t) a[k] = mid + 1; else b[k] = mid;
              more |= a[k] < b[k];
            }
          }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const double x0 = loc[k][a[k] - 1], x1 = loc[k][a[k]];
          const double y0 = val[k][a[k] - 1], y1 = val[k][a[k]];
          const double s = (t - x0) / (x1 - x0);
          track[k] = y0 + s * (y1 - y0);
        }
      } else {
        for (int k = 0; k < 4; ++k) {
          const double* e = ev[k];
          int a = lo[k], b = hi[k];
          while (a < b) {
            const int mid = (a + b) >> 1;
            if ((e[mid] + e[mid + 1]) / 2.0 / fs <= t) a = mid + 1; else b = mid;
          }
          const double x0 = (e[a - 1] + e[a]) / 2.0 / fs;
          const double x1 = (e[a] + e[a + 1]) / 2.0 / fs;
          const double y0 = fs / (e[a] - e[a - 1]);
          const double y1 = fs / (e[a + 1] - e[a]);
          const double s = (t - x0) / (x1 - x0);
          track[k] = y0 + s * (y1 - y0);
        }
      }
      double val = (track[0] + track[1] + track[2] + track[3]) / 4.0;
      if (val > upper || val < lower || val > B.f0_ceil || val < B.f0_floor) val = 0.0;
      out[f] = val;
    }
  }
}

}  // namespace hv
