// Adjoint of the band-pass bank and interval detectors for the per-band
// candidates (a5-a9): dL/draw[band][frame] -> dL/dy, with every discrete
// choice held fixed (which events exist, each frame's histc segments, the
// range checks that zero a candidate).
//
// Forward, per band b of a clip (harvest.cpp:99-293, GetFilteredSignal,
// ZeroCrossingEngine, GetFourZeroCrossingIntervals, interp1,
// GetF0CandidateContourSub):
//   f_b[i]  = sum_j y[j] h_b[i + H_b + 1 - j]               (taps h_b, 2 H_b + 1 long)
//   e       = i + 1 - s0 / (s1 - s0)                        (fine edge; (s0, s1) from f_b
//             at i, i + 1 for the two zero-crossing kinds, from its first
//             difference at i .. i + 2 for the peak and dip kinds)
//   x_m     = (e_m + e_{m+1}) / 2 / fs,  y_m = fs / (e_{m+1} - e_m)
//   track   = y_{k-1} + s (y_k - y_{k-1}),  s = (t - x_{k-1}) / (x_k - x_{k-1})
//   raw     = (track_0 + track_1 + track_2 + track_3) / 4
// The backward pass reruns the band bank with its dump (each block's
// filtered samples exactly as its event scan read them), re-detects the same
// events from them, walks the frames as band_contour_walk does, and chains
// the derivatives back to f_b and then, through the transpose of the
// filter (a correlation with h_b), to y. WORLD's final-bin term (the two
// spectrum bins its in-place product overwrites) is held fixed: it scales
// with each band's filter response at the Nyquist frequency and the
// waveform's content there, both negligible for these band-pass filters.
#include "hv_events.cuh"
#include "hv_stages.cuh"

namespace hv {

namespace {

constexpr int kAdjointThreads = 256;

__global__ void __launch_bounds__(kAdjointThreads)
raw_adjoint(RawAdjointView v) {
  __shared__ int item_slot;
  __shared__ unsigned long long scan_scratch[kAdjointThreads / 32];
  const BatchView& B = v.batch;
  const FftBankGeometry& g = v.geo;
  const int tid = threadIdx.x;
  const int stride = g.valid + 2;
  const int run = g.run;
  const int64_t cap = v.slot_capacity;
  double* edge[4];
  long long* where[4];
  double* grad[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int64_t base = (static_cast<int64_t>(blockIdx.x) * 4 + k) * cap;
    edge[k] = v.edges + base;
    where[k] = v.where + base;
    grad[k] = v.grad_edges + base;
  }
  const double fs = B.fs_r;
  for (;;) {
    if (tid == 0) item_slot = atomicAdd(v.queue, 1);
    __syncthreads();
    const int item = item_slot;
    __syncthreads();
    if (item >= v.item_count) return;
    const int c = v.items[item].x, b = v.items[item].y;
    const int64_t y0 = B.y_off[c], y_len = B.y_off[c + 1] - y0;
    const int64_t blk0 = g.blk_off[c], blocks = g.blk_off[c + 1] - blk0;
    const double* dump = v.dump + (static_cast<int64_t>(b) * g.total_blocks + blk0) * stride;
    // 1. The events, in the forward's order and with its expressions.
    int count[4] = {0, 0, 0, 0};
    for (int64_t j = 0; j < blocks; ++j) {
      const int64_t o = j * g.valid;
      const int edge_end = static_cast<int>(min(static_cast<int64_t>(g.valid), y_len - 1 - o));
      const int peak_end = static_cast<int>(min(static_cast<int64_t>(g.valid), y_len - 2 - o));
      const double* d = dump + j * stride;
      const int q_lo = min(tid * run, edge_end), q_hi = min(q_lo + run, edge_end);
      const int len = q_hi - q_lo;
      unsigned hits[4] = {0u, 0u, 0u, 0u};
      for (int i = 0; i < len; ++i) {
        const double f0 = d[q_lo + i], f1 = d[q_lo + i + 1], f2 = d[q_lo + i + 2];
        const double a0 = -f0, a1 = -f1, a2 = -f2;
        const double d0 = a0 - a1, d1 = a1 - a2;
        hits[0] |= (0.0 < f0 && f1 <= 0.0) ? 1u << i : 0u;
        hits[1] |= (0.0 < a0 && a1 <= 0.0) ? 1u << i : 0u;
        if (q_lo + i < peak_end) {
          hits[2] |= (0.0 < d0 && d1 <= 0.0) ? 1u << i : 0u;
          hits[3] |= (0.0 < -d0 && -d1 <= 0.0) ? 1u << i : 0u;
        }
      }
      const unsigned long long mine = static_cast<unsigned long long>(__popc(hits[0])) |
                                      static_cast<unsigned long long>(__popc(hits[1])) << 16 |
                                      static_cast<unsigned long long>(__popc(hits[2])) << 32 |
                                      static_cast<unsigned long long>(__popc(hits[3])) << 48;
      unsigned long long total;
      const unsigned long long before = block_scan_packed(mine, scan_scratch, total);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        int64_t at = count[k] + static_cast<int>((before >> (16 * k)) & 0xffff);
        for (unsigned m = hits[k]; m; m &= m - 1) {
          const int i = __ffs(m) - 1;
          const double f0 = d[q_lo + i], f1 = d[q_lo + i + 1];
          double s0, s1;
          if (k < 2) {
            s0 = k == 0 ? f0 : -f0;
            s1 = k == 0 ? f1 : -f1;
          } else {
            const double a0 = -f0, a1 = -f1, a2 = -d[q_lo + i + 2];
            const double d0 = a0 - a1, d1 = a1 - a2;
            s0 = k == 2 ? d0 : -d0;
            s1 = k == 2 ? d1 : -d1;
          }
          edge[k][at] = fine_edge(o + q_lo + i + 1, s0, s1);
          where[k][at] = j * stride + q_lo + i;
          grad[k][at] = 0.0;
          ++at;
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) count[k] += static_cast<int>((total >> (16 * k)) & 0xffff);
    }
    __syncthreads();
    // 2. Frames: the forward's walk, adding g / 4 dtrack / de to the three
    // edges each track uses.
    const int64_t f_begin = B.frame_off[c];
    const int frames = static_cast<int>(B.frame_off[c + 1] - f_begin);
    const bool usable = count[0] - 1 > 2 && count[1] - 1 > 2 && count[2] - 1 > 2 && count[3] - 1 > 2;
    const int per = (frames + kAdjointThreads - 1) / kAdjointThreads;
    const int fa = imin(tid * per, frames), fb = imin(fa + per, frames);
    if (usable && fa < fb) {
      const double centre = v.centre[b];
      const double upper = centre * 1.1, lower = centre * 0.9;
      const double* gr = v.grad_raw + static_cast<int64_t>(b) * v.total_frames + f_begin;
      int seg[4], last[4], lo[4], hi[4];
      double x0[4], x1[4], y0v[4], y1v[4], ez[4], ea[4], eb[4];
      const double t0 = frame_seconds(fa);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        last[k] = count[k] - 2;
        lo[k] = 0;
        hi[k] = count[k] - 1;
      }
      for (bool more = true; more;) {
        more = false;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          if (lo[k] >= hi[k]) continue;
          const int mid = (lo[k] + hi[k]) >> 1;
          if ((edge[k][mid] + edge[k][mid + 1]) * (0.5 / fs) <= t0) lo[k] = mid + 1; else hi[k] = mid;
          more |= lo[k] < hi[k];
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        seg[k] = imin(imax(lo[k], 1), last[k]);
        const double* e = edge[k] + seg[k];
        ez[k] = e[-1];
        ea[k] = e[0];
        eb[k] = e[1];
        x0[k] = (ez[k] + ea[k]) * (0.5 / fs);
        x1[k] = (ea[k] + eb[k]) * (0.5 / fs);
        y0v[k] = fs / (ea[k] - ez[k]);
        y1v[k] = fs / (eb[k] - ea[k]);
      }
      for (int f = fa; f < fb; ++f) {
        const double t = frame_seconds(f);
        for (;;) {
          bool any = false;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            if (!(seg[k] < last[k] && x1[k] <= t)) continue;
            any = true;
            ++seg[k];
            ez[k] = ea[k];
            ea[k] = eb[k];
            eb[k] = edge[k][seg[k] + 1];
            x0[k] = x1[k];
            y0v[k] = y1v[k];
            x1[k] = (ea[k] + eb[k]) * (0.5 / fs);
            y1v[k] = fs / (eb[k] - ea[k]);
          }
          if (!any) break;
        }
        double track[4], s[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          s[k] = (t - x0[k]) / (x1[k] - x0[k]);
          track[k] = y0v[k] + s[k] * (y1v[k] - y0v[k]);
        }
        const double val = (track[0] + track[1] + track[2] + track[3]) / 4.0;
        if (val > upper || val < lower || val > B.f0_ceil || val < B.f0_floor) continue;
        const double gv = gr[f];
        if (gv == 0.0) continue;
        const double gk = gv / 4.0, half_fs = 0.5 / fs;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const double h = x1[k] - x0[k];
          const double ds0 = (s[k] - 1.0) / h, ds1 = -s[k] / h;     // ds/dx0, ds/dx1
          const double dy = y1v[k] - y0v[k];
          const double d_y0 = y0v[k] * y0v[k] / fs, d_y1 = y1v[k] * y1v[k] / fs;
          // x0 = (ez + ea) / 2 / fs, x1 = (ea + eb) / 2 / fs,
          // y0 = fs / (ea - ez), y1 = fs / (eb - ea).
          const double dz = (1.0 - s[k]) * d_y0 + dy * ds0 * half_fs;
          const double da = -(1.0 - s[k]) * d_y0 + s[k] * d_y1 + dy * (ds0 + ds1) * half_fs;
          const double db = -s[k] * d_y1 + dy * ds1 * half_fs;
          atomicAdd(grad[k] + seg[k] - 1, gk * dz);
          atomicAdd(grad[k] + seg[k], gk * da);
          atomicAdd(grad[k] + seg[k] + 1, gk * db);
        }
      }
    }
    __syncthreads();
    // 3. Each edge e = i + 1 - s0 / (s1 - s0): de/ds0 = -s1 / D^2,
    // de/ds1 = s0 / D^2 with D = s1 - s0, then (s0, s1) back to f_b.
    double* gf = v.grad_f + static_cast<int64_t>(b) * v.y_total + y0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      for (int n = tid; n < count[k]; n += kAdjointThreads) {
        const double ge = grad[k][n];
        if (ge == 0.0) continue;
        const long long w = where[k][n];
        const int64_t j = w / stride;
        const int q = static_cast<int>(w - j * stride);
        const double* d = dump + w;
        const int64_t i = j * g.valid + q;          // sample index of f0 in the clip's y
        const double f0 = d[0], f1 = d[1];
        double s0, s1;
        if (k < 2) {
          s0 = k == 0 ? f0 : -f0;
          s1 = k == 0 ? f1 : -f1;
        } else {
          const double a0 = -f0, a1 = -f1, a2 = -d[2];
          s0 = k == 2 ? a0 - a1 : -(a0 - a1);
          s1 = k == 2 ? a1 - a2 : -(a1 - a2);
        }
        const double den = s1 - s0;
        const double g0 = ge * (-s1 / (den * den)), g1 = ge * (s0 / (den * den));   // dL/ds0, dL/ds1
        if (k == 0) {
          atomicAdd(gf + i, g0);
          atomicAdd(gf + i + 1, g1);
        } else if (k == 1) {
          atomicAdd(gf + i, -g0);
          atomicAdd(gf + i + 1, -g1);
        } else {
          // s0 = f1 - f0, s1 = f2 - f1 (kind 2); negated for kind 3.
          const double sg = k == 2 ? 1.0 : -1.0;
          atomicAdd(gf + i, -sg * g0);
          atomicAdd(gf + i + 1, sg * (g0 - g1));
          atomicAdd(gf + i + 2, sg * g1);
        }
      }
    }
    __syncthreads();
  }
}

// Transpose of the filter: dL/dy[j] = scale sum_b sum_m dL/df_b[j + m - H_b - 1] h_b[m],
// with h_b[m] = taps_rev[b][2 H_b - m]. The band bank's block transforms
// leave their outputs `scale` (the real block length) times the
// convolution, and the events were read from those outputs. One thread per
// sample.
__global__ void __launch_bounds__(256)
band_correlate(BatchView v, const double* __restrict__ grad_f, int64_t y_total, const int* __restrict__ half,
               const int64_t* __restrict__ tap_off, const double* __restrict__ taps_rev, double scale,
               double* __restrict__ grad_y) {
  const int64_t gy = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gy >= y_total) return;
  const int c = owner(v.y_off, v.clips, gy);
  const int64_t y0 = v.y_off[c];
  const int64_t j = gy - y0, y_len = v.y_off[c + 1] - y0;
  double acc = 0.0;
  for (int b = 0; b < v.bands; ++b) {
    const int h = half[b];
    const double* taps = taps_rev + tap_off[b];
    const double* gf = grad_f + static_cast<int64_t>(b) * y_total + y0;
    const int m_lo = static_cast<int>(max(static_cast<int64_t>(0), h + 1 - j));
    const int m_hi = static_cast<int>(min(static_cast<int64_t>(2 * h), y_len - 1 - j + h + 1));
    for (int m = m_lo; m <= m_hi; ++m) acc = fma(gf[j + m - h - 1], taps[2 * h - m], acc);
  }
  grad_y[gy] = scale * acc;
}

}  // namespace

cudaError_t launch_raw_adjoint(const RawAdjointView& v, int ctas, cudaStream_t stream) {
  raw_adjoint<<<ctas, kAdjointThreads, 0, stream>>>(v);
  return cudaGetLastError();
}

cudaError_t launch_band_correlate(const BatchView& v, const double* grad_f, int64_t y_total, const int* half,
                                  const int64_t* tap_off, const double* taps_rev, double* grad_y,
                                  cudaStream_t stream) {
  band_correlate<<<static_cast<unsigned>((y_total + 255) / 256), 256, 0, stream>>>(
      v, grad_f, y_total, half, tap_off, taps_rev, static_cast<double>(fft_bank_block_length()), grad_y);
  return cudaGetLastError();
}

}  // namespace hv
