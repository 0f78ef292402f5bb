// a4-a9 by overlap-save FFT convolution: the band-pass bank, the four
// interval detectors and the per-band candidates.
//
// WORLD filters every band with one whole-signal FFT of size n
// (GetFilteredSignal, harvest.cpp:99-148). Here the convolution is split
// into real blocks of B = 8192 samples that overlap by 2H + 2 (H the
// largest filter half length), so every transform fits in shared memory:
//   * block_spectra: the forward spectrum of every block of every clip,
//     computed once and shared by all bands;
//   * filter_spectra: per band the spectrum of its taps, placed so that the
//     valid outputs of every band start at the same block offset 2H;
//   * band_bank_fft: persistent CTAs take (clip, band) items longest first
//     and walk the clip block by block: spectrum product, inverse transform,
//     WORLD's final-bin correction, event detection and ordered compaction,
//     then interp1 of the four interval tracks at every 1 ms frame.
// The block outputs equal B times the linear convolution; WORLD's equal n
// times it; both scales are powers of two, so zero crossings are unchanged
// and the correction is added scaled by B / n.
#include "fft4096.cuh"
#include "hv_events.cuh"

namespace hv {

constexpr int kHalfN = kFftN;  // M: complex points per real block

// tw[t] = e^{-2 pi i t / 8192}. The refinement reads the same table.
static_assert(kRealN == kTwiddleN, "the twiddle table has one entry per real block sample");
__global__ void make_twiddles(double2* __restrict__ tw) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kRealN) return;
  double s, c;
  sincospi(2.0 * t / kRealN, &s, &c);
  tw[t] = make_double2(c, -s);
}

// Forward real FFT of the 8192 samples in `buf` (packed as z[m] = x[2m] +
// i x[2m+1]): emit(k, X[k]) for k = 0..4096.
template <class Emit>
__device__ void real_forward(double2* buf, const double2* __restrict__ tw, Emit emit) {
  __syncthreads();
  fft4096<-1>(buf, tw);
  for (int k = threadIdx.x; k <= kHalfN; k += kFftThreads) {
    const double2 a = buf[fpad(k & (kHalfN - 1))];
    const double2 b = conj2(buf[fpad((kHalfN - k) & (kHalfN - 1))]);
    const double2 e = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
    const double2 d = csub(a, b);
    const double2 o = make_double2(0.5 * d.y, -0.5 * d.x);  // d / (2i)
    emit(k, cadd(e, cmul(twiddle<-1>(tw, k), o)));
  }
}

// One spectrum per block of every clip; block j of clip c holds
// y[j V - H + 1 + p], p < 8192 (zero outside the clip). Each bin is turned by
// e^{-2 pi i k H / 8192}, the linear phase of every band's filter (below),
// so that the bands' products need only real amplitudes.
__global__ void __launch_bounds__(kFftThreads)
block_spectra(BatchView v, FftBankGeometry g, const double* __restrict__ y,
              const double2* __restrict__ tw, double2* __restrict__ spectra) {
  extern __shared__ double2 buf[];
  const int blk = blockIdx.x;
  const int c = owner(g.blk_off, v.clips, blk);
  const int64_t j = blk - g.blk_off[c];
  const int64_t y0 = v.y_off[c];
  const int64_t y_len = v.y_off[c + 1] - y0;
  const int64_t start = j * g.valid - g.max_half + 1;
  for (int m = threadIdx.x; m < kHalfN; m += kFftThreads) {
    const int64_t p0 = start + 2 * m, p1 = p0 + 1;
    buf[fpad(m)] = make_double2(p0 >= 0 && p0 < y_len ? y[y0 + p0] : 0.0,
                                p1 >= 0 && p1 < y_len ? y[y0 + p1] : 0.0);
  }
  double2* out = spectra + static_cast<int64_t>(blk) * (kHalfN + 1);
  const int H = g.max_half;
  real_forward(buf, tw, [&](int k, double2 x) { out[k] = cmul(x, twiddle<-1>(tw, k * H)); });
}

// Per band the spectrum of g_b[p] = h_b[p - (H - h_b)], p in [H - h_b, H + h_b].
// g_b is symmetric about p = H (h_b is a window times a cosine centred on its
// middle tap), so G_b[k] = A_b[k] e^{-2 pi i k H / 8192} with A_b real; the
// amplitudes A_b[k] (the real part after removing the phase; the imaginary
// part is rounding) are stored.
__global__ void __launch_bounds__(kFftThreads)
filter_spectra(const int* __restrict__ half, const int64_t* __restrict__ tap_off,
               const double* __restrict__ taps_rev, int max_half, const double2* __restrict__ tw,
               double* __restrict__ amps) {
  extern __shared__ double2 buf[];
  const int b = blockIdx.x;
  const int h = half[b];
  const double* taps = taps_rev + tap_off[b];   // taps_rev[j] = h_b[2h - j]
  auto tap = [&](int p) -> double {
    const int m = p - (max_half - h);
    return m >= 0 && m <= 2 * h ? taps[2 * h - m] : 0.0;
  };
  for (int m = threadIdx.x; m < kHalfN; m += kFftThreads) buf[fpad(m)] = make_double2(tap(2 * m), tap(2 * m + 1));
  double* out = amps + static_cast<int64_t>(b) * (kHalfN + 1);
  real_forward(buf, tw, [&](int k, double2 x) { out[k] = cmul(x, twiddle<+1>(tw, k * max_half)).x; });
}

__global__ void __launch_bounds__(kFftThreads, 2)
band_bank_fft(BankView v, FftBankGeometry g, const double2* __restrict__ spectra,
              const double* __restrict__ amps, const double2* __restrict__ tw,
              const double* __restrict__ edge_bins, int* __restrict__ queue, double* __restrict__ slots,
              double* __restrict__ raw) {
  extern __shared__ double2 buf[];
  __shared__ int item_slot;
  __shared__ double red[3 * (kFftThreads / 32)];
  __shared__ unsigned long long scan_scratch[kFftThreads / 32];
  const BatchView& B = v.batch;
  const int tid = threadIdx.x;
  double* xs = reinterpret_cast<double*>(buf);
  double* events = slots + blockIdx.x * (4 * v.slot_capacity);
  double* const ev[4] = {events, events + v.slot_capacity, events + 2 * v.slot_capacity,
                         events + 3 * v.slot_capacity};
  const int H = g.max_half;
  const int run = g.run;   // positions per thread in the event scan (even)
  const RunDivider div_run{run, 1.0f / run};
  for (;;) {
    if (tid == 0) item_slot = atomicAdd(queue, 1);
    __syncthreads();
    const int item = item_slot;
    __syncthreads();
    if (item >= v.item_count) return;
    const int c = v.items[item].x, b = v.items[item].y;
    const int half = v.half[b];
    const int64_t y_len = B.y_off[c + 1] - B.y_off[c];
    const int n = B.nfft[c];
    double c0, c1r, c1i;
    final_bin_terms(v.taps_rev + v.tap_off[b], half, n, edge_bins + 3 * c,
                    static_cast<double>(kRealN) / n, red, c0, c1r, c1i);
    const double* A = amps + static_cast<int64_t>(b) * (kHalfN + 1);
    const int64_t blk0 = g.blk_off[c], blocks = g.blk_off[c + 1] - blk0;
    FinalBinTerm fb;
    fb.c0 = c0;
    fb.c1r = c1r;
    fb.c1i = c1i;
    fb.n = n;
    sincospi(2.0 / n, &fb.step1_s, &fb.step1_c);
    sincospi(2.0 * 512 / n, &fb.step512_s, &fb.step512_c);
    int count[4] = {0, 0, 0, 0};
    for (int64_t j = 0; j < blocks; ++j) {
      const double2* Y = spectra + (blk0 + j) * (kHalfN + 1);
      __syncthreads();
      // Spectrum product and packing for the inverse real transform:
      // Z[k] = (X[k] + conj X[M-k]) + i e^{+2 pi i k / 8192} (X[k] - conj X[M-k]).
      for (int k = tid; k <= kHalfN / 2; k += kFftThreads) {
        const double2 yk = Y[k], ym = Y[kHalfN - k];
        const double ak = A[k], am = A[kHalfN - k];
        const double2 xk = make_double2(yk.x * ak, yk.y * ak);
        const double2 xm = make_double2(ym.x * am, ym.y * am);
        const double2 w = twiddle<+1>(tw, k);
        buf[fpad(k)] = cadd(cadd(xk, conj2(xm)), rot90<+1>(cmul(w, csub(xk, conj2(xm)))));
        if (k != 0 && k != kHalfN / 2) {
          const double2 w2 = make_double2(-w.x, w.y);   // e^{+2 pi i (M - k) / 8192}
          buf[fpad(kHalfN - k)] = cadd(cadd(xm, conj2(xk)), rot90<+1>(cmul(w2, csub(xm, conj2(xk)))));
        }
      }
      __syncthreads();
      stockham_pass<+1>(buf, tw, 1);
      stockham_pass<+1>(buf, tw, 16);
      // Output i = j V + q (block sample 2H + q) lands at lin[q + q / run],
      // plus WORLD's final-bin term at its unnormalised index i + half + 1.
      const int64_t o = j * g.valid;
      const int edge_end = static_cast<int>(min(static_cast<int64_t>(g.valid), y_len - 1 - o));
      const int peak_end = static_cast<int>(min(static_cast<int64_t>(g.valid), y_len - 2 - o));
      fb.origin = o + half + 1;
      fb.limit = edge_end + 2;
      inverse_last_pass_to_runs(buf, tw, 2 * H, div_run, fb);
      if (v.dump) {
        double* d = v.dump + (static_cast<int64_t>(b) * g.total_blocks + blk0 + j) * (g.valid + 2);
        for (int q = tid; q < edge_end + 2; q += kFftThreads) d[q] = xs[q + div_run(q)];
      }
      // Events: each thread scans a contiguous run of positions, counting in
      // the first pass; a block scan of the packed counts orders the runs;
      // the second pass writes the sub-sample edges of its hits.
      const int q_lo = min(tid * run, edge_end), q_hi = min(q_lo + run, edge_end);
      // Within this thread's run, sample q_lo + i sits at lin[q_lo + i + tid]
      // (i < run) and the two lookahead samples one slot further.
      const double* mine_lin = xs + q_lo + min(tid, edge_end / run + 1);
      auto X = [&](int i) -> double { return mine_lin[i + (i >= run ? 1 : 0)]; };
      const int len = q_hi - q_lo;   // run <= 32: hits fit one bit mask per kind
      // The four detectors compare each sample with zero and with its
      // neighbour: a sample is > 0 (pos) or < 0 (neg) by its sign and
      // magnitude bits, and a difference of two samples, rounded, has the
      // sign of their comparison. So with bit i of pos/neg for sample i and
      // of up/down for sample i + 1 > / < sample i, a hit at i is a set bit
      // i whose bit i + 1 is clear: pos then not pos (0 < f0, f1 <= 0), neg
      // then not neg, up then not up (0 < f1 - f0, f2 - f1 <= 0), down then
      // not down. Bits past sample len + 1 are never used.
      unsigned hits[4] = {0u, 0u, 0u, 0u};
      if (len > 0) {
        unsigned long long pos, neg, up = 0, down = 0;
        double prev = X(0);
        {
          const long long b = __double_as_longlong(prev);
          pos = b > 0 ? 1ull : 0ull;
          neg = static_cast<unsigned long long>(b) > 0x8000000000000000ull ? 1ull : 0ull;
        }
        for (int i0 = 0; i0 <= len; i0 += 8) {
          double v[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) v[u] = X(i0 + 1 + u);
          unsigned gp = 0u, gn = 0u, gu = 0u, gd = 0u;
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const double cur = v[u];
            const long long b = __double_as_longlong(cur);
            gp |= (b > 0 ? 1u : 0u) << u;
            gn |= (static_cast<unsigned long long>(b) > 0x8000000000000000ull ? 1u : 0u) << u;
            gu |= (cur > prev ? 1u : 0u) << u;
            gd |= (cur < prev ? 1u : 0u) << u;
            prev = cur;
          }
          pos |= static_cast<unsigned long long>(gp) << (i0 + 1);
          neg |= static_cast<unsigned long long>(gn) << (i0 + 1);
          up |= static_cast<unsigned long long>(gu) << i0;
          down |= static_cast<unsigned long long>(gd) << i0;
        }
        const unsigned len_mask = len >= 32 ? ~0u : (1u << len) - 1u;
        const int pk = imax(0, imin(len, peak_end - q_lo));
        const unsigned peak_mask = pk >= 32 ? ~0u : (1u << pk) - 1u;
        hits[0] = static_cast<unsigned>(pos & ~(pos >> 1)) & len_mask;
        hits[1] = static_cast<unsigned>(neg & ~(neg >> 1)) & len_mask;
        hits[2] = static_cast<unsigned>(up & ~(up >> 1)) & peak_mask;
        hits[3] = static_cast<unsigned>(down & ~(down >> 1)) & peak_mask;
      }
      const unsigned long long mine = static_cast<unsigned long long>(__popc(hits[0])) |
                                      static_cast<unsigned long long>(__popc(hits[1])) << 16 |
                                      static_cast<unsigned long long>(__popc(hits[2])) << 32 |
                                      static_cast<unsigned long long>(__popc(hits[3])) << 48;
      unsigned long long total;
      const unsigned long long before = block_scan_packed(mine, scan_scratch, total);
      // Second pass over the hits only: a warp runs each kind's loop as many
      // times as its busiest lane has hits, so the division of every edge is
      // issued once per hit rather than once per sample any lane hits.
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        double* dst = ev[k] + count[k] + static_cast<int>((before >> (16 * k)) & 0xffff);
        for (unsigned m = hits[k]; m; m &= m - 1) {
          const int i = __ffs(m) - 1;
          const double f0 = X(i), f1 = X(i + 1);
          double s0, s1;
          if (k < 2) {
            s0 = k == 0 ? f0 : -f0;
            s1 = k == 0 ? f1 : -f1;
          } else {
            const double a0 = -f0, a1 = -f1, a2 = -X(i + 2);
            const double d0 = a0 - a1, d1 = a1 - a2;
            s0 = k == 2 ? d0 : -d0;
            s1 = k == 2 ? d1 : -d1;
          }
          *dst++ = fine_edge(o + q_lo + i + 1, s0, s1);
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) count[k] += static_cast<int>((total >> (16 * k)) & 0xffff);
    }
    __syncthreads();
    const int64_t f_begin = B.frame_off[c];
    band_contour_walk(B, ev, count, v.centre[b], raw + b * v.total_frames + f_begin,
                      static_cast<int>(B.frame_off[c + 1] - f_begin));
  }
}

// Host side --------------------------------------------------------------

size_t fft_bank_smem_bytes() { return sizeof(double2) * kFftPadded; }

int fft_bank_block_length() { return kRealN; }

int fft_bank_ctas_per_sm() {
  const size_t smem = fft_bank_smem_bytes();
  if (cudaFuncSetAttribute(band_bank_fft, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
          cudaSuccess ||
      cudaFuncSetAttribute(block_spectra, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
          cudaSuccess ||
      cudaFuncSetAttribute(filter_spectra, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
          cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, band_bank_fft, kFftThreads, smem) != cudaSuccess)
    blocks = 0;
  cudaGetLastError();
  return blocks;
}

cudaError_t launch_twiddles(double2* tw, cudaStream_t stream) {
  make_twiddles<<<kRealN / 256, 256, 0, stream>>>(tw);
  return cudaGetLastError();
}

cudaError_t launch_filter_spectra(const int* half, const int64_t* tap_off, const double* taps_rev, int bands,
                                  int max_half, const double2* tw, double* amps, cudaStream_t stream) {
  filter_spectra<<<bands, kFftThreads, fft_bank_smem_bytes(), stream>>>(half, tap_off, taps_rev, max_half, tw,
                                                                         amps);
  return cudaGetLastError();
}

cudaError_t launch_fft_bank(const BankView& v, const FftBankGeometry& g, const double* y, const double* edge_bins,
                            const double2* tw, const double* amps, double2* spectra, int* queue,
                            double* slots, int ctas, double* raw, cudaStream_t stream) {
  block_spectra<<<static_cast<unsigned>(g.total_blocks), kFftThreads, fft_bank_smem_bytes(), stream>>>(
      v.batch, g, y, tw, spectra);
  band_bank_fft<<<ctas, kFftThreads, fft_bank_smem_bytes(), stream>>>(v, g, spectra, amps, tw, edge_bins,
                                                                      queue, slots, raw);
  return cudaGetLastError();
}

}  // namespace hv
