// a5-a9: band-pass bank, four interval detectors and per-band candidates.
//
// One persistent kernel. Its work items are (clip, band) pairs, handed out
// longest first through an atomic counter. For one item a CTA walks the clip
// in tiles of kTile outputs:
//   * filters the tile with the band's Nuttall-windowed cosine
//     (GetFilteredSignal, harvest.cpp:99-148) as a direct FIR from shared
//     memory, adds WORLD's final-bin correction (see below) and keeps the
//     result in shared memory;
//   * flags the four event kinds (ZeroCrossingEngine and
//     GetFourZeroCrossingIntervals, harvest.cpp:162-238), computes their
//     sub-sample positions, and appends them in order to the CTA's private
//     event lists with a block-wide scan;
// and after the last tile interpolates the four interval tracks at every
// 1 ms frame (interp1 with histc clamping, matlabfunctions.cpp:136-176;
// GetF0CandidateContour(Sub), harvest.cpp:240-293) into raw[band][frame].
//
// Final-bin correction. WORLD multiplies spectra in place while mirroring
// each product into bin n-i-1, so bins n/2-1 and n/2 both end up holding
// H[n/2-1] Y[n/2-1] Y[n/2] (harvest.cpp:116-133). Relative to the plain
// convolution this adds, at output index q of the unnormalised inverse,
//   (-1)^q [c0 + 2 (Re c1 cos(2 pi q/n) + Im c1 sin(2 pi q/n))]
// with P = H[n/2-1] Y[n/2-1], Q = Y[n/2] P, c0 = Re Q - H[n/2] Y[n/2] and
// c1 = Q - P. The FIR computes the convolution divided by n (n is a power of
// two, so the scale is exact and zero crossings are unchanged); the
// correction is added divided by n as well.
#include "hv_events.cuh"

namespace hv {

constexpr int kFirR = 8;                    // outputs per thread
constexpr int kBankThreads = 128;
constexpr int kTile = kFirR * kBankThreads; // outputs per tile
constexpr int kStep = kTile - 2;            // event positions per tile


__device__ __forceinline__ int win_index(int j, int pitch) {
  return (j % kFirR) * pitch + j / kFirR;
}

// Exclusive block scan of four 16-bit counters packed in one 64-bit word.
__device__ __forceinline__ unsigned long long block_scan4(unsigned long long v,
                                                          unsigned long long* scratch,
                                                          unsigned long long& total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long n = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += n;
  }
  if (lane == 31) scratch[warp] = inc;
  __syncthreads();
  unsigned long long before = 0, all = 0;
  for (int w = 0; w < kBankThreads / 32; ++w) {
    if (w < warp) before += scratch[w];
    all += scratch[w];
  }
  __syncthreads();
  total = all;
  return before + inc - v;
}

__global__ void __launch_bounds__(kBankThreads)
band_bank_fir(BankView v, const double* __restrict__ y, const double* __restrict__ edge_bins,
              int* __restrict__ queue, double* __restrict__ slots, double* __restrict__ raw) {
  extern __shared__ double smem[];
  __shared__ unsigned long long scan_scratch[kBankThreads / 32];
  __shared__ int item_slot;
  __shared__ double red[3][kBankThreads / 32];
  const BatchView& B = v.batch;
  const int win_len = kTile + v.max_pad_taps + kFirR;
  const int pitch = (win_len + kFirR - 1) / kFirR + 1;
  double* s_taps = smem;
  double* s_win = s_taps + v.max_pad_taps;
  double* s_tile = s_win + pitch * kFirR;
  double* events = slots + blockIdx.x * (4 * v.slot_capacity);
  const int tid = threadIdx.x;

  for (;;) {
    if (tid == 0) item_slot = atomicAdd(queue, 1);
    __syncthreads();
    int item = item_slot;
    __syncthreads();
    if (item >= v.item_count) return;
    const int c = v.items[item].x, b = v.items[item].y;
    const int half = v.half[b];
    const int64_t y0 = B.y_off[c];
    const int y_len = static_cast<int>(B.y_off[c + 1] - y0);
    const int n = B.nfft[c];
    const int pad_taps = static_cast<int>(v.tap_off[b + 1] - v.tap_off[b]);
    const double* taps = v.taps_rev + v.tap_off[b];
    for (int i = tid; i < pad_taps; i += kBankThreads) s_taps[i] = taps[i];

    // Final-bin correction, divided by n like the FIR's convolution.
    double c0, c1r, c1i;
    final_bin_terms(taps, half, n, edge_bins + 3 * c, 1.0 / n, &red[0][0], c0, c1r, c1i);

    int count[4] = {0, 0, 0, 0};
    double* ev[4] = {events, events + v.slot_capacity, events + 2 * v.slot_capacity,
                     events + 3 * v.slot_capacity};
    const int last_edge_pos = y_len - 2;   // negative/positive crossings: i <= y_len-2
    const int last_peak_pos = y_len - 3;   // peak/dip crossings of the difference

    for (int s = 0; s <= last_edge_pos; s += kStep) {
      __syncthreads();
      // Window w[j] = y[s - half + 1 + j], zero outside the clip.
      const int64_t ws = static_cast<int64_t>(s) - half + 1;
      for (int j = tid; j < win_len; j += kBankThreads) {
        int64_t k = ws + j;
        s_win[win_index(j, pitch)] = (k >= 0 && k < y_len) ? y[y0 + k] : 0.0;
      }
      __syncthreads();
      double acc[kFirR], win[2 * kFirR];
#pragma unroll
      for (int q = 0; q < kFirR; ++q) { acc[q] = 0.0; win[q] = s_win[q * pitch + tid]; }
      for (int m0 = 0; m0 < pad_taps; m0 += kFirR) {
        const int base = tid + (m0 + kFirR) / kFirR;
#pragma unroll
        for (int u = 0; u < kFirR; ++u) win[kFirR + u] = s_win[u * pitch + base];
#pragma unroll
        for (int u = 0; u < kFirR; ++u) {
          const double hv = s_taps[m0 + u];
#pragma unroll
          for (int q = 0; q < kFirR; ++q) acc[q] = fma(hv, win[q + u], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < kFirR; ++q) win[q] = win[kFirR + q];
      }
#pragma unroll
      for (int q = 0; q < kFirR; ++q) {
        int o = tid * kFirR + q;
        int64_t qidx = static_cast<int64_t>(s) + o + half + 1;  // unnormalised output index
        double sn, cs;
        sincospi(2.0 * static_cast<double>(qidx % n) / n, &sn, &cs);
        double corr = c0 + 2.0 * (c1r * cs + c1i * sn);
        s_tile[o] = acc[q] + ((qidx & 1) ? -corr : corr);
      }
      __syncthreads();

      // Events at positions p = s + k, k in [0, kStep).
      double fine[4][kFirR];
      unsigned long long mine = 0;
      int local[4] = {0, 0, 0, 0};
#pragma unroll
      for (int q = 0; q < kFirR; ++q) {
        int k = tid * kFirR + q;
        int p = s + k;
        if (k >= kStep) break;
        double f0 = s_tile[k], f1 = s_tile[k + 1], f2 = s_tile[k + 2];
        if (p <= last_edge_pos) {
          if (0.0 < f0 && f1 <= 0.0) fine[0][local[0]++] = fine_edge(p + 1, f0, f1);
          double a0 = -f0, a1 = -f1;
          if (0.0 < a0 && a1 <= 0.0) fine[1][local[1]++] = fine_edge(p + 1, a0, a1);
          if (p <= last_peak_pos) {
            double a2 = -f2;
            double d0 = a0 - a1, d1 = a1 - a2;
            if (0.0 < d0 && d1 <= 0.0) fine[2][local[2]++] = fine_edge(p + 1, d0, d1);
            double e0 = -d0, e1 = -d1;
            if (0.0 < e0 && e1 <= 0.0) fine[3][local[3]++] = fine_edge(p + 1, e0, e1);
          }
        }
      }
      mine = static_cast<unsigned long long>(local[0]) |
             (static_cast<unsigned long long>(local[1]) << 16) |
             (static_cast<unsigned long long>(local[2]) << 32) |
             (static_cast<unsigned long long>(local[3]) << 48);
      unsigned long long total;
      unsigned long long before = block_scan4(mine, scan_scratch, total);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        int at = count[k] + static_cast<int>((before >> (16 * k)) & 0xffff);
#pragma unroll
        for (int q = 0; q < kFirR; ++q)
          if (q < local[k]) ev[k][at + q] = fine[k][q];
        count[k] += static_cast<int>((total >> (16 * k)) & 0xffff);
      }
    }
    __syncthreads();

    // Interpolate the four interval tracks at every 1 ms frame.
    const int64_t f_begin = B.frame_off[c];
    band_contour_walk(B, ev, count, v.centre[b], raw + b * v.total_frames + f_begin,
                      static_cast<int>(B.frame_off[c + 1] - f_begin));
  }
}

size_t band_bank_smem_bytes(int max_pad_taps) {
  int win_len = kTile + max_pad_taps + kFirR;
  int pitch = (win_len + kFirR - 1) / kFirR + 1;
  return sizeof(double) * (static_cast<size_t>(max_pad_taps) + static_cast<size_t>(pitch) * kFirR + kTile);
}

int band_bank_tap_multiple() { return kFirR; }
int band_bank_threads() { return kBankThreads; }

cudaError_t launch_band_bank(const BankView& v, const double* y, const double* edge_bins,
                             int* queue, double* slots, int ctas, double* raw,
                             cudaStream_t stream) {
  size_t smem = band_bank_smem_bytes(v.max_pad_taps);
  band_bank_fir<<<ctas, kBankThreads, smem, stream>>>(v, y, edge_bins, queue, slots, raw);
  return cudaGetLastError();
}

int band_bank_ctas_per_sm(int max_pad_taps) {
  // Allow the largest opt-in dynamic shared memory once, so every plan's
  // launch (and graph replay) fits whatever its tap count.
  int device = 0, optin = 0, blocks = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  cudaFuncAttributes attr{};
  if (cudaFuncGetAttributes(&attr, band_bank_fir) != cudaSuccess) return 0;
  const int dynamic_max = optin - static_cast<int>(attr.sharedSizeBytes);
  size_t smem = band_bank_smem_bytes(max_pad_taps);
  if (smem > static_cast<size_t>(dynamic_max)) return 0;
  if (cudaFuncSetAttribute(band_bank_fir, cudaFuncAttributeMaxDynamicSharedMemorySize, dynamic_max) !=
      cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, band_bank_fir, kBankThreads, smem) != cudaSuccess)
    blocks = 0;
  cudaGetLastError();  // leave no stale error for the next launch check
  return blocks;
}

}  // namespace hv
