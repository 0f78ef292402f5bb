// a10-a13: channel aggregation, candidate overlap, instantaneous-frequency
// refinement, pruning and the best candidate per frame.
#include "hv_stages.cuh"

namespace hv {

// a10: DetectOfficialF0Candidates(Sub1/Sub2) (harvest.cpp:348-412). One
// thread per frame walks the bands: runs of at least 10 voiced channels
// (first and last channel forced unvoiced) become one candidate, their mean
// summed in channel order. `cand` is [frame][per_group]; per-clip maxima go
// to count[] (zeroed by the caller).
__global__ void official_candidates(BatchView v, const double* __restrict__ raw,
                                    int64_t total_frames, double* __restrict__ cand,
                                    int* __restrict__ count) {
  int64_t gf = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gf >= total_frames) return;
  double* row = cand + gf * v.per_group;
  int found = 0, start = 0, prev = 0;
  for (int b = 1; b < v.bands; ++b) {
    int now = (b == v.bands - 1) ? 0 : (raw[b * total_frames + gf] > 0 ? 1 : 0);
    if (now - prev == 1) start = b;
    if (now - prev == -1 && b - start >= 10) {
      double sum = 0.0;
      for (int j = start; j < b; ++j) sum += raw[j * total_frames + gf];
      sum /= (b - start);
      if (found < v.per_group) row[found] = sum;
      ++found;
    }
    prev = now;
  }
  for (int j = found; j < v.per_group; ++j) row[j] = 0.0;
  // At most (bands - 1) / 11 runs fit, fewer than per_group; the clamp only
  // keeps later column arithmetic in bounds.
  if (found) atomicMax(count + owner(v.frame_off, v.clips, gf), imin(found, v.per_group));
}

// a12: GetRefinedF0 / GetMeanF0 / FixF0 (harvest.cpp:434-617) for one
// candidate. The reference windows the waveform (Blackman window and its
// centred difference), takes two zero-padded FFTs of size n and reads at
// most six harmonic bins. Only those bins are needed, so they are evaluated
// directly as DFT sums; window and twiddle phasors advance by rotation and
// are re-anchored exactly every 32 samples.
__device__ void refine_candidate(const double* __restrict__ y, int y_len, double fs, double t,
                                 double f0c, double f0_floor, double f0_ceil, double& out_f0,
                                 double& out_score) {
  if (f0c <= 0.0) { out_f0 = 0.0; out_score = 0.0; return; }
  const int half = static_cast<int>(1.5 * fs / f0c + 1.0);
  const int len = 2 * half + 1;
  const double span = (2.0 * half + 1.0) / fs;
  const int n = 1 << (2 + (31 - __clz(len)));      // 2^(2 + floor(log2 len))
  const int base = matlab_round((t + (-half) / fs) * fs + 0.001);
  const int harmonics = imin(static_cast<int>(fs / 2.0 / f0c), 6);
  int bin[6];
  double mr[6], mi[6], dr[6], di[6], tr[6], ti[6], sr[6], si[6];
#pragma unroll
  for (int h = 0; h < 6; ++h) {
    bin[h] = h < harmonics ? matlab_round(f0c * n / fs * (h + 1)) : 0;
    mr[h] = mi[h] = dr[h] = di[h] = 0.0;
    double s, c;
    sincospi(-2.0 * bin[h] / n, &s, &c);
    sr[h] = c; si[h] = s;
  }
  // Window phase advances by 2 pi / len per sample (span * fs == len).
  double ds, dc;
  sincospi(2.0 / len, &ds, &dc);
  auto window_at = [&](int i, double& c1, double& s1) {
    double tmp = (base + i - 1.0) / fs - t;
    sincos(2.0 * kPi * tmp / span, &s1, &c1);
  };
  double c1, s1;
  window_at(0, c1, s1);
  double w_prev = 0.0;
  double w_cur = 0.42 + 0.5 * c1 + 0.08 * (2.0 * c1 * c1 - 1.0);
  for (int i0 = 0; i0 < len; i0 += 32) {
    // Exact anchors for the twiddles at i0 and the window at i0 + 1.
#pragma unroll
    for (int h = 0; h < 6; ++h) {
      long long m = (static_cast<long long>(bin[h]) * i0) % n;
      double s, c;
      sincospi(-2.0 * static_cast<double>(m) / n, &s, &c);
      tr[h] = c; ti[h] = s;
    }
    double nc, ns;
    window_at(i0 + 1, nc, ns);
    const int i1 = imin(i0 + 32, len);
    for (int i = i0; i < i1; ++i) {
      double w_next = 0.0;
      if (i + 1 < len) w_next = 0.42 + 0.5 * nc + 0.08 * (2.0 * nc * nc - 1.0);
      double dw = -(w_next - w_prev) / 2.0;
      int idx = imax(0, imin(y_len - 1, base + i - 1));
      double xs = y[idx];
      double a = xs * w_cur, d = xs * dw;
#pragma unroll
      for (int h = 0; h < 6; ++h) {
        mr[h] = fma(a, tr[h], mr[h]); mi[h] = fma(a, ti[h], mi[h]);
        dr[h] = fma(d, tr[h], dr[h]); di[h] = fma(d, ti[h], di[h]);
        double r = tr[h] * sr[h] - ti[h] * si[h];
        ti[h] = fma(tr[h], si[h], ti[h] * sr[h]);
        tr[h] = r;
      }
      double rc = nc * dc - ns * ds;
      ns = fma(nc, ds, ns * dc);
      nc = rc;
      w_prev = w_cur;
      w_cur = w_next;
    }
  }
  // FixF0 (harvest.cpp:507-536).
  double num = 0.0, den = 0.0, err = 0.0;
#pragma unroll
  for (int h = 0; h < 6; ++h) {
    if (h >= harmonics) break;
    double power = mr[h] * mr[h] + mi[h] * mi[h];
    double cross = mr[h] * di[h] - mi[h] * dr[h];
    double inst = power == 0.0 ? 0.0
                               : static_cast<double>(bin[h]) * fs / n + cross / power * fs / 2.0 / kPi;
    double amp = sqrt(power);
    num += amp * inst;
    den += amp * (h + 1.0);
    err += fabs((inst / (h + 1.0) - f0c) / f0c);
  }
  double refined = num / (den + kGuard);
  double score = 1.0 / (err / harmonics + kGuard);
  if (refined < f0_floor || refined > f0_ceil || score < 2.5) refined = score = 0.0;
  out_f0 = refined;
  out_score = score;
}

// a11 + a12: one thread per (frame, column). OverlapF0Candidates
// (harvest.cpp:417-429) is applied on the fly: column g*K + j of frame f
// holds candidate j of frame f (g = 0), f - g (g = 1..3) or f + g - 3
// (g = 4..6); columns past 7K are zero.
__global__ void refine_candidates(BatchView v, const double* __restrict__ y,
                                  const double* __restrict__ cand, const int* __restrict__ count,
                                  int64_t total_frames, double* __restrict__ refined,
                                  double* __restrict__ scores) {
  int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (cell >= total_frames * v.capacity) return;
  int64_t gf = cell / v.capacity;
  int col = static_cast<int>(cell - gf * v.capacity);
  int c = owner(v.frame_off, v.clips, gf);
  int64_t f0_row = v.frame_off[c];
  int frames = static_cast<int>(v.frame_off[c + 1] - f0_row);
  int f = static_cast<int>(gf - f0_row);
  int k = count[c];
  double f0c = 0.0;
  if (col < 7 * k) {
    int g = col / k, j = col - g * k;
    int src = g == 0 ? f : (g <= 3 ? f - g : f + (g - 3));
    if (src >= 0 && src < frames) f0c = cand[(f0_row + src) * v.per_group + j];
  }
  double out_f0 = 0.0, out_score = 0.0;
  if (f0c > 0.0) {
    int64_t y0 = v.y_off[c];
    int y_len = static_cast<int>(v.y_off[c + 1] - y0);
    refine_candidate(y + y0, y_len, v.fs_r, f * 1 / 1000.0, f0c, v.f0_floor, v.f0_ceil, out_f0,
                     out_score);
  }
  refined[cell] = out_f0;
  scores[cell] = out_score;
}

// a13: RemoveUnreliableCandidates(Sub) with SelectBestF0 (harvest.cpp:636-688)
// and SearchF0Base (harvest.cpp:693-705). One thread per (frame, column)
// writes the pruned pair; neighbours are read from the unpruned arrays.
__global__ void prune_candidates(BatchView v, const double* __restrict__ refined,
                                 const double* __restrict__ scores, const int* __restrict__ count,
                                 int64_t total_frames, double* __restrict__ pruned,
                                 double* __restrict__ pruned_scores) {
  int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (cell >= total_frames * v.capacity) return;
  int64_t gf = cell / v.capacity;
  int col = static_cast<int>(cell - gf * v.capacity);
  int c = owner(v.frame_off, v.clips, gf);
  int64_t f0_row = v.frame_off[c];
  int frames = static_cast<int>(v.frame_off[c + 1] - f0_row);
  int f = static_cast<int>(gf - f0_row);
  int columns = 7 * count[c];
  double ref = refined[cell], sc = scores[cell];
  if (col < columns && f >= 1 && f <= frames - 2 && ref != 0) {
    double e1 = 1.0, e2 = 1.0;
    const double* next = refined + (gf + 1) * v.capacity;
    const double* prev = refined + (gf - 1) * v.capacity;
    for (int j = 0; j < columns; ++j) {
      double tmp = fabs(ref - next[j]) / ref;
      if (!(tmp > e1)) e1 = tmp;
    }
    for (int j = 0; j < columns; ++j) {
      double tmp = fabs(ref - prev[j]) / ref;
      if (!(tmp > e2)) e2 = tmp;
    }
    double e = e1 < e2 ? e1 : e2;
    if (!(e <= 0.05)) ref = sc = 0.0;
  }
  pruned[cell] = ref;
  pruned_scores[cell] = sc;
}

__global__ void best_candidates(BatchView v, const double* __restrict__ pruned,
                                const double* __restrict__ pruned_scores,
                                const int* __restrict__ count, int64_t total_frames,
                                double* __restrict__ best) {
  int64_t gf = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gf >= total_frames) return;
  int columns = 7 * count[owner(v.frame_off, v.clips, gf)];
  double top = 0.0, pick = 0.0;
  for (int j = 0; j < columns; ++j) {
    double s = pruned_scores[gf * v.capacity + j];
    if (s > top) { top = s; pick = pruned[gf * v.capacity + j]; }
  }
  best[gf] = pick;
}

cudaError_t launch_candidates(const BatchView& v, const double* raw, int64_t total_frames,
                              double* cand, int* count, cudaStream_t stream) {
  const int threads = 128;
  official_candidates<<<static_cast<unsigned>((total_frames + threads - 1) / threads), threads, 0,
                        stream>>>(v, raw, total_frames, cand, count);
  return cudaGetLastError();
}

cudaError_t launch_refine(const BatchView& v, const double* y, const double* cand,
                          const int* count, int64_t total_frames, double* refined,
                          double* scores, cudaStream_t stream) {
  const int threads = 128;
  int64_t cells = total_frames * v.capacity;
  refine_candidates<<<static_cast<unsigned>((cells + threads - 1) / threads), threads, 0, stream>>>(
      v, y, cand, count, total_frames, refined, scores);
  return cudaGetLastError();
}

cudaError_t launch_prune(const BatchView& v, const double* refined, const double* scores,
                         const int* count, int64_t total_frames, double* pruned,
                         double* pruned_scores, double* best, cudaStream_t stream) {
  const int threads = 128;
  int64_t cells = total_frames * v.capacity;
  prune_candidates<<<static_cast<unsigned>((cells + threads - 1) / threads), threads, 0, stream>>>(
      v, refined, scores, count, total_frames, pruned, pruned_scores);
  best_candidates<<<static_cast<unsigned>((total_frames + threads - 1) / threads), threads, 0,
                    stream>>>(v, pruned, pruned_scores, count, total_frames, best);
  return cudaGetLastError();
}

}  // namespace hv
