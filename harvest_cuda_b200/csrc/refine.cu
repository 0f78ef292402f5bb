// a11-a12: candidate overlap and instantaneous-frequency refinement.
//
// RefineF0Candidates (harvest.cpp:622-631) refines every nonzero candidate of
// every frame with a Blackman window of about 3 fs / f0 samples, so the work
// per candidate varies by two orders of magnitude. The stage therefore runs
// as three steps:
//   1. bucket: every (frame, column) slot applies OverlapF0Candidates
//      (harvest.cpp:417-429) on the fly and counts its nonzero candidate in
//      a quarter-octave class of its window length;
//   2. scatter: the same walk writes (f0, frame, column) jobs into one list
//      ordered by class, longest windows first;
//   3. refine: one thread per job, so the 32 lanes of a warp run windows of
//      nearly the same length; outputs go to the job's own slot.
#include "hv_stages.cuh"

namespace hv {

// Window length class: four classes per octave.
__device__ __forceinline__ int size_class(int len) {
  int e = 31 - __clz(len);
  return e < 2 ? 4 * e : 4 * e + ((len >> (e - 2)) & 3);
}

// Candidate in column `col` of frame `gf` after overlap: column g*K + j of
// frame f holds candidate j of frame f (g = 0), f - g (g = 1..3) or
// f + g - 3 (g = 4..6); other columns are zero.
__device__ __forceinline__ double overlapped_candidate(const BatchView& v, const double* cand,
                                                       const int* count, int64_t gf, int col) {
  int c = owner(v.frame_off, v.clips, gf);
  int64_t row0 = v.frame_off[c];
  int frames = static_cast<int>(v.frame_off[c + 1] - row0);
  int f = static_cast<int>(gf - row0);
  int k = count[c];
  if (col >= 7 * k) return 0.0;
  int g = col / k, j = col - g * k;
  int src = g == 0 ? f : (g <= 3 ? f - g : f + (g - 3));
  if (src < 0 || src >= frames) return 0.0;
  return cand[(row0 + src) * v.per_group + j];
}

template <bool kScatter>
__global__ void __launch_bounds__(256)
refine_bucket(BatchView v, const double* __restrict__ cand, const int* __restrict__ count,
              int64_t total_frames, int* __restrict__ class_count, int* __restrict__ class_cursor,
              RefineJob* __restrict__ jobs) {
  __shared__ int s_count[kRefineClasses], s_base[kRefineClasses];
  for (int i = threadIdx.x; i < kRefineClasses; i += blockDim.x) s_count[i] = 0;
  __syncthreads();
  int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int cls = -1, rank = 0;
  double f0c = 0.0;
  int64_t gf = 0;
  int col = 0;
  if (cell < total_frames * v.capacity) {
    gf = cell / v.capacity;
    col = static_cast<int>(cell - gf * v.capacity);
    f0c = overlapped_candidate(v, cand, count, gf, col);
    if (f0c > 0.0) {
      int half = static_cast<int>(1.5 * v.fs_r / f0c + 1.0);
      cls = imin(size_class(2 * half + 1), kRefineClasses - 1);
      rank = atomicAdd(&s_count[cls], 1);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kRefineClasses; i += blockDim.x) {
    if (!s_count[i]) continue;
    if (kScatter) s_base[i] = atomicAdd(&class_cursor[i], s_count[i]);
    else atomicAdd(&class_count[i], s_count[i]);
  }
  if (!kScatter) return;
  __syncthreads();
  if (cls >= 0) {
    RefineJob job;
    job.f0c = f0c;
    job.key = gf * kRefineColumns + col;
    jobs[s_base[cls] + rank] = job;
  }
}

// Exclusive scan of the class counts, largest class first.
__global__ void refine_offsets(const int* __restrict__ class_count, int* __restrict__ class_cursor,
                               int* __restrict__ total) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int run = 0;
  for (int c = kRefineClasses - 1; c >= 0; --c) {
    class_cursor[c] = run;
    run += class_count[c];
  }
  *total = run;
}

// GetRefinedF0 / GetMeanF0 / GetBaseIndex / GetMainWindow / GetDiffWindow /
// GetSpectra / FixF0 (harvest.cpp:434-617) for one candidate. The reference
// windows the waveform with a Blackman window and its centred difference,
// takes two zero-padded FFTs of size n and reads at most six harmonic bins.
// Only those bins are needed, so they are evaluated directly as DFT sums.
// The window phasor advances by 2 pi / len per sample and each twiddle by
// 2 pi k / n; both are re-anchored from exact values every kAnchor samples.
constexpr int kAnchor = 64;

__device__ void refine_candidate(const double* __restrict__ y, int y_len, double fs, double t,
                                 double f0c, double f0_floor, double f0_ceil, double& out_f0,
                                 double& out_score) {
  const int half = static_cast<int>(1.5 * fs / f0c + 1.0);
  const int len = 2 * half + 1;
  const double span = (2.0 * half + 1.0) / fs;
  const int n = 1 << (2 + (31 - __clz(len)));        // 2^(2 + floor(log2 len)), len odd
  const int base = matlab_round((t + (-half) / fs) * fs + 0.001);
  const int harmonics = imin(static_cast<int>(fs / 2.0 / f0c), 6);
  int bin[6];
  double mr[6], mi[6], dr[6], di[6], tr[6], ti[6], sr[6], si[6];
#pragma unroll
  for (int h = 0; h < 6; ++h) {
    bin[h] = h < harmonics ? matlab_round(f0c * n / fs * (h + 1)) : 0;
    mr[h] = mi[h] = dr[h] = di[h] = 0.0;
    sincospi(-2.0 * bin[h] / n, &si[h], &sr[h]);
  }
  double ds, dc;
  sincospi(2.0 / len, &ds, &dc);
  // Window phase of sample i: 2 pi ((base + i - 1) / fs - t) / span, as in
  // GetMainWindow (harvest.cpp:449-455).
  auto phase = [&](int i, double& c1, double& s1) {
    double tmp = (base + i - 1.0) / fs - t;
    sincos(2.0 * kPi * tmp / span, &s1, &c1);
  };
  double nc, ns;
  phase(0, nc, ns);
  double w_prev = 0.0;
  double w_cur = 0.42 + 0.5 * nc + 0.08 * (2.0 * nc * nc - 1.0);
  const bool inside = base - 1 >= 0 && base - 1 + len <= y_len;
  const double* yb = y + (base - 1);
  for (int i0 = 0; i0 < len; i0 += kAnchor) {
#pragma unroll
    for (int h = 0; h < 6; ++h) {
      long long m = (static_cast<long long>(bin[h]) * i0) % n;
      sincospi(-2.0 * static_cast<double>(m) / n, &ti[h], &tr[h]);
    }
    phase(i0 + 1, nc, ns);
    const int i1 = imin(i0 + kAnchor, len);
    for (int i = i0; i < i1; ++i) {
      const double w_next = (i + 1 < len) ? 0.42 + 0.5 * nc + 0.08 * (2.0 * nc * nc - 1.0) : 0.0;
      const double dw = -(w_next - w_prev) / 2.0;
      const double xs = inside ? yb[i] : y[imax(0, imin(y_len - 1, base + i - 1))];
      const double a = xs * w_cur, d = xs * dw;
#pragma unroll
      for (int h = 0; h < 6; ++h) {
        mr[h] = fma(a, tr[h], mr[h]);
        mi[h] = fma(a, ti[h], mi[h]);
        dr[h] = fma(d, tr[h], dr[h]);
        di[h] = fma(d, ti[h], di[h]);
        const double r = fma(tr[h], sr[h], -ti[h] * si[h]);
        ti[h] = fma(tr[h], si[h], ti[h] * sr[h]);
        tr[h] = r;
      }
      const double rc = fma(nc, dc, -ns * ds);
      ns = fma(nc, ds, ns * dc);
      nc = rc;
      w_prev = w_cur;
      w_cur = w_next;
    }
  }
  // FixF0 (harvest.cpp:507-536), same evaluation order.
  double num = 0.0, den = 0.0, err = 0.0;
#pragma unroll
  for (int h = 0; h < 6; ++h) {
    if (h >= harmonics) break;
    const double power = mr[h] * mr[h] + mi[h] * mi[h];
    const double cross = mr[h] * di[h] - mi[h] * dr[h];
    const double inst =
        power == 0.0 ? 0.0 : static_cast<double>(bin[h]) * fs / n + cross / power * fs / 2.0 / kPi;
    const double amp = sqrt(power);
    num += amp * inst;
    den += amp * (h + 1.0);
    err += fabs((inst / (h + 1.0) - f0c) / f0c);
  }
  double refined = num / (den + kGuard);
  double score = 1.0 / (err / harmonics + kGuard);
  if (refined < f0_floor || refined > f0_ceil || score < 2.5) refined = score = 0.0;  // :610-614
  out_f0 = refined;
  out_score = score;
}

// One thread per job, grid-stride over the job list (longest windows first).
__global__ void __launch_bounds__(128)
refine_jobs(BatchView v, const double* __restrict__ y, const RefineJob* __restrict__ jobs,
            const int* __restrict__ total, double* __restrict__ refined, double* __restrict__ scores) {
  const int count = *total;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
    const RefineJob job = jobs[idx];
    const int64_t gf = job.key / kRefineColumns;
    const int col = static_cast<int>(job.key - gf * kRefineColumns);
    const int c = owner(v.frame_off, v.clips, gf);
    const int f = static_cast<int>(gf - v.frame_off[c]);
    const int64_t y0 = v.y_off[c];
    double f0 = 0.0, score = 0.0;
    refine_candidate(y + y0, static_cast<int>(v.y_off[c + 1] - y0), v.fs_r, f * 1 / 1000.0, job.f0c,
                     v.f0_floor, v.f0_ceil, f0, score);
    refined[gf * v.capacity + col] = f0;
    scores[gf * v.capacity + col] = score;
  }
}

cudaError_t launch_refine(const BatchView& v, const RefineBuffers& b, const double* y,
                          const double* cand, const int* count, int64_t total_frames, double* refined,
                          double* scores, int sms, cudaStream_t stream) {
  const int64_t cells = total_frames * v.capacity;
  cudaError_t e;
  if ((e = cudaMemsetAsync(b.class_count, 0, sizeof(int) * kRefineClasses, stream)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(refined, 0, sizeof(double) * cells, stream)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(scores, 0, sizeof(double) * cells, stream)) != cudaSuccess) return e;
  const unsigned grid = static_cast<unsigned>((cells + 255) / 256);
  refine_bucket<false><<<grid, 256, 0, stream>>>(v, cand, count, total_frames, b.class_count,
                                                 b.class_cursor, b.jobs);
  refine_offsets<<<1, 32, 0, stream>>>(b.class_count, b.class_cursor, b.total);
  refine_bucket<true><<<grid, 256, 0, stream>>>(v, cand, count, total_frames, b.class_count,
                                                b.class_cursor, b.jobs);
  refine_jobs<<<sms * 16, 128, 0, stream>>>(v, y, b.jobs, b.total, refined, scores);
  return cudaGetLastError();
}

}  // namespace hv
