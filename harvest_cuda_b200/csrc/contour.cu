// a14-a16: FixF0Contour, SmoothF0Contour and resampling to frame_period.
//
// These stages are sequential within a clip (each voiced section extends
// through candidate lists frame by frame and sections merge in order), so
// one thread owns one clip and clips run in parallel. The code follows the
// reference step by step with the same comparisons and evaluation order, so
// given the same candidates it reproduces WORLD bit for bit.
#include "hv_stages.cuh"

namespace hv {

constexpr int kExtend = 101;   // ExtendF0 reaches at most 101 frames (threshold 100 + 1)


// Doubles of scratch one clip of `frames` frames needs.
__host__ __device__ inline int64_t contour_scratch_doubles(int64_t frames) {
  int64_t sections = (frames + 1) / 8 + 2;
  // s1..s4, extension values, section records (8 ints), smoothing work,
  // boundary list (up to frames + 600 ints).
  return 4 * frames + 2 * kExtend * sections + 4 * sections + (frames + 600) + (frames + 602) + 64;
}

// GetBoundaryList (harvest.cpp:727-743) over f(0..len).
template <class F>
__device__ int boundary_list(F f, int len, int* out) {
  int count = 0, prev = 0;
  for (int i = 1; i < len; ++i) {
    int v = (i == len - 1) ? 0 : (f(i) > 0 ? 1 : 0);
    if (v != prev) { out[count] = i - count % 2; ++count; }
    prev = v;
  }
  return count;
}

// SelectBestF0 (harvest.cpp:636-650).
__device__ __forceinline__ double select_best(double ref, const double* cand, int count,
                                              double allowed) {
  double best = 0.0, err = allowed;
  for (int i = 0; i < count; ++i) {
    double e = fabs(ref - cand[i]) / ref;
    if (e > err) continue;
    best = cand[i];
    err = e;
  }
  return best;
}

// SearchScore (harvest.cpp:901-907).
__device__ __forceinline__ double search_score(double f0, const double* cand, const double* score,
                                               int count) {
  double s = 0.0;
  for (int i = 0; i < count; ++i)
    if (f0 == cand[i] && s < score[i]) s = score[i];
  return s;
}

// One step of the zero-lag Butterworth pass of FilteringF0
// (harvest.cpp:1058-1063).
struct Butter {
  double w0 = 0.0, w1 = 0.0;
  __device__ __forceinline__ double step(double x) {
    const double b0 = 0.0078202080334971724, b1 = 0.015640416066994345;
    const double a0 = 1.7347257688092754, a1 = -0.76600660094326412;
    double wt = x + a0 * w0 + a1 * w1;
    double out = b0 * wt + b1 * w0 + b0 * w1;
    w1 = w0;
    w0 = wt;
    return out;
  }
  // Runs `steps` steps on a constant input. Once a step leaves the state
  // unchanged, every later step repeats it, so the rest is skipped; the
  // result is identical to running all steps. Returns the last output.
  __device__ double run_constant(double x, int64_t steps) {
    double out = 0.0;
    for (int64_t k = 0; k < steps; ++k) {
      double p0 = w0, p1 = w1;
      out = step(x);
      if (w0 == p0 && w1 == p1) break;
    }
    return out;
  }
};

__global__ void contour_clips(ContourView v) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const BatchView& B = v.batch;
  if (c >= B.clips) return;
  const int64_t row0 = B.frame_off[c];
  const int F = static_cast<int>(B.frame_off[c + 1] - row0);
  const int columns = 7 * v.count[c];
  const int stride = B.capacity;
  const double* cand = v.pruned + row0 * stride;
  const double* score = v.pruned_scores + row0 * stride;
  const double* base = v.best + row0;

  // Scratch layout (doubles): s1 | s2 | s3 | s4 | ext | sec | smooth | bl
  double* sc = v.scratch + v.scratch_off[c];
  const int64_t sections_cap = (F + 1) / 8 + 2;
  double* s1 = sc;
  double* s2 = s1 + F;
  double* s3 = s2 + F;
  double* s4 = s3 + F;
  double* ext = s4 + F;                                  // [sections][2][kExtend]
  int* sec = reinterpret_cast<int*>(ext + 2 * kExtend * sections_cap);  // 8 ints per section
  double* work = reinterpret_cast<double*>(sec + 8 * sections_cap);      // F + 600
  int* bl = reinterpret_cast<int*>(work + F + 600);                     // F + 601 ints

  // FixStep1 (harvest.cpp:710-722), allowed range 0.008.
  for (int i = 0; i < F; ++i) s1[i] = 0.0;
  for (int i = 2; i < F; ++i) {
    if (base[i] == 0.0) continue;
    double ref = base[i - 1] * 2 - base[i - 2];
    s1[i] = fabs((base[i] - ref) / ref) > 0.008 &&
            fabs((base[i] - base[i - 1])) / base[i - 1] > 0.008 ? 0.0 : base[i];
  }
  // FixStep2 (harvest.cpp:748-762), minimum 6.
  for (int i = 0; i < F; ++i) s2[i] = s1[i];
  {
    int nb = boundary_list([&](int i) { return s1[i]; }, F, bl);
    for (int i = 0; i < nb / 2; ++i) {
      if (bl[2 * i + 1] - bl[2 * i] >= 6) continue;
      for (int j = bl[2 * i]; j <= bl[2 * i + 1]; ++j) s2[j] = 0.0;
    }
  }
  // FixStep3 (harvest.cpp:968-995) with Extend/ExtendF0/ExtendSub/
  // MakeSortedOrder/MergeF0/MergeF0Sub (harvest.cpp:791-963). Each
  // section keeps only its body (from s2) and the at most 101 values its
  // extension wrote on either side.
  for (int i = 0; i < F; ++i) s3[i] = s2[i];
  int nb = boundary_list([&](int i) { return s2[i]; }, F, bl);
  // Sections of FixStep2's output span at least 7 frames with gaps between
  // them, so (F + 1) / 8 + 2 records always suffice; the clamp is a guard.
  int sections = imin(nb / 2, static_cast<int>(sections_cap));
  // sec[8*i + ...]: 0 st, 1 ed (body), 2 st', 3 ed' (extended), 4 kept order
  for (int i = 0; i < sections; ++i) {
    int st = bl[2 * i], ed = bl[2 * i + 1];
    double* fwd = ext + (2 * i) * kExtend;
    double* bwd = fwd + kExtend;
    for (int k = 0; k < kExtend; ++k) fwd[k] = bwd[k] = 0.0;
    // Forward from the end.
    {
      int last = imin(F - 2, ed + 100);
      double cur = s2[ed];
      int reached = ed, misses = 0;
      for (int k = 0; k <= last - ed; ++k) {
        int idx = ed + k + 1;
        double val = select_best(cur, cand + static_cast<int64_t>(idx) * stride, columns, 0.18);
        fwd[k] = val;
        if (val == 0.0) ++misses; else { cur = val; misses = 0; reached = idx; }
        if (misses == 4) break;
      }
      sec[8 * i + 3] = reached;
    }
    // Backward from the start.
    {
      int last = imax(1, st - 100);
      double cur = s2[st];
      int reached = st, misses = 0;
      for (int k = 0; k <= st - last; ++k) {
        int idx = st - k - 1;
        double val = select_best(cur, cand + static_cast<int64_t>(idx) * stride, columns, 0.18);
        bwd[k] = val;
        if (val == 0.0) ++misses; else { cur = val; misses = 0; reached = idx; }
        if (misses == 4) break;
      }
      sec[8 * i + 2] = reached;
    }
    sec[8 * i + 0] = st;
    sec[8 * i + 1] = ed;
  }
  auto channel = [&](int i, int j) -> double {
    int st = sec[8 * i], ed = sec[8 * i + 1];
    if (j >= st && j <= ed) return s2[j];
    if (j > ed && j - ed - 1 < kExtend) return ext[(2 * i) * kExtend + (j - ed - 1)];
    if (j < st && st - 1 - j < kExtend) return ext[(2 * i + 1) * kExtend + (st - 1 - j)];
    return 0.0;
  };
  // ExtendSub (harvest.cpp:840-856): the running mean is never reset; the
  // kept sections keep their original order. Their extended bounds go to
  // bl[2k], bl[2k+1] and the section index to sec[8k + 4].
  int kept = 0;
  {
    double mean = 0.0;
    for (int i = 0; i < sections; ++i) {
      int st = sec[8 * i + 2], ed = sec[8 * i + 3];
      for (int j = st; j < ed; ++j) mean += channel(i, j);
      mean /= ed - st;
      if (2200.0 / mean < ed - st) {
        sec[8 * kept + 4] = i;
        ++kept;
      }
    }
    for (int k = 0; k < kept; ++k) {
      int i = sec[8 * k + 4];
      bl[2 * k] = sec[8 * i + 2];
      bl[2 * k + 1] = sec[8 * i + 3];
    }
  }
  if (kept != 0) {
    // MakeSortedOrder (harvest.cpp:883-896) as written, order in sec[8k + 5].
    for (int k = 0; k < kept; ++k) sec[8 * k + 5] = k;
    for (int i = 1; i < kept; ++i)
      for (int j = i - 1; j >= 0; --j) {
        int oi = sec[8 * i + 5], oj = sec[8 * j + 5];
        if (bl[oj * 2] > bl[oi * 2]) { sec[8 * i + 5] = oj; sec[8 * j + 5] = oi; }
        else break;
      }
    // MergeF0 (harvest.cpp:937-963); pair 0 of bl is the running extent.
    for (int j = 0; j < F; ++j) s3[j] = channel(sec[4], j);
    for (int i = 1; i < kept; ++i) {
      int o = sec[8 * i + 5];
      int ch = sec[8 * o + 4];
      int st2 = bl[2 * o], ed2 = bl[2 * o + 1];
      if (st2 - bl[1] > 0) {
        for (int j = st2; j <= ed2; ++j) s3[j] = channel(ch, j);
        bl[0] = st2;
        bl[1] = ed2;
      } else {
        int st1 = bl[0], ed1 = bl[1];
        if (st1 <= st2 && ed1 >= ed2) { bl[1] = ed1; continue; }
        double sc1 = 0.0, sc2 = 0.0;
        for (int j = st2; j <= ed1; ++j) {
          sc1 += search_score(s3[j], cand + static_cast<int64_t>(j) * stride,
                              score + static_cast<int64_t>(j) * stride, columns);
          sc2 += search_score(channel(ch, j), cand + static_cast<int64_t>(j) * stride,
                              score + static_cast<int64_t>(j) * stride, columns);
        }
        int from = sc1 > sc2 ? ed1 : st2;
        for (int j = from; j <= ed2; ++j) s3[j] = channel(ch, j);
        bl[1] = ed2;
      }
    }
  }
  // FixStep4 (harvest.cpp:1000-1022), threshold 9.
  for (int i = 0; i < F; ++i) s4[i] = s3[i];
  {
    int nb4 = boundary_list([&](int i) { return s3[i]; }, F, bl);
    for (int i = 0; i < nb4 / 2 - 1; ++i) {
      int distance = bl[2 * (i + 1)] - bl[2 * i + 1] - 1;
      if (distance >= 9) continue;
      double v0 = s3[bl[2 * i + 1]] + 1;
      double v1 = s3[bl[2 * (i + 1)]] - 1;
      double slope = (v1 - v0) / (distance + 1.0);
      int cnt = 1;
      for (int j = bl[2 * i + 1] + 1; j <= bl[2 * (i + 1)] - 1; ++j) s4[j] = v0 + slope * cnt++;
    }
  }
  // SmoothF0Contour (harvest.cpp:1079-1113): each voiced section of the
  // contour padded by 300 zero frames is filtered forward and backward over
  // the whole padded length with its end values held. The constant runs
  // are evaluated with Butter::run_constant, which is exact.
  double* sm = v.smoothed + row0;
  for (int i = 0; i < F; ++i) sm[i] = 0.0;
  {
    const int lag = 300;
    const int64_t len = F + 2 * lag;
    auto padded = [&](int j) -> double { return (j >= lag && j < lag + F) ? s4[j - lag] : 0.0; };
    int nbs = boundary_list(padded, static_cast<int>(len), bl);
    for (int s = 0; s < nbs / 2; ++s) {
      const int st = bl[2 * s], ed = bl[2 * s + 1];
      const double head = padded(st), tail = padded(ed);
      Butter fw;
      fw.run_constant(head, st);
      const int body = ed - st + 1;
      for (int j = st; j <= ed; ++j) work[j - st] = fw.step(padded(j));
      // Trailing run of the forward pass, stored until its state settles.
      const int64_t trailing = len - 1 - ed;
      int64_t stored = 0;
      double settled = 0.0;
      bool fixed = false;
      for (int64_t k = 0; k < trailing; ++k) {
        double p0 = fw.w0, p1 = fw.w1;
        double out = fw.step(tail);
        if (fw.w0 == p0 && fw.w1 == p1) { settled = out; fixed = true; break; }
        work[body + stored++] = out;
      }
      Butter bw;
      if (fixed) bw.run_constant(settled, trailing - stored);
      for (int64_t k = stored - 1; k >= 0; --k) bw.step(work[body + k]);
      for (int j = ed; j >= st; --j) sm[j - lag] = bw.step(work[j - st]);
    }
  }
  // Resampling (harvest.cpp:1246-1251); for frame_period 1 the same
  // expression reproduces the direct branch (harvest.cpp:1230-1235).
  const int64_t o0 = v.out_off[c];
  const int out_len = static_cast<int>(v.out_off[c + 1] - o0);
  for (int i = 0; i < out_len; ++i) {
    double t = i * v.period / 1000.0;
    v.t_out[o0 + i] = t;
    v.f0_out[o0 + i] = sm[imin(F - 1, matlab_round(t * 1000.0))];
  }
}

cudaError_t launch_contour(const ContourView& v, cudaStream_t stream) {
  const int threads = 32;
  contour_clips<<<(v.batch.clips + threads - 1) / threads, threads, 0, stream>>>(v);
  return cudaGetLastError();
}

int64_t contour_scratch(int64_t frames) { return contour_scratch_doubles(frames); }

}  // namespace hv
