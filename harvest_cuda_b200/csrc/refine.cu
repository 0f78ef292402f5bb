// a11-a12: candidate overlap and instantaneous-frequency refinement.
//
// RefineF0Candidates (harvest.cpp:622-631) refines every nonzero candidate of
// every frame with a Blackman window of about 3 fs / f0 samples, so the work
// per candidate varies by two orders of magnitude. The stage therefore runs
// as three steps:
//   1. bucket: one thread per (frame, official candidate) applies
//      OverlapF0Candidates (harvest.cpp:417-429) on the fly to that
//      candidate's seven overlap cells and counts each cell that needs its
//      own spectra in a quarter-octave class of its window length;
//   2. scatter: the same walk writes (f0, frame, column) jobs into one list
//      ordered by class, longest windows first;
//   3. refine: one thread per job, so the 32 lanes of a warp run windows of
//      nearly the same length; outputs go to the job's own cell.
#include "hv_stages.cuh"

namespace hv {

// Window length class: four classes per octave.
__device__ __forceinline__ int size_class(int len) {
  int e = 31 - __clz(len);
  return e < 2 ? 4 * e : 4 * e + ((len >> (e - 2)) & 3);
}

// GetRefinedF0 / GetMeanF0 / GetBaseIndex / GetMainWindow / GetDiffWindow /
// GetSpectra / FixF0 (harvest.cpp:434-617) for one candidate. The reference
// windows the waveform with a Blackman window and its centred difference,
// takes two zero-padded FFTs of size n and reads at most six harmonic bins.
// Only those bins are needed, so they are evaluated directly as DFT sums.
// The window phasor advances by 2 pi / len per sample and each twiddle by
// 2 pi k / n; both are re-anchored from exact values every kAnchor samples.
constexpr int kAnchor = 256;

// The discrete parameters of one candidate's refinement: window half length,
// FFT size, first waveform index and the harmonic bins.
struct CandidateWindow {
  int half, len, n, base, harmonics;
  int bin[6];
  __device__ __forceinline__ CandidateWindow(double fs, double t, double f0c) {
    half = static_cast<int>(1.5 * fs / f0c + 1.0);
    len = 2 * half + 1;
    n = 1 << (2 + (31 - __clz(len)));        // 2^(2 + floor(log2 len)), len odd
    base = matlab_round((t + (-half) / fs) * fs + 0.001);
    harmonics = imin(static_cast<int>(fs / 2.0 / f0c), 6);
#pragma unroll
    for (int h = 0; h < 6; ++h) bin[h] = h < harmonics ? matlab_round(f0c * n / fs * (h + 1)) : 0;
  }
};

// Slot (row * per_group + j) of candidate j of frame f after overlap group
// g (OverlapF0Candidates, harvest.cpp:417-429): from frame f (g = 0),
// f - g (g = 1..3) or f + g - 3 (g = 4..6); -1 outside the clip.
__device__ __forceinline__ int64_t sibling_slot(const BatchView& v, int64_t row0, int frames, int f, int g,
                                                int j) {
  const int src = g == 0 ? f : (g <= 3 ? f - g : f + (g - 3));
  return src < 0 || src >= frames ? -1 : (row0 + src) * v.per_group + j;
}

// Refinement key of a candidate F0: its window half length, harmonic count
// and bins, packed exactly. x = half << 32 | bin_0; y holds the harmonic
// count and, per harmonic h >= 1, bin_h - (h + 1) bin_0 (within +-3, since
// every bin rounds (h + 1) f0c n / fs) offset by 8 in 4 bits. Equal keys mean
// equal windows and bins, hence bit-identical spectra at one frame. A delta
// outside its field sets bit 63, and such keys are never taken as equal.
__device__ __forceinline__ ulonglong2 refine_key(double fs, double f0c) {
  const CandidateWindow cw(fs, 0.0, f0c);
  unsigned long long y = static_cast<unsigned long long>(cw.harmonics);
#pragma unroll
  for (int h = 1; h < 6; ++h) {
    const int delta = h < cw.harmonics ? cw.bin[h] - (h + 1) * cw.bin[0] : 0;
    if (delta < -8 || delta > 7) y |= 1ull << 63;
    y |= static_cast<unsigned long long>((delta + 8) & 15) << (4 * h);
  }
  return make_ulonglong2(static_cast<unsigned long long>(cw.half) << 32 | static_cast<unsigned int>(cw.bin[0]), y);
}

__device__ __forceinline__ bool same_key(ulonglong2 a, ulonglong2 b) {
  return a.x == b.x && a.y == b.y && !(a.y >> 63);
}

// item_off[c] = sum over clips c' < c of frames(c') * count[c']: the items of
// the bucket passes are the (frame, official candidate j < count) pairs,
// numbered clip by clip, frame-major. One block; blockDim.x <= 256.
__device__ void clip_item_offsets(const BatchView& v, const int* __restrict__ count,
                                  int64_t* __restrict__ item_off) {
  __shared__ long long part[256];
  const int nt = blockDim.x, t = threadIdx.x;
  const int per = (v.clips + nt - 1) / nt;
  const int c0 = imin(t * per, v.clips), c1 = imin(c0 + per, v.clips);
  long long sum = 0;
  for (int c = c0; c < c1; ++c) sum += (v.frame_off[c + 1] - v.frame_off[c]) * count[c];
  part[t] = sum;
  __syncthreads();
  for (int d = 1; d < nt; d <<= 1) {   // inclusive scan of the parts
    const long long x = t >= d ? part[t - d] : 0;
    __syncthreads();
    part[t] += x;
    __syncthreads();
  }
  long long run = part[t] - sum;
  for (int c = c0; c < c1; ++c) {
    item_off[c] = run;
    run += (v.frame_off[c + 1] - v.frame_off[c]) * count[c];
  }
  if (t == nt - 1) item_off[v.clips] = part[t];
}

// Refinement keys of every official candidate slot; block 0 also writes the
// bucket passes' item offsets.
__global__ void candidate_keys(BatchView v, const double* __restrict__ cand, const int* __restrict__ count,
                               int64_t slots, ulonglong2* __restrict__ keys, int64_t* __restrict__ item_off) {
  if (blockIdx.x == 0) clip_item_offsets(v, count, item_off);
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= slots) return;
  const double f0c = cand[i];
  // Keys are read only for nonzero candidates (the bucket pass's live cells).
  if (f0c > 0.0) keys[i] = refine_key(v.fs_r, f0c);
}

// One thread per (frame, official candidate j < count) item (numbered by
// item_off, so no lane waits on a column past its clip's count): the seven
// overlap cells of column j (groups g = 0..6) at this frame. A cell is a job when its
// candidate is nonzero and no lower group of the same j holds a candidate
// with the same key; the leader's job also serves those later siblings.
// Pass 1 (kScatter = false) finds the jobs, counts them per window-length
// class, records each cell's class + 1 (0: no job) in byte g of
// leaders[2 item] and each job's siblings (the later groups with the same
// key) as bits g2 of the 7-bit field g of leaders[2 item + 1], and zeroes the
// refined F0 and score of cells without a candidate (cells of siblings are
// written by their leader's job); pass 2 reads the records and writes the
// jobs at the class offsets, the sibling bits in the job key's bits 41-47.
// Columns from 7 count on are left as they are: nothing reads them.
template <bool kScatter>
__global__ void __launch_bounds__(256)
refine_bucket(BatchView v, const double* __restrict__ cand, const int* __restrict__ count,
              const ulonglong2* __restrict__ keys, const int64_t* __restrict__ item_off,
              unsigned long long* __restrict__ leaders,
              int* __restrict__ class_count, int* __restrict__ class_cursor, RefineJob* __restrict__ jobs,
              double* __restrict__ refined, double* __restrict__ scores) {
  __shared__ int s_count[kRefineClasses], s_base[kRefineClasses];
  for (int i = threadIdx.x; i < kRefineClasses; i += blockDim.x) s_count[i] = 0;
  __syncthreads();
  const int64_t item = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool valid = item < item_off[v.clips];
  // Clip, count, frame and column of the item (a clip with count 0 has no
  // items, so K >= 1 here).
  int c = 0, K = 1, f = 0, j = 0;
  if (valid) {
    c = owner(item_off, v.clips, item);
    K = count[c];
    const int64_t local = item - item_off[c];
    if (local < 0x7fffffff) {
      const int l = static_cast<int>(local);
      f = l / K;
      j = l - f * K;
    } else {
      f = static_cast<int>(local / K);
      j = static_cast<int>(local - static_cast<int64_t>(f) * K);
    }
  }
  const int64_t row0 = v.frame_off[c];
  const int frames = static_cast<int>(v.frame_off[c + 1] - row0);
  const int64_t gf = row0 + f;
  int cls[7], rank[7];
#pragma unroll
  for (int g = 0; g < 7; ++g) cls[g] = -1;
  if (valid) {
    if (!kScatter) {
      unsigned long long record = 0, sibling_record = 0;
      {
        ulonglong2 key[7];
        bool live[7];
#pragma unroll
        for (int g = 0; g < 7; ++g) {
          const int64_t slot = sibling_slot(v, row0, frames, f, g, j);
          live[g] = slot >= 0 && cand[slot] > 0.0;
          if (!live[g]) {
            refined[gf * v.capacity + g * K + j] = 0.0;
            scores[gf * v.capacity + g * K + j] = 0.0;
          }
          key[g] = live[g] ? keys[slot] : make_ulonglong2(0ull, 0ull);
          bool leader = live[g];
#pragma unroll
          for (int g2 = 0; g2 < g; ++g2)
            if (live[g2] && same_key(key[g], key[g2])) leader = false;
          if (leader) {
            const int half = static_cast<int>(key[g].x >> 32);
            cls[g] = imin(size_class(2 * half + 1), kRefineClasses - 1);
            rank[g] = atomicAdd(&s_count[cls[g]], 1);
            record |= static_cast<unsigned long long>(cls[g] + 1) << (8 * g);
          }
        }
#pragma unroll
        for (int g = 0; g < 7; ++g) {
          if (cls[g] < 0) continue;
          unsigned long long m = 0;
#pragma unroll
          for (int g2 = g + 1; g2 < 7; ++g2)
            if (live[g2] && same_key(key[g], key[g2])) m |= 1ull << g2;
          sibling_record |= m << (7 * g);
        }
      }
      leaders[2 * item] = record;
      leaders[2 * item + 1] = sibling_record;
    } else {
      const unsigned long long record = leaders[2 * item];
#pragma unroll
      for (int g = 0; g < 7; ++g) {
        const int b = static_cast<int>((record >> (8 * g)) & 0xff);
        if (b) {
          cls[g] = b - 1;
          rank[g] = atomicAdd(&s_count[cls[g]], 1);
        }
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kRefineClasses; i += blockDim.x) {
    if (!s_count[i]) continue;
    if (kScatter) s_base[i] = atomicAdd(&class_cursor[i], s_count[i]);
    else atomicAdd(&class_count[i], s_count[i]);
  }
  if (!kScatter || !valid) return;
  __syncthreads();
  bool any = false;
#pragma unroll
  for (int g = 0; g < 7; ++g) any |= cls[g] >= 0;
  if (!any) return;
  const unsigned long long sibling_record = leaders[2 * item + 1];
#pragma unroll
  for (int g = 0; g < 7; ++g) {
    if (cls[g] < 0) continue;
    RefineJob job;
    job.f0c = cand[sibling_slot(v, row0, frames, f, g, j)];
    job.key = static_cast<long long>(gf * kRefineColumns + g * K + j) |
              static_cast<long long>((sibling_record >> (7 * g)) & 0x7f) << kJobSiblingShift;
    jobs[s_base[cls[g]] + rank[g]] = job;
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

// Visits the window's samples in order: body(i, w, dw, tr, ti) receives the
// Blackman window w, the centred difference window dw and, per harmonic,
// the twiddle e^{-2 pi i bin i / n} as (tr, ti).
template <class Body>
__device__ __forceinline__ void walk_window(const CandidateWindow& cw, double fs, double t, Body&& body) {
  const int len = cw.len, n = cw.n;
  const double span = (2.0 * cw.half + 1.0) / fs;
  double tr[6], ti[6], sr[6], si[6];
#pragma unroll
  for (int h = 0; h < 6; ++h) sincospi(-2.0 * cw.bin[h] / n, &si[h], &sr[h]);
  double ds, dc;
  sincospi(2.0 / len, &ds, &dc);
  // Window phase of sample i: 2 pi ((base + i - 1) / fs - t) / span, as in
  // GetMainWindow (harvest.cpp:449-455).
  auto phase = [&](int i, double& c1, double& s1) {
    double tmp = (cw.base + i - 1.0) / fs - t;
    sincos(2.0 * kPi * tmp / span, &s1, &c1);
  };
  double nc, ns;
  phase(0, nc, ns);
  // The Blackman window as candidate_spectra forms it.
  auto blackman = [](double c) { return fma(fma(0.16, c, 0.5), c, 0.34); };
  double w_prev = 0.0;
  double w_cur = blackman(nc);
  for (int i0 = 0; i0 < len; i0 += kAnchor) {
#pragma unroll
    for (int h = 0; h < 6; ++h) {
      long long m = (static_cast<long long>(cw.bin[h]) * i0) & (n - 1);
      sincospi(-2.0 * static_cast<double>(m) / n, &ti[h], &tr[h]);
    }
    phase(i0 + 1, nc, ns);
    const int i1 = imin(i0 + kAnchor, len);
    for (int i = i0; i < i1; ++i) {
      const double w_next = (i + 1 < len) ? blackman(nc) : 0.0;
      const double dw = -(w_next - w_prev) / 2.0;
      body(i, w_cur, dw, tr, ti);
#pragma unroll
      for (int h = 0; h < 6; ++h) {
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
}

// Main- and difference-window spectra of one candidate at its harmonic bins
// (GetSpectra, harvest.cpp:461-505, at those bins only).
struct HarmonicSpectra {
  double mr[6], mi[6], dr[6], di[6];
};

// e^{-2 pi i m / n} for 0 <= m < n, n a power of two: from the workspace
// table tw[t] = e^{-2 pi i t / kTwiddleN} when n <= kTwiddleN (the argument
// 2 m / n is then exactly 2 t / kTwiddleN, so the entry is the value sincospi
// would give), else computed.
__device__ __forceinline__ double2 bin_twiddle(const double2* __restrict__ tw, long long m, int n) {
  if (n <= kTwiddleN) return __ldg(&tw[m * (kTwiddleN / n)]);
  double s, c;
  sincospi(2.0 * static_cast<double>(m) / n, &s, &c);
  return make_double2(c, -s);
}

// The bin sums are Goertzel recurrences, one for the windowed and one for
// the difference-windowed waveform per harmonic: with theta = 2 pi bin / n,
//   s_i = x_i + 2 cos(theta) s_{i-1} - s_{i-2},
//   X = e^{-i theta (N-1)} (s_{N-1} - e^{-i theta} s_{N-2}).
// Per harmonic and sample that is 2 operations per sequence, one multiply-add
// on the dependency chain. The rounding error grows as theta nears 0; at the
// longest windows of a 50 Hz floor at 8 kHz (483 samples, n = 1024) it stays
// below 2.5e-13 of sum |x| (against an extended-precision sum), far inside
// the F0 tolerance, and the refined F0 moves by less than that.
__device__ __forceinline__ void candidate_spectra(const double* __restrict__ y, int y_len, double fs,
                                                  double t, const CandidateWindow& cw,
                                                  const double2* __restrict__ tw, HarmonicSpectra& sp) {
  const int len = cw.len, n = cw.n;
  double c2[6], a1[6], a2[6], d1[6], d2[6];
#pragma unroll
  for (int h = 0; h < 6; ++h) {
    c2[h] = 2.0 * bin_twiddle(tw, cw.bin[h], n).x;
    a1[h] = a2[h] = d1[h] = d2[h] = 0.0;
  }
  const double span = (2.0 * cw.half + 1.0) / fs;
  double ds, dc;
  sincospi(2.0 / len, &ds, &dc);
  auto phase = [&](int i, double& c1, double& s1) {
    double tmp = (cw.base + i - 1.0) / fs - t;
    sincos(2.0 * kPi * tmp / span, &s1, &c1);
  };
  double nc, ns;
  phase(0, nc, ns);
  // Blackman window 0.42 + 0.5 cos + 0.08 cos 2 as 0.34 + 0.5 cos + 0.16 cos^2.
  auto blackman = [](double c) { return fma(fma(0.16, c, 0.5), c, 0.34); };
  double w_prev = 0.0;
  double w_cur = blackman(nc);
  const bool inside = cw.base - 1 >= 0 && cw.base - 1 + len <= y_len;
  const double* yb = y + (cw.base - 1);
  auto accumulate = [&](int i, double w, double dw) {
    const double xs = inside ? yb[i] : y[imax(0, imin(y_len - 1, cw.base + i - 1))];
    const double a = xs * w, d = xs * dw;
#pragma unroll
    for (int h = 0; h < 6; ++h) {
      const double na = fma(c2[h], a1[h], a - a2[h]);
      a2[h] = a1[h];
      a1[h] = na;
      const double nd = fma(c2[h], d1[h], d - d2[h]);
      d2[h] = d1[h];
      d1[h] = nd;
    }
  };
  // Samples 0 .. len - 2; the last one, whose next window value is 0, after.
  // Between anchors the window cosine follows the Chebyshev recurrence
  // cos((k + 1) d) = 2 cos d cos(k d) - cos((k - 1) d): one multiply-add per
  // sample instead of a four-operation rotation. Its rounding error grows
  // as k / sin d over the 256 samples between exact anchors: at most about
  // 2e-12 of the window, at the longest windows (483 samples, d = 2 pi /
  // 483), far below the F0 tolerance; the refined F0 moves by about 1e-13
  // relative (against anchors every 64 samples, on the 16 kHz batch).
  const double k2 = 2.0 * dc;
  for (int i0 = 0; i0 < len - 1; i0 += kAnchor) {
    phase(i0 + 1, nc, ns);
    double cp = fma(nc, dc, ns * ds);   // cos of the previous sample's phase
    const int i1 = imin(i0 + kAnchor, len - 1);
    // Four samples per iteration: their loads issue together (2, 3, 6 and
    // 8 were 1-14 % slower on the 16 kHz batch; 1 was 19 % slower).
#pragma unroll 4
    for (int i = i0; i < i1; ++i) {
      const double w_next = blackman(nc);
      accumulate(i, w_cur, w_prev - w_next);
      const double cn = fma(k2, nc, -cp);
      cp = nc;
      nc = cn;
      w_prev = w_cur;
      w_cur = w_next;
    }
  }
  accumulate(len - 1, w_cur, w_prev);
#pragma unroll
  for (int h = 0; h < 6; ++h) {
    const double2 step = bin_twiddle(tw, cw.bin[h], n);                        // e^{-i theta}
    const double2 rot = bin_twiddle(tw, (static_cast<long long>(cw.bin[h]) * (len - 1)) & (n - 1), n);
    const double ct = step.x, st = -step.y, cp = rot.x, sp_ = rot.y;
    // a sequence
    double s2 = a2[h];
    double re = a1[h] - ct * s2, im = st * s2;
    sp.mr[h] = re * cp - im * sp_;
    sp.mi[h] = re * sp_ + im * cp;
    // d sequence, accumulated with twice the difference window
    s2 = d2[h];
    re = d1[h] - ct * s2;
    im = st * s2;
    sp.dr[h] = 0.5 * (re * cp - im * sp_);
    sp.di[h] = 0.5 * (re * sp_ + im * cp);
  }
}

// FixF0 (harvest.cpp:507-536) split in two, each sum in the reference's
// order: the instantaneous frequencies and the refined F0 depend only on the
// spectra; the score also depends on the candidate's initial F0. The
// zeroing of RefineF0Candidates (harvest.cpp:610-614) follows the score.
__device__ __forceinline__ double fix_f0_frequencies(const HarmonicSpectra& sp, const CandidateWindow& cw,
                                                     double fs, double inst[6]) {
  double num = 0.0, den = 0.0;
  // Rolled: the per-job code stays small (instruction fetch limits the
  // refinement more than these few iterations do).
#pragma unroll 1
  for (int h = 0; h < 6; ++h) {
    inst[h] = 0.0;
    if (h >= cw.harmonics) continue;
    const double power = sp.mr[h] * sp.mr[h] + sp.mi[h] * sp.mi[h];
    const double cross = sp.mr[h] * sp.di[h] - sp.mi[h] * sp.dr[h];
    inst[h] = power == 0.0 ? 0.0 : static_cast<double>(cw.bin[h]) * fs / cw.n + cross / power * fs / 2.0 / kPi;
    const double amp = sqrt(power);
    num += amp * inst[h];
    den += amp * (h + 1.0);
  }
  return num / (den + kGuard);
}

__device__ __forceinline__ void fix_f0_score(const double inst[6], int harmonics, double refined, double f0c,
                                             double f0_floor, double f0_ceil, double& out_f0, double& out_score) {
  double err = 0.0;
#pragma unroll 1
  for (int h = 0; h < harmonics; ++h) err += fabs((inst[h] / (h + 1.0) - f0c) / f0c);
  double score = 1.0 / (err / harmonics + kGuard);
  if (refined < f0_floor || refined > f0_ceil || score < 2.5) refined = score = 0.0;
  out_f0 = refined;
  out_score = score;
}

// One thread per job, grid-stride over the job list (longest windows first).
// A job's spectra also serve the later overlap siblings (same candidate,
// group g2 > g) with the same window and bins, named by the job key's sibling
// bits: those cells get FixF0 with their own initial F0, which changes only
// the score. kMinBlocks caps registers so that that many 128-thread blocks
// fit on an SM; the autotuner picks the instance and the grid (RefineShape).
template <int kMinBlocks>
__global__ void __launch_bounds__(128, kMinBlocks)
refine_jobs(BatchView v, const double* __restrict__ y, const RefineJob* __restrict__ jobs,
            const int* __restrict__ total, const double* __restrict__ cand, const int* __restrict__ count,
            const double2* __restrict__ tw, double* __restrict__ refined, double* __restrict__ scores) {
  const int total_jobs = *total;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total_jobs; idx += gridDim.x * blockDim.x) {
    const RefineJob job = jobs[idx];
    const long long cell = job.key & ((1ll << kJobSiblingShift) - 1);
    const unsigned siblings = static_cast<unsigned>(job.key >> kJobSiblingShift);
    const int64_t gf = cell / kRefineColumns;
    const int col = static_cast<int>(cell - gf * kRefineColumns);
    const int c = owner(v.frame_off, v.clips, gf);
    const int64_t row0 = v.frame_off[c];
    const int f = static_cast<int>(gf - row0);
    const int64_t y0 = v.y_off[c];
    const double t = frame_seconds(f);
    const CandidateWindow cw(v.fs_r, t, job.f0c);
    HarmonicSpectra sp;
    candidate_spectra(y + y0, static_cast<int>(v.y_off[c + 1] - y0), v.fs_r, t, cw, tw, sp);
    double inst[6];
    const double value = fix_f0_frequencies(sp, cw, v.fs_r, inst);
    const int harmonics = cw.harmonics;
    double f0 = 0.0, score = 0.0;
    fix_f0_score(inst, harmonics, value, job.f0c, v.f0_floor, v.f0_ceil, f0, score);
    refined[gf * v.capacity + col] = f0;
    scores[gf * v.capacity + col] = score;
    const int frames = static_cast<int>(v.frame_off[c + 1] - row0);
    const int K = count[c], g = col / K, j = col - g * K;
    for (unsigned m = siblings; m; m &= m - 1) {
      const int g2 = __ffs(m) - 1;
      const double other = cand[sibling_slot(v, row0, frames, f, g2, j)];
      fix_f0_score(inst, harmonics, value, other, v.f0_floor, v.f0_ceil, f0, score);
      refined[gf * v.capacity + g2 * K + j] = f0;
      scores[gf * v.capacity + g2 * K + j] = score;
    }
  }
}

// Adjoint of the refinement for the F0 gradient, with every discrete choice
// held fixed. For each frame whose FixF0Contour step-3 value is a refined
// candidate, FixF0's result f = sum_h A_h IF_h / (sum_h (h + 1) A_h + guard),
// with A_h = |M_h| and IF_h = bin_h fs / n + (Mr Di - Mi Dr) / |M_h|^2 fs / 2 pi,
// is differentiated through the main and difference spectra M_h, D_h, which
// are linear in the waveform. The spectra are recomputed from y and the
// candidate F0 on the tape (nothing per frame is stored by the forward
// pass); the frame's share of dL/dy is added with atomics.
__global__ void __launch_bounds__(128)
refine_adjoint(BatchView v, const double* __restrict__ y, const double* __restrict__ tape,
               const double* __restrict__ grad_fixed, int64_t total_frames, const double2* __restrict__ tw,
               double* __restrict__ grad_y) {
  for (int64_t gf = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; gf < total_frames;
       gf += (int64_t)gridDim.x * blockDim.x) {
    const double g = grad_fixed[gf];
    const double f0c = tape[2 * gf + 1];
    // A tape from the forward pass holds candidates within [f0_floor, f0_ceil];
    // anything outside [1, fs_r] Hz is not one and is skipped.
    if (g == 0.0 || !(f0c >= 1.0 && f0c <= v.fs_r)) continue;
    const int c = owner(v.frame_off, v.clips, gf);
    const int f = static_cast<int>(gf - v.frame_off[c]);
    const int64_t y0 = v.y_off[c];
    const int y_len = static_cast<int>(v.y_off[c + 1] - y0);
    const double fs = v.fs_r, t = frame_seconds(f);
    const CandidateWindow cw(fs, t, f0c);
    HarmonicSpectra sp;
    candidate_spectra(y + y0, y_len, fs, t, cw, tw, sp);
    double num = 0.0, den = 0.0, amp[6], inst[6];
#pragma unroll
    for (int h = 0; h < 6; ++h) {
      amp[h] = inst[h] = 0.0;
      if (h >= cw.harmonics) continue;
      const double power = sp.mr[h] * sp.mr[h] + sp.mi[h] * sp.mi[h];
      const double cross = sp.mr[h] * sp.di[h] - sp.mi[h] * sp.dr[h];
      inst[h] = power == 0.0 ? 0.0 : static_cast<double>(cw.bin[h]) * fs / cw.n + cross / power * fs / 2.0 / kPi;
      amp[h] = sqrt(power);
      num += amp[h] * inst[h];
      den += amp[h] * (h + 1.0);
    }
    const double e = den + kGuard, refined = num / e, kappa = fs / 2.0 / kPi;
    // g * df/dMr_h, df/dMi_h, df/dDr_h, df/dDi_h.
    double cmr[6], cmi[6], cdr[6], cdi[6];
#pragma unroll
    for (int h = 0; h < 6; ++h) {
      cmr[h] = cmi[h] = cdr[h] = cdi[h] = 0.0;
      const double power = amp[h] * amp[h];
      if (h >= cw.harmonics || !(amp[h] > 0.0)) continue;
      const double cross = sp.mr[h] * sp.di[h] - sp.mi[h] * sp.dr[h];
      const double g_amp = (inst[h] - refined * (h + 1.0)) / e;
      const double g_inst = amp[h] / e;
      const double g_power = g_amp / (2.0 * amp[h]) - g_inst * kappa * cross / (power * power);
      const double g_cross = g_inst * kappa / power;
      cmr[h] = g * (2.0 * sp.mr[h] * g_power + sp.di[h] * g_cross);
      cmi[h] = g * (2.0 * sp.mi[h] * g_power - sp.dr[h] * g_cross);
      cdr[h] = -g * sp.mi[h] * g_cross;
      cdi[h] = g * sp.mr[h] * g_cross;
    }
    double* gy = grad_y + y0;
    walk_window(cw, fs, t, [&](int i, double w, double dw, const double* tr, const double* ti) {
      double sm = 0.0, sd = 0.0;
#pragma unroll
      for (int h = 0; h < 6; ++h) {
        sm += cmr[h] * tr[h] + cmi[h] * ti[h];
        sd += cdr[h] * tr[h] + cdi[h] * ti[h];
      }
      atomicAdd(gy + imax(0, imin(y_len - 1, cw.base + i - 1)), w * sm + dw * sd);
    });
  }
}

cudaError_t launch_refine(const BatchView& v, const RefineBuffers& b, const double* y,
                          const double* cand, const int* count, int64_t total_frames, double* refined,
                          double* scores, int sms, RefineShape shape, cudaStream_t stream) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(b.class_count, 0, sizeof(int) * kRefineClasses, stream)) != cudaSuccess) return e;
  const int64_t slots = total_frames * v.per_group;
  const unsigned grid = static_cast<unsigned>((slots + 255) / 256);
  candidate_keys<<<grid, 256, 0, stream>>>(v, cand, count, slots, b.keys, b.item_off);
  // Items number at most frames * per_group, the slots.
  refine_bucket<false><<<grid, 256, 0, stream>>>(v, cand, count, b.keys, b.item_off, b.leaders, b.class_count,
                                                 b.class_cursor, b.jobs, refined, scores);
  refine_offsets<<<1, 32, 0, stream>>>(b.class_count, b.class_cursor, b.total);
  refine_bucket<true><<<grid, 256, 0, stream>>>(v, cand, count, b.keys, b.item_off, b.leaders, b.class_count,
                                                b.class_cursor, b.jobs, refined, scores);
  const unsigned job_grid = static_cast<unsigned>(sms * shape.blocks_per_sm);
  auto kernel = shape.min_blocks == 4 ? refine_jobs<4> : (shape.min_blocks == 5 ? refine_jobs<5> : refine_jobs<1>);
  kernel<<<job_grid, 128, 0, stream>>>(v, y, b.jobs, b.total, cand, count, b.twiddles, refined, scores);
  return cudaGetLastError();
}

cudaError_t launch_refine_adjoint(const BatchView& v, const double* y, const double* tape,
                                  const double* grad_fixed, int64_t total_frames, const double2* tw,
                                  double* grad_y, int sms, cudaStream_t stream) {
  const int64_t blocks = (total_frames + 127) / 128;
  refine_adjoint<<<static_cast<unsigned>(blocks < sms * 8 ? blocks : sms * 8), 128, 0, stream>>>(
      v, y, tape, grad_fixed, total_frames, tw, grad_y);
  return cudaGetLastError();
}

}  // namespace hv
