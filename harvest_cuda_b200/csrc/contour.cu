// a14-a16: FixF0Contour, SmoothF0Contour and resampling to frame_period.
//
// Three kernels per batch (contour_prepare, contour_extend, contour_finish,
// below). The steps whose result depends on order run exactly as the
// reference writes them, on one warp of the clip's block: ExtendSub's
// carried mean, MakeSortedOrder, and MergeF0 with MergeF0Sub's score sums.
// Everything else runs across many threads: FixStep1, the boundary lists
// (warp ballots and a block scan), FixStep2's pruning, the two ExtendF0 runs
// of every voiced section (a warp per section, many blocks per clip),
// FixStep4's gap filling, the zero-lag smoothing of every voiced section and
// the resampling. Given the same candidates the kernels reproduce WORLD bit
// for bit, except for the smoothing of sections of 2048 frames or more.
#include <math_constants.h>

#include "hv_events.cuh"   // block_scan_packed (and hv_stages.cuh)

namespace hv {

constexpr int kExtend = 101;      // ExtendF0 writes at most 101 frames per side
constexpr int kTransient = 1024;  // per-lane buffer for a smoothing tail
// Free-response steps the smoothing adjoint follows past a section's ends:
// the filter's poles have radius 0.875, so the rest is below 0.875^512
// (1e-30) of the response's peak.
constexpr int kAdjointTail = 512;
constexpr unsigned kAll = 0xffffffffu;

constexpr int kContourThreads = 256;   // threads of a clip's block in contour_prepare / contour_finish
constexpr int kContourWarps = kContourThreads / 32;
constexpr int kZone = 100;             // body frames at each end whose SearchScore contour_extend records

// Doubles of scratch one clip of `frames` frames needs (contour_adjoint
// reuses the same space with a layout of its own).
// `threads`: the block size contour_finish runs with (per-thread smoothing
// tails, per-warp long buffers).
__host__ __device__ inline int64_t contour_scratch_doubles(int64_t frames, int threads) {
  const int64_t cap = (frames + 1) / 8 + 2;   // voiced sections: runs of >= 7 frames
  return 4 * frames + 4 * kExtend * cap + 2 * kZone * cap + 4 * cap + (frames + 602) +
         int64_t(threads) * kTransient + (threads / 32) * (frames + 600) + (frames + 602) / 2 +
         frames + 8 + 64;
}

// One clip's scratch as the three contour kernels use it.
struct ContourScratch {
  double *s1, *s2, *s3, *s4;   // FixStep1 .. FixStep4 contours (record_tape reads s3)
  double* ext;                 // [cap][2][kExtend] forward and backward extension values
  double* ext_sc;              // [cap][2][kExtend] their SearchScore values
  double* zone_sc;             // [cap][2][kZone] SearchScore of the first and last kZone body frames
  int* sec;                    // [cap][8] st, ed, extended st, extended ed, kept section, order,
                               //          frames examined backward, forward
  int* bl;                     // boundary lists, up to 2 (F + 602) ints
  double* tails;               // threads x kTransient smoothing tails
  double* shared_tail;         // warps x (F + 600)
  int* deferred;               // sections whose tail needs the long buffer
  double* ms;                  // [F] recorded SearchScore of merged frame j's value, NaN if none
  int* meta;                   // [0] sections, [1] kept sections
  int64_t cap;
  __device__ ContourScratch(double* sc, int F, int threads) {
    cap = (F + 1) / 8 + 2;
    s1 = sc;
    s2 = s1 + F;
    s3 = s2 + F;
    s4 = s3 + F;
    ext = s4 + F;
    ext_sc = ext + 2 * kExtend * cap;
    zone_sc = ext_sc + 2 * kExtend * cap;
    sec = reinterpret_cast<int*>(zone_sc + 2 * kZone * cap);
    bl = sec + 8 * cap;
    tails = reinterpret_cast<double*>(bl) + (F + 602);
    shared_tail = tails + static_cast<int64_t>(threads) * kTransient;
    deferred = reinterpret_cast<int*>(shared_tail + static_cast<int64_t>(threads / 32) * (F + 600));
    ms = reinterpret_cast<double*>(deferred + 2 * ((F + 602) / 2));
    meta = reinterpret_cast<int*>(ms + F);
  }
};

// One voiced section's extended row and the SearchScores contour_extend
// recorded for it, with its bounds held in registers.
struct SectionRow {
  int st, ed, examined_back, examined_fwd;
  const double *fwd, *bwd, *fwd_sc, *bwd_sc, *head_sc, *tail_sc;
  // The section's value at frame j: its body from the step-2 contour, the
  // extension values beside it, 0 elsewhere.
  __device__ __forceinline__ double value(const double* s2, int j) const {
    if (j >= st && j <= ed) return s2[j];
    if (j > ed && j - ed - 1 < kExtend) return fwd[j - ed - 1];
    if (j < st && st - 1 - j < kExtend) return bwd[st - 1 - j];
    return 0.0;
  }
  // The recorded SearchScore of value(j), or NaN if none was recorded.
  __device__ __forceinline__ double recorded(int j) const {
    if (j > ed) return j - ed - 1 < examined_fwd ? fwd_sc[j - ed - 1] : CUDART_NAN;
    if (j < st) return st - 1 - j < examined_back ? bwd_sc[st - 1 - j] : CUDART_NAN;
    if (j - st < kZone) return head_sc[j - st];
    if (ed - j < kZone) return tail_sc[kZone - 1 - (ed - j)];
    return CUDART_NAN;
  }
};
__device__ __forceinline__ SectionRow section_row(const ContourScratch& S, int i, int st, int ed, int examined_back,
                                                  int examined_fwd) {
  SectionRow r;
  r.st = st;
  r.ed = ed;
  r.examined_back = examined_back;
  r.examined_fwd = examined_fwd;
  r.fwd = S.ext + (2 * i) * kExtend;
  r.bwd = r.fwd + kExtend;
  r.fwd_sc = S.ext_sc + (2 * i) * kExtend;
  r.bwd_sc = r.fwd_sc + kExtend;
  r.head_sc = S.zone_sc + (2 * i) * kZone;
  r.tail_sc = r.head_sc + kZone;
  return r;
}
__device__ __forceinline__ SectionRow section_row(const ContourScratch& S, int i) {
  return section_row(S, i, S.sec[8 * i], S.sec[8 * i + 1], S.sec[8 * i + 6], S.sec[8 * i + 7]);
}

// GetBoundaryList (harvest.cpp:727-743) over f(0..len), by all 32 lanes:
// voicing changes are found 32 frames at a time with a ballot, and change
// number idx is stored as i - idx % 2. Four groups of 32 frames are loaded
// before their ballots are taken in order. Returns the count on every lane.
template <class F>
__device__ int warp_boundary_list(F f, int len, int* out) {
  constexpr int kGroups = 4;
  const int lane = threadIdx.x & 31;
  int count = 0;
  for (int base = 1; base < len; base += 32 * kGroups) {
    bool change[kGroups];
#pragma unroll
    for (int u = 0; u < kGroups; ++u) {
      const int i = base + 32 * u + lane;
      change[u] = false;
      if (i < len) {
        int now = (i == len - 1) ? 0 : (f(i) > 0 ? 1 : 0);
        int before = (i - 1 == 0) ? 0 : (f(i - 1) > 0 ? 1 : 0);
        change[u] = now != before;
      }
    }
#pragma unroll
    for (int u = 0; u < kGroups; ++u) {
      const int i = base + 32 * u + lane;
      const unsigned mask = __ballot_sync(kAll, change[u]);
      if (change[u]) {
        int idx = count + __popc(mask & ((1u << lane) - 1));
        out[idx] = i - idx % 2;
      }
      count += __popc(mask);
    }
  }
  __syncwarp();
  return count;
}

// GetBoundaryList by the whole block: each warp takes a contiguous part of
// 1 .. len - 1 and counts its voicing changes with ballots; a scan over the
// warps' counts places each warp's changes, which a second pass writes.
// Returns the count on every thread. `red` is shared scratch of one int per
// warp; the function starts and ends with a barrier.
template <class F>
__device__ int block_boundary_list(F f, int len, int* out, int* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int per = ((len - 1 + nw - 1) / nw + 31) / 32 * 32;
  const int i_begin = 1 + warp * per, i_end = imin(len, i_begin + per);
  auto change_at = [&](int i) -> bool {
    const int now = (i == len - 1) ? 0 : (f(i) > 0 ? 1 : 0);
    const int before = (i - 1 == 0) ? 0 : (f(i - 1) > 0 ? 1 : 0);
    return now != before;
  };
  __syncthreads();
  int count = 0;
  for (int b = i_begin; b < i_end; b += 32) {
    const int i = b + lane;
    count += __popc(__ballot_sync(kAll, i < i_end && change_at(i)));
  }
  if (lane == 0) red[warp] = count;
  __syncthreads();
  int idx0 = 0, all = 0;
  for (int w = 0; w < nw; ++w) {
    if (w < warp) idx0 += red[w];
    all += red[w];
  }
  for (int b = i_begin; b < i_end; b += 32) {
    const int i = b + lane;
    const bool ch = i < i_end && change_at(i);
    const unsigned mask = __ballot_sync(kAll, ch);
    if (ch) {
      const int idx = idx0 + __popc(mask & ((1u << lane) - 1));
      out[idx] = i - idx % 2;
    }
    idx0 += __popc(mask);
  }
  __syncthreads();
  return all;
}

// The sequential loops below load kChunk values ahead into registers and
// then consume them in the reference's order.
constexpr int kChunk = 8;

// Warp arg-min of SelectBestF0 over the lanes' picks (error best_e of
// column best_i holding val; best_i < 0: none): the smallest error, the
// later column on ties, whose value every lane returns (0 if no lane has a
// pick). Column i sits in lane i % 32. The errors map to unsigned keys in the
// same order (-0 as +0, which the comparison holds equal); the minimum key is
// found by its high and then its low word, the column by a maximum over the
// lanes holding that key: three dependent reductions and one shuffle, where
// five rounds of shuffles and FP64 compares would chain twice as long.
__device__ __forceinline__ double warp_pick(double best_e, int best_i, double val) {
  unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(best_e + 0.0));
  b = (b >> 63) ? ~b : (b | 0x8000000000000000ull);
  const unsigned long long key = best_i >= 0 ? b : ~0ull;
  const unsigned hi = static_cast<unsigned>(key >> 32), lo = static_cast<unsigned>(key);
  const unsigned min_hi = __reduce_min_sync(kAll, hi);
  const unsigned min_lo = __reduce_min_sync(kAll, hi == min_hi ? lo : ~0u);
  const bool at_min = best_i >= 0 && hi == min_hi && lo == min_lo;
  const unsigned top = __reduce_max_sync(kAll, at_min ? static_cast<unsigned>(best_i) + 1u : 0u);
  const double won = __shfl_sync(kAll, val, static_cast<int>((top - 1u) & 31u));
  return top ? won : 0.0;
}

// Warp maximum of SearchScore partial maxima, which are +0 or larger and
// never NaN (a lane takes a score only when it exceeds its current maximum):
// their bit patterns order as unsigned integers, so the maximum is found by
// its high and then its low word.
__device__ __forceinline__ double warp_max_score(double s) {
  const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(s));
  const unsigned hi = static_cast<unsigned>(b >> 32), lo = static_cast<unsigned>(b);
  const unsigned max_hi = __reduce_max_sync(kAll, hi);
  const unsigned max_lo = __reduce_max_sync(kAll, hi == max_hi ? lo : 0u);
  return __longlong_as_double(static_cast<long long>((static_cast<unsigned long long>(max_hi) << 32) | max_lo));
}

// SelectBestF0 (harvest.cpp:636-650) with the columns spread over the lanes
// of a warp. The
// reference's loop keeps a candidate whenever its error is at most the
// running minimum (which starts at `allowed`), so it returns the candidate
// of smallest error, the later column on ties, or 0 if none is within
// `allowed`; the warp arg-min below picks the same one. Every lane returns it.
__device__ __forceinline__ double warp_select_best(double ref, const double* cand, int count,
                                                   double allowed) {
  const int lane = threadIdx.x & 31;
  double best_e = allowed, best_v = 0.0;
  int best_i = -1;
  for (int i = lane; i < count; i += 32) {
    const double c = cand[i];
    const double e = fabs(ref - c) / ref;
    if (e <= best_e) { best_e = e; best_i = i; best_v = c; }
  }
  return warp_pick(best_e, best_i, best_v);
}

// A candidate row held in registers, column lane + 32 k in slot k, for
// rows of at most kRowSlots * 32 columns; loading the next frame's row
// before selecting in the current one hides its latency.
constexpr int kRowSlots = 8;
struct CandRow {
  double c[kRowSlots];
  __device__ __forceinline__ void load(const double* cand, int count) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < kRowSlots; ++k) c[k] = lane + 32 * k < count ? cand[lane + 32 * k] : 0.0;
  }
};

// warp_select_best on a row in registers: the same columns in the same order
// per lane and the same reduction, so the same candidate.
__device__ __forceinline__ double warp_select_best(double ref, const CandRow& row, int count, double allowed) {
  const int lane = threadIdx.x & 31;
  double best_e = allowed, best_v = 0.0;
  int best_i = -1;
#pragma unroll
  for (int k = 0; k < kRowSlots; ++k) {
    const int i = lane + 32 * k;
    if (i >= count) break;
    const double c = row.c[k];
    const double e = fabs(ref - c) / ref;
    if (e <= best_e) { best_e = e; best_i = i; best_v = c; }
  }
  return warp_pick(best_e, best_i, best_v);
}

// One direction of ExtendF0 (harvest.cpp:791-824) from frame `from` with
// value `cur`: frames from + dir, from + 2 dir, ... up to `steps` of them,
// each SelectBestF0 against the last accepted value, stopping after four
// misses in a row. Values go to out[k] (lane 0); returns the last frame
// that took a value.
__device__ __forceinline__ int extend_f0(const double* cand, int64_t stride, int columns, int from, int dir,
                                         int steps, double cur, double* out) {
  const int lane = threadIdx.x & 31;
  int reached = from, misses = 0;
  if (columns <= kRowSlots * 32) {
    CandRow row, next;
    if (steps > 0) row.load(cand + static_cast<int64_t>(from + dir) * stride, columns);
    for (int k = 0; k < steps; ++k) {
      const int idx = from + dir * (k + 1);
      if (k + 1 < steps) next.load(cand + static_cast<int64_t>(idx + dir) * stride, columns);
      const double val = warp_select_best(cur, row, columns, 0.18);
      if (lane == 0) out[k] = val;
      if (val == 0.0) ++misses; else { cur = val; misses = 0; reached = idx; }
      if (misses == 4) break;
      row = next;
    }
  } else {
    for (int k = 0; k < steps; ++k) {
      const int idx = from + dir * (k + 1);
      const double val = warp_select_best(cur, cand + static_cast<int64_t>(idx) * stride, columns, 0.18);
      if (lane == 0) out[k] = val;
      if (val == 0.0) ++misses; else { cur = val; misses = 0; reached = idx; }
      if (misses == 4) break;
    }
  }
  return reached;
}

// SearchScore (harvest.cpp:901-907).
__device__ __forceinline__ double search_score(double f0, const double* cand, const double* score,
                                               int count) {
  double s = 0.0;
  for (int i0 = 0; i0 < count; i0 += kChunk) {
    double c[kChunk], v[kChunk];
#pragma unroll
    for (int k = 0; k < kChunk; ++k) {
      c[k] = i0 + k < count ? cand[i0 + k] : 0.0;
      v[k] = i0 + k < count ? score[i0 + k] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < kChunk; ++k)
      if (i0 + k < count && f0 == c[k] && s < v[k]) s = v[k];
  }
  return s;
}

// One step of the Butterworth pass of FilteringF0 (harvest.cpp:1058-1063).
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
  // `steps` steps on a constant input. The state (w0, w1) then evolves by a
  // fixed map, so once it equals an earlier state it repeats with that
  // period, and the whole periods left are skipped: the result equals
  // running all steps. A state settles within a few hundred steps into a
  // fixed point or a rounding limit cycle (periods 4 and 8, rarely a few
  // dozen). Each state is compared with the previous one and with a
  // reference re-taken after 1, 2, 4, ..., 64 steps and then every 64 steps,
  // which finds every period up to 64.
  __device__ __forceinline__ void run_constant(double x, int64_t steps) {
    run_rounds([x](int) { return x; }, 1, steps);
  }

  // `steps` steps on the inputs pat[0], ..., pat[p - 1], pat[0], ... The
  // state after each round of p steps evolves by a fixed map; repeats of it
  // are skipped as in run_constant.
  __device__ __forceinline__ void run_periodic(const double* pat, int p, int64_t steps) {
    run_rounds([pat](int i) { return pat[i]; }, p, steps);
  }

  template <class In>
  __device__ __forceinline__ void run_rounds(In in, int p, int64_t steps) {
    const int64_t rounds = steps / p;
    double s0 = w0, s1 = w1;
    int since = 0, every = 1;
    for (int64_t r = 0; r < rounds; ++r) {
      const double p0 = w0, p1 = w1;
      for (int i = 0; i < p; ++i) step(in(i));
      ++since;
      int period = 0;
      if (w0 == p0 && w1 == p1) period = 1;
      else if (w0 == s0 && w1 == s1) period = since;
      if (period) {
        for (int64_t q = (rounds - r - 1) % period; q > 0; --q)
          for (int i = 0; i < p; ++i) step(in(i));
        break;
      }
      if (since == every) {
        s0 = w0;
        s1 = w1;
        since = 0;
        every = every < 64 ? 2 * every : 64;
      }
    }
    for (int64_t i = 0; i < steps % p; ++i) step(in(static_cast<int>(i)));
  }
};

// The held tail of a section: the forward filter `fw` runs `trailing` steps
// on tail_value, then the backward filter `bw` runs over those outputs in
// reverse. The forward state settles into a fixed point or a limit cycle of
// period <= 64 (see run_constant); from there its outputs repeat with that
// period, kept in the first 64 doubles of `tail`, and the backward pass over
// them runs as run_periodic. The outputs before that are recomputed stretch
// by stretch, newest first, from states checkpointed every `cap` / 2 steps
// in the second half of `tail`, into its first half; recomputation from a
// saved state repeats the same steps. So `bw` ends as if every output had
// been stored. Returns false if more than cap / 4 checkpoints are needed.
__device__ __noinline__ bool held_tail(Butter fw, double tail_value, int64_t trailing, double* tail,
                                       int64_t cap, Butter& bw) {
  constexpr int kAhead = 2 * kChunk;
  constexpr int kRing = 64;
  const int64_t stretch = cap / 2;
  double* saved = tail + stretch;   // (w0, w1) before steps 0, stretch, 2 stretch, ...
  double* ring = tail;              // output k at ring[k % kRing]
  double* rpat = tail + kRing;      // the periodic outputs in reverse order
  int64_t stored = trailing;        // outputs before the periodic part
  int period = 0;
  double s0 = fw.w0, s1 = fw.w1;
  int since = 0, every = 1;
  for (int64_t k = 0; k < trailing; ++k) {
    if (k % stretch == 0) {
      const int64_t c = k / stretch;
      if (2 * c + 1 >= stretch) return false;
      saved[2 * c] = fw.w0;
      saved[2 * c + 1] = fw.w1;
    }
    const double p0 = fw.w0, p1 = fw.w1;
    ring[k % kRing] = fw.step(tail_value);
    ++since;
    if (fw.w0 == p0 && fw.w1 == p1) period = 1;
    else if (fw.w0 == s0 && fw.w1 == s1) period = since;
    if (period) {
      // Outputs stored .. k are one period; every later output repeats them.
      stored = k + 1 - period;
      break;
    }
    if (since == every) {
      s0 = fw.w0;
      s1 = fw.w1;
      since = 0;
      every = every < 64 ? 2 * every : 64;
    }
  }
  if (period) {
    for (int i = 0; i < period; ++i) {
      const int64_t rel = (trailing - 1 - stored - i) % period;   // output trailing - 1 - i
      rpat[i] = ring[(stored + rel) % kRing];
    }
    bw.run_periodic(rpat, period, trailing - stored);
  }
  for (int64_t first = (stored > 0 ? (stored - 1) / stretch : -1) * stretch; first >= 0; first -= stretch) {
    const int64_t n = stored - first < stretch ? stored - first : stretch;
    Butter re;
    re.w0 = saved[2 * (first / stretch)];
    re.w1 = saved[2 * (first / stretch) + 1];
    for (int64_t k = 0; k < n; ++k) tail[k] = re.step(tail_value);
    for (int64_t k0 = n - 1; k0 >= 0; k0 -= kAhead) {
      double in[kAhead];
#pragma unroll
      for (int k = 0; k < kAhead; ++k) in[k] = k0 - k >= 0 ? tail[k0 - k] : 0.0;
#pragma unroll
      for (int k = 0; k < kAhead; ++k)
        if (k0 - k >= 0) bw.step(in[k]);
    }
  }
  return true;
}

// Smooths the voiced section [st, ed] of the padded contour (lag 300) as
// FilteringF0 does over the whole padded length: the held head, the body
// and the held tail forward, then everything backward. Body outputs go to
// out[j - lag]. The held head runs as run_constant and the held tail as
// held_tail (in `tail`, cap doubles), both equal to running every step.
// Returns false if the tail needs more than cap / 4 checkpoints.
template <class P>
__device__ bool smooth_section(P padded, int st, int ed, int64_t len, double* out, double* tail,
                               int64_t cap) {
  const int lag = 300;
  const double head = padded(st), tail_value = padded(ed);
  constexpr int kAhead = 2 * kChunk;
  Butter fw;
  fw.run_constant(head, st);
  for (int j0 = st; j0 <= ed; j0 += kAhead) {
    double in[kAhead];
#pragma unroll
    for (int k = 0; k < kAhead; ++k) in[k] = j0 + k <= ed ? padded(j0 + k) : 0.0;
#pragma unroll
    for (int k = 0; k < kAhead; ++k)
      if (j0 + k <= ed) out[j0 + k - lag] = fw.step(in[k]);
  }
  Butter bw;
  if (!held_tail(fw, tail_value, len - 1 - ed, tail, cap, bw)) return false;
  for (int j0 = ed; j0 >= st; j0 -= kAhead) {
    double in[kAhead];
#pragma unroll
    for (int k = 0; k < kAhead; ++k) in[k] = j0 - k >= st ? out[j0 - k - lag] : 0.0;
#pragma unroll
    for (int k = 0; k < kAhead; ++k)
      if (j0 - k >= st) out[j0 - k - lag] = bw.step(in[k]);
  }
  return true;
}

// Sections at least this long are smoothed by the whole warp.
constexpr int kLongSection = 2048;
// Steps a lane runs from a zero state before its chunk: the filter's poles
// have radius sqrt(0.766) = 0.875, so a state's influence falls below
// 0.875^512 (1e-30) of it.
constexpr int kWarm = 512;

// smooth_section for a long section [st, ed], by the whole warp. The held
// head and tail run as in smooth_section (every lane computes the head's
// constant-input steps; lane 0 runs the tail and its checkpointed backward
// pass in `tail`, cap doubles). The body, forward and then backward, is cut
// into 32 chunks, one per lane; a lane starts kWarm steps before its chunk
// from a zero state, or from the exact state where that reaches the end of
// the body. Its chunk's outputs then differ from a single pass's only by
// rounding (a few units in the last place).
template <class P>
__device__ void smooth_section_warp(P padded, int st, int ed, int64_t len, double* out, double* tail,
                                    int64_t cap) {
  const int lag = 300, lane = threadIdx.x & 31;
  const double head = padded(st), tail_value = padded(ed);
  const int n = ed - st + 1, chunk = (n + 31) / 32;
  const int c0 = imin(st + lane * chunk, ed + 1), c1 = imin(c0 + chunk, ed + 1);   // this lane's [c0, c1)
  constexpr int kAhead = 2 * kChunk;   // inputs loaded ahead into registers
  // Forward body.
  Butter fw;
  auto forward = [&](int from, int to, bool store) {   // steps from .. to - 1
    for (int j0 = from; j0 < to; j0 += kAhead) {
      double in[kAhead];
#pragma unroll
      for (int k = 0; k < kAhead; ++k) in[k] = j0 + k < to ? padded(j0 + k) : 0.0;
#pragma unroll
      for (int k = 0; k < kAhead; ++k) {
        if (j0 + k >= to) break;
        const double o = fw.step(in[k]);
        if (store) out[j0 + k - lag] = o;
      }
    }
  };
  int j = c0 - kWarm;
  if (j <= st) {
    fw.run_constant(head, st);
    j = st;
  }
  forward(j, c0, false);
  forward(c0, c1, true);
  __syncwarp();                        // forward outputs visible to every lane
  const int owner = (n - 1) / chunk;   // lane whose chunk ends at ed
  fw.w0 = __shfl_sync(kAll, fw.w0, owner);
  fw.w1 = __shfl_sync(kAll, fw.w1, owner);
  // Held tail, forward and backward, on lane 0 (as in smooth_section).
  Butter bw;
  // cap is the padded length, so the checkpoints always fit.
  if (lane == 0) held_tail(fw, tail_value, len - 1 - ed, tail, cap, bw);
  const double t0 = __shfl_sync(kAll, bw.w0, 0), t1 = __shfl_sync(kAll, bw.w1, 0);
  // Backward body: every lane first runs its warm-up over forward outputs of
  // later chunks, then (after all have) overwrites its own chunk.
  Butter b;
  auto backward = [&](int from, int to, bool store) {   // steps from down to to
    for (int j0 = from; j0 >= to; j0 -= kAhead) {
      double in[kAhead];
#pragma unroll
      for (int k = 0; k < kAhead; ++k) in[k] = j0 - k >= to ? out[j0 - k - lag] : 0.0;
#pragma unroll
      for (int k = 0; k < kAhead; ++k) {
        if (j0 - k < to) break;
        const double o = b.step(in[k]);
        if (store) out[j0 - k - lag] = o;
      }
    }
  };
  j = c1 - 1 + kWarm;
  if (j >= ed) {
    b.w0 = t0;
    b.w1 = t1;
    j = ed;
  }
  backward(j, c1, false);
  __syncwarp();
  backward(c1 - 1, c0, true);
  __syncwarp();
}

// The contour stage runs as three kernels per batch. Each keeps WORLD's
// order wherever a result depends on it; the work that does not is spread
// over many threads:
//   contour_prepare  (a block of 8 warps per clip): FixStep1, FixStep2 and
//                    the voiced sections of the step-2 contour;
//   contour_extend   (many blocks per clip, a warp per section): both
//                    ExtendF0 runs of every section, recording with every
//                    value it writes that value's SearchScore, and the
//                    SearchScore of the first and last kZone body frames;
//   contour_finish   (a block of 8 or 16 warps per clip): ExtendSub's
//                    carried mean, MergeF0 (in parallel when the sections
//                    come sorted; MergeF0Sub's score sums read the recorded
//                    SearchScores), FixStep4, SmoothF0Contour and the
//                    resampling.
__global__ void __launch_bounds__(kContourThreads) contour_prepare(ContourView v) {
  __shared__ int red[kContourWarps];
  const int c = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const BatchView& B = v.batch;
  const int64_t row0 = B.frame_off[c];
  const int F = static_cast<int>(B.frame_off[c + 1] - row0);
  const ContourScratch S(v.scratch + v.scratch_off[c], F, v.finish_threads);
  const double* base = v.best + row0;
  // FixStep1 (harvest.cpp:710-722), allowed range 0.008.
  for (int i = tid; i < F; i += nt) {
    double out = 0.0;
    const double b0 = base[i];
    if (i >= 2 && b0 != 0.0) {
      const double b1 = base[i - 1], b2 = base[i - 2];
      const double ref = b1 * 2 - b2;
      out = fabs((b0 - ref) / ref) > 0.008 && fabs((b0 - b1)) / b1 > 0.008 ? 0.0 : b0;
    }
    S.s1[i] = out;
    S.s2[i] = out;
  }
  __syncthreads();
  // FixStep2 (harvest.cpp:748-762): voiced runs shorter than 7 frames go.
  int nb = block_boundary_list([&](int i) { return S.s1[i]; }, F, S.bl, red);
  for (int i = tid; i < nb / 2; i += nt) {
    if (S.bl[2 * i + 1] - S.bl[2 * i] >= 6) continue;
    for (int j = S.bl[2 * i]; j <= S.bl[2 * i + 1]; ++j) S.s2[j] = 0.0;
  }
  __syncthreads();
  for (int i = tid; i < F; i += nt) S.s3[i] = S.s2[i];
  // The voiced sections of FixStep3 (harvest.cpp:968-975).
  nb = block_boundary_list([&](int i) { return S.s2[i]; }, F, S.bl, red);
  const int sections = imin(nb / 2, static_cast<int>(S.cap));
  for (int i = tid; i < sections; i += nt) {
    S.sec[8 * i + 0] = S.bl[2 * i];
    S.sec[8 * i + 1] = S.bl[2 * i + 1];
  }
  if (tid == 0) S.meta[0] = sections;
}

// SearchScore (harvest.cpp:901-907) of `value` in one frame's row, by the
// whole warp: each lane keeps the reference's running maximum over its
// columns (a NaN score never replaces it), and the lanes' maxima combine
// into the same value. Every lane returns it.
__device__ __forceinline__ double warp_search_score(double value, const double* cand, const double* score,
                                                    int columns) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int i = lane; i < columns; i += 32)
    if (value == cand[i] && s < score[i]) s = score[i];
  return warp_max_score(s);
}

// One direction of ExtendF0 as extend_f0, also recording the SearchScore of
// every value written (out_score[k]) from the same rows, and the number of
// frames examined. Rows of at most 32 NS columns are held in registers, D
// frames ahead (the rows do not depend on the chain of picks), so a step
// waits for no load. The pick and its score are the warp reductions of
// warp_select_best and warp_search_score. Returns the last frame that took
// a value.
template <int NS, int D>
__device__ int extend_f0_ahead(const double* cand, const double* score, int64_t stride, int columns, int from,
                               int dir, int steps, double cur, double* out, double* out_score, int& examined) {
  const int lane = threadIdx.x & 31;
  int reached = from, misses = 0;
  examined = 0;
  double rc[D][NS], rs[D][NS];
  auto load = [&](double (&c)[NS], double (&sc)[NS], int k) {   // the row of step k
    const bool live = k < steps;
    const int64_t row = live ? static_cast<int64_t>(from + dir * (k + 1)) * stride : 0;
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      const bool ok = live && lane + 32 * q < columns;
      c[q] = ok ? cand[row + lane + 32 * q] : 0.0;
      sc[q] = ok ? score[row + lane + 32 * q] : 0.0;
    }
  };
#pragma unroll
  for (int u = 0; u < D; ++u) load(rc[u], rs[u], u);
  bool done = false;
  for (int k0 = 0; k0 < steps && !done; k0 += D) {
#pragma unroll
    for (int u = 0; u < D; ++u) {
      const int k = k0 + u;
      if (k >= steps) {
        done = true;
        break;
      }
      // SelectBestF0 (harvest.cpp:636-650): smallest error within 0.18, the
      // later column on ties.
      double best_e = 0.18, val = 0.0;
      int best_i = -1;
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        const int i = lane + 32 * q;
        if (i >= columns) break;
        const double e = fabs(cur - rc[u][q]) / cur;
        if (e <= best_e) { best_e = e; best_i = i; val = rc[u][q]; }
      }
      val = warp_pick(best_e, best_i, val);
      // SearchScore (harvest.cpp:901-907) of the pick in the same row.
      double sc = 0.0;
#pragma unroll
      for (int q = 0; q < NS; ++q)
        if (lane + 32 * q < columns && val == rc[u][q] && sc < rs[u][q]) sc = rs[u][q];
      sc = warp_max_score(sc);
      load(rc[u], rs[u], k + D);
      if (lane == 0) {
        out[k] = val;
        out_score[k] = sc;
      }
      examined = k + 1;
      if (val == 0.0) ++misses; else { cur = val; misses = 0; reached = from + dir * (k + 1); }
      if (misses == 4) {
        done = true;
        break;
      }
    }
  }
  return reached;
}

// The same for rows wider than 256 columns, read from memory at each step.
__device__ int extend_f0_wide(const double* cand, const double* score, int64_t stride, int columns, int from,
                              int dir, int steps, double cur, double* out, double* out_score, int& examined) {
  const int lane = threadIdx.x & 31;
  int reached = from, misses = 0;
  examined = 0;
  for (int k = 0; k < steps; ++k) {
    const int idx = from + dir * (k + 1);
    const double* crow = cand + static_cast<int64_t>(idx) * stride;
    const double val = warp_select_best(cur, crow, columns, 0.18);
    const double s = warp_search_score(val, crow, score + static_cast<int64_t>(idx) * stride, columns);
    if (lane == 0) {
      out[k] = val;
      out_score[k] = s;
    }
    examined = k + 1;
    if (val == 0.0) ++misses; else { cur = val; misses = 0; reached = idx; }
    if (misses == 4) break;
  }
  return reached;
}

// SearchScore of the step-2 value of frames j_lo .. j_hi (out[j - j_lo]),
// by the warp, the rows of F frames loaded before any is reduced.
template <int NS, int FR>
__device__ void body_scores(const double* s2, const double* cand, const double* score, int64_t stride, int columns,
                            int j_lo, int j_hi, double* out) {
  const int lane = threadIdx.x & 31;
  for (int j0 = j_lo; j0 <= j_hi; j0 += FR) {
    double c[FR][NS], sc[FR][NS], v[FR];
#pragma unroll
    for (int f = 0; f < FR; ++f) {
      const int j = j0 + f;
      const bool live = j <= j_hi;
      v[f] = live ? s2[j] : 0.0;
      const int64_t row = live ? static_cast<int64_t>(j) * stride : 0;
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        const bool ok = live && lane + 32 * q < columns;
        c[f][q] = ok ? cand[row + lane + 32 * q] : 0.0;
        sc[f][q] = ok ? score[row + lane + 32 * q] : 0.0;
      }
    }
#pragma unroll
    for (int f = 0; f < FR; ++f) {
      double s = 0.0;
#pragma unroll
      for (int q = 0; q < NS; ++q)
        if (lane + 32 * q < columns && v[f] == c[f][q] && s < sc[f][q]) s = sc[f][q];
      s = warp_max_score(s);
      if (lane == 0 && j0 + f <= j_hi) out[j0 + f - j_lo] = s;
    }
  }
}

// Both ExtendF0 runs of section i and the SearchScores of its first and
// last kZone body frames, by one warp.
template <int NS, int D, int FR>
__device__ void extend_section(const ContourScratch& S, int i, int F, const double* cand, const double* score,
                               int stride, int columns) {
  const int lane = threadIdx.x & 31;
  const int st = S.sec[8 * i], ed = S.sec[8 * i + 1];
  double* fwd = S.ext + (2 * i) * kExtend;
  double* bwd = fwd + kExtend;
  double* fsc = S.ext_sc + (2 * i) * kExtend;
  double* bsc = fsc + kExtend;
  for (int k = lane; k < kExtend; k += 32) fwd[k] = bwd[k] = 0.0;
  __syncwarp();
  int ef = 0, eb = 0, rf, rb;
  // ExtendF0 forward from the end, then backward from the start (harvest.cpp:867-873).
  const int steps_f = imin(F - 2, ed + 100) - ed + 1, steps_b = st - imax(1, st - 100) + 1;
  if constexpr (NS > 0) {
    rf = extend_f0_ahead<NS, D>(cand, score, stride, columns, ed, 1, steps_f, S.s2[ed], fwd, fsc, ef);
    rb = extend_f0_ahead<NS, D>(cand, score, stride, columns, st, -1, steps_b, S.s2[st], bwd, bsc, eb);
    body_scores<NS, FR>(S.s2, cand, score, stride, columns, st, imin(ed, st + kZone - 1), S.zone_sc + (2 * i) * kZone);
    const int t_lo = imax(st, ed - kZone + 1);
    body_scores<NS, FR>(S.s2, cand, score, stride, columns, t_lo, ed,
                        S.zone_sc + (2 * i + 1) * kZone + (t_lo - (ed - kZone + 1)));
  } else {
    rf = extend_f0_wide(cand, score, stride, columns, ed, 1, steps_f, S.s2[ed], fwd, fsc, ef);
    rb = extend_f0_wide(cand, score, stride, columns, st, -1, steps_b, S.s2[st], bwd, bsc, eb);
    double* head = S.zone_sc + (2 * i) * kZone;
    double* tail = head + kZone;
    for (int j = st; j <= imin(ed, st + kZone - 1); ++j) {
      const double s = warp_search_score(S.s2[j], cand + static_cast<int64_t>(j) * stride,
                                         score + static_cast<int64_t>(j) * stride, columns);
      if (lane == 0) head[j - st] = s;
    }
    for (int j = imax(st, ed - kZone + 1); j <= ed; ++j) {
      const double s = warp_search_score(S.s2[j], cand + static_cast<int64_t>(j) * stride,
                                         score + static_cast<int64_t>(j) * stride, columns);
      if (lane == 0) tail[kZone - 1 - (ed - j)] = s;
    }
  }
  if (lane == 0) {
    S.sec[8 * i + 2] = rb;
    S.sec[8 * i + 3] = rf;
    S.sec[8 * i + 6] = eb;
    S.sec[8 * i + 7] = ef;
  }
}

__global__ void __launch_bounds__(kContourThreads, 2) contour_extend(ContourView v) {
  const int c = blockIdx.x;
  const int gw = blockIdx.y * kContourWarps + (threadIdx.x >> 5);
  const int nw = gridDim.y * kContourWarps;
  const BatchView& B = v.batch;
  const int64_t row0 = B.frame_off[c];
  const int F = static_cast<int>(B.frame_off[c + 1] - row0);
  const int columns = v.column_multiple * v.count[c];
  const int stride = B.capacity;
  const double* cand = v.pruned + row0 * stride;
  const double* score = v.pruned_scores + row0 * stride;
  const ContourScratch S(v.scratch + v.scratch_off[c], F, v.finish_threads);
  const int sections = S.meta[0];
  for (int i = gw; i < sections; i += nw) {
    if (columns <= 128) extend_section<4, 4, 4>(S, i, F, cand, score, stride, columns);
    else if (columns <= 256) extend_section<8, 2, 2>(S, i, F, cand, score, stride, columns);
    else extend_section<0, 1, 1>(S, i, F, cand, score, stride, columns);
  }
}

// MergeF0Sub's comparison (harvest.cpp:919-927), by all 32 lanes: whether
// the sum of fetch(j).a over j in [lo, hi] is larger than that of
// fetch(j).b, each added in frame order as the reference does; fetch returns
// 0, 0 for j > hi. Scores are nonnegative, so each ordered sum lies within
// (n - 1) u relative of the exact one, as does the warp's sum in any order:
// each lane adds its frames (up to 8 rounds of 32 fetched at once) and the
// lanes' sums are reduced by one tree. The decision is taken from those
// sums when they differ by more than both errors can explain; when the two
// sides hold the same score at every frame the reference's sums are equal
// (not larger); otherwise (or if a sum is not finite) the warp repeats the
// ordered sums exactly.
template <class Fetch>
__device__ bool merge_sum_larger(int lo, int hi, Fetch fetch) {
  constexpr int kRounds = 8;   // rounds of 32 frames loaded before any is added
  const int lane = threadIdx.x & 31;
  double t1 = 0.0, t2 = 0.0;   // this lane's partial sums, reduced once at the end
  bool mine = false;
  for (int c0 = lo; c0 <= hi; c0 += 32 * kRounds) {
    double a[kRounds], b[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; ++r) fetch(c0 + 32 * r + lane, a[r], b[r]);
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      mine |= a[r] != b[r];
      t1 += a[r];
      t2 += b[r];
    }
  }
  for (int o = 16; o; o >>= 1) {
    t1 += __shfl_xor_sync(kAll, t1, o);
    t2 += __shfl_xor_sync(kAll, t2, o);
  }
  if (!__any_sync(kAll, mine)) return false;
  const double n = hi - lo + 1;
  constexpr double u = 1.1102230246251565e-16;   // 2^-53
  if (fabs(t1 - t2) > 4.0 * (n + 2.0) * u * (t1 + t2) && t1 + t2 <= 1.0e300) return t1 > t2;
  // The reference's ordered sums: 32 frames a round from shuffles.
  double sc1 = 0.0, sc2 = 0.0, a, b;
  fetch(lo + lane, a, b);
  for (int j0 = lo; j0 <= hi; j0 += 32) {
    double na, nb;
    fetch(j0 + 32 + lane, na, nb);
    const int m = imin(32, hi - j0 + 1);
    for (int k = 0; k < m; ++k) {
      sc1 += __shfl_sync(kAll, a, k);
      sc2 += __shfl_sync(kAll, b, k);
    }
    a = na;
    b = nb;
  }
  return sc1 > sc2;
}

// MergeF0 (harvest.cpp:937-963) in parallel, for a sort order (sec[8i + 5],
// from MakeSortedOrder) that leaves the extended starts non-decreasing and
// keeps kept section 0 first: the reference reads
// position i's bounds from boundary pair order[i], which aliases the running
// extent (pair 0) only for section 0, and starts the merged contour from
// section 0. Position i stands for kept section order[i]. With
// position i's extended bounds st_i, ed_i, the running extent's end before
// merge i is ed1_i = max_{k<i} ed_k: a merge that changes it (a gap, st_i >
// ed1_i, or a MergeF0Sub that is not contained) sets it to ed_i > ed1_i, and
// a contained one (ed_i <= ed1_i; the running start never exceeds st_i)
// leaves it. So every merge's kind and sum range [st_i, ed1_i] are known up
// front. The merged contour over that range was last written by p_i, the
// first position reaching the maximum (no merge between p_i and i writes),
// from the start of p_i's copy on; before that by what p_i's own merge saw,
// p_(p_i) from its copy start on, and so on down to position 0, whose values
// cover every frame. A MergeF0Sub decision (copy from ed1_i if the merged
// side's score sum is larger, else from st_i) is thus a function of the copy
// starts along its p chain, and the copy starts solve a triangular system.
// The block
//   1. scans the maxima (warp 0);
//   2. runs up to kIterations parallel rounds: every MergeF0Sub is decided
//      by a warp from the current copy starts, and decided again only when
//      a copy start on its chain changed since it was last decided. A round
//      that changes no copy start means every decision used the final
//      starts of its chain, i.e. the sequential solution;
//   3. otherwise walks the merges in order on warp 0 and decides again
//      every decision whose chain changed since it was taken;
//   4. copies each merge's values over the frames no later merge writes:
//      [from_i, min(ed_i, min_{k>i} from_k - 1)] (later copies end later).
// The merged contour is S.s3, filled beforehand with position 0's values.
struct MergeScores {
  const double *cand, *score;
  int stride, columns;
};
__device__ __forceinline__ double section_score(const ContourScratch& S, const SectionRow& r, const MergeScores& q,
                                                int j) {
  const double rec = r.recorded(j);
  if (rec == rec) return rec;
  return search_score(r.value(S.s2, j), q.cand + static_cast<int64_t>(j) * q.stride,
                      q.score + static_cast<int64_t>(j) * q.stride, q.columns);
}

// The MergeF0Sub decision of position i (by all 32 lanes) from the copy
// starts in `from`: whether the merged side's sum over [st, e1] is larger.
// Unless `force`, it is only recomputed (`fresh`) if a copy start on the
// chain was changed at or after iteration `since` (stamp), i.e. possibly
// after the decision was last taken; otherwise it returns false. The chain's
// last writers are held as up to kChain segments; a longer chain resolves
// each frame's writer on its own.
__device__ __forceinline__ bool merge_decision(const ContourScratch& S, const MergeScores& q, const int* from,
                                               const int* prev, const int* stamp, const int* pch, int i, int st,
                                               int e1, bool force, int since, bool& fresh) {
  constexpr int kChain = 4;
  int seg_lo[kChain], seg_ch[kChain], n = 0, w = prev[i];
  fresh = force;
  for (;;) {
    const int fw = w == 0 ? INT_MIN : from[w];
    if (w != 0 && stamp[w] >= since) fresh = true;
    if (n < kChain) {
      seg_lo[n] = fw;
      seg_ch[n] = pch[w];
    }
    ++n;
    if (w == 0 || fw <= st) break;
    w = prev[w];
  }
  if (!fresh) return false;
  const SectionRow ri = section_row(S, pch[i]);
  return merge_sum_larger(st, e1, [&](int j, double& a, double& b) {
    a = b = 0.0;
    if (j > e1) return;
    int ch = -1;
    if (n <= kChain) {
      for (int g = 0; g < n; ++g)
        if (ch < 0 && j >= seg_lo[g]) ch = seg_ch[g];
    } else {
      int x = prev[i];
      while (x != 0 && j < from[x]) x = prev[x];
      ch = pch[x];
    }
    a = section_score(S, section_row(S, ch), q, j);
    b = section_score(S, ri, q, j);
  });
}

__device__ void merge_sorted(const ContourScratch& S, int kept, const MergeScores& q) {
  constexpr int kGap = 1, kContained = 2, kSub = 3;
  constexpr int kIterations = 4;         // parallel rounds before the ordered pass
  constexpr int kOrdered = 1 << 30;      // stamp of a change made by the ordered pass
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  const int* sec = S.sec;
  int* bl = S.bl;
  int* ed1 = reinterpret_cast<int*>(S.shared_tail);   // free until the smoothing
  int* prev = ed1 + kept;
  int* kind = prev + kept;
  int* from = kind + kept;
  int* stamp = from + kept;      // round of the last change of from[i]
  int* computed = stamp + kept;  // round in which decision i was last taken
  int* until = computed + kept;
  int* pst = until + kept;       // position i's extended bounds and section
  int* ped = pst + kept;
  int* pch = ped + kept;
  for (int i = threadIdx.x; i < kept; i += blockDim.x) {
    const int o = sec[8 * i + 5];
    pst[i] = bl[2 * o];
    ped[i] = bl[2 * o + 1];
    pch[i] = sec[8 * o + 4];
  }
  __syncthreads();
  // 1. Running maxima of the extended ends (first position on ties), the
  // merge kinds and the initial copy starts (each MergeF0Sub from st_i).
  if (warp == 0) {
    int cv = ped[0], ci = 0, last_gap = 0;
    for (int i0 = 1; i0 < kept; i0 += 32) {
      const int i = i0 + lane;
      const int e = i < kept ? ped[i] : INT_MIN;
      int v = e, x = i;
      for (int o = 1; o < 32; o <<= 1) {
        const int ov = __shfl_up_sync(kAll, v, o), ox = __shfl_up_sync(kAll, x, o);
        if (lane >= o && !(v > ov)) {
          v = ov;
          x = ox;
        }
      }
      int pv = __shfl_up_sync(kAll, v, 1), px = __shfl_up_sync(kAll, x, 1);
      if (lane == 0) pv = INT_MIN;
      const int mv = pv > cv ? pv : cv, mx = pv > cv ? px : ci;
      if (i < kept) {
        const int st = pst[i];
        const int kd = st > mv ? kGap : (e <= mv ? kContained : kSub);
        ed1[i] = mv;
        prev[i] = mx;
        kind[i] = kd;
        from[i] = kd == kContained ? -1 : st;
        stamp[i] = -1;
        computed[i] = -1;
        if (kd == kGap) last_gap = i;
      }
      const int lv = __shfl_sync(kAll, v, 31), lx = __shfl_sync(kAll, x, 31);
      if (lv > cv) {
        cv = lv;
        ci = lx;
      }
    }
    // The reference leaves the running extent in boundary pair 0.
    last_gap = __reduce_max_sync(kAll, last_gap);
    const int st1 = last_gap > 0 ? pst[last_gap] : pst[0];
    __syncwarp();
    if (lane == 0) {
      bl[0] = st1;
      bl[1] = cv;
    }
  }
  __syncthreads();
  // 2. Parallel rounds: each MergeF0Sub decided from the current copy
  // starts, and again whenever one on its chain changed since. Each warp
  // takes a contiguous run of positions and walks it in order, so a chain
  // inside the run sees the copy starts its warp has just set (p_i is
  // nearly always one or two positions back); only chains reaching into
  // another warp's run can need a later round.
  bool settled = false;
  const int per_warp = (kept - 1 + warps - 1) / warps;
  const int run_lo = 1 + warp * per_warp, run_hi = imin(kept, run_lo + per_warp);
  for (int t = 0; t < kIterations && !settled; ++t) {
    int mine = 0;   // this thread changed a copy start this round
    for (int i = run_lo; i < run_hi; ++i) {
      if (kind[i] != kSub) continue;
      const int st = pst[i], e1 = ed1[i];
      bool fresh;
      const bool larger = merge_decision(S, q, from, prev, stamp, pch, i, st, e1, t == 0, computed[i], fresh);
      if (!fresh) continue;
      const int fr = larger ? e1 : st;
      if (lane == 0) {
        computed[i] = t;
        if (fr != from[i]) {
          from[i] = fr;
          stamp[i] = t;
          mine = 1;
        }
      }
      __syncwarp();
    }
    // One barrier that also tells every thread whether any changed.
    settled = !__syncthreads_or(mine);
  }
  // 3. If the last round still changed something: the ordered pass, which
  // decides again every decision a change on its chain may have reached.
  if (!settled && warp == 0) {
    for (int i = 1; i < kept; ++i) {
      if (kind[i] != kSub) continue;
      const int st = pst[i], e1 = ed1[i];
      bool fresh;
      const bool larger = merge_decision(S, q, from, prev, stamp, pch, i, st, e1, false, computed[i], fresh);
      if (fresh) {
        const int fr = larger ? e1 : st;
        if (lane == 0 && fr != from[i]) {
          from[i] = fr;
          stamp[i] = kOrdered;
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  // 4a. Where each copy ends: before the earliest later copy start.
  if (warp == 0) {
    int carry = INT_MAX;
    for (int i1 = kept - 1; i1 >= 1; i1 -= 32) {
      const int i = i1 - lane;
      const int f = i >= 1 ? from[i] : -1;
      int v = f >= 0 ? f : INT_MAX;
      for (int o = 1; o < 32; o <<= 1) {
        const int ov = __shfl_up_sync(kAll, v, o);
        if (lane >= o) v = imin(v, ov);
      }
      int later = __shfl_up_sync(kAll, v, 1);
      if (lane == 0) later = INT_MAX;
      later = imin(later, carry);
      if (i >= 1 && f >= 0) until[i] = imin(ped[i], later == INT_MAX ? INT_MAX : later - 1);
      carry = imin(carry, __shfl_sync(kAll, v, 31));
    }
  }
  __syncthreads();
  // 4b. The copies, a warp per merge.
  for (int i = 1 + warp; i < kept; i += warps) {
    const int fr = from[i];
    if (fr < 0) continue;
    const int to = until[i];
    const SectionRow r = section_row(S, pch[i]);
    for (int j = fr + lane; j <= to; j += 32) S.s3[j] = r.value(S.s2, j);
  }
  __syncthreads();
}

// kThreads: 256, or 512 when the batch has fewer clips than the GPU has SMs
// (one block per clip, so the larger block only adds warps to the
// block-parallel parts: ExtendSub's sums, MergeF0's decisions, smoothing).
template <int kThreads>
__global__ void __launch_bounds__(kThreads) contour_finish(ContourView v) {
  constexpr int kWarps = kThreads / 32;
  __shared__ int red[kWarps];
  __shared__ int deferred_count;
  const int c = blockIdx.x;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const BatchView& B = v.batch;
  const int64_t row0 = B.frame_off[c];
  const int F = static_cast<int>(B.frame_off[c + 1] - row0);
  const int columns = v.column_multiple * v.count[c];
  const int stride = B.capacity;
  const double* cand = v.pruned + row0 * stride;
  const double* score = v.pruned_scores + row0 * stride;
  const ContourScratch S(v.scratch + v.scratch_off[c], F, v.finish_threads);
  const int sections = S.meta[0];
  int* sec = S.sec;
  int* bl = S.bl;
  // A section's extended row: its body from s2 plus the extension values.
  auto channel = [&](int i, int j) -> double {
    const int st = sec[8 * i], ed = sec[8 * i + 1];
    if (j >= st && j <= ed) return S.s2[j];
    if (j > ed && j - ed - 1 < kExtend) return S.ext[(2 * i) * kExtend + (j - ed - 1)];
    if (j < st && st - 1 - j < kExtend) return S.ext[(2 * i + 1) * kExtend + (st - 1 - j)];
    return 0.0;
  };
  // ExtendSub (harvest.cpp:840-856): section i is kept when 2200 / mean_i
  // < n_i, where mean_i = (mean_(i-1) + its n_i extended values, added in
  // order) / n_i and the running mean is never reset. Only the decisions
  // are used. Each warp first sums its sections' values in any order; with
  // every value nonnegative, that sum and the reference's ordered one are
  // both within (n_i + 1) u relative of the exact sum. The recurrence then
  // runs on those sums (below), carrying a bound on the relative error of
  // its mean and of the reference's, and takes a decision only if
  // 2200 / mean lies farther from n_i than that bound can move it. If any
  // decision is that close, or any value is negative or not finite, warp 0
  // repeats the reference's ordered sum exactly. Kept sections keep their
  // order; their section index goes to sec[8k + 4].
  // sums[2i], sums[2i + 1]: section i's sum and its length n_i.
  double* sums = S.shared_tail;   // free until the smoothing
  __shared__ int unsafe;
  if (tid == 0) unsafe = 0;
  __syncthreads();
  __shared__ double warp_max[kWarps];
  double vmax = 0.0;
  for (int i = warp; i < sections; i += nt / 32) {
    const SectionRow r = section_row(S, i);
    const int st = sec[8 * i + 2], ed = sec[8 * i + 3];
    double part = 0.0;
    bool bad = false;
    for (int j = st + lane; j < ed; j += 32) {
      const double x = r.value(S.s2, j);
      bad |= !(x >= 0.0 && x <= 1.0e300);
      part += x;
      vmax = fmax(vmax, x);
    }
    for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(kAll, part, o);
    if (__any_sync(kAll, bad) && lane == 0) unsafe = 1;
    if (lane == 0) {
      sums[2 * i] = part;
      sums[2 * i + 1] = ed - st;
    }
  }
  for (int o = 16; o; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(kAll, vmax, o));
  if (lane == 0) warp_max[warp] = vmax;
  __syncthreads();
  // Each thread takes sections; section i's mean is the recurrence run over
  // the last kWindow sections from a zero mean. With every n >= 2 (else the
  // exact path runs) a mean never exceeds twice the largest value, so the
  // mean carried into the window adds at most (2 max value) times the
  // product of 1/n over the window, below 1e-20 of the mean on real
  // sections; that bound joins the carried rounding bound. Sections within
  // kWindow of the start run the whole recurrence, in the same order.
  if (!unsafe) {
    constexpr double u = 1.1102230246251565e-16;   // 2^-53
    constexpr int kWindow = 32;
    double top = 0.0;
    for (int w = 0; w < kWarps; ++w) top = fmax(top, warp_max[w]);
    int* keep = reinterpret_cast<int*>(sums + 2 * static_cast<int64_t>(sections));
    for (int i = tid; i < sections; i += nt) {
      const int k0 = imax(0, i - kWindow + 1);
      double mean = 0.0, err = 0.0, carried = 1.0, sum = 0.0;
      bool ok = true;
      for (int k = k0; k <= i; ++k) {
        const double n = sums[2 * k + 1];
        ok &= n >= 2.0;
        sum = mean + sums[2 * k];
        const double rho = sum > 0.0 ? mean / sum : 0.0;
        err = err * rho + (n + 3.0) * u * 1.0001;
        mean = sum / n;
        carried /= n;
      }
      int decision = 0;
      if (!ok) unsafe = 1;                            // the bound below needs every n >= 2
      if (sum != 0.0) {                               // exactly zero for both: never kept
        const double n = sums[2 * i + 1];
        const double ratio = 2200.0 / mean;
        const double bound = err + (k0 > 0 ? 2.01 * top * carried / mean : 0.0);
        if (!(fabs(ratio - n) > ratio * (4.0 * bound + 8.0 * u))) unsafe = 1;
        else decision = ratio < n;
      }
      keep[i] = decision;
    }
    __syncthreads();
    if (!unsafe) {
      // Kept sections in order: a block scan of the flags, a block at a time.
      __shared__ unsigned long long scan_scratch[kWarps];
      int running = 0;
      for (int b0 = 0; b0 < sections; b0 += nt) {
        const int i = b0 + tid;
        const unsigned long long f = i < sections && keep[i] ? 1ull : 0ull;
        unsigned long long total;
        const unsigned long long before = block_scan_packed(f, scan_scratch, total);
        if (f) sec[8 * (running + static_cast<int>(before)) + 4] = i;
        running += static_cast<int>(total);
      }
      if (tid == 0) S.meta[1] = running;
    }
  }
  __syncthreads();
  // The exact ordered sum, when a decision was too close to call: warp 0
  // walks (section, 32 frames) chunks; each lane loads its value of the next
  // chunk before the current one is summed, and every lane adds the current
  // chunk's 32 values in order from shuffles, so all lanes hold the
  // reference's sum.
  if (unsafe && warp == 0) {
    int kept = 0;
    double mean = 0.0;
    int i = 0, st = 0, ed = 0, j0 = 0;
    double val = 0.0;
    if (sections > 0) {
      st = sec[2];
      ed = sec[3];
      j0 = st;
      val = j0 + lane < ed ? channel(0, j0 + lane) : 0.0;
    }
    while (i < sections) {
      int ni = i, nst = st, ned = ed, nj0 = j0 + 32;
      if (nj0 >= ed) {
        ni = i + 1;
        if (ni < sections) {
          nst = sec[8 * ni + 2];
          ned = sec[8 * ni + 3];
          nj0 = nst;
        }
      }
      const double nval = ni < sections && nj0 + lane < ned ? channel(ni, nj0 + lane) : 0.0;
      const int m = imin(32, ed - j0);
      for (int k = 0; k < m; ++k) mean += __shfl_sync(kAll, val, k);
      if (ni != i) {
        mean /= ed - st;
        if (2200.0 / mean < ed - st) {
          if (lane == 0) sec[8 * kept + 4] = i;
          ++kept;
        }
      }
      i = ni;
      st = nst;
      ed = ned;
      j0 = nj0;
      val = nval;
    }
    if (lane == 0) S.meta[1] = kept;
  }
  __syncthreads();
  const int kept = S.meta[1];
  // MakeSortedOrder (harvest.cpp:883-896): extended bounds of the kept
  // sections go to bl[2k], bl[2k+1] (every thread) and the sort order to
  // sec[8k + 5]. Kept sections come in order, and their extended starts
  // nearly always are; only if some are not does thread 0 run the
  // reference's insertion sort.
  for (int k = tid; k < kept; k += nt) {
    const int i = sec[8 * k + 4];
    bl[2 * k] = sec[8 * i + 2];
    bl[2 * k + 1] = sec[8 * i + 3];
    sec[8 * k + 5] = k;
  }
  __syncthreads();
  int inversions = 0;
  for (int k = tid; k + 1 < kept; k += nt) inversions |= bl[2 * k] > bl[2 * (k + 1)];
  const bool sorted = !__syncthreads_or(inversions);
  if (!sorted && tid == 0) {
    for (int i = 1; i < kept; ++i)
      for (int j = i - 1; j >= 0; --j) {
        const int oi = sec[8 * i + 5], oj = sec[8 * j + 5];
        if (bl[oj * 2] > bl[oi * 2]) { sec[8 * i + 5] = oj; sec[8 * j + 5] = oi; }
        else break;
      }
  }
  __syncthreads();
  // The parallel merge needs the order MakeSortedOrder produced to keep
  // section 0 first and to leave the extended starts non-decreasing: its
  // insertion sort swaps order[i] with order[j] rather than shifting, so its
  // result need not be sorted.
  bool parallel = sorted;
  if (!sorted) {
    int bad = 0;
    for (int k = tid; k + 1 < kept; k += nt) bad |= bl[2 * sec[8 * k + 5]] > bl[2 * sec[8 * (k + 1) + 5]];
    parallel = !__syncthreads_or(bad) && sec[5] == 0;
  }
  if (kept != 0 && parallel) {
    const SectionRow first = section_row(S, sec[4]);
    for (int j = tid; j < F; j += nt) S.s3[j] = first.value(S.s2, j);
    merge_sorted(S, kept, MergeScores{cand, score, stride, columns});
  } else if (kept != 0) {
    // MergeF0 (harvest.cpp:937-963) in the reference's order, when
    // MakeSortedOrder moves kept section 0 from first place or leaves the
    // starts unsorted: start from section 0 (every thread), then warp 0
    // merges in that order. ms[j] holds the
    // SearchScore of merged frame j's value where contour_extend recorded it
    // and NaN where it did not (a SearchScore is never NaN); MergeF0Sub's
    // sums compute the missing ones.
    //
    // A merged section's values are copied over [from, ed2]. MergeF0Sub's
    // sums of later merges read frames within 100 frames before a later
    // section's body (extended starts are at most 101 frames before a body,
    // and the running extent ends at most 101 frames after an earlier body);
    // bodies do not overlap, so a later merge reads or overwrites at most
    // this section's last 100 body frames and its extension. That part is
    // copied at once; the rest of the range (its body before them) is
    // copied by every thread after the last merge.
    //
    // recs[i] for sorted position i: section, extended bounds (bl), and
    // the body start and end, filled in parallel; the sequential loop loads
    // the next merge's record before it works on the current one.
    int* recs = reinterpret_cast<int*>(sums);     // 8 ints per kept section
    int* lazy = recs + 8 * static_cast<int64_t>(kept);   // per merge: deferred copy [from, to], section
    for (int i = tid; i < kept; i += nt) {
      const int o = sec[8 * i + 5], ch = sec[8 * o + 4];
      recs[8 * i + 0] = ch;
      recs[8 * i + 1] = o;
      recs[8 * i + 2] = bl[2 * o];
      recs[8 * i + 3] = bl[2 * o + 1];
      recs[8 * i + 4] = sec[8 * ch];
      recs[8 * i + 5] = sec[8 * ch + 1];
      recs[8 * i + 6] = sec[8 * ch + 6];
      recs[8 * i + 7] = sec[8 * ch + 7];
      lazy[4 * i + 0] = 0;
      lazy[4 * i + 1] = -1;
    }
    const SectionRow first = section_row(S, sec[4]);
    for (int j = tid; j < F; j += nt) {
      S.s3[j] = first.value(S.s2, j);
      S.ms[j] = first.recorded(j);
    }
    __syncthreads();
    if (warp == 0) {
      auto search = [&](double value, int j) {
        return search_score(value, cand + static_cast<int64_t>(j) * stride,
                            score + static_cast<int64_t>(j) * stride, columns);
      };
      int st1 = bl[0], ed1 = bl[1];   // the running extent (bl[0], bl[1] in the reference)
      int next[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (kept > 1)
        for (int q = 0; q < 8; ++q) next[q] = recs[8 + q];
      for (int i = 1; i < kept; ++i) {
        const int ch = next[0], o = next[1];
        // A section whose bounds are pair 0 reads the running extent, as the
        // reference's boundary_list[order[i] * 2] does after earlier merges.
        const int st2 = o == 0 ? st1 : next[2], ed2 = o == 0 ? ed1 : next[3];
        const SectionRow row = section_row(S, ch, next[4], next[5], next[6], next[7]);
        if (i + 1 < kept)
          for (int q = 0; q < 8; ++q) next[q] = recs[8 * (i + 1) + q];
        int from = 0, to = -1;
        if (st2 - ed1 > 0) {
          from = st2;
          to = ed2;
        } else if (!(st1 <= st2 && ed1 >= ed2)) {   // MergeF0Sub (harvest.cpp:912-932)
          const bool larger = merge_sum_larger(st2, ed1, [&](int j, double& a, double& b) {
            a = b = 0.0;
            if (j > ed1) return;
            a = S.ms[j];
            if (a != a) a = search(S.s3[j], j);
            b = row.recorded(j);
            if (b != b) b = search(row.value(S.s2, j), j);
          });
          from = larger ? ed1 : st2;
          to = ed2;
        }
        if (to >= 0) {
          if (st2 - ed1 > 0) st1 = st2;
          ed1 = ed2;
          // The part later merges may read or overwrite now (values loaded
          // for the whole stretch before any is stored), the rest later.
          const int now = imax(from, row.ed - 99);
          if (lane == 0 && now > from) {
            lazy[4 * i + 0] = from;
            lazy[4 * i + 1] = now - 1;
            lazy[4 * i + 2] = ch;
          }
          for (int j0 = now; j0 <= to; j0 += 128) {
            double v[4], r[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int j = j0 + 32 * q + lane;
              v[q] = j <= to ? row.value(S.s2, j) : 0.0;
              r[q] = j <= to ? row.recorded(j) : 0.0;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int j = j0 + 32 * q + lane;
              if (j <= to) {
                S.s3[j] = v[q];
                S.ms[j] = r[q];
              }
            }
          }
        }
        __syncwarp();
      }
      if (lane == 0) {
        bl[0] = st1;
        bl[1] = ed1;
      }
    }
    __syncthreads();
    // The deferred body copies, one merge per warp; no later merge read or
    // wrote those frames.
    for (int i = 1 + warp; i < kept; i += nt / 32) {
      const int from = lazy[4 * i + 0], to = lazy[4 * i + 1];
      if (to < from) continue;
      const SectionRow row = section_row(S, lazy[4 * i + 2]);
      for (int j = from + lane; j <= to; j += 32) S.s3[j] = row.value(S.s2, j);
    }
    __syncthreads();
  }
  // FixStep4 (harvest.cpp:1000-1022), threshold 9.
  for (int i = tid; i < F; i += nt) S.s4[i] = S.s3[i];
  __syncthreads();
  int nb = block_boundary_list([&](int i) { return S.s3[i]; }, F, bl, red);
  for (int i = tid; i < nb / 2 - 1; i += nt) {
    const int distance = bl[2 * (i + 1)] - bl[2 * i + 1] - 1;
    if (distance >= 9) continue;
    const double v0 = S.s3[bl[2 * i + 1]] + 1;
    const double v1 = S.s3[bl[2 * (i + 1)]] - 1;
    const double slope = (v1 - v0) / (distance + 1.0);
    int cnt = 1;
    for (int j = bl[2 * i + 1] + 1; j <= bl[2 * (i + 1)] - 1; ++j) S.s4[j] = v0 + slope * cnt++;
  }
  __syncthreads();
  if (v.fixed_out)
    for (int i = tid; i < F; i += nt) v.fixed_out[row0 + i] = S.s4[i];
  // SmoothF0Contour (harvest.cpp:1079-1113): short sections one per
  // thread, long ones one per warp.
  double* sm = v.smoothed + row0;
  for (int i = tid; i < F; i += nt) sm[i] = 0.0;
  const int lag = 300;
  const int64_t len = F + 2 * lag;
  const double* s4 = S.s4;
  auto padded = [&](int j) -> double { return (j >= lag && j < lag + F) ? s4[j - lag] : 0.0; };
  const int nbs = block_boundary_list(padded, static_cast<int>(len), bl, red);
  if (tid == 0) deferred_count = 0;
  __syncthreads();
  for (int s = tid; s < nbs / 2; s += nt) {
    if (bl[2 * s + 1] - bl[2 * s] + 1 >= kLongSection) continue;
    if (!smooth_section(padded, bl[2 * s], bl[2 * s + 1], len, sm, S.tails + tid * kTransient, kTransient))
      S.deferred[atomicAdd(&deferred_count, 1)] = s;
  }
  __syncthreads();
  // Tails that had not settled within the thread's buffer: redo with room
  // for the whole padded length.
  if (tid == 0)
    for (int k = 0; k < deferred_count; ++k) {
      const int s = S.deferred[k];
      smooth_section(padded, bl[2 * s], bl[2 * s + 1], len, sm, S.shared_tail, len);
    }
  __syncthreads();
  // Long sections, one per warp.
  int long_index = 0;
  for (int s = 0; s < nbs / 2; ++s)
    if (bl[2 * s + 1] - bl[2 * s] + 1 >= kLongSection) {
      if (long_index % kWarps == warp)
        smooth_section_warp(padded, bl[2 * s], bl[2 * s + 1], len, sm, S.shared_tail + warp * (F + 600), len);
      ++long_index;
    }
  __syncthreads();
  // Resampling (harvest.cpp:1246-1251); for frame_period 1 the same
  // expression reproduces the direct branch (harvest.cpp:1230-1235).
  if (!v.f0_out) return;
  const int64_t o0 = v.out_off[c];
  const int out_len = static_cast<int>(v.out_off[c + 1] - o0);
  for (int i = tid; i < out_len; i += nt) {
    const double t = i * v.period / 1000.0;
    v.t_out[o0 + i] = t;
    v.f0_out[o0 + i] = sm[imin(F - 1, matlab_round(t * 1000.0))];
  }
}

// Tape of the F0 gradient, written after contour_finish while its scratch is
// live: per frame the step-3 value and the initial F0 of the candidate it
// copies. Every nonzero step-3 value is a copy of a pruned candidate of its
// own frame (FixStep1 keeps SearchF0Base's pick; ExtendF0 and MergeF0 copy
// candidates), so the first column holding that value identifies it; a
// candidate's refined F0 depends on its initial F0 only through discrete
// choices (window length, bins), so any column holding the same value
// reproduces the same refinement.
__global__ void record_tape(ContourView v, const double* __restrict__ cand, int64_t total_frames,
                            double* __restrict__ tape) {
  const int64_t gf = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gf >= total_frames) return;
  const BatchView& B = v.batch;
  const int c = owner(B.frame_off, B.clips, gf);
  const int64_t row0 = B.frame_off[c];
  const int F = static_cast<int>(B.frame_off[c + 1] - row0);
  const double fixed = v.scratch[v.scratch_off[c] + 2 * F + (gf - row0)];   // s3 of the contour kernels
  double f0c = 0.0;
  if (fixed > 0.0) {
    const double* row = v.pruned + gf * B.capacity;
    const int columns = 7 * v.count[c];
    for (int col = 0; col < columns; ++col)
      if (row[col] == fixed) { f0c = overlapped_candidate(B, cand, v.count, gf, col); break; }
  }
  tape[2 * gf] = fixed;
  tape[2 * gf + 1] = f0c;
}

// Sections at least this long have their smoothing adjoint run by the whole
// warp; shorter ones run one per lane.
constexpr int kAdjointLong = 1024;
// Steps a lane of adjoint_section_warp runs from a zero state before its
// chunk: the skipped state's influence falls below 0.875^256 (1.5e-15) of it.
constexpr int kAdjointWarm = 256;

// The smoothing adjoint of one long section [st, ed] by the whole warp. The
// forward pass runs over [st, ed + trailing] (the section's gradient, then
// zeros), its outputs past ed going to `tail` (kAdjointTail doubles); the
// backward pass runs over [st - leading, ed + trailing] on the forward
// outputs (zero before st), its outputs past either end summed into the end
// frames. Each pass is cut into 32 chunks, one per lane; a lane starts
// kAdjointWarm steps before its chunk from a zero state, or from the pass's
// own zero start where that is reached, so the result equals the one-lane
// loop of contour_adjoint up to rounding and terms below 0.875^kAdjointWarm.
__device__ void adjoint_section_warp(const double* __restrict__ g_sm, double* __restrict__ body,
                                     double* __restrict__ g_s4, double* __restrict__ tail, int st, int ed,
                                     int leading, int trailing) {
  const int lag = 300, lane = threadIdx.x & 31;
  constexpr int kAhead = 2 * kChunk;   // inputs loaded ahead into registers
  const int e = ed + trailing;
  {
    const int n = e - st + 1, chunk = (n + 31) / 32;
    const int c0 = imin(st + lane * chunk, e + 1), c1 = imin(c0 + chunk, e + 1);   // this lane's [c0, c1)
    Butter fw;
    auto run = [&](int from, int to, bool store) {   // steps from .. to - 1
      for (int j0 = from; j0 < to; j0 += kAhead) {
        double in[kAhead];
#pragma unroll
        for (int k = 0; k < kAhead; ++k) in[k] = j0 + k < to && j0 + k <= ed ? g_sm[j0 + k - lag] : 0.0;
#pragma unroll
        for (int k = 0; k < kAhead; ++k) {
          const int j = j0 + k;
          if (j >= to) break;
          const double o = fw.step(in[k]);
          if (store) {
            if (j <= ed) body[j - lag] = o;
            else tail[j - ed - 1] = o;
          }
        }
      }
    };
    run(imax(st, c0 - kAdjointWarm), c0, false);
    run(c0, c1, true);
  }
  __syncwarp();
  const int s = st - leading;
  double held_st = 0.0, held_ed = 0.0;
  {
    const int n = e - s + 1, chunk = (n + 31) / 32;
    const int c0 = imin(s + lane * chunk, e + 1), c1 = imin(c0 + chunk, e + 1);
    Butter bw;
    auto run = [&](int from, int to, bool store) {   // steps from down to to
      for (int j0 = from; j0 >= to; j0 -= kAhead) {
        double in[kAhead];
#pragma unroll
        for (int k = 0; k < kAhead; ++k) {
          const int j = j0 - k;
          in[k] = j < to || j < st ? 0.0 : j <= ed ? body[j - lag] : tail[j - ed - 1];
        }
#pragma unroll
        for (int k = 0; k < kAhead; ++k) {
          const int j = j0 - k;
          if (j < to) break;
          const double o = bw.step(in[k]);
          if (store) {
            if (j > ed) held_ed += o;
            else if (j >= st) g_s4[j - lag] = o;
            else held_st += o;
          }
        }
      }
    };
    run(imin(e, c1 - 1 + kAdjointWarm), c1, false);
    run(c1 - 1, c0, true);
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    held_st += __shfl_xor_sync(kAll, held_st, o);
    held_ed += __shfl_xor_sync(kAll, held_ed, o);
  }
  __syncwarp();
  if (lane == 0) {
    g_s4[ed - lag] += held_ed;
    g_s4[st - lag] += held_st;
  }
  __syncwarp();
}

// Transpose of the resampling, SmoothF0Contour and FixStep4 for the F0
// gradient, with the voicing held fixed; one warp per clip. From dL/df0 at
// the output frames it forms dL/d(step-3 value) per 1 ms frame:
//   * resampling: an output frame's gradient goes to the frame it copies;
//   * smoothing: each voiced section is smoothed by a linear map (held
//     padding, Butterworth pass, reversal, pass, reversal); its transpose is
//     the same two passes over the section's gradient, zero outside it,
//     followed by summing the held regions into the section's end frames.
//     The free response beyond kAdjointTail samples past either end
//     (below 0.875^512 of the peak) is dropped;
//   * FixStep4: a frame filled cnt frames into a gap of d frames between
//     sections ending at a and starting at b depends on the step-3 values
//     at a and b with weights 1 - cnt / (d + 1) and cnt / (d + 1).
__global__ void __launch_bounds__(32) contour_adjoint(GradView v) {
  const int c = blockIdx.x;
  const int lane = threadIdx.x;
  const BatchView& B = v.batch;
  const int64_t row0 = B.frame_off[c];
  const int F = static_cast<int>(B.frame_off[c + 1] - row0);
  double* s3 = v.scratch + v.scratch_off[c];
  double* s4 = s3 + F;
  double* g_sm = s4 + F;
  double* g_s4 = g_sm + F;
  double* g_s3 = g_s4 + F;
  double* weight = g_s3 + F;        // cnt / (d + 1) of a filled frame, -1 elsewhere
  double* body = weight + F;        // a section's gradient after the first pass
  double* tails = body + F;         // 32 x kTransient
  int* bl = reinterpret_cast<int*>(tails + 32 * kTransient);   // up to F + 602 ints
  for (int i = lane; i < F; i += 32) {
    s3[i] = s4[i] = v.tape[2 * (row0 + i)];
    g_sm[i] = g_s4[i] = g_s3[i] = 0.0;
    weight[i] = -1.0;
  }
  __syncwarp();
  const int64_t o0 = v.out_off[c];
  const int out_len = static_cast<int>(v.out_off[c + 1] - o0);
  for (int i = lane; i < out_len; i += 32) {
    const double t = i * v.period / 1000.0;
    atomicAdd(g_sm + imin(F - 1, matlab_round(t * 1000.0)), v.grad_f0[o0 + i]);
  }
  // FixStep4's fills, as contour_finish computes them.
  int nb = warp_boundary_list([&](int i) { return s3[i]; }, F, bl);
  for (int i = lane; i < nb / 2 - 1; i += 32) {
    const int a = bl[2 * i + 1], b = bl[2 * (i + 1)];
    const int distance = b - a - 1;
    if (distance >= 9) continue;
    const double v0 = s3[a] + 1;
    const double v1 = s3[b] - 1;
    const double slope = (v1 - v0) / (distance + 1.0);
    int cnt = 1;
    for (int j = a + 1; j <= b - 1; ++j) {
      weight[j] = (j - a) / (distance + 1.0);
      s4[j] = v0 + slope * cnt++;
    }
  }
  __syncwarp();
  // Smoothing: each voiced section of the padded contour shorter than
  // kAdjointLong on one lane, the longer ones by the whole warp after them.
  // The lanes' free responses past their sections' ends sit interleaved in
  // `tails` (step k of lane l at k * 32 + l), so their stores and loads
  // coalesce; the sequential loops load kAhead inputs ahead into registers.
  const int lag = 300;
  const int len = F + 2 * lag;
  constexpr int kAhead = 2 * kChunk;
  auto padded = [&](int j) -> double { return (j >= lag && j < lag + F) ? s4[j - lag] : 0.0; };
  const int nbs = warp_boundary_list(padded, len, bl);
  for (int sec = lane; sec < nbs / 2; sec += 32) {
    const int st = bl[2 * sec], ed = bl[2 * sec + 1];
    if (ed - st + 1 >= kAdjointLong) continue;
    Butter fw;
    for (int j0 = st; j0 <= ed; j0 += kAhead) {
      double in[kAhead];
#pragma unroll
      for (int k = 0; k < kAhead; ++k) in[k] = j0 + k <= ed ? g_sm[j0 + k - lag] : 0.0;
#pragma unroll
      for (int k = 0; k < kAhead; ++k) {
        if (j0 + k > ed) break;
        body[j0 + k - lag] = fw.step(in[k]);
      }
    }
    const int trailing = imin(len - 1 - ed, kAdjointTail);
    for (int k = 0; k < trailing; ++k) tails[k * 32 + lane] = fw.step(0.0);
    Butter bw;
    double held = 0.0;
    for (int k0 = trailing - 1; k0 >= 0; k0 -= kAhead) {
      double in[kAhead];
#pragma unroll
      for (int k = 0; k < kAhead; ++k) in[k] = k0 - k >= 0 ? tails[(k0 - k) * 32 + lane] : 0.0;
#pragma unroll
      for (int k = 0; k < kAhead; ++k) {
        if (k0 - k < 0) break;
        held += bw.step(in[k]);
      }
    }
    for (int j0 = ed; j0 >= st; j0 -= kAhead) {
      double in[kAhead];
#pragma unroll
      for (int k = 0; k < kAhead; ++k) in[k] = j0 - k >= st ? body[j0 - k - lag] : 0.0;
#pragma unroll
      for (int k = 0; k < kAhead; ++k) {
        if (j0 - k < st) break;
        g_s4[j0 - k - lag] = bw.step(in[k]);
      }
    }
    g_s4[ed - lag] += held;
    held = 0.0;
    const int leading = imin(st, kAdjointTail);
    for (int k = 0; k < leading; ++k) held += bw.step(0.0);
    g_s4[st - lag] += held;
  }
  __syncwarp();
  for (int sec = 0; sec < nbs / 2; ++sec) {
    const int st = bl[2 * sec], ed = bl[2 * sec + 1];
    if (ed - st + 1 < kAdjointLong) continue;
    adjoint_section_warp(g_sm, body, g_s4, tails, st, ed, imin(st, kAdjointTail),
                         imin(len - 1 - ed, kAdjointTail));
  }
  __syncwarp();
  // FixStep4: unfilled frames pass through; each gap then adds to its left
  // end, and (after a barrier, since one frame can end one gap and start the
  // next) to its right end.
  for (int i = lane; i < F; i += 32)
    if (weight[i] < 0.0) g_s3[i] = g_s4[i];
  __syncwarp();
  nb = warp_boundary_list([&](int i) { return s3[i]; }, F, bl);
  for (int side = 0; side < 2; ++side) {
    for (int i = lane; i < nb / 2 - 1; i += 32) {
      const int a = bl[2 * i + 1], b = bl[2 * (i + 1)];
      if (b - a - 1 >= 9) continue;
      double acc = 0.0;
      for (int j = a + 1; j <= b - 1; ++j) acc += (side ? weight[j] : 1.0 - weight[j]) * g_s4[j];
      g_s3[side ? b : a] += acc;
    }
    __syncwarp();
  }
  for (int i = lane; i < F; i += 32) v.grad_fixed[row0 + i] = s3[i] > 0.0 ? g_s3[i] : 0.0;
}

cudaError_t launch_tape(const ContourView& v, const double* cand, int64_t total_frames, double* tape,
                        cudaStream_t stream) {
  record_tape<<<static_cast<unsigned>((total_frames + 255) / 256), 256, 0, stream>>>(v, cand, total_frames, tape);
  return cudaGetLastError();
}

cudaError_t launch_contour_adjoint(const GradView& v, cudaStream_t stream) {
  contour_adjoint<<<v.batch.clips, 32, 0, stream>>>(v);
  return cudaGetLastError();
}

cudaError_t launch_contour(const ContourView& v, cudaStream_t stream) {
  contour_prepare<<<v.batch.clips, kContourThreads, 0, stream>>>(v);
  contour_extend<<<dim3(v.batch.clips, v.extend_blocks > 1 ? v.extend_blocks : 1), kContourThreads, 0, stream>>>(v);
  if (v.finish_threads == 512) contour_finish<512><<<v.batch.clips, 512, 0, stream>>>(v);
  else contour_finish<kContourThreads><<<v.batch.clips, kContourThreads, 0, stream>>>(v);
  return cudaGetLastError();
}

// SearchF0Base (harvest.cpp:693-705) per frame: the candidate of the first
// highest score strictly above zero (a NaN score never wins), else 0. One
// thread per frame; rows are [frames][stride], clip c has columns[c].
__global__ void search_base(const double* __restrict__ cand, const double* __restrict__ scores,
                            int64_t total_frames, int stride, const int64_t* __restrict__ frame_off, int clips,
                            const int* __restrict__ columns, double* __restrict__ base) {
  const int64_t f = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (f >= total_frames) return;
  const int cols = columns[owner(frame_off, clips, f)];
  const double* c = cand + f * stride;
  const double* s = scores + f * stride;
  double best = 0.0, best_score = 0.0;
  for (int j = 0; j < cols; ++j)
    if (s[j] > best_score) {
      best = c[j];
      best_score = s[j];
    }
  base[f] = best;
}

cudaError_t launch_search_base(const double* cand, const double* scores, int64_t total_frames, int stride,
                               const int64_t* frame_off, int clips, const int* columns, double* base,
                               cudaStream_t stream) {
  if (total_frames <= 0) return cudaSuccess;
  const int threads = 256;
  search_base<<<static_cast<unsigned>((total_frames + threads - 1) / threads), threads, 0, stream>>>(
      cand, scores, total_frames, stride, frame_off, clips, columns, base);
  return cudaGetLastError();
}

int64_t contour_scratch(int64_t frames, int finish_threads) { return contour_scratch_doubles(frames, finish_threads); }

}  // namespace hv
