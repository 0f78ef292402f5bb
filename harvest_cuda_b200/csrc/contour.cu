// a14-a16: FixF0Contour, SmoothF0Contour and resampling to frame_period.
//
// One warp owns one clip; clips run in parallel. Within a clip the
// data-parallel parts run across the 32 lanes: FixStep1, the boundary lists
// (warp ballots over the voicing changes), FixStep2's pruning, the extension
// of every voiced section, FixStep4's gap filling, the zero-lag smoothing of
// every voiced section and the resampling. The steps whose result depends on
// order stay in lane 0, exactly as the reference writes them: ExtendSub's
// carried mean, MakeSortedOrder, and MergeF0's score sums. Given the same
// candidates the warp reproduces WORLD bit for bit.
#include "hv_stages.cuh"

namespace hv {

constexpr int kExtend = 101;      // ExtendF0 writes at most 101 frames per side
constexpr int kTransient = 1024;  // per-lane buffer for a smoothing tail
constexpr unsigned kAll = 0xffffffffu;

// Doubles of scratch one clip of `frames` frames needs.
__host__ __device__ inline int64_t contour_scratch_doubles(int64_t frames) {
  int64_t sections = (frames + 1) / 8 + 2;
  // s1..s4, extension values, section records (8 ints each), boundary list
  // (up to frames + 600 ints), per-lane smoothing tails, the shared tail for
  // deferred sections, deferred-section list.
  return 4 * frames + 2 * kExtend * sections + 4 * sections + (frames + 602) +
         32 * kTransient + (frames + 600) + (frames + 602) / 2 + 64;
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

// The contour stage runs one warp per clip and is bound by the latency of
// dependent loads, so the sequential loops below load kChunk values ahead
// into registers and then consume them in the reference's order.
constexpr int kChunk = 8;

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
  for (int o = 16; o; o >>= 1) {
    const double oe = __shfl_xor_sync(kAll, best_e, o), ov = __shfl_xor_sync(kAll, best_v, o);
    const int oi = __shfl_xor_sync(kAll, best_i, o);
    if (oi >= 0 && (best_i < 0 || oe < best_e || (oe == best_e && oi > best_i))) {
      best_e = oe; best_i = oi; best_v = ov;
    }
  }
  return best_v;
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
  for (int o = 16; o; o >>= 1) {
    const double oe = __shfl_xor_sync(kAll, best_e, o), ov = __shfl_xor_sync(kAll, best_v, o);
    const int oi = __shfl_xor_sync(kAll, best_i, o);
    if (oi >= 0 && (best_i < 0 || oe < best_e || (oe == best_e && oi > best_i))) {
      best_e = oe; best_i = oi; best_v = ov;
    }
  }
  return best_v;
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

__global__ void __launch_bounds__(32) contour_clips(ContourView v) {
  const int c = blockIdx.x;
  const int lane = threadIdx.x;
  const BatchView& B = v.batch;
  const int64_t row0 = B.frame_off[c];
  const int F = static_cast<int>(B.frame_off[c + 1] - row0);
  const int columns = v.column_multiple * v.count[c];
  const int stride = B.capacity;
  const double* cand = v.pruned + row0 * stride;
  const double* score = v.pruned_scores + row0 * stride;
  const double* base = v.best + row0;

  double* sc = v.scratch + v.scratch_off[c];
  const int64_t sections_cap = (F + 1) / 8 + 2;
  double* s1 = sc;
  double* s2 = s1 + F;
  double* s3 = s2 + F;
  double* s4 = s3 + F;
  double* ext = s4 + F;                                              // [sections][2][kExtend]
  int* sec = reinterpret_cast<int*>(ext + 2 * kExtend * sections_cap);  // 8 ints per section
  int* bl = sec + 8 * sections_cap;                                  // F + 602 doubles of ints
  double* tails = reinterpret_cast<double*>(bl) + (F + 602);         // 32 x kTransient
  double* shared_tail = tails + 32 * kTransient;                     // F + 600
  int* deferred = reinterpret_cast<int*>(shared_tail + F + 600);     // (F + 602) ints

  // FixStep1 (harvest.cpp:710-722), allowed range 0.008; four groups of 32
  // frames per iteration.
  for (int i0 = lane; i0 < F; i0 += 128) {
    double b0[4], b1[4], b2[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + 32 * u;
      b0[u] = i < F ? base[i] : 0.0;
      b1[u] = i < F && i >= 2 ? base[i - 1] : 0.0;
      b2[u] = i < F && i >= 2 ? base[i - 2] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + 32 * u;
      if (i >= F) break;
      double out = 0.0;
      if (i >= 2 && b0[u] != 0.0) {
        double ref = b1[u] * 2 - b2[u];
        out = fabs((b0[u] - ref) / ref) > 0.008 && fabs((b0[u] - b1[u])) / b1[u] > 0.008 ? 0.0 : b0[u];
      }
      s1[i] = out;
      s2[i] = out;
    }
  }
  __syncwarp();
  // FixStep2 (harvest.cpp:748-762): voiced runs shorter than 7 frames go.
  int nb = warp_boundary_list([&](int i) { return s1[i]; }, F, bl);
  for (int i = lane; i < nb / 2; i += 32) {
    if (bl[2 * i + 1] - bl[2 * i] >= 6) continue;
    for (int j = bl[2 * i]; j <= bl[2 * i + 1]; ++j) s2[j] = 0.0;
  }
  __syncwarp();
  for (int i = lane; i < F; i += 32) s3[i] = s2[i];
  // FixStep3 (harvest.cpp:968-995): Extend/ExtendF0, one section at a time
  // with the whole warp (each frame's SelectBestF0 across the lanes).
  nb = warp_boundary_list([&](int i) { return s2[i]; }, F, bl);
  const int sections = imin(nb / 2, static_cast<int>(sections_cap));
  for (int i = 0; i < sections; ++i) {
    const int st = bl[2 * i], ed = bl[2 * i + 1];
    double* fwd = ext + (2 * i) * kExtend;
    double* bwd = fwd + kExtend;
    for (int k = lane; k < kExtend; k += 32) fwd[k] = bwd[k] = 0.0;
    __syncwarp();
    {  // ExtendF0 forward from the end (harvest.cpp:867-870)
      const int reached = extend_f0(cand, stride, columns, ed, 1, imin(F - 2, ed + 100) - ed + 1, s2[ed], fwd);
      if (lane == 0) sec[8 * i + 3] = reached;
    }
    {  // ExtendF0 backward from the start (harvest.cpp:871-873)
      const int reached = extend_f0(cand, stride, columns, st, -1, st - imax(1, st - 100) + 1, s2[st], bwd);
      if (lane == 0) sec[8 * i + 2] = reached;
    }
    if (lane == 0) {
      sec[8 * i + 0] = st;
      sec[8 * i + 1] = ed;
    }
  }
  __syncwarp();
  // A section's extended row: its body from s2 plus the extension values.
  auto channel = [&](int i, int j) -> double {
    const int st = sec[8 * i], ed = sec[8 * i + 1];
    if (j >= st && j <= ed) return s2[j];
    if (j > ed && j - ed - 1 < kExtend) return ext[(2 * i) * kExtend + (j - ed - 1)];
    if (j < st && st - 1 - j < kExtend) return ext[(2 * i + 1) * kExtend + (st - 1 - j)];
    return 0.0;
  };
  // ExtendSub (harvest.cpp:840-856): the running mean is never reset. The
  // lanes load 32 channel values at a time and every lane adds them in
  // order from shuffles, so all lanes hold the reference's sum. Kept
  // sections keep their order; their section index goes to sec[8k + 4].
  int kept = 0;
  {
    double mean = 0.0;
    for (int i = 0; i < sections; ++i) {
      const int st = sec[8 * i + 2], ed = sec[8 * i + 3];
      for (int j0 = st; j0 < ed; j0 += 32) {
        const double v = j0 + lane < ed ? channel(i, j0 + lane) : 0.0;
        const int m = imin(32, ed - j0);
        for (int k = 0; k < m; ++k) mean += __shfl_sync(kAll, v, k);
      }
      mean /= ed - st;
      if (2200.0 / mean < ed - st) {
        if (lane == 0) sec[8 * kept + 4] = i;
        ++kept;
      }
    }
  }
  __syncwarp();
  // MakeSortedOrder (harvest.cpp:883-896) in lane 0: extended bounds of the
  // kept sections go to bl[2k], bl[2k+1] and the sort order to sec[8k + 5].
  if (lane == 0) {
    for (int k = 0; k < kept; ++k) {
      const int i = sec[8 * k + 4];
      bl[2 * k] = sec[8 * i + 2];
      bl[2 * k + 1] = sec[8 * i + 3];
      sec[8 * k + 5] = k;
    }
    for (int i = 1; i < kept; ++i)
      for (int j = i - 1; j >= 0; --j) {
        const int oi = sec[8 * i + 5], oj = sec[8 * j + 5];
        if (bl[oj * 2] > bl[oi * 2]) { sec[8 * i + 5] = oj; sec[8 * j + 5] = oi; }
        else break;
      }
  }
  __syncwarp();
  if (kept != 0) {
    // MergeF0 (harvest.cpp:937-963): start from the first kept section, then
    // lane 0 decides each merge (pair 0 of bl is the running extent) and
    // the warp copies the chosen range.
    const int first = sec[4];
    for (int j = lane; j < F; j += 32) s3[j] = channel(first, j);
    __syncwarp();
    for (int i = 1; i < kept; ++i) {
      const int o = sec[8 * i + 5];
      const int ch = sec[8 * o + 4];
      const int st2 = bl[2 * o], ed2 = bl[2 * o + 1];
      const int st1 = bl[0], ed1 = bl[1];
      int from = 0, to = -1;
      if (st2 - ed1 > 0) {
        from = st2;
        to = ed2;
      } else if (!(st1 <= st2 && ed1 >= ed2)) {   // MergeF0Sub (harvest.cpp:912-932)
        // Scores of 32 frames at a time, one per lane, summed in order by
        // every lane from shuffles.
        double sc1 = 0.0, sc2 = 0.0;
        for (int j0 = st2; j0 <= ed1; j0 += 32) {
          const int j = j0 + lane;
          double a = 0.0, b = 0.0;
          if (j <= ed1) {
            a = search_score(s3[j], cand + static_cast<int64_t>(j) * stride,
                             score + static_cast<int64_t>(j) * stride, columns);
            b = search_score(channel(ch, j), cand + static_cast<int64_t>(j) * stride,
                             score + static_cast<int64_t>(j) * stride, columns);
          }
          const int m = imin(32, ed1 - j0 + 1);
          for (int k = 0; k < m; ++k) {
            sc1 += __shfl_sync(kAll, a, k);
            sc2 += __shfl_sync(kAll, b, k);
          }
        }
        from = sc1 > sc2 ? ed1 : st2;
        to = ed2;
      }
      __syncwarp();
      if (lane == 0 && to >= 0) {
        if (st2 - ed1 > 0) bl[0] = st2;
        bl[1] = ed2;
      }
      for (int j = from + lane; j <= to; j += 32) s3[j] = channel(ch, j);
      __syncwarp();
    }
  }
  // FixStep4 (harvest.cpp:1000-1022), threshold 9.
  for (int i = lane; i < F; i += 32) s4[i] = s3[i];
  __syncwarp();
  nb = warp_boundary_list([&](int i) { return s3[i]; }, F, bl);
  for (int i = lane; i < nb / 2 - 1; i += 32) {
    const int distance = bl[2 * (i + 1)] - bl[2 * i + 1] - 1;
    if (distance >= 9) continue;
    const double v0 = s3[bl[2 * i + 1]] + 1;
    const double v1 = s3[bl[2 * (i + 1)]] - 1;
    const double slope = (v1 - v0) / (distance + 1.0);
    int cnt = 1;
    for (int j = bl[2 * i + 1] + 1; j <= bl[2 * (i + 1)] - 1; ++j) s4[j] = v0 + slope * cnt++;
  }
  __syncwarp();
  if (v.fixed_out)
    for (int i = lane; i < F; i += 32) v.fixed_out[row0 + i] = s4[i];
  // SmoothF0Contour (harvest.cpp:1079-1113), one voiced section per lane.
  double* sm = v.smoothed + row0;
  for (int i = lane; i < F; i += 32) sm[i] = 0.0;
  __syncwarp();
  const int lag = 300;
  const int64_t len = F + 2 * lag;
  auto padded = [&](int j) -> double { return (j >= lag && j < lag + F) ? s4[j - lag] : 0.0; };
  const int nbs = warp_boundary_list(padded, static_cast<int>(len), bl);
  __shared__ int deferred_count;
  if (lane == 0) deferred_count = 0;
  __syncwarp();
  for (int s = lane; s < nbs / 2; s += 32) {
    if (bl[2 * s + 1] - bl[2 * s] + 1 >= kLongSection) continue;
    if (!smooth_section(padded, bl[2 * s], bl[2 * s + 1], len, sm, tails + lane * kTransient, kTransient))
      deferred[atomicAdd(&deferred_count, 1)] = s;
  }
  __syncwarp();
  // Tails that had not settled within the lane buffer: redo with room for
  // the whole padded length.
  if (lane == 0)
    for (int k = 0; k < deferred_count; ++k) {
      const int s = deferred[k];
      smooth_section(padded, bl[2 * s], bl[2 * s + 1], len, sm, shared_tail, len);
    }
  __syncwarp();
  // Long sections, one at a time with the whole warp.
  for (int s = 0; s < nbs / 2; ++s)
    if (bl[2 * s + 1] - bl[2 * s] + 1 >= kLongSection)
      smooth_section_warp(padded, bl[2 * s], bl[2 * s + 1], len, sm, shared_tail, len);
  // Resampling (harvest.cpp:1246-1251); for frame_period 1 the same
  // expression reproduces the direct branch (harvest.cpp:1230-1235).
  if (!v.f0_out) return;
  const int64_t o0 = v.out_off[c];
  const int out_len = static_cast<int>(v.out_off[c + 1] - o0);
  for (int i = lane; i < out_len; i += 32) {
    const double t = i * v.period / 1000.0;
    v.t_out[o0 + i] = t;
    v.f0_out[o0 + i] = sm[imin(F - 1, matlab_round(t * 1000.0))];
  }
}

// Tape of the F0 gradient, written after contour_clips while its scratch is
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
  const double fixed = v.scratch[v.scratch_off[c] + 2 * F + (gf - row0)];   // s3 of contour_clips
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

// Transpose of the resampling, SmoothF0Contour and FixStep4 for the F0
// gradient, with the voicing held fixed; one warp per clip. From dL/df0 at
// the output frames it forms dL/d(step-3 value) per 1 ms frame:
//   * resampling: an output frame's gradient goes to the frame it copies;
//   * smoothing: each voiced section is smoothed by a linear map (held
//     padding, Butterworth pass, reversal, pass, reversal); its transpose is
//     the same two passes over the section's gradient, zero outside it,
//     followed by summing the held regions into the section's end frames.
//     The free response beyond kTransient samples past either end
//     (below 0.88^1024 of the peak) is dropped;
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
  // FixStep4's fills, as contour_clips computes them.
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
  // Smoothing, one voiced section of the padded contour per lane.
  const int lag = 300;
  const int64_t len = F + 2 * lag;
  auto padded = [&](int j) -> double { return (j >= lag && j < lag + F) ? s4[j - lag] : 0.0; };
  const int nbs = warp_boundary_list(padded, static_cast<int>(len), bl);
  for (int sec = lane; sec < nbs / 2; sec += 32) {
    const int st = bl[2 * sec], ed = bl[2 * sec + 1];
    Butter fw;
    for (int j = st; j <= ed; ++j) body[j - lag] = fw.step(g_sm[j - lag]);
    double* tail = tails + lane * kTransient;
    const int64_t trailing = len - 1 - ed < kTransient ? len - 1 - ed : kTransient;
    for (int64_t k = 0; k < trailing; ++k) tail[k] = fw.step(0.0);
    Butter bw;
    double held = 0.0;
    for (int64_t k = trailing - 1; k >= 0; --k) held += bw.step(tail[k]);
    for (int j = ed; j >= st; --j) g_s4[j - lag] = bw.step(body[j - lag]);
    g_s4[ed - lag] += held;
    held = 0.0;
    const int leading = st < kTransient ? st : kTransient;
    for (int k = 0; k < leading; ++k) held += bw.step(0.0);
    g_s4[st - lag] += held;
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
  contour_clips<<<v.batch.clips, 32, 0, stream>>>(v);
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

int64_t contour_scratch(int64_t frames) { return contour_scratch_doubles(frames); }

}  // namespace hv
