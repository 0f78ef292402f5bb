// a10 and a13: channel aggregation, pruning and the best candidate per frame.
#include <algorithm>

#include "hv_stages.cuh"

namespace hv {

// a10: DetectOfficialF0Candidates(Sub1/Sub2) (harvest.cpp:348-412). One
// thread per frame walks the bands: runs of at least 10 voiced channels
// (first and last channel forced unvoiced) become one candidate, their mean
// summed in channel order. `cand` is [frame][per_group]; per-clip maxima go
// to count[] (zeroed by the caller), one atomic per clip per warp. Bands are
// loaded 16 at a time (the loads of a group are independent), and each run's sum is carried along the walk:
// the same additions, from 0, in channel order, as the reference's loop.
__global__ void official_candidates(BatchView v, const double* __restrict__ raw,
                                    int64_t total_frames, double* __restrict__ cand,
                                    int* __restrict__ count) {
  int64_t gf = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gf >= total_frames) return;
  double* row = cand + gf * v.per_group;
  int found = 0, start = 0, prev = 0;
  double run = 0.0;
  for (int b0 = 1; b0 < v.bands; b0 += 16) {
    double r[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int b = b0 + u;
      r[u] = b < v.bands - 1 ? raw[b * total_frames + gf] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int b = b0 + u;
      if (b >= v.bands) break;
      const int now = (b == v.bands - 1) ? 0 : (r[u] > 0 ? 1 : 0);
      if (now - prev == 1) {
        start = b;
        run = 0.0;
      }
      if (now - prev == -1 && b - start >= 10) {
        if (found < v.per_group) row[found] = run / (b - start);
        ++found;
      }
      if (now) run += r[u];
      prev = now;
    }
  }
  for (int j = found; j < v.per_group; ++j) row[j] = 0.0;
  // At most (bands - 1) / 11 runs fit, fewer than per_group; the clamp only
  // keeps later column arithmetic in bounds.
  // Lanes of the same clip take their maximum first (the counters only
  // grow, so the order of the atomics does not matter).
  const int c = owner(v.frame_off, v.clips, gf);
  const unsigned peers = __match_any_sync(__activemask(), c);
  const int m = __reduce_max_sync(peers, static_cast<unsigned>(imin(found, v.per_group)));
  if (m > 0 && (threadIdx.x & 31) == __ffs(peers) - 1) atomicMax(count + c, m);
}

// a13: RemoveUnreliableCandidates(Sub) with SelectBestF0 (harvest.cpp:636-688)
// and SearchF0Base (harvest.cpp:693-705). One warp per frame: lanes take
// columns, neighbour rows are read from the unpruned arrays, and the best
// candidate is the first column holding the highest pruned score. The warp
// first packs the nonzero candidates of the two neighbour rows into shared
// memory, so each candidate's two minima run over those only (a zero
// candidate c gives |ref - c| / ref = 1 for ref > 0, which the error's cap
// at 1 already covers), and packs this row's nonzero candidates, so that a
// lane checks one of them at a time: about half of the 7 count columns are
// zero, and with one lane per column the warp ran the minima once per 32
// columns with most lanes idle. Per warp 2 capacity doubles and capacity
// ints of shared memory (the packed columns; their values are re-read from
// the row).
__global__ void __launch_bounds__(128)
prune_frames(BatchView v, const double* __restrict__ refined, const double* __restrict__ scores,
             const int* __restrict__ count, int64_t total_frames, double* __restrict__ pruned,
             double* __restrict__ pruned_scores, double* __restrict__ best) {
  extern __shared__ double s_rows[];
  const int lane = threadIdx.x & 31;
  const int64_t gf = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
  if (gf >= total_frames) return;   // uniform per warp
  const int c = owner(v.frame_off, v.clips, gf);
  const int64_t row0 = v.frame_off[c];
  const int frames = static_cast<int>(v.frame_off[c + 1] - row0);
  const int f = static_cast<int>(gf - row0);
  const int columns = 7 * count[c];
  const int cap = v.capacity;
  const double* row = refined + gf * cap;
  const bool interior = f >= 1 && f <= frames - 2;
  double* s_next = s_rows + (threadIdx.x >> 5) * (2 * cap + (cap + 1) / 2);
  double* s_prev = s_next + cap;
  int* s_col = reinterpret_cast<int*>(s_prev + cap);   // this row's columns to check, packed
  const unsigned below = (1u << lane) - 1u;
  int n_next = 0, n_prev = 0, n_cur = 0;
  double top = 0.0, pick = 0.0;
  int top_col = cap;
  // Highest pruned score, first column on ties.
  auto consider = [&](double sc, double ref, int col) {
    if (sc > top || (sc == top && col < top_col)) {
      top = sc;
      pick = ref;
      top_col = col;
    }
  };
  // Columns from 7 count on hold no candidate; they are neither read nor
  // written (every reader stops at 7 count). Columns that need no check are
  // written here; the others are packed, so that the checks below keep
  // every lane busy.
  for (int base = 0; base < columns; base += 32) {
    const int j = base + lane;
    const bool in = j < columns;
    const double ref = in ? row[j] : 0.0, sc = in ? scores[gf * cap + j] : 0.0;
    if (interior) {
      const double a = in ? row[cap + j] : 0.0;
      const double b = in ? row[j - cap] : 0.0;
      const unsigned ma = __ballot_sync(0xffffffffu, a != 0.0), mb = __ballot_sync(0xffffffffu, b != 0.0);
      if (a != 0.0) s_next[n_next + __popc(ma & below)] = a;
      if (b != 0.0) s_prev[n_prev + __popc(mb & below)] = b;
      n_next += __popc(ma);
      n_prev += __popc(mb);
    }
    const bool check = in && interior && ref != 0.0;
    const unsigned mc = __ballot_sync(0xffffffffu, check);
    if (check) {
      s_col[n_cur + __popc(mc & below)] = j;
    } else if (in) {
      pruned[gf * cap + j] = ref;
      pruned_scores[gf * cap + j] = sc;
      consider(sc, ref, j);
    }
    n_cur += __popc(mc);
  }
  __syncwarp();
  for (int k = lane; k < n_cur; k += 32) {
    const int col = s_col[k];
    double ref = row[col], sc = scores[gf * cap + col];
    // SelectBestF0 leaves min(1, min_j |ref - c_j| / ref) as the error.
    // Correctly rounded division by the same positive ref is monotone, so
    // the smaller of the two rows' errors is the quotient of the smaller
    // difference: one division, bit-identical, and the cap at 1 does not
    // change the test. With no nonzero neighbour the quotient is infinite.
    double d1 = __longlong_as_double(0x7ff0000000000000ll), d2 = d1;
    for (int j = 0; j < n_next; ++j) d1 = fmin(d1, fabs(ref - s_next[j]));
    for (int j = 0; j < n_prev; ++j) d2 = fmin(d2, fabs(ref - s_prev[j]));
    const double e = fmin(d1, d2) / ref;
    if (!(e <= 0.05)) ref = sc = 0.0;
    pruned[gf * cap + col] = ref;
    pruned_scores[gf * cap + col] = sc;
    consider(sc, ref, col);
  }
  for (int o = 16; o; o >>= 1) {
    double ot = __shfl_down_sync(0xffffffffu, top, o);
    double op = __shfl_down_sync(0xffffffffu, pick, o);
    int oc = __shfl_down_sync(0xffffffffu, top_col, o);
    if (ot > top || (ot == top && oc < top_col)) { top = ot; pick = op; top_col = oc; }
  }
  if (lane == 0) best[gf] = top > 0.0 ? pick : 0.0;
}

cudaError_t launch_candidates(const BatchView& v, const double* raw, int64_t total_frames,
                              double* cand, int* count, cudaStream_t stream) {
  const int threads = 128;
  official_candidates<<<static_cast<unsigned>((total_frames + threads - 1) / threads), threads, 0,
                        stream>>>(v, raw, total_frames, cand, count);
  return cudaGetLastError();
}

cudaError_t launch_prune(const BatchView& v, const double* refined, const double* scores,
                         const int* count, int64_t total_frames, double* pruned,
                         double* pruned_scores, double* best, cudaStream_t stream) {
  // Up to 4 warps per block, each with 2.5 capacity doubles of shared
  // memory, within the default 48 KB.
  const size_t per_warp = sizeof(double) * (2 * static_cast<size_t>(v.capacity) + (v.capacity + 1) / 2);
  const int warps = static_cast<int>(std::max<size_t>(1, std::min<size_t>(4, 49152 / per_warp)));
  prune_frames<<<static_cast<unsigned>((total_frames + warps - 1) / warps), 32 * warps, warps * per_warp, stream>>>(
      v, refined, scores, count, total_frames, pruned, pruned_scores, best);
  return cudaGetLastError();
}

}  // namespace hv
