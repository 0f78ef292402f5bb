// a10 and a13: channel aggregation, pruning and the best candidate per frame.
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
