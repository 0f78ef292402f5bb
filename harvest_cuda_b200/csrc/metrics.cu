// Accuracy metrics of one F0 track against another, per clip of a ragged
// batch, on the device: the statistics of the reference's benchmark
// comparison (benchmarks/benchmark.py:20-37) for large-batch evaluation
// without copying the tracks to the host.
//
// One CTA per clip. Per clip, over frames i of the clip's output range:
//   voiced_ref = #(ref > 0), joint = #(ref > 0 and f0 > 0),
//   disagree = #((ref > 0) != (f0 > 0)),
//   cents_i = |1200 log2(f0_i / ref_i)| over jointly voiced frames,
//   cents_max, over_600 = #(cents > 600), and cents_p99 with numpy's default
//   ("linear") quantile: position h = 0.99 (m - 1) between the floor(h)-th
//   and the next order statistic. The order statistics come from a radix
//   select on the IEEE bit patterns, which for non-negative doubles sort
//   like the values: eight passes of 8-bit digits, most significant first.
#include "hv_stages.cuh"

namespace hv {

namespace {

constexpr int kMetricThreads = 256;

__device__ __forceinline__ bool cents_at(const double* ref, const double* f0, int64_t i, double& cents) {
  const double r = ref[i], a = f0[i];
  if (!(r > 0.0 && a > 0.0)) return false;
  cents = fabs(1200.0 * log2(a / r));
  return true;
}

template <class T, class Op>
__device__ T block_reduce(T v, Op op, T identity, T* shared) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o; o >>= 1) v = op(v, __shfl_down_sync(0xffffffffu, v, o));
  if (lane == 0) shared[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < (kMetricThreads >> 5) ? shared[lane] : identity;
    for (int o = 16; o; o >>= 1) v = op(v, __shfl_down_sync(0xffffffffu, v, o));
    if (lane == 0) shared[0] = v;
  }
  __syncthreads();
  T out = shared[0];
  __syncthreads();
  return out;
}

// The rank-th smallest (0-based) jointly voiced cents value of [begin, end).
__device__ unsigned long long select_rank(const double* ref, const double* f0, int64_t begin, int64_t end,
                                          long long rank, unsigned int* hist, long long* scan) {
  unsigned long long prefix = 0, mask = 0;
  for (int shift = 56; shift >= 0; shift -= 8) {
    for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[d] = 0;
    __syncthreads();
    for (int64_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
      double c;
      if (!cents_at(ref, f0, i, c)) continue;
      const unsigned long long key = static_cast<unsigned long long>(__double_as_longlong(c));
      if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      long long below = 0;
      int d = 0;
      for (; d < 255; ++d) {
        if (below + hist[d] > rank) break;
        below += hist[d];
      }
      scan[0] = d;
      scan[1] = rank - below;
    }
    __syncthreads();
    prefix |= static_cast<unsigned long long>(scan[0]) << shift;
    mask |= 255ull << shift;
    rank = scan[1];
    __syncthreads();
  }
  return prefix;
}

// stats per clip: frames, voiced_ref, joint, vuv_disagreement, cents_p99,
// cents_max, over_600 (cents values are NaN where the clip has no jointly
// voiced frame).
__global__ void __launch_bounds__(kMetricThreads)
compare_clips(const double* __restrict__ ref, const double* __restrict__ f0, const int64_t* __restrict__ off,
              double* __restrict__ stats) {
  __shared__ long long s_count[32];
  __shared__ double s_max[32];
  __shared__ unsigned int hist[256];
  __shared__ long long scan[2];
  const int c = blockIdx.x;
  const int64_t begin = off[c], end = off[c + 1];
  long long voiced = 0, joint = 0, disagree = 0, over = 0;
  double mx = 0.0;
  for (int64_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
    const bool rv = ref[i] > 0.0, av = f0[i] > 0.0;
    voiced += rv;
    disagree += rv != av;
    double cts;
    if (cents_at(ref, f0, i, cts)) {
      ++joint;
      mx = fmax(mx, cts);
      over += cts > 600.0;
    }
  }
  auto add = [](long long a, long long b) { return a + b; };
  voiced = block_reduce(voiced, add, 0ll, s_count);
  joint = block_reduce(joint, add, 0ll, s_count);
  disagree = block_reduce(disagree, add, 0ll, s_count);
  over = block_reduce(over, add, 0ll, s_count);
  mx = block_reduce(mx, [](double a, double b) { return fmax(a, b); }, 0.0, s_max);
  const int64_t frames = end - begin;
  double p99 = __longlong_as_double(0x7ff8000000000000ll), cmax = p99;
  if (joint > 0) {
    const double h = 0.99 * static_cast<double>(joint - 1);
    const long long k = static_cast<long long>(floor(h));
    const double lo = __longlong_as_double(static_cast<long long>(select_rank(ref, f0, begin, end, k, hist, scan)));
    double hi = lo;
    if (k + 1 < joint)
      hi = __longlong_as_double(static_cast<long long>(select_rank(ref, f0, begin, end, k + 1, hist, scan)));
    p99 = lo + (h - static_cast<double>(k)) * (hi - lo);
    cmax = mx;
  }
  if (threadIdx.x == 0) {
    double* out = stats + 7 * static_cast<int64_t>(c);
    out[0] = static_cast<double>(frames);
    out[1] = static_cast<double>(voiced);
    out[2] = static_cast<double>(joint);
    out[3] = frames ? static_cast<double>(disagree) / static_cast<double>(frames) : 0.0;
    out[4] = p99;
    out[5] = cmax;
    out[6] = static_cast<double>(over);
  }
}

}  // namespace

cudaError_t launch_compare(const double* ref, const double* f0, const int64_t* off, int clips, double* stats,
                           cudaStream_t stream) {
  compare_clips<<<clips, kMetricThreads, 0, stream>>>(ref, f0, off, stats);
  return cudaGetLastError();
}

}  // namespace hv
