// a2-a3: decimation of every clip to the internal rate and DC removal.
//
// WORLD's path (harvest.cpp:43-66, matlabfunctions.cpp:178-204) edge-holds the
// clip by lag = ceil(140/r)*r samples, reflects 9 more samples at each end
// (which, because lag > 9, reproduces the held value exactly), runs the order-3
// low-pass of FilterForDecimate forward and then backward, and keeps every r-th
// sample. The recurrence is sequential, so it is evaluated here as a blocked
// state-passing scan:
//   1. every segment of S samples computes its zero-state final state;
//   2. every segment's initial state is chained from the zero-state results
//      of the segments before it with the exact 3x3 transition matrix
//      T = A^S (precomputed on the host), one thread per segment;
//   3. every segment reruns from its true initial state and writes outputs.
// Each output therefore follows the reference recurrence sample by sample,
// differing only by the rounding of the chained initial state.
#include "hv_stages.cuh"

namespace hv {


__device__ __forceinline__ void clip_of_segment(const DecimateView& v, int64_t seg, int& c,
                                                int64_t& begin, int64_t& end) {
  c = owner(v.seg_off, v.clips, seg);
  int64_t k = seg - v.seg_off[c];
  int64_t total = v.t_off[c + 1] - v.t_off[c];
  begin = k * v.seg_len;
  end = begin + v.seg_len < total ? begin + v.seg_len : total;
}

// Input of the forward pass at padded index i: the held and reflected clip
// (xc: the clip's samples, n of them).
__device__ __forceinline__ double forward_input(const double* xc, int64_t n, int lag, int64_t i) {
  int64_t j = i - 9 - lag;
  j = j < 0 ? 0 : (j > n - 1 ? n - 1 : j);
  return xc[j];
}

// One step of FilterForDecimate (matlabfunctions.cpp:118-124); the expression
// order matches the reference so the step is bit-identical given its state.
__device__ __forceinline__ double lowpass_step(const DecimateView& v, double in, double& s0,
                                               double& s1, double& s2) {
  double w = in + v.a[0] * s0 + v.a[1] * s1 + v.a[2] * s2;
  double out = v.b[0] * w + v.b[1] * s0 + v.b[1] * s1 + v.b[0] * s2;
  s2 = s1; s1 = s0; s0 = w;
  return out;
}

// Pass 0 reads the padded clip; pass 1 reads the forward output reversed.
template <int kPass>
__global__ void decimate_segment_states(DecimateView v, const double* __restrict__ x,
                                        const double* __restrict__ u, int64_t segments,
                                        double* __restrict__ states) {
  int64_t seg = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (seg >= segments) return;
  int c; int64_t begin, end;
  clip_of_segment(v, seg, c, begin, end);
  int64_t total = v.t_off[c + 1] - v.t_off[c];
  const double* uc = u + v.t_off[c];
  const double* xc = x + v.x_off[c];
  const int64_t n = v.x_off[c + 1] - v.x_off[c];
  const int lag = v.lag;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int64_t i = begin; i < end; ++i) {
    double in = kPass == 0 ? forward_input(xc, n, lag, i) : uc[total - 1 - i];
    lowpass_step(v, in, s0, s1, s2);
  }
  states[3 * seg + 0] = s0;
  states[3 * seg + 1] = s1;
  states[3 * seg + 2] = s2;
}

// The initial state of every segment from the zero-state results z of the
// segments before it: s_k = T s_(k-1) + z_(k-1) from s = 0 at the clip's
// first segment, unrolled over the last kChainDepth segments (Horner's
// order, the expressions of the sequential chain). The filters' poles lie
// within radius 0.89 (ratio 12; 0.66 at ratio 2), so |T| <= 7e-13 and the
// dropped term T^3 s_(k-3) is below 1e-36 of the state: the rounded result
// is that of the full chain. One thread per segment.
constexpr int kChainDepth = 3;
__global__ void decimate_chain(DecimateView v, const double* __restrict__ z, int64_t segments,
                               double* __restrict__ entry) {
  const int64_t seg = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (seg >= segments) return;
  const int64_t first = v.seg_off[owner(v.seg_off, v.clips, seg)];
  const double* m = v.trans;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
  for (int d = kChainDepth; d >= 1; --d) {
    const int64_t k = seg - d;
    if (k < first) continue;
    const double n0 = m[0] * s0 + m[1] * s1 + m[2] * s2 + z[3 * k];
    const double n1 = m[3] * s0 + m[4] * s1 + m[5] * s2 + z[3 * k + 1];
    const double n2 = m[6] * s0 + m[7] * s1 + m[8] * s2 + z[3 * k + 2];
    s0 = n0; s1 = n1; s2 = n2;
  }
  entry[3 * seg] = s0;
  entry[3 * seg + 1] = s1;
  entry[3 * seg + 2] = s2;
}

// The backward pass (kPass 1): writes the kept samples of the backward
// output into y (before DC removal). The forward pass is
// decimate_forward_staged, below.
constexpr int kDecimateThreads = 128;

template <int kPass>
__global__ void decimate_segment_run(DecimateView v, const double* __restrict__ x, double* __restrict__ u,
                                     int64_t segments, const double* __restrict__ states, double* __restrict__ y) {
  int64_t seg = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (seg >= segments) return;
  int c; int64_t begin, end;
  clip_of_segment(v, seg, c, begin, end);
  int64_t total = v.t_off[c + 1] - v.t_off[c];
  double* uc = u + v.t_off[c];
  double s0 = states[3 * seg], s1 = states[3 * seg + 1], s2 = states[3 * seg + 2];
  // Kept sample k of the decimated clip sits at backward index
  // total - 9 - nbeg - (skip + k) * r (matlabfunctions.cpp:195-200).
  const int r = v.ratio;
  int64_t m = total - 18;
  int64_t nout = (m - 1) / r + 1;
  int64_t nbeg = r - r * nout + m;
  int64_t skip = v.lag / r;
  int64_t y_len = v.y_off[c + 1] - v.y_off[c];
  int64_t anchor = total - 9 - nbeg;  // backward index of decimated sample 0
  double* yc = y + v.y_off[c];
  // Kept indices j <= anchor with anchor - j a multiple of r, walked down
  // from the last one: the first kept index at or after begin, then every
  // r-th (one division per segment instead of one per sample).
  int64_t keep = begin <= anchor ? begin + (anchor - begin) % r : end;
  int64_t k = (anchor - keep) / r - skip;
  const double* in = uc + (total - 1);
  for (int64_t j = begin; j < end; ++j) {
    const double out = lowpass_step(v, in[-j], s0, s1, s2);
    if (j == keep) {
      if (k >= 0 && k < y_len) yc[k] = out;
      keep += r;
      --k;
    }
  }
}

// Adjoint of the decimation for the F0 gradient. The forward map is
// y = S F R F P x: P edge-holds the clip, F is the causal low-pass with
// zero initial state, R reverses, S keeps every r-th sample. With
// F^T = R F R its transpose is P^T R F R F S^T: the kept-sample gradient is
// spread onto the padded grid, reversed and low-passed (pass 0), reversed
// and low-passed again (pass 1), and the held regions are summed into the
// clip's first and last samples. Both passes reuse the blocked
// state-passing scan of the forward decimation.

// Pass 0 input at padded index i: S^T dL/dy read in reverse.
__device__ __forceinline__ double kept_gradient(const DecimateView& v, const double* gy, int c, int64_t total,
                                                int64_t i) {
  const int r = v.ratio;
  const int64_t m = total - 18;
  const int64_t nout = (m - 1) / r + 1;
  const int64_t nbeg = r - r * nout + m;
  const int64_t dist = (total - 9 - nbeg) - (total - 1 - i);
  if (dist < 0 || dist % r) return 0.0;
  const int64_t k = dist / r - v.lag / r;
  return k >= 0 && k < v.y_off[c + 1] - v.y_off[c] ? gy[v.y_off[c] + k] : 0.0;
}

template <int kPass>
__global__ void adjoint_segment_states(DecimateView v, const double* __restrict__ gy,
                                       const double* __restrict__ u, int64_t segments,
                                       double* __restrict__ states) {
  int64_t seg = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (seg >= segments) return;
  int c; int64_t begin, end;
  clip_of_segment(v, seg, c, begin, end);
  int64_t total = v.t_off[c + 1] - v.t_off[c];
  const double* uc = u + v.t_off[c];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int64_t i = begin; i < end; ++i) {
    double in = kPass == 0 ? kept_gradient(v, gy, c, total, i) : uc[total - 1 - i];
    lowpass_step(v, in, s0, s1, s2);
  }
  states[3 * seg + 0] = s0;
  states[3 * seg + 1] = s1;
  states[3 * seg + 2] = s2;
}

// Pass 0 writes the first low-passed sequence into u. Pass 1 writes the
// gradient of every clip sample that is not held (indices 1 .. n-2) and
// leaves the segment's sums over the held regions in its state slots.
template <int kPass>
__global__ void adjoint_segment_run(DecimateView v, const double* __restrict__ gy, double* __restrict__ u,
                                    int64_t segments, double* __restrict__ states, double* __restrict__ gx) {
  int64_t seg = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (seg >= segments) return;
  int c; int64_t begin, end;
  clip_of_segment(v, seg, c, begin, end);
  int64_t total = v.t_off[c + 1] - v.t_off[c];
  double* uc = u + v.t_off[c];
  double s0 = states[3 * seg], s1 = states[3 * seg + 1], s2 = states[3 * seg + 2];
  if (kPass == 0) {
    for (int64_t i = begin; i < end; ++i) uc[i] = lowpass_step(v, kept_gradient(v, gy, c, total, i), s0, s1, s2);
    return;
  }
  const int64_t n = v.x_off[c + 1] - v.x_off[c];
  double* gxc = gx + v.x_off[c];
  double first = 0.0, last = 0.0;
  for (int64_t j = begin; j < end; ++j) {
    const double out = lowpass_step(v, uc[total - 1 - j], s0, s1, s2);
    const int64_t xi = total - 1 - j - 9 - v.lag;
    if (xi <= 0) first += out;
    else if (xi >= n - 1) last += out;
    else gxc[xi] = out;
  }
  states[3 * seg] = first;
  states[3 * seg + 1] = last;
}

// Sums the held-region partials of every segment, in segment order.
__global__ void adjoint_edges(DecimateView v, const double* __restrict__ states, double* __restrict__ gx) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= v.clips) return;
  double first = 0.0, last = 0.0;
  for (int64_t seg = v.seg_off[c]; seg < v.seg_off[c + 1]; ++seg) {
    first += states[3 * seg];
    last += states[3 * seg + 1];
  }
  const int64_t n = v.x_off[c + 1] - v.x_off[c];
  gx[v.x_off[c]] = first;
  if (n > 1) gx[v.x_off[c] + n - 1] = last;
}

constexpr int kDcThreads = 256;

// Sum over the block of each thread's kN values, in a fixed tree (warp
// shuffles, then the warps' sums by warp 0); the sums are valid in thread 0.
template <int kN>
__device__ __forceinline__ void block_sum(double (&v)[kN], double (*part)[kDcThreads / 32]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < kN; ++j)
    for (int o = 16; o; o >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], o);
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < kN; ++j) part[j][warp] = v[j];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int j = 0; j < kN; ++j) {
      v[j] = lane < kDcThreads / 32 ? part[j][lane] : 0.0;
      for (int o = 16; o; o >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], o);
    }
  }
}

// Word w of clip c's chunk parts added over its chunks by one full warp
// (lane l takes chunks l, l + 32, ... in order, then a shuffle tree); every
// lane returns the sum, the same in every block that asks.
__device__ __forceinline__ double clip_chunk_sum(const DcChunks& d, int c, int w) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int64_t j = d.chunk_off[c] + lane; j < d.chunk_off[c + 1]; j += 32) s += d.parts[4 * j + w];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// Transpose of the DC removal: g -= mean(g) per clip, the mean formed from
// dc_chunk_sums' chunk sums as dc_remove forms it.
__global__ void __launch_bounds__(kDcThreads) dc_subtract(const BatchView v, DcChunks d, double* __restrict__ g) {
  __shared__ double s_mean;
  const int64_t k = blockIdx.x;
  const int c = owner(d.chunk_off, v.clips, k);
  const int64_t begin = v.y_off[c], len = v.y_off[c + 1] - begin;
  if (threadIdx.x < 32) {
    const double sum = clip_chunk_sum(d, c, 0);
    if (threadIdx.x == 0) s_mean = sum / len;
  }
  __syncthreads();
  const double mean = s_mean;
  const int64_t lo = (k - d.chunk_off[c]) * kDcChunk, hi = lo + kDcChunk < len ? lo + kDcChunk : len;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kDcThreads) g[begin + i] -= mean;
}

// Sets *flag if any sample is not finite (the reference rejects such input,
// src/bindings.cpp:36-38); checked by the host before results are copied.
__global__ void flag_nonfinite(const double* __restrict__ x, int64_t total, int* __restrict__ flag) {
  bool bad = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x)
    bad |= !isfinite(x[i]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) *flag = 1;
}

// PCM16 ingestion: sample / 32768, exact in float64 (the conversion of the
// reference's benchmark for mono PCM16 WAV input, benchmarks/benchmark.py:80-84).
__global__ void pcm16_to_double(const int16_t* __restrict__ in, int64_t total, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = static_cast<double>(in[i]) / 32768.0;
}

// Ratio 1: the waveform is used as is (harvest.cpp:45-48).
__global__ void copy_clips(const double* __restrict__ x, int64_t total, double* __restrict__ y) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < total) y[i] = x[i];
}

// a3 (harvest.cpp:82-86): y -= mean(y). Also the two spectrum bins that
// WORLD's band filter overwrites (harvest.cpp:116-133): Y[n/2] and Y[n/2-1]
// of the zero-padded n-point transform, for the final-bin correction. Each
// clip is cut into chunks of kDcChunk samples, a block per chunk, so that a
// long clip spreads over many SMs; every sum has a fixed order (a tree
// within a chunk, then the clip's chunks by lane and a shuffle tree), so a
// clip's results do not depend on the batch around it:
//   dc_chunk_sums: parts[4 k] = the sum of chunk k's samples;
//   dc_remove:     each block forms its clip's mean from the chunk sums (the
//                  same additions in every block), subtracts it and writes
//                  its chunk's three bin sums to parts[4 k + 1 .. 3];
//   dc_edge_bins:  a warp per clip adds its chunks' bin sums.
__global__ void __launch_bounds__(kDcThreads) dc_chunk_sums(const BatchView v, DcChunks d,
                                                             const double* __restrict__ y) {
  __shared__ double part[1][kDcThreads / 32];
  const int64_t k = blockIdx.x;
  const int c = owner(d.chunk_off, v.clips, k);
  const int64_t begin = v.y_off[c], len = v.y_off[c + 1] - begin;
  const int64_t lo = (k - d.chunk_off[c]) * kDcChunk, hi = lo + kDcChunk < len ? lo + kDcChunk : len;
  double acc[1] = {0.0};
  for (int64_t i = lo + threadIdx.x; i < hi; i += kDcThreads) acc[0] += y[begin + i];
  block_sum(acc, part);
  if (threadIdx.x == 0) d.parts[4 * k] = acc[0];
}

__global__ void __launch_bounds__(kDcThreads) dc_remove(const BatchView v, DcChunks d, double* __restrict__ y) {
  __shared__ double part[3][kDcThreads / 32];
  __shared__ double s_mean;
  const int64_t k = blockIdx.x;
  const int c = owner(d.chunk_off, v.clips, k);
  const int64_t begin = v.y_off[c], len = v.y_off[c + 1] - begin;
  if (threadIdx.x < 32) {
    const double sum = clip_chunk_sum(d, c, 0);
    if (threadIdx.x == 0) s_mean = sum / len;
  }
  __syncthreads();
  const double mean = s_mean;
  const int n = v.nfft[c];
  const int64_t lo = (k - d.chunk_off[c]) * kDcChunk, hi = lo + kDcChunk < len ? lo + kDcChunk : len;
  // Y[n/2] = sum y_j (-1)^j and Y[n/2-1] = sum y_j (-1)^j e^{+2 pi i j / n}.
  double acc[3] = {0.0, 0.0, 0.0};
  for (int64_t i = lo + threadIdx.x; i < hi; i += kDcThreads) {
    const double val = y[begin + i] - mean;
    y[begin + i] = val;
    const double sg = (i & 1) ? -val : val;
    acc[0] += sg;
    double sn, cs;
    sincospi(2.0 * static_cast<double>(i) / n, &sn, &cs);
    acc[1] += sg * cs;
    acc[2] += sg * sn;
  }
  block_sum(acc, part);
  if (threadIdx.x == 0) {
    d.parts[4 * k + 1] = acc[0];
    d.parts[4 * k + 2] = acc[1];
    d.parts[4 * k + 3] = acc[2];
  }
}

__global__ void dc_edge_bins(const BatchView v, DcChunks d, double* __restrict__ bins /* 3 per clip */) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (c >= v.clips) return;   // uniform per warp
  const double ny = clip_chunk_sum(d, c, 1), br = clip_chunk_sum(d, c, 2), bi = clip_chunk_sum(d, c, 3);
  if ((threadIdx.x & 31) == 0) {
    bins[3 * c] = ny;
    bins[3 * c + 1] = br;
    bins[3 * c + 2] = bi;
  }
}

// Pass 0 with coalesced stores: each thread runs its own segment, 32 steps
// at a time, into its row of a shared tile; each warp then stores its 32
// threads' rows, each row one contiguous run of u. Every thread of the block
// takes part in every barrier.
__global__ void __launch_bounds__(kDecimateThreads)
decimate_forward_staged(DecimateView v, const double* __restrict__ x, double* __restrict__ u, int64_t segments,
                        const double* __restrict__ states) {
  __shared__ double tile[kDecimateThreads][33];
  __shared__ long long base[kDecimateThreads];
  __shared__ int length[kDecimateThreads];
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int64_t seg = blockIdx.x * (int64_t)blockDim.x + t;
  const bool live = seg < segments;
  int c = 0;
  int64_t begin = 0, end = 0, n = 0;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  const double* xc = x;
  if (live) {
    clip_of_segment(v, seg, c, begin, end);
    s0 = states[3 * seg];
    s1 = states[3 * seg + 1];
    s2 = states[3 * seg + 2];
    xc = x + v.x_off[c];
    n = v.x_off[c + 1] - v.x_off[c];
  }
  base[t] = live ? v.t_off[c] + begin : 0;
  length[t] = live ? static_cast<int>(end - begin) : 0;
  const int lag = v.lag;
  for (int t0 = 0; t0 < v.seg_len; t0 += 32) {
    for (int k = 0; k < 32; ++k) {
      const int64_t i = begin + t0 + k;
      if (live && i < end) tile[t][k] = lowpass_step(v, forward_input(xc, n, lag, i), s0, s1, s2);
    }
    __syncthreads();
    for (int r = 0; r < 32; ++r) {
      const int row = 32 * w + r;
      if (t0 + lane < length[row]) u[base[row] + t0 + lane] = tile[row][lane];
    }
    __syncthreads();
  }
}

// Host-side launchers -------------------------------------------------------

// `states` holds 6 doubles per segment: the zero-state results, then the
// chained initial states.
cudaError_t launch_decimate(const DecimateView& v, const double* x, double* u, double* states,
                            int64_t segments, double* y, cudaStream_t stream) {
  const int threads = kDecimateThreads;
  unsigned grid = static_cast<unsigned>((segments + threads - 1) / threads);
  double* entry = states + 3 * segments;
  decimate_segment_states<0><<<grid, threads, 0, stream>>>(v, x, u, segments, states);
  decimate_chain<<<grid, threads, 0, stream>>>(v, states, segments, entry);
  decimate_forward_staged<<<grid, threads, 0, stream>>>(v, x, u, segments, entry);
  decimate_segment_states<1><<<grid, threads, 0, stream>>>(v, x, u, segments, states);
  decimate_chain<<<grid, threads, 0, stream>>>(v, states, segments, entry);
  decimate_segment_run<1><<<grid, threads, 0, stream>>>(v, x, u, segments, entry, y);
  return cudaGetLastError();
}

// Loads the module code of every kernel that launch_decimate, launch_copy
// and launch_remove_mean start (lazy loading would otherwise load them, and
// may allocate, at their first launch).
cudaError_t preload_decimation_kernels() {
  cudaFuncAttributes a;
  cudaError_t e = cudaSuccess;
  auto load = [&](const void* fn) { if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, fn); };
  load(reinterpret_cast<const void*>(decimate_segment_states<0>));
  load(reinterpret_cast<const void*>(decimate_segment_states<1>));
  load(reinterpret_cast<const void*>(decimate_chain));
  load(reinterpret_cast<const void*>(decimate_forward_staged));
  load(reinterpret_cast<const void*>(decimate_segment_run<1>));
  load(reinterpret_cast<const void*>(copy_clips));
  load(reinterpret_cast<const void*>(dc_chunk_sums));
  load(reinterpret_cast<const void*>(dc_remove));
  load(reinterpret_cast<const void*>(dc_edge_bins));
  return e;
}

cudaError_t launch_check_finite(const double* x, int64_t total, int* flag, int sms, cudaStream_t stream) {
  flag_nonfinite<<<sms * 4, 256, 0, stream>>>(x, total, flag);
  return cudaGetLastError();
}

cudaError_t launch_copy(const double* x, int64_t total, double* y, cudaStream_t stream) {
  const int threads = 256;
  copy_clips<<<static_cast<unsigned>((total + threads - 1) / threads), threads, 0, stream>>>(x, total, y);
  return cudaGetLastError();
}

cudaError_t launch_remove_mean(const BatchView& v, const DcChunks& d, double* y, double* bins, cudaStream_t stream) {
  const unsigned chunks = static_cast<unsigned>(d.total);
  dc_chunk_sums<<<chunks, kDcThreads, 0, stream>>>(v, d, y);
  dc_remove<<<chunks, kDcThreads, 0, stream>>>(v, d, y);
  dc_edge_bins<<<(v.clips + 7) / 8, 256, 0, stream>>>(v, d, bins);
  return cudaGetLastError();
}

cudaError_t launch_remove_mean_adjoint(const BatchView& v, const DcChunks& d, double* grad_y, cudaStream_t stream) {
  const unsigned chunks = static_cast<unsigned>(d.total);
  dc_chunk_sums<<<chunks, kDcThreads, 0, stream>>>(v, d, grad_y);
  dc_subtract<<<chunks, kDcThreads, 0, stream>>>(v, d, grad_y);
  return cudaGetLastError();
}

cudaError_t launch_decimate_adjoint(const DecimateView& v, const double* grad_y, double* u, double* states,
                                    int64_t segments, double* grad_x, cudaStream_t stream) {
  const int threads = 128;
  unsigned grid = static_cast<unsigned>((segments + threads - 1) / threads);
  unsigned cgrid = static_cast<unsigned>((v.clips + threads - 1) / threads);
  double* entry = states + 3 * segments;
  adjoint_segment_states<0><<<grid, threads, 0, stream>>>(v, grad_y, u, segments, states);
  decimate_chain<<<grid, threads, 0, stream>>>(v, states, segments, entry);
  adjoint_segment_run<0><<<grid, threads, 0, stream>>>(v, grad_y, u, segments, entry, grad_x);
  adjoint_segment_states<1><<<grid, threads, 0, stream>>>(v, grad_y, u, segments, states);
  decimate_chain<<<grid, threads, 0, stream>>>(v, states, segments, entry);
  adjoint_segment_run<1><<<grid, threads, 0, stream>>>(v, grad_y, u, segments, entry, grad_x);
  adjoint_edges<<<cgrid, threads, 0, stream>>>(v, entry, grad_x);
  return cudaGetLastError();
}

cudaError_t launch_pcm16(const int16_t* in, int64_t total, double* out, int sms, cudaStream_t stream) {
  pcm16_to_double<<<sms * 8, 256, 0, stream>>>(in, total, out);
  return cudaGetLastError();
}

}  // namespace hv
