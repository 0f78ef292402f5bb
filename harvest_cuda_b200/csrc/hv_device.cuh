// Device-side helpers and the batch layout shared by all Harvest kernels.
//
// A batch is B clips of one sampling rate and one analysis setting, packed
// ragged: clip c owns x[x_off[c] .. x_off[c+1]), its decimated waveform owns
// y[y_off[c] .. y_off[c+1]) and its 1 ms analysis frames own rows
// frame_off[c] .. frame_off[c+1] of every per-frame array. All kernels are
// FP64 and are compiled with --fmad=false so that threshold arithmetic
// follows the reference's evaluation order (its CMakeLists.txt:40-41).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hv {

constexpr double kPi = 3.1415926535897932384;      // world::kPi
constexpr double kGuard = 0.000000000001;          // kMySafeGuardMinimum

// Read-only description of a batch, passed by value to kernels.
struct BatchView {
  int clips;
  int ratio;          // decimation ratio r
  int bands;          // band-pass channels
  int capacity;       // candidate columns per frame (7 * round(bands / 10))
  int per_group;      // capacity / 7: candidates per frame before overlap
  double fs_r;        // internal sampling rate fs / r
  double f0_floor, f0_ceil;
  const int64_t* x_off;      // [clips + 1]
  const int64_t* y_off;      // [clips + 1]
  const int64_t* frame_off;  // [clips + 1]
  const int* nfft;           // [clips] WORLD's whole-signal FFT size per clip
};

// matlab_round (matlabfunctions.cpp:206-208): half away from zero.
__device__ __forceinline__ int matlab_round(double v) {
  return v > 0 ? static_cast<int>(v + 0.5) : static_cast<int>(v - 0.5);
}

// Clip index owning a flattened row, by binary search over offsets.
__device__ __forceinline__ int owner(const int64_t* off, int clips, int64_t row) {
  int lo = 0, hi = clips - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= row) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }
__device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }

// Time of 1 ms frame f in seconds: f / 1000.0 correctly rounded (WORLD's
// `i * 1 / 1000.0`), without a division. q = RN(f * RN(1/1000)) is
// corrected once by its exact remainder RN(f - 1000 q) (Markstein's scheme
// for a constant divisor); the result equals the IEEE quotient for every
// int f >= 0.
__device__ __forceinline__ double frame_seconds(int f) {
  constexpr double kInv = 1.0 / 1000.0;
  const double x = static_cast<double>(f);
  const double q = __dmul_rn(x, kInv);
  return __fma_rn(__fma_rn(-q, 1000.0, x), kInv, q);
}

}  // namespace hv
