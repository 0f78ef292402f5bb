// C-ABI shim over the reference's own CUDA path, for timing and parity
// checks only (test infrastructure; the engine never loads it).
//
// The reference's Python binding validates its arguments and calls
// harvest_cuda::analyze() with a cached GpuWorkspace (src/bindings.cpp:60-80,
// src/workspace_cache.h); analyze() decimates and runs the band bank,
// candidates, refinement and pruning on the GPU through src/cuda_backend.cu
// and the contour stages on the host (src/engine.cpp:240-333). This shim
// makes the same calls, one workspace per device kept for the process.
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>

#include "engine.h"

namespace {
std::string g_error;
struct WorkspaceDeleter {
  void operator()(harvest_cuda::GpuWorkspace* w) const { harvest_cuda::delete_gpu_workspace(w); }
};
std::map<int, std::unique_ptr<harvest_cuda::GpuWorkspace, WorkspaceDeleter>> g_workspaces;
std::once_flag g_host_cache;
}  // namespace

extern "C" {

const char* refcuda_last_error(void) { return g_error.c_str(); }

int refcuda_available(int device) { return harvest_cuda::cuda_available(device) ? 1 : 0; }

// f0 and times receive out_len values (GetSamplesForHarvest(fs, n, period)).
int refcuda_harvest(const double* x, int n, int fs, double f0_floor, double f0_ceil, double period,
                    int device, double* f0, double* times, int out_len) {
  try {
    std::call_once(g_host_cache, [] { harvest_cuda::initialize_host_cache(); });
    auto& w = g_workspaces[device];
    if (!w) w.reset(harvest_cuda::create_gpu_workspace(device));
    harvest_cuda::Result r = harvest_cuda::analyze(x, n, fs, f0_floor, f0_ceil, period, w.get());
    if (static_cast<int>(r.f0.size()) != out_len) throw std::invalid_argument("output length mismatch");
    std::memcpy(f0, r.f0.data(), sizeof(double) * out_len);
    std::memcpy(times, r.times.data(), sizeof(double) * out_len);
    g_error.clear();
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 2;
  }
}

void refcuda_release(void) { g_workspaces.clear(); }

}  // extern "C"
