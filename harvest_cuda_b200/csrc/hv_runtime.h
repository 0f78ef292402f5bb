// Host runtime of the engine: CUDA error mapping, the device check, the
// primary-context owner, the context guard and the per-device workspace
// cache. Host C++ only, written against the CUDA runtime and driver headers
// alone, so that the tests can compile it against fake headers whose calls
// fail on demand (no GPU involved).
//
// Contracts kept from the reference:
//   * the device check and its messages (src/cuda_device.h:26-39);
//   * the caller's current context is restored exactly, also when a call
//     fails half-way (src/cuda_device.h:74-108);
//   * one workspace per device, calls on one device take turns, calls on
//     different devices do not wait, and clear() never invalidates a call in
//     flight nor lets a workspace created across it be cached
//     (src/workspace_cache.h:10-70).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace hv {

struct InvalidArgument : std::runtime_error { using std::runtime_error::runtime_error; };
struct RuntimeFailure : std::runtime_error { using std::runtime_error::runtime_error; };

// Throws RuntimeFailure for a failed runtime call, naming the call and the
// error, with a hint for the two failures a user can act on.
inline void check(cudaError_t code, const char* what) {
  if (code == cudaSuccess) return;
  const char* name = cudaGetErrorName(code);
  const char* text = cudaGetErrorString(code);
  std::string msg = std::string("CUDA: ") + what + ": " + (name ? name : std::to_string(int(code)));
  if (text) msg += std::string(": ") + text;
  if (code == cudaErrorMemoryAllocation)
    msg += ". GPU memory allocation failed; try shorter or fewer clips.";
  if (code == cudaErrorNoDevice || code == cudaErrorInsufficientDriver)
    msg += ". Check the NVIDIA driver and CUDA_VISIBLE_DEVICES.";
  throw RuntimeFailure(msg);
}

// Driver entry points, resolved through the runtime so that the library has
// no link-time dependency on libcuda (it loads on machines without a GPU
// driver).
struct Driver {
  decltype(&cuInit) init = nullptr;
  decltype(&cuDevicePrimaryCtxRetain) retain = nullptr;
  decltype(&cuDevicePrimaryCtxRelease) release = nullptr;
  decltype(&cuCtxGetCurrent) get_current = nullptr;
  decltype(&cuCtxSetCurrent) set_current = nullptr;
  bool ok = false;
  Driver() {
    auto get = [](const char* name, void** fn) {
      cudaDriverEntryPointQueryResult q;
      return cudaGetDriverEntryPoint(name, fn, cudaEnableDefault, &q) == cudaSuccess && *fn &&
             q == cudaDriverEntryPointSuccess;
    };
    ok = get("cuInit", reinterpret_cast<void**>(&init)) &&
         get("cuDevicePrimaryCtxRetain", reinterpret_cast<void**>(&retain)) &&
         get("cuDevicePrimaryCtxRelease", reinterpret_cast<void**>(&release)) &&
         get("cuCtxGetCurrent", reinterpret_cast<void**>(&get_current)) &&
         get("cuCtxSetCurrent", reinterpret_cast<void**>(&set_current));
  }
};
inline const Driver& driver() {
  static Driver d;
  return d;
}

// Rejects a negative or invisible device index (InvalidArgument) and a
// missing driver or GPU, or a GPU older than sm_100 (RuntimeFailure). One
// attribute query on the good path: cudaGetDeviceProperties fills every
// property through the driver and took milliseconds (at times over 100 ms)
// per call.
inline void check_device(int device) {
  if (device < 0) throw InvalidArgument("device must be a nonnegative visible GPU index");
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    const char* why = e == cudaSuccess ? "no devices" : cudaGetErrorString(e);
    throw RuntimeFailure("CUDA: no usable GPU is visible (" +
                         std::string(why ? why : std::to_string(int(e))) +
                         "). Check the NVIDIA driver and CUDA_VISIBLE_DEVICES.");
  }
  if (device >= count)
    throw InvalidArgument("device " + std::to_string(device) + " is out of range; " +
                          std::to_string(count) + " GPU(s) are visible through CUDA_VISIBLE_DEVICES");
  int major = 0;
  check(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device), "cudaDeviceGetAttribute");
  if (major < 10) {
    cudaDeviceProp p{};
    check(cudaGetDeviceProperties(&p, device), "cudaGetDeviceProperties");
    throw RuntimeFailure("this build targets sm_100a (B200); device " + std::to_string(device) +
                         " (" + p.name + ") has compute capability " + std::to_string(p.major) +
                         "." + std::to_string(p.minor));
  }
}

// Keeps a device's primary context retained while its owner lives.
class PrimaryContext {
 public:
  explicit PrimaryContext(int device) : device_(device) {
    const Driver& d = driver();
    if (!d.ok) throw RuntimeFailure("CUDA driver entry points unavailable");
    if (d.init(0) != CUDA_SUCCESS) throw RuntimeFailure("cuInit failed");
    if (d.retain(&ctx_, device) != CUDA_SUCCESS) throw RuntimeFailure("cuDevicePrimaryCtxRetain failed");
  }
  PrimaryContext(const PrimaryContext&) = delete;
  PrimaryContext& operator=(const PrimaryContext&) = delete;
  ~PrimaryContext() { driver().release(device_); }
  CUcontext get() const { return ctx_; }

 private:
  int device_;
  CUcontext ctx_ = nullptr;
};

// Makes `target` current for its scope and puts the caller's context back on
// exit, whether or not the scope ends by an exception. If the switch itself
// fails, the caller's context was never changed.
class ContextGuard {
 public:
  explicit ContextGuard(CUcontext target) {
    const Driver& d = driver();
    if (d.get_current(&prev_) != CUDA_SUCCESS) throw RuntimeFailure("cuCtxGetCurrent failed");
    switched_ = prev_ != target;
    if (switched_ && d.set_current(target) != CUDA_SUCCESS) throw RuntimeFailure("cuCtxSetCurrent failed");
  }
  ContextGuard(const ContextGuard&) = delete;
  ContextGuard& operator=(const ContextGuard&) = delete;
  ~ContextGuard() {
    if (switched_) driver().set_current(prev_);
  }

 private:
  CUcontext prev_ = nullptr;
  bool switched_ = false;
};

// Device memory that only grows. A request larger than the block waits for
// the GPU work that may still read it (the event `last` and `stream`), frees
// it and allocates the request, plus min(request, 512 MB) of headroom when
// asked, so that a run of calls with growing sizes reallocates only a few
// times. On a failed allocation the buffer is left empty (and the error
// thrown), so that a later, smaller request can still succeed.
struct GrowingBuffer {
  void* ptr = nullptr;
  size_t size = 0;

  // Returns true when the block was reallocated: anything that captured its
  // address (a CUDA graph) must be rebuilt.
  bool reserve(size_t bytes, cudaEvent_t last, cudaStream_t stream, bool headroom, const char* what) {
    if (bytes <= size) return false;
    check(cudaEventSynchronize(last), "cudaEventSynchronize");
    check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    release();
    const size_t extra = headroom ? (bytes < (size_t(512) << 20) ? bytes : (size_t(512) << 20)) : 0;
    void* p = nullptr;
    check(cudaMalloc(&p, bytes + extra), what);
    ptr = p;
    size = bytes + extra;
    return true;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    size = 0;
  }
};

// One workspace per device, handed out by exclusive ownership.
//
// A Lease takes the device's idle workspace out of the cache (or builds one
// when there is none) and owns it until it ends; it then hands it back. While
// a lease of the current epoch holds or is building a device's workspace,
// other leases of that device wait; leases of other devices never do.
//
// clear() starts a new epoch: idle workspaces are destroyed at once, and a
// workspace that is in use (or being built) when clear() runs stays with its
// lease and is destroyed when that lease ends, instead of going back to the
// cache. A lease that starts after clear() no longer waits for leases of the
// old epoch: it builds a fresh workspace.
//
// Workspaces are built and destroyed outside the cache's lock (their
// constructors and destructors synchronise with the GPU).
template <class W>
class DeviceCache {
 public:
  using Factory = std::function<std::unique_ptr<W>(int)>;

  explicit DeviceCache(Factory make) : make_(std::move(make)) {}
  DeviceCache(const DeviceCache&) = delete;
  DeviceCache& operator=(const DeviceCache&) = delete;
  ~DeviceCache() { clear(); }

  class Lease {
   public:
    Lease(DeviceCache& cache, int device) : cache_(cache), device_(device) {
      std::unique_lock<std::mutex> lock(cache.mutex_);
      State& st = cache.state_[device];
      // Wait while a lease of the current epoch owns this device.
      cache.changed_.wait(lock, [&] { return !(st.held && st.held_epoch == cache.epoch_); });
      epoch_ = cache.epoch_;
      st.held = true;
      st.held_epoch = epoch_;
      ws_ = std::move(st.idle);
      if (ws_) return;
      lock.unlock();
      try {
        ws_ = cache.make_(device);
      } catch (...) {
        cache.release(device_, epoch_, nullptr);
        throw;
      }
      if (!ws_) {
        cache.release(device_, epoch_, nullptr);
        throw RuntimeFailure("workspace construction returned nothing");
      }
    }
    Lease(const Lease&) = delete;
    Lease& operator=(const Lease&) = delete;
    ~Lease() { cache_.release(device_, epoch_, std::move(ws_)); }
    W& get() const { return *ws_; }

   private:
    DeviceCache& cache_;
    int device_;
    uint64_t epoch_ = 0;
    std::unique_ptr<W> ws_;
  };

  void clear() {
    std::vector<std::unique_ptr<W>> retired;
    {
      std::lock_guard<std::mutex> lock(mutex_);
      ++epoch_;
      for (auto& kv : state_)
        if (kv.second.idle) retired.push_back(std::move(kv.second.idle));
    }
    changed_.notify_all();
    // `retired` is destroyed here, outside the lock.
  }

  // Workspaces currently idle in the cache (for tests and diagnostics).
  int idle_count() {
    std::lock_guard<std::mutex> lock(mutex_);
    int n = 0;
    for (auto& kv : state_) n += kv.second.idle ? 1 : 0;
    return n;
  }

 private:
  struct State {
    std::unique_ptr<W> idle;     // the device's workspace while no lease holds it
    bool held = false;           // a lease holds or is building the workspace
    uint64_t held_epoch = 0;     // the epoch of that lease
  };

  // Ends a lease of `epoch` on `device`: its workspace goes back to the cache
  // if no clear() ran since the lease began; otherwise it is destroyed after
  // the lock is released.
  void release(int device, uint64_t epoch, std::unique_ptr<W> ws) {
    std::unique_ptr<W> retired;
    {
      std::lock_guard<std::mutex> lock(mutex_);
      State& st = state_[device];
      if (epoch == epoch_) {
        st.held = false;
        st.idle = std::move(ws);
      } else {
        retired = std::move(ws);
        if (st.held && st.held_epoch == epoch) st.held = false;
      }
    }
    changed_.notify_all();
  }

  Factory make_;
  std::mutex mutex_;
  std::condition_variable changed_;
  std::map<int, State> state_;
  uint64_t epoch_ = 0;
};

}  // namespace hv
