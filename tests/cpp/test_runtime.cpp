// Host-side fault injection for the engine's runtime
// (harvest_cuda_b200/csrc/hv_runtime.h), compiled against the fake CUDA
// headers in fake_cuda/ whose calls fail on demand: no GPU, no driver.
//
// Covers the reference's host tests in kind (tests/cpp/test_cuda_device.cpp,
// tests/cpp/test_workspace_cache.cpp): the device check (no devices, a
// driver error, compute capability below 10, bad indices), error messages,
// the primary context's reference count, the context guard restoring the
// caller's context on every path (nested guards, an exception in the scope,
// a failed query, a failed switch), the growing device buffer under an
// allocation failure, and the workspace cache: reuse, per-device waiting, a
// failed construction, clear() while idle, during use and during
// construction, destruction outside the lock, and 4 threads x 500 calls with
// clears in between.
//
// Usage: test_runtime            (everything that shares one process)
//        test_runtime no-driver  (driver entry points missing: a fresh
//                                 process, because they are resolved once)
#include "hv_runtime.h"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <future>
#include <string>
#include <thread>
#include <vector>

struct FakeCudaContext {
  int device;
};

namespace fake {
int device_count = 1;
cudaError_t count_status = cudaSuccess;
int major[4] = {10, 10, 10, 10};
int minor[4] = {0, 0, 0, 0};
int last_attribute_device = -1;
bool error_strings = true;
bool entry_points = true;
CUresult init_status = CUDA_SUCCESS;
bool fail_retain = false;
bool fail_get = false;
CUcontext fail_set = nullptr;
FakeCudaContext primary[4] = {{0}, {1}, {2}, {3}};
FakeCudaContext callers_own{-1};
CUcontext current = &callers_own;
int refs[4] = {0, 0, 0, 0};
std::vector<CUcontext> switches;
size_t malloc_limit = ~size_t(0);
long live_blocks = 0;
int syncs = 0;
}  // namespace fake

// ------------------------------------------------------------ fake runtime --
const char* cudaGetErrorName(cudaError_t e) {
  if (!fake::error_strings) return nullptr;
  switch (e) {
    case cudaSuccess: return "cudaSuccess";
    case cudaErrorMemoryAllocation: return "cudaErrorMemoryAllocation";
    case cudaErrorInsufficientDriver: return "cudaErrorInsufficientDriver";
    case cudaErrorNoDevice: return "cudaErrorNoDevice";
  }
  return "cudaErrorUnknown";
}
const char* cudaGetErrorString(cudaError_t e) {
  if (!fake::error_strings) return nullptr;
  switch (e) {
    case cudaSuccess: return "no error";
    case cudaErrorMemoryAllocation: return "out of memory";
    case cudaErrorInsufficientDriver: return "CUDA driver version is insufficient for CUDA runtime version";
    case cudaErrorNoDevice: return "no CUDA-capable device is detected";
  }
  return "unknown error";
}
cudaError_t cudaGetLastError(void) { return cudaSuccess; }
cudaError_t cudaGetDeviceCount(int* count) {
  *count = fake::count_status == cudaSuccess ? fake::device_count : 0;
  return fake::count_status;
}
cudaError_t cudaDeviceGetAttribute(int* value, cudaDeviceAttr attr, int device) {
  fake::last_attribute_device = device;
  *value = attr == cudaDevAttrComputeCapabilityMajor ? fake::major[device] : 148;
  return cudaSuccess;
}
cudaError_t cudaGetDeviceProperties(cudaDeviceProp* p, int device) {
  std::snprintf(p->name, sizeof p->name, "fake GPU %d", device);
  p->major = fake::major[device];
  p->minor = fake::minor[device];
  return cudaSuccess;
}
cudaError_t cudaMalloc(void** ptr, size_t bytes) {
  if (bytes > fake::malloc_limit) return cudaErrorMemoryAllocation;
  *ptr = std::malloc(1);
  ++fake::live_blocks;
  return cudaSuccess;
}
cudaError_t cudaFree(void* ptr) {
  if (ptr) {
    std::free(ptr);
    --fake::live_blocks;
  }
  return cudaSuccess;
}
cudaError_t cudaEventSynchronize(cudaEvent_t) { ++fake::syncs; return cudaSuccess; }
cudaError_t cudaStreamSynchronize(cudaStream_t) { ++fake::syncs; return cudaSuccess; }

CUresult cuInit(unsigned int) { return fake::init_status; }
CUresult cuDevicePrimaryCtxRetain(CUcontext* ctx, CUdevice device) {
  if (fake::fail_retain) return 1;
  ++fake::refs[device];
  *ctx = &fake::primary[device];
  return CUDA_SUCCESS;
}
CUresult cuDevicePrimaryCtxRelease(CUdevice device) {
  --fake::refs[device];
  return CUDA_SUCCESS;
}
CUresult cuCtxGetCurrent(CUcontext* ctx) {
  if (fake::fail_get) return 1;
  *ctx = fake::current;
  return CUDA_SUCCESS;
}
CUresult cuCtxSetCurrent(CUcontext ctx) {
  fake::switches.push_back(ctx);
  if (fake::fail_set && ctx == fake::fail_set) return 1;
  fake::current = ctx;
  return CUDA_SUCCESS;
}
cudaError_t cudaGetDriverEntryPoint(const char* symbol, void** fn, unsigned long long,
                                    cudaDriverEntryPointQueryResult* status) {
  *fn = nullptr;
  *status = cudaDriverEntryPointSymbolNotFound;
  if (!fake::entry_points) return cudaSuccess;
  const struct { const char* name; void* fn; } table[] = {
      {"cuInit", reinterpret_cast<void*>(&cuInit)},
      {"cuDevicePrimaryCtxRetain", reinterpret_cast<void*>(&cuDevicePrimaryCtxRetain)},
      {"cuDevicePrimaryCtxRelease", reinterpret_cast<void*>(&cuDevicePrimaryCtxRelease)},
      {"cuCtxGetCurrent", reinterpret_cast<void*>(&cuCtxGetCurrent)},
      {"cuCtxSetCurrent", reinterpret_cast<void*>(&cuCtxSetCurrent)},
  };
  for (const auto& e : table)
    if (!std::strcmp(symbol, e.name)) {
      *fn = e.fn;
      *status = cudaDriverEntryPointSuccess;
    }
  return cudaSuccess;
}

// ------------------------------------------------------------------ checks --
static int failures = 0;
#define EXPECT(cond)                                                         \
  do {                                                                       \
    if (!(cond)) {                                                           \
      ++failures;                                                            \
      std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
    }                                                                        \
  } while (0)

// The exception `body` throws, or "" when it returns; `kind` names its type.
template <class F>
std::string thrown(F&& body, std::string* kind = nullptr) {
  try {
    body();
  } catch (const hv::InvalidArgument& e) {
    if (kind) *kind = "InvalidArgument";
    return e.what();
  } catch (const hv::RuntimeFailure& e) {
    if (kind) *kind = "RuntimeFailure";
    return e.what();
  } catch (const std::exception& e) {
    if (kind) *kind = "other";
    return e.what();
  }
  if (kind) *kind = "";
  return "";
}
bool has(const std::string& s, const char* part) { return s.find(part) != std::string::npos; }

// Runs `body` on a thread and fails the whole program if it has not ended
// within `seconds` (a deadlock would otherwise hang the test).
template <class F>
void within(double seconds, F body, const char* what) {
  auto f = std::async(std::launch::async, body);
  if (f.wait_for(std::chrono::duration<double>(seconds)) != std::future_status::ready) {
    std::fprintf(stderr, "FAILED: %s did not finish within %.1f s\n", what, seconds);
    std::fflush(stderr);
    std::_Exit(3);
  }
  f.get();
}

// ------------------------------------------------------------ device check --
void test_device_check() {
  std::string kind;
  EXPECT(thrown([] { hv::check_device(0); }).empty());
  EXPECT(fake::last_attribute_device == 0);

  fake::major[0] = 9;
  fake::minor[0] = 0;
  std::string m = thrown([] { hv::check_device(0); }, &kind);
  EXPECT(kind == "RuntimeFailure" && has(m, "sm_100a") && has(m, "fake GPU 0") && has(m, "9.0"));
  fake::major[0] = 10;

  fake::device_count = 0;
  m = thrown([] { hv::check_device(0); }, &kind);
  EXPECT(kind == "RuntimeFailure" && has(m, "no usable GPU") && has(m, "CUDA_VISIBLE_DEVICES"));
  fake::device_count = 1;

  fake::count_status = cudaErrorInsufficientDriver;
  m = thrown([] { hv::check_device(0); }, &kind);
  EXPECT(kind == "RuntimeFailure" && has(m, "driver version is insufficient"));
  fake::error_strings = false;   // messages still carry the numeric code
  m = thrown([] { hv::check_device(0); }, &kind);
  EXPECT(kind == "RuntimeFailure" && has(m, "(35)"));
  fake::error_strings = true;
  fake::count_status = cudaSuccess;

  m = thrown([] { hv::check_device(-1); }, &kind);
  EXPECT(kind == "InvalidArgument" && has(m, "nonnegative"));
  m = thrown([] { hv::check_device(1); }, &kind);
  EXPECT(kind == "InvalidArgument" && has(m, "out of range"));

  // The capability check reads the requested device, not device 0.
  fake::device_count = 2;
  fake::major[0] = 8;
  EXPECT(thrown([] { hv::check_device(1); }).empty());
  EXPECT(fake::last_attribute_device == 1);
  m = thrown([] { hv::check_device(0); }, &kind);
  EXPECT(kind == "RuntimeFailure" && has(m, "device 0"));
  fake::major[0] = 10;
  fake::device_count = 1;
}

void test_error_messages() {
  std::string kind;
  std::string m = thrown([] { hv::check(cudaErrorMemoryAllocation, "cudaMalloc(workspace)"); }, &kind);
  EXPECT(kind == "RuntimeFailure" && has(m, "cudaMalloc(workspace)") && has(m, "cudaErrorMemoryAllocation") &&
         has(m, "GPU memory allocation failed"));
  m = thrown([] { hv::check(cudaErrorNoDevice, "query"); }, &kind);
  EXPECT(has(m, "CUDA_VISIBLE_DEVICES"));
  fake::error_strings = false;
  m = thrown([] { hv::check(cudaErrorMemoryAllocation, "cudaMalloc"); }, &kind);
  EXPECT(has(m, "CUDA: cudaMalloc: 2"));
  fake::error_strings = true;
  EXPECT(thrown([] { hv::check(cudaSuccess, "fine"); }).empty());
}

// ---------------------------------------------------------------- contexts --
void test_contexts() {
  CUcontext own = &fake::callers_own;
  CUcontext p0 = &fake::primary[0], p2 = &fake::primary[2];
  fake::current = own;
  fake::switches.clear();
  {
    hv::PrimaryContext owner(0);
    EXPECT(fake::refs[0] == 1 && fake::current == own && owner.get() == p0);
    {
      hv::ContextGuard guard(owner.get());
      EXPECT(fake::current == p0);
      {
        hv::PrimaryContext other(2);
        hv::ContextGuard nested(other.get());
        EXPECT(fake::current == p2);
      }
      EXPECT(fake::current == p0 && fake::refs[2] == 0);
    }
    EXPECT(fake::current == own);
    EXPECT((fake::switches == std::vector<CUcontext>{p0, p2, p0, own}));

    // An exception inside the guarded scope still restores the caller's context.
    fake::switches.clear();
    std::string m = thrown([&] {
      hv::ContextGuard guard(p0);
      hv::check(cudaErrorMemoryAllocation, "cudaMalloc(workspace)");
    });
    EXPECT(has(m, "GPU memory allocation failed"));
    EXPECT(fake::current == own && (fake::switches == std::vector<CUcontext>{p0, own}));

    // Already current: no switch at all.
    fake::switches.clear();
    fake::current = p0;
    { hv::ContextGuard guard(p0); }
    EXPECT(fake::switches.empty() && fake::current == p0);

    // No context current: restored to none.
    fake::current = nullptr;
    { hv::ContextGuard guard(p0); }
    EXPECT(fake::current == nullptr && (fake::switches == std::vector<CUcontext>{p0, nullptr}));

    // A failed query throws before any switch.
    fake::switches.clear();
    fake::current = own;
    fake::fail_get = true;
    m = thrown([&] { hv::ContextGuard guard(p0); });
    EXPECT(has(m, "cuCtxGetCurrent") && fake::current == own && fake::switches.empty());
    fake::fail_get = false;

    // A failed switch throws and leaves the caller's context current.
    fake::fail_set = p0;
    m = thrown([&] { hv::ContextGuard guard(p0); });
    EXPECT(has(m, "cuCtxSetCurrent") && fake::current == own &&
           (fake::switches == std::vector<CUcontext>{p0}));
    fake::fail_set = nullptr;
  }
  EXPECT(fake::refs[0] == 0);

  fake::fail_retain = true;
  std::string m = thrown([] { hv::PrimaryContext owner(0); });
  EXPECT(has(m, "cuDevicePrimaryCtxRetain") && fake::refs[0] == 0);
  fake::fail_retain = false;

  fake::init_status = 3;
  m = thrown([] { hv::PrimaryContext owner(0); });
  EXPECT(has(m, "cuInit") && fake::refs[0] == 0);
  fake::init_status = CUDA_SUCCESS;
}

// ------------------------------------------------------------ device memory --
void test_growing_buffer() {
  hv::GrowingBuffer b;
  fake::syncs = 0;
  EXPECT(b.reserve(100, nullptr, nullptr, true, "cudaMalloc(workspace)"));
  EXPECT(b.ptr && b.size == 200 && fake::live_blocks == 1 && fake::syncs == 2);
  EXPECT(!b.reserve(150, nullptr, nullptr, true, "cudaMalloc(workspace)"));   // fits: nothing moves
  EXPECT(fake::syncs == 2);
  // Headroom is capped at 512 MB.
  EXPECT(b.reserve(size_t(2) << 30, nullptr, nullptr, true, "cudaMalloc(workspace)"));
  EXPECT(b.size == (size_t(2) << 30) + (size_t(512) << 20) && fake::live_blocks == 1);
  // Growth fails: the old block is gone, the buffer is empty, the error says so.
  fake::malloc_limit = size_t(3) << 30;
  std::string kind;
  std::string m = thrown([&] { b.reserve(size_t(4) << 30, nullptr, nullptr, true, "cudaMalloc(workspace)"); },
                         &kind);
  EXPECT(kind == "RuntimeFailure" && has(m, "cudaMalloc(workspace)") && has(m, "GPU memory allocation failed"));
  EXPECT(b.ptr == nullptr && b.size == 0 && fake::live_blocks == 0);
  // A later request that fits is served.
  EXPECT(b.reserve(1000, nullptr, nullptr, false, "cudaMalloc(metrics)"));
  EXPECT(b.ptr && b.size == 1000 && fake::live_blocks == 1);
  fake::malloc_limit = ~size_t(0);
  b.release();
  EXPECT(fake::live_blocks == 0 && b.size == 0);
}

// ---------------------------------------------------------- workspace cache --
struct FakeWorkspace;
std::atomic<int> live[2];
std::atomic<int> built{0};
std::function<void()> on_build, on_destroy;

struct FakeWorkspace {
  int device, id;
  std::atomic<int> users{0};
  FakeWorkspace(int d, int i) : device(d), id(i) { ++live[d]; }
  ~FakeWorkspace() {
    --live[device];
    if (on_destroy) on_destroy();
  }
};

using Cache = hv::DeviceCache<FakeWorkspace>;
std::unique_ptr<FakeWorkspace> build_workspace(int device) {
  if (device < 0 || device >= 2) throw hv::InvalidArgument("device out of range");
  if (on_build) on_build();
  return std::make_unique<FakeWorkspace>(device, ++built);
}

void test_cache_reuse_and_waiting() {
  Cache cache(build_workspace);
  int first;
  { Cache::Lease a(cache, 0); first = a.get().id; }
  within(5, [&] {
    { Cache::Lease a(cache, 0); EXPECT(a.get().id == first); }
    { Cache::Lease b(cache, 1); EXPECT(b.get().device == 1); }
    { Cache::Lease a(cache, 0); EXPECT(a.get().id == first); }
  }, "reuse from another thread");
  EXPECT(live[0] == 1 && live[1] == 1 && cache.idle_count() == 2);
  std::string kind;
  thrown([&] { Cache::Lease bad(cache, 2); }, &kind);
  EXPECT(kind == "InvalidArgument");

  // A second call on a busy device waits for it; other devices do not wait.
  std::promise<void> started;
  std::future<int> waiting;
  {
    Cache::Lease holder(cache, 0);
    waiting = std::async(std::launch::async, [&] {
      started.set_value();
      Cache::Lease second(cache, 0);
      return second.get().id;
    });
    started.get_future().wait();
    EXPECT(waiting.wait_for(std::chrono::milliseconds(100)) == std::future_status::timeout);
    within(5, [&] { Cache::Lease other(cache, 1); EXPECT(other.get().device == 1); }, "other device");
  }
  EXPECT(waiting.get() == first && live[0] == 1);

  // clear() with nothing in use destroys every idle workspace at once.
  within(5, [&] { cache.clear(); }, "clear from another thread");
  EXPECT(live[0] == 0 && live[1] == 0 && cache.idle_count() == 0);
  { Cache::Lease a(cache, 0); EXPECT(a.get().id != first); }
  cache.clear();
  EXPECT(live[0] == 0);
}

void test_cache_failed_build() {
  Cache cache(build_workspace);
  // Construction fails (an allocation failure on the GPU): the error reaches
  // the caller, nothing is cached, and the device is not left busy.
  on_build = [] { hv::check(cudaErrorMemoryAllocation, "cudaMalloc(twiddles)"); };
  std::string m = thrown([&] { Cache::Lease a(cache, 0); });
  EXPECT(has(m, "GPU memory allocation failed") && live[0] == 0 && cache.idle_count() == 0);
  on_build = {};
  within(5, [&] { Cache::Lease a(cache, 0); EXPECT(a.get().device == 0); }, "lease after a failed build");
  EXPECT(live[0] == 1 && cache.idle_count() == 1);

  // A call that fails while it holds the workspace (under a context guard)
  // restores the caller's context and returns the workspace to the cache.
  CUcontext own = &fake::callers_own;
  fake::current = own;
  m = thrown([&] {
    Cache::Lease a(cache, 0);
    hv::PrimaryContext ctx(0);
    hv::ContextGuard guard(ctx.get());
    hv::GrowingBuffer arena;
    fake::malloc_limit = 10;
    arena.reserve(1 << 20, nullptr, nullptr, true, "cudaMalloc(workspace)");
  });
  fake::malloc_limit = ~size_t(0);
  EXPECT(has(m, "cudaMalloc(workspace)") && fake::current == own && fake::refs[0] == 0);
  EXPECT(live[0] == 1 && cache.idle_count() == 1 && fake::live_blocks == 0);
  cache.clear();
  EXPECT(live[0] == 0);
}

void test_cache_clear_during_use() {
  Cache cache(build_workspace);
  int newer_id = -1;
  {
    Cache::Lease in_use(cache, 0);
    FakeWorkspace* old = &in_use.get();
    within(5, [&] { cache.clear(); }, "clear during use");
    // The call in flight keeps its workspace.
    EXPECT(live[0] == 1 && in_use.get().device == 0 && &in_use.get() == old);
    // A call after clear() does not wait for it and gets a new workspace.
    within(5, [&] {
      Cache::Lease newer(cache, 0);
      EXPECT(&newer.get() != old);
      newer_id = newer.get().id;
    }, "lease after clear");
    EXPECT(live[0] == 2);
  }
  // The old call cannot put its workspace back into a cleared cache: the
  // cached workspace is the newer one.
  EXPECT(live[0] == 1 && cache.idle_count() == 1);
  { Cache::Lease again(cache, 0); EXPECT(again.get().id == newer_id); }
  cache.clear();
  EXPECT(live[0] == 0);

  // Destroying workspaces does not hold the cache's lock.
  { Cache::Lease a(cache, 0); }
  on_destroy = [&] { cache.clear(); };
  within(5, [&] { cache.clear(); }, "clear from a workspace destructor");
  on_destroy = {};
  EXPECT(live[0] == 0);
}

void test_cache_clear_during_build() {
  Cache cache(build_workspace);
  std::promise<void> building, proceed;
  auto resume = proceed.get_future().share();
  std::atomic<bool> hold_first{true};
  on_build = [&] {   // the first build blocks until told to go on
    if (hold_first.exchange(false)) {
      building.set_value();
      resume.wait();
    }
  };
  auto worker = std::async(std::launch::async, [&] { Cache::Lease a(cache, 0); });
  building.get_future().wait();
  within(5, [&] { cache.clear(); }, "clear during a build");
  // A lease after the clear does not wait for the build of the old epoch.
  int newer_id = -1;
  within(5, [&] { Cache::Lease b(cache, 0); newer_id = b.get().id; }, "lease while an old-epoch build runs");
  proceed.set_value();
  worker.get();
  on_build = {};
  // The workspace built across the clear was not cached; the newer one was.
  EXPECT(live[0] == 1 && cache.idle_count() == 1);
  { Cache::Lease again(cache, 0); EXPECT(again.get().id == newer_id); }
  cache.clear();
  EXPECT(live[0] == 0);
}

void test_cache_threads() {
  Cache cache(build_workspace);
  std::atomic<int> overlap{0};
  std::vector<std::future<void>> workers;
  for (int w = 0; w < 4; ++w)
    workers.push_back(std::async(std::launch::async, [&, w] {
      for (int call = 0; call < 500; ++call) {
        Cache::Lease lease(cache, w % 2);
        FakeWorkspace& ws = lease.get();
        if (ws.device != w % 2) ++overlap;
        if (++ws.users != 1) ++overlap;   // one call per workspace at a time
        if (call % 17 == 0) cache.clear();
        std::this_thread::yield();
        --ws.users;
      }
    }));
  within(60, [&] { for (auto& f : workers) f.get(); }, "4 threads x 500 calls");
  EXPECT(overlap == 0);
  EXPECT(live[0] <= 1 && live[1] <= 1);
  cache.clear();
  EXPECT(live[0] == 0 && live[1] == 0);
}

int main(int argc, char** argv) {
  if (argc > 1 && !std::strcmp(argv[1], "no-driver")) {
    fake::entry_points = false;
    std::string m = thrown([] { hv::PrimaryContext owner(0); });
    EXPECT(has(m, "driver entry points unavailable") && fake::refs[0] == 0);
  } else {
    test_device_check();
    test_error_messages();
    test_contexts();
    test_growing_buffer();
    test_cache_reuse_and_waiting();
    test_cache_failed_build();
    test_cache_clear_during_use();
    test_cache_clear_during_build();
    test_cache_threads();
    EXPECT(live[0] == 0 && live[1] == 0);
  }
  if (failures) {
    std::fprintf(stderr, "%d check(s) failed\n", failures);
    return 1;
  }
  std::printf("runtime host tests passed (%s)\n", argc > 1 ? argv[1] : "all");
  return 0;
}
