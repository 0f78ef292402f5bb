// Host engine and C ABI of the B200 Harvest engine.
//
//   * validation identical to the reference's bindings (src/bindings.cpp:18-39);
//   * the per-device workspace cache, device check and context handling of
//     hv_runtime.h;
//   * batch planning (parameters of src/engine.cpp:255-266 per clip), one
//     device arena per workspace, and the launch sequence of the stages,
//     captured once per batch shape into a CUDA graph and replayed.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "harvest_b200.h"
#include "hv_runtime.h"
#include "hv_stages.cuh"

namespace hv {
namespace {

// ---------------------------------------------------------------- errors --
thread_local std::string g_error;
thread_local double g_stage_ms[HV_STAGE_COUNT] = {};
thread_local int g_tuning[3] = {0, 0, 0};   // refinement shape of the last call, and whether it tuned

template <class F>
int guarded(F&& body) {
  try {
    body();
    g_error.clear();
    return HV_OK;
  } catch (const InvalidArgument& e) {
    g_error = e.what();
    return HV_INVALID_ARGUMENT;
  } catch (const std::bad_alloc&) {
    g_error = "host memory allocation failed";
    return HV_RUNTIME_ERROR;
  } catch (const std::exception& e) {
    g_error = e.what();
    return HV_RUNTIME_ERROR;
  }
}

// ------------------------------------------------------------- WORLD maths --
constexpr double kLog2 = 0.69314718055994529;  // world::kLog2

int matlab_round_host(double v) { return v > 0 ? static_cast<int>(v + 0.5) : static_cast<int>(v - 0.5); }
int suitable_fft_size(int samples) {  // common.cpp:51-54
  return static_cast<int>(std::pow(2.0, static_cast<int>(std::log(static_cast<double>(samples)) / kLog2) + 1.0));
}
int samples_for(int fs, int64_t n, double period) {  // harvest.cpp:1219-1221
  return static_cast<int>(1000.0 * n / fs / period) + 1;
}
int ratio_for(int fs) { return std::min(12, std::max(1, matlab_round_host(fs / 8000.0))); }

// FilterForDecimate coefficients (matlabfunctions.cpp:27-113), rows by ratio.
const double kLowA[13][3] = {
    {0, 0, 0}, {0, 0, 0},
    {0.041156734567757189, -0.42599112459189636, 0.041037215479961225},
    {0.95039378983237421, -0.67429146741526791, 0.15412211621346475},
    {1.4499664446880227, -0.98943497080950582, 0.24578252340690215},
    {1.7610939654280557, -1.2554914843859768, 0.3237186507788215},
    {1.9715352749512141, -1.4686795689225347, 0.3893908434965701},
    {2.1225239019534703, -1.6395144861046302, 0.44469707800587366},
    {2.2357462340187593, -1.7780899984041358, 0.49152555365968692},
    {2.3236003491759578, -1.8921545617463598, 0.53148928133729068},
    {2.3936475118069387, -1.9873904075111861, 0.5658879979027055},
    {2.450743295230728, -2.06794904601978, 0.59574774438332101},
    {2.4981398605924205, -2.1368928194784025, 0.62187513816221485}};
const double kLowB[13][2] = {
    {0, 0}, {0, 0},
    {0.16797464681802227, 0.50392394045406674},
    {0.071221945171178636, 0.21366583551353591},
    {0.036710750339322612, 0.11013225101796784},
    {0.021334858522387423, 0.06400457556716227},
    {0.013469181309343825, 0.040407543928031475},
    {0.0090366882681608418, 0.027110064804482525},
    {0.0063522763407111993, 0.019056829022133598},
    {0.0046331164041389372, 0.013899349212416812},
    {0.0034818622251927556, 0.010445586675578267},
    {0.0026822508007163792, 0.0080467524021491377},
    {0.0021097275904709001, 0.0063291827714127002}};

// validate() of the reference (src/bindings.cpp:18-39), per clip.
void validate_settings(int64_t n, int fs, double floor, double ceil, double period) {
  if (n <= 0 || n > INT_MAX) throw InvalidArgument("x must be nonempty and contain at most INT_MAX samples");
  if (fs < 8000 || fs > 192000) throw InvalidArgument("fs must be between 8000 and 192000 Hz");
  if (!std::isfinite(floor) || !std::isfinite(ceil) || floor <= 0 || ceil <= floor)
    throw InvalidArgument("require finite 0 < f0_floor < f0_ceil");
  int ratio = std::min(12, std::max(1, int(fs / 8000.0 + 0.5)));
  if (n < int64_t(2) * ratio)
    throw InvalidArgument("x is too short: require at least two samples after internal decimation");
  if (ceil >= double(fs) / ratio / 2) throw InvalidArgument("f0_ceil must be below the internal Nyquist frequency");
  if (!std::isfinite(period) || period <= 0)
    throw InvalidArgument("frame_period must be finite and positive (milliseconds)");
  if (1000.0 * n / fs / period >= INT_MAX || 1000.0 * n / fs >= INT_MAX ||
      double(n) / ratio + 10.0 * fs / ratio / floor >= (1 << 28))
    throw InvalidArgument("input or analysis settings exceed supported allocation sizes");
}
void validate_samples(const double* x, int64_t n) {
  bool finite = true;
  for (int64_t i = 0; i < n; ++i) finite &= std::isfinite(x[i]);
  if (!finite) throw InvalidArgument("x must contain only finite samples");
}

// ------------------------------------------------------------------- plan --
struct Settings {
  int fs;
  double floor, ceil, period;
  bool operator<(const Settings& o) const {
    return std::tie(fs, floor, ceil, period) < std::tie(o.fs, o.floor, o.ceil, o.period);
  }
};

// Band-bank tables for one (fs, floor, ceil): centres, half lengths and the
// reversed, padded taps of GetFilteredSignal (harvest.cpp:101-108) computed
// with the host's libm exactly as the reference does.
struct BankTables {
  int bands = 0, max_pad_taps = 0, max_half = 0;
  std::vector<double> centre;
  std::vector<int> half;
  std::vector<int64_t> tap_off;
  std::vector<double> taps_rev;
};

// Band-pass channels of HarvestGeneralBody (harvest.cpp:1161-1162): 40 per
// octave between 0.9 f0_floor and 1.1 f0_ceil.
int band_count(double floor, double ceil) {
  const double lo = floor * 0.9, hi = ceil * 1.1;
  return 1 + static_cast<int>(std::log(hi / lo) / kLog2 * 40.0);
}

BankTables make_bank(int fs, double floor, double ceil) {
  BankTables t;
  const int ratio = ratio_for(fs);
  const double fs_r = double(fs) / ratio;
  const double lo = floor * 0.9;
  t.bands = band_count(floor, ceil);
  const int mult = band_bank_tap_multiple();
  t.tap_off.push_back(0);
  for (int b = 0; b < t.bands; ++b) {
    double c = lo * std::pow(2.0, (b + 1) / 40.0);
    int h = matlab_round_host(fs_r / c * 2.0);
    int len = 2 * h + 1;
    std::vector<double> taps(len);
    for (int i = 0; i < len; ++i) {
      double tmp = i / (len - 1.0);
      taps[i] = 0.355768 - 0.487396 * std::cos(2.0 * kPi * tmp) + 0.144232 * std::cos(4.0 * kPi * tmp) -
                0.012604 * std::cos(6.0 * kPi * tmp);
    }
    for (int i = -h; i <= h; ++i) taps[i + h] *= std::cos(2 * kPi * c * i / fs_r);
    int padded = (len + mult - 1) / mult * mult;
    for (int j = 0; j < padded; ++j) t.taps_rev.push_back(j < len ? taps[len - 1 - j] : 0.0);
    t.tap_off.push_back(t.tap_off.back() + padded);
    t.centre.push_back(c);
    t.half.push_back(h);
    t.max_pad_taps = std::max(t.max_pad_taps, padded);
    t.max_half = std::max(t.max_half, h);
  }
  return t;
}

struct Plan {
  Settings s;
  std::vector<int64_t> lengths;
  int clips = 0, ratio = 1, bands = 0, capacity = 0, per_group = 0, lag = 0;
  double fs_r = 0;
  std::shared_ptr<const BankTables> bank;
  // Host copies of the per-clip tables.
  std::vector<int64_t> x_off, y_off, t_off, seg_off, frame_off, out_off, scratch_off;
  std::vector<int64_t> dc_off;   // the DC removal's chunks per clip (kDcChunk samples of y each)
  std::vector<int> nfft;
  std::vector<int2> items;
  int64_t slot_capacity = 0, total_seg = 0;
  double trans[9];
  // FFT band bank (overlap-save blocks), used unless the filters are too long.
  bool use_fft = false;
  int fft_valid = 0;
  std::vector<int64_t> blk_off;
  int64_t total_blocks = 0;
  // Per-plan tables (offsets, work items, block offsets), uploaded to the
  // head of the arena by Workspace::prepare when another plan used it last.
  uint64_t id = 0;
  std::vector<char> meta;
  size_t o_x = 0, o_y = 0, o_t = 0, o_s = 0, o_f = 0, o_o = 0, o_sc = 0, o_n = 0, o_it = 0, o_bo = 0, o_dc = 0;
  size_t arena_bytes = 0;
  struct Layout {
    size_t meta, pcm, x, u, states, y, bins, queue, flag, slots, spectra, raw, cand, count, jobs, classes, refined, scores,
        pruned, pruned_scores, best, smoothed, scratch, f0, times, grad_y, grad_fixed, keys, leaders, item_off,
        dc_parts;
  } at{};
  int bank_ctas = 0;
  // Device pointers, set by Workspace::prepare: into the arena's copy of
  // `meta`, and into the workspace's device copy of the band tables.
  int64_t *d_x_off, *d_y_off, *d_t_off, *d_seg_off, *d_frame_off, *d_out_off, *d_scratch_off, *d_tap_off;
  int* d_nfft;
  int* d_half;
  double *d_centre, *d_taps;
  int2* d_items;
  int64_t* d_blk_off = nullptr;
  int64_t* d_dc_off = nullptr;
  double* filters = nullptr;   // [bands][4097] filter amplitudes of the FFT bank
  // Refinement launch shape and contour extension blocks per clip, chosen by
  // the autotuner on the plan's first run (extend_blocks 0: the default).
  RefineShape refine_shape;
  int extend_blocks = 0;
  bool tuned = false;
  // contour_finish's block size: 512 when the batch has fewer clips than
  // the GPU has SMs (a block per clip), else 256.
  int contour_threads = 256;
  // Captured launch sequence for this plan at a given arena base.
  cudaGraphExec_t graph = nullptr;
  void* graph_arena = nullptr;
  ~Plan() {
    if (graph) cudaGraphExecDestroy(graph);
  }
};

// Device copy of one (fs, f0_floor, f0_ceil)'s band tables and, once the FFT
// bank needs them, its filter spectra; shared by every plan with those
// settings, so that planning a new batch shape allocates nothing on the device.
struct DeviceBank {
  void* tables = nullptr;
  double* filters = nullptr;        // [bands][block / 2 + 1] real amplitudes
  double* centre = nullptr;
  int* half = nullptr;
  int64_t* tap_off = nullptr;
  double* taps = nullptr;
  DeviceBank() = default;
  DeviceBank(const DeviceBank&) = delete;
  DeviceBank& operator=(const DeviceBank&) = delete;
  ~DeviceBank() {
    if (tables) cudaFree(tables);
    if (filters) cudaFree(filters);
  }
};

constexpr int kSegment = 256;   // decimation scan segment length

// Edge padding of GetWaveformAndSpectrumSub (harvest.cpp:50-51): ceil(140 / r) r samples.
constexpr int decimation_lag(int ratio) { return (140 + ratio - 1) / ratio * ratio; }

void mat3_mul(const double* a, const double* b, double* out) {
  double r[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
  std::memcpy(out, r, sizeof r);
}

size_t align_up(size_t v) { return (v + 255) / 256 * 256; }

// ------------------------------------------------------------- workspace --
struct Workspace {
  int device;
  PrimaryContext ctx;
  cudaStream_t stream = nullptr;
  cudaEvent_t marks[HV_STAGE_COUNT + 1] = {};
  cudaEvent_t last = nullptr;  // completion of the previous call's work
  cudaEvent_t fork = nullptr, join = nullptr;   // the backward pass's side branch on `stream`
  GrowingBuffer arena;          // the plans' device arena
  int sms = 0;
  double2* twiddles = nullptr;  // e^{-2 pi i t / 8192}, t < 8192
  int* host_flag = nullptr;      // pinned word for the non-finite-sample flag
  std::map<Settings, std::shared_ptr<const BankTables>> banks;
  // Autotuned refinement shapes by (fs, f0_floor, f0_ceil, log2 of the
  // batch's total samples).
  struct Tuning {
    RefineShape refine;
    int extend_blocks;
  };
  std::map<std::tuple<int, double, double, int, int>, Tuning> tuned_shapes;
  std::list<std::unique_ptr<Plan>> plans;  // most recent first
  std::map<Settings, std::unique_ptr<DeviceBank>> device_banks;
  uint64_t next_plan_id = 1;
  uint64_t meta_owner = 0;   // plan whose tables are at the head of the arena
  GrowingBuffer metric_buf;     // inputs and offsets of hv_compare_batch
  GrowingBuffer raw_buf;        // band-bank dump and adjoint scratch of the per-band-candidate gradient
  GrowingBuffer contour_buf;    // tables, copies and scratch of hv_contour_batch

  explicit Workspace(int dev) : device(dev), ctx(dev) {
    ContextGuard g(ctx.get());
    check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto& e : marks) check(cudaEventCreate(&e), "cudaEventCreate");
    check(cudaEventCreateWithFlags(&last, cudaEventDisableTiming), "cudaEventCreate");
    check(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "cudaEventCreate");
    check(cudaEventCreateWithFlags(&join, cudaEventDisableTiming), "cudaEventCreate");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    check(cudaMalloc(&twiddles, sizeof(double2) * fft_bank_block_length()), "cudaMalloc(twiddles)");
    check(cudaHostAlloc(reinterpret_cast<void**>(&host_flag), sizeof(int), cudaHostAllocDefault), "cudaHostAlloc");
    check(launch_twiddles(twiddles, stream), "twiddles");
    check(cudaStreamSynchronize(stream), "twiddles");
  }
  ~Workspace() {
    try {
      ContextGuard g(ctx.get());
      if (last) cudaEventSynchronize(last);
      if (stream) cudaStreamSynchronize(stream);
      plans.clear();
      device_banks.clear();
      arena.release();
      metric_buf.release();
      raw_buf.release();
      contour_buf.release();
      if (twiddles) cudaFree(twiddles);
      if (host_flag) cudaFreeHost(host_flag);
      for (auto& e : marks) if (e) cudaEventDestroy(e);
      if (last) cudaEventDestroy(last);
      if (fork) cudaEventDestroy(fork);
      if (join) cudaEventDestroy(join);
      if (stream) cudaStreamDestroy(stream);
    } catch (...) {
    }
  }

  void ensure_arena(size_t bytes) {
    if (bytes <= arena.size) return;
    // Graphs captured the old arena's addresses.
    for (auto& p : plans) {
      if (p->graph) { cudaGraphExecDestroy(p->graph); p->graph = nullptr; }
    }
    meta_owner = 0;
    arena.reserve(bytes, last, stream, true, "cudaMalloc(workspace)");
  }

  // The device band tables of `s`, with filter spectra when `spectra`.
  DeviceBank& device_bank(const Settings& s, const BankTables& bank, bool spectra) {
    Settings key{s.fs, s.floor, s.ceil, 0.0};
    auto it = device_banks.find(key);
    if (it == device_banks.end()) {
      if (device_banks.size() >= 16) {
        // Bounded: once the GPU is done, drop every bank and the graphs that
        // captured their addresses (plans take the pointers anew each call).
        check(cudaEventSynchronize(last), "cudaEventSynchronize");
        check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
        for (auto& q : plans)
          if (q->graph) { cudaGraphExecDestroy(q->graph); q->graph = nullptr; }
        device_banks.clear();
      }
      auto b = std::make_unique<DeviceBank>();
      std::vector<char> blob;
      auto put = [&](const void* src, size_t bytes) {
        size_t at = align_up(blob.size());
        blob.resize(at + bytes);
        if (bytes) std::memcpy(blob.data() + at, src, bytes);
        return at;
      };
      size_t o_c = put(bank.centre.data(), 8 * bank.centre.size());
      size_t o_h = put(bank.half.data(), 4 * bank.half.size());
      size_t o_to = put(bank.tap_off.data(), 8 * bank.tap_off.size());
      size_t o_tp = put(bank.taps_rev.data(), 8 * bank.taps_rev.size());
      check(cudaMalloc(&b->tables, blob.size()), "cudaMalloc(bank)");
      check(cudaMemcpy(b->tables, blob.data(), blob.size(), cudaMemcpyHostToDevice), "cudaMemcpy(bank)");
      char* m = static_cast<char*>(b->tables);
      b->centre = reinterpret_cast<double*>(m + o_c);
      b->half = reinterpret_cast<int*>(m + o_h);
      b->tap_off = reinterpret_cast<int64_t*>(m + o_to);
      b->taps = reinterpret_cast<double*>(m + o_tp);
      it = device_banks.emplace(key, std::move(b)).first;
    }
    DeviceBank& b = *it->second;
    if (spectra && !b.filters) {
      if (fft_bank_ctas_per_sm() < 1) throw RuntimeFailure("FFT band-bank kernel does not fit on this device");
      const int block = fft_bank_block_length();
      check(cudaMalloc(&b.filters, sizeof(double) * (block / 2 + 1) * bank.bands), "cudaMalloc(filters)");
      check(launch_filter_spectra(b.half, b.tap_off, b.taps, bank.bands, bank.max_half, twiddles, b.filters,
                                  stream),
            "filter_spectra");
      check(cudaStreamSynchronize(stream), "filter_spectra");
    }
    return b;
  }

  // Plan lookup, arena sizing, ordering after the previous call on `st`, and
  // the plan's tables at the head of the arena (uploaded only when another
  // plan used the arena last). Every entry point goes through here.
  Plan& prepare(const Settings& s, const int64_t* offsets, int clips, cudaStream_t st) {
    Plan& p = plan_for(s, offsets, clips);
    ensure_arena(p.arena_bytes);
    check(cudaStreamWaitEvent(st, last, 0), "cudaStreamWaitEvent");
    if (meta_owner != p.id) {
      check(cudaMemcpyAsync(ptr<char>(p.at.meta), p.meta.data(), p.meta.size(), cudaMemcpyHostToDevice, st),
            "cudaMemcpy(plan)");
      meta_owner = p.id;
    }
    char* m = ptr<char>(p.at.meta);
    p.d_x_off = reinterpret_cast<int64_t*>(m + p.o_x);
    p.d_y_off = reinterpret_cast<int64_t*>(m + p.o_y);
    p.d_t_off = reinterpret_cast<int64_t*>(m + p.o_t);
    p.d_seg_off = reinterpret_cast<int64_t*>(m + p.o_s);
    p.d_frame_off = reinterpret_cast<int64_t*>(m + p.o_f);
    p.d_out_off = reinterpret_cast<int64_t*>(m + p.o_o);
    p.d_scratch_off = reinterpret_cast<int64_t*>(m + p.o_sc);
    p.d_nfft = reinterpret_cast<int*>(m + p.o_n);
    p.d_items = reinterpret_cast<int2*>(m + p.o_it);
    p.d_blk_off = reinterpret_cast<int64_t*>(m + p.o_bo);
    p.d_dc_off = reinterpret_cast<int64_t*>(m + p.o_dc);
    DeviceBank& b = device_bank(s, *p.bank, p.use_fft);
    p.d_centre = b.centre;
    p.d_half = b.half;
    p.d_tap_off = b.tap_off;
    p.d_taps = b.taps;
    p.filters = b.filters;
    return p;
  }

  std::shared_ptr<const BankTables> bank_for(const Settings& s) {
    Settings key{s.fs, s.floor, s.ceil, 0.0};
    auto it = banks.find(key);
    if (it != banks.end()) return it->second;
    auto t = std::make_shared<const BankTables>(make_bank(s.fs, s.floor, s.ceil));
    if (banks.size() > 8) banks.clear();
    banks[key] = t;
    return t;
  }

  Plan& plan_for(const Settings& s, const int64_t* offsets, int clips) {
    std::vector<int64_t> lengths(clips);
    for (int c = 0; c < clips; ++c) lengths[c] = offsets[c + 1] - offsets[c];
    for (auto it = plans.begin(); it != plans.end(); ++it) {
      Plan& p = **it;
      if (p.s.fs == s.fs && p.s.floor == s.floor && p.s.ceil == s.ceil && p.s.period == s.period &&
          p.lengths == lengths) {
        plans.splice(plans.begin(), plans, it);
        return *plans.front();
      }
    }
    auto plan = build_plan(s, std::move(lengths));
    plans.push_front(std::move(plan));
    while (plans.size() > 8) plans.pop_back();
    return *plans.front();
  }

  std::unique_ptr<Plan> build_plan(const Settings& s, std::vector<int64_t> lengths) {
    auto p = std::make_unique<Plan>();
    p->s = s;
    p->lengths = std::move(lengths);
    const int B = p->clips = static_cast<int>(p->lengths.size());
    p->contour_threads = B < sms ? 512 : 256;
    p->ratio = ratio_for(s.fs);
    p->fs_r = double(s.fs) / p->ratio;
    p->bank = bank_for(s);
    p->bands = p->bank->bands;
    p->per_group = matlab_round_host(p->bands / 10.0);
    p->capacity = p->per_group * 7;
    if (p->capacity >= kRefineColumns)
      throw InvalidArgument("f0_floor/f0_ceil span too many band-pass channels");
    p->lag = decimation_lag(p->ratio);
    const double first = p->bank->centre[0];
    p->x_off.assign(B + 1, 0); p->y_off.assign(B + 1, 0); p->t_off.assign(B + 1, 0);
    p->seg_off.assign(B + 1, 0); p->frame_off.assign(B + 1, 0); p->out_off.assign(B + 1, 0);
    p->scratch_off.assign(B + 1, 0);
    p->dc_off.assign(B + 1, 0);
    p->nfft.assign(B, 0);
    for (int c = 0; c < B; ++c) {
      int64_t n = p->lengths[c];
      int y_len = static_cast<int>(std::ceil(double(n) / p->ratio));
      int64_t total = n + 2 * p->lag + 18;
      int frames = samples_for(s.fs, n, 1.0);
      p->x_off[c + 1] = p->x_off[c] + n;
      p->y_off[c + 1] = p->y_off[c] + y_len;
      p->dc_off[c + 1] = p->dc_off[c] + dc_chunk_count(y_len);
      p->t_off[c + 1] = p->t_off[c] + (p->ratio > 1 ? total : 0);
      p->seg_off[c + 1] = p->seg_off[c] + (p->ratio > 1 ? (total + kSegment - 1) / kSegment : 0);
      p->frame_off[c + 1] = p->frame_off[c] + frames;
      p->out_off[c + 1] = p->out_off[c] + samples_for(s.fs, n, s.period);
      p->scratch_off[c + 1] = p->scratch_off[c] + contour_scratch(frames, p->contour_threads);
      p->nfft[c] = suitable_fft_size(y_len + 5 + 2 * static_cast<int>(2.0 * p->fs_r / first));
      p->slot_capacity = std::max<int64_t>(p->slot_capacity, y_len / 2 + 2);
    }
    p->total_seg = p->seg_off[B];
    const BankTables& bank = *p->bank;
    // The FFT bank needs its overlap (2 H + 2) to fit in half a block; the
    // direct FIR covers longer filters. HARVEST_B200_BANK=fir|fft overrides.
    const int block = fft_bank_block_length();
    p->use_fft = 2 * bank.max_half + 2 <= block / 2;
    if (const char* force = std::getenv("HARVEST_B200_BANK")) {
      if (!std::strcmp(force, "fir")) p->use_fft = false;
      if (!std::strcmp(force, "fft") && 2 * bank.max_half + 2 < block) p->use_fft = true;
    }
    p->blk_off.assign(B + 1, 0);
    if (p->use_fft) {
      p->fft_valid = block - 2 - 2 * bank.max_half;
      for (int c = 0; c < B; ++c) {
        int64_t positions = p->y_off[c + 1] - p->y_off[c] - 1;   // event positions 0..y_len-2
        p->blk_off[c + 1] = p->blk_off[c] + (positions + p->fft_valid - 1) / p->fft_valid;
      }
      p->total_blocks = p->blk_off[B];
    }
    // Work items longest first.
    std::vector<std::pair<int64_t, int2>> items;
    items.reserve(size_t(B) * p->bands);
    for (int c = 0; c < B; ++c)
      for (int b = 0; b < p->bands; ++b) {
        int64_t y_len = p->y_off[c + 1] - p->y_off[c];
        int64_t taps = bank.tap_off[b + 1] - bank.tap_off[b];
        int64_t cost = p->use_fft ? (p->blk_off[c + 1] - p->blk_off[c]) : y_len * (taps + 16);
        items.push_back({cost, make_int2(c, b)});
      }
    std::stable_sort(items.begin(), items.end(),
                     [](const auto& a, const auto& b) { return a.first > b.first; });
    for (auto& it : items) p->items.push_back(it.second);
    // A^S for the decimation scan.
    if (p->ratio > 1) {
      const double* a = kLowA[p->ratio];
      double A[9] = {a[0], a[1], a[2], 1, 0, 0, 0, 1, 0};
      double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
      for (int e = kSegment; e; e >>= 1) {
        if (e & 1) mat3_mul(R, A, R);
        mat3_mul(A, A, A);
      }
      std::memcpy(p->trans, R, sizeof R);
    }
    // Per-plan tables, uploaded to the head of the arena by prepare().
    p->id = next_plan_id++;
    auto put = [&](const void* src, size_t bytes) {
      size_t at = align_up(p->meta.size());
      p->meta.resize(at + bytes);
      if (bytes) std::memcpy(p->meta.data() + at, src, bytes);
      return at;
    };
    p->o_x = put(p->x_off.data(), 8 * (B + 1));
    p->o_y = put(p->y_off.data(), 8 * (B + 1));
    p->o_t = put(p->t_off.data(), 8 * (B + 1));
    p->o_s = put(p->seg_off.data(), 8 * (B + 1));
    p->o_f = put(p->frame_off.data(), 8 * (B + 1));
    p->o_o = put(p->out_off.data(), 8 * (B + 1));
    p->o_sc = put(p->scratch_off.data(), 8 * (B + 1));
    p->o_n = put(p->nfft.data(), 4 * B);
    p->o_it = put(p->items.data(), sizeof(int2) * p->items.size());
    p->o_bo = put(p->blk_off.data(), 8 * (B + 1));
    p->o_dc = put(p->dc_off.data(), 8 * (B + 1));
    if (p->use_fft && fft_bank_ctas_per_sm() < 1)
      throw RuntimeFailure("FFT band-bank kernel does not fit on this device");
    // Arena layout.
    int per_sm = p->use_fft ? fft_bank_ctas_per_sm() : band_bank_ctas_per_sm(bank.max_pad_taps);
    if (per_sm < 1) throw RuntimeFailure("band-bank kernel does not fit on this device");
    int items_n = static_cast<int>(p->items.size());
    p->bank_ctas = std::max(1, std::min(items_n, sms * per_sm));
    const int64_t F = p->frame_off[B];
    if (F >= (int64_t(1) << kJobSiblingShift) / kRefineColumns)
      throw InvalidArgument("batch too long: more than 2^31 analysis frames");
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t at = off; off = align_up(off + bytes); return at; };
    p->at.meta = take(p->meta.size());
    p->at.pcm = take(2 * p->x_off[B]);
    p->at.x = take(8 * p->x_off[B]);
    p->at.u = take(8 * p->t_off[B]);
    p->at.states = take(8 * 6 * p->total_seg);   // zero-state results, chained initial states
    p->at.y = take(8 * p->y_off[B]);
    p->at.bins = take(8 * 3 * B);
    p->at.dc_parts = take(8 * 4 * p->dc_off[B]);
    p->at.queue = take(16);
    p->at.flag = take(16);
    p->at.slots = take(8 * 4 * p->slot_capacity * p->bank_ctas);
    p->at.spectra = take(sizeof(double2) * (block / 2 + 1) * p->total_blocks);
    p->at.raw = take(8 * size_t(p->bands) * F);
    p->at.cand = take(8 * size_t(p->per_group) * F);
    p->at.count = take(4 * B);
    p->at.jobs = take(sizeof(RefineJob) * size_t(p->capacity) * F);
    p->at.classes = take(sizeof(int) * (2 * kRefineClasses + 1));
    p->at.keys = take(sizeof(ulonglong2) * size_t(p->per_group) * F);
    p->at.leaders = take(2 * sizeof(unsigned long long) * size_t(p->per_group) * F);
    p->at.item_off = take(sizeof(int64_t) * (size_t(B) + 1));
    p->at.refined = take(8 * size_t(p->capacity) * F);
    p->at.scores = take(8 * size_t(p->capacity) * F);
    p->at.pruned = take(8 * size_t(p->capacity) * F);
    p->at.pruned_scores = take(8 * size_t(p->capacity) * F);
    p->at.best = take(8 * F);
    p->at.smoothed = take(8 * F);
    p->at.scratch = take(8 * p->scratch_off[B]);
    p->at.f0 = take(8 * p->out_off[B]);
    p->at.times = take(8 * p->out_off[B]);
    p->at.grad_y = take(8 * p->y_off[B]);
    p->at.grad_fixed = take(8 * F);
    p->arena_bytes = off;
    return p;
  }

  template <class T>
  T* ptr(size_t at) const { return reinterpret_cast<T*>(static_cast<char*>(arena.ptr) + at); }

  DcChunks dc_view(const Plan& p) const {
    return DcChunks{p.d_dc_off, p.dc_off[p.clips], ptr<double>(p.at.dc_parts)};
  }

  static BatchView batch_view(const Plan& p) {
    BatchView bv{};
    bv.clips = p.clips; bv.ratio = p.ratio; bv.bands = p.bands; bv.capacity = p.capacity;
    bv.per_group = p.per_group; bv.fs_r = p.fs_r; bv.f0_floor = p.s.floor; bv.f0_ceil = p.s.ceil;
    bv.x_off = p.d_x_off; bv.y_off = p.d_y_off; bv.frame_off = p.d_frame_off; bv.nfft = p.d_nfft;
    return bv;
  }

  static DecimateView decimate_view(const Plan& p) {
    DecimateView dv{};
    dv.clips = p.clips; dv.ratio = p.ratio; dv.lag = p.lag; dv.seg_len = kSegment;
    std::memcpy(dv.a, kLowA[p.ratio], sizeof dv.a);
    std::memcpy(dv.b, kLowB[p.ratio], sizeof dv.b);
    std::memcpy(dv.trans, p.trans, sizeof dv.trans);
    dv.x_off = p.d_x_off; dv.y_off = p.d_y_off; dv.t_off = p.d_t_off; dv.seg_off = p.d_seg_off;
    return dv;
  }

  static BankView bank_view(const Plan& p) {
    BankView kv{};
    kv.batch = batch_view(p);
    kv.centre = p.d_centre; kv.half = p.d_half; kv.tap_off = p.d_tap_off; kv.taps_rev = p.d_taps;
    kv.items = p.d_items; kv.item_count = static_cast<int>(p.items.size());
    kv.max_pad_taps = p.bank->max_pad_taps; kv.total_frames = p.frame_off[p.clips];
    kv.slot_capacity = p.slot_capacity;
    return kv;
  }

  static FftBankGeometry fft_geometry(const Plan& p) {
    const int run = 2 * ((p.fft_valid + 2 + 2 * 256 - 1) / (2 * 256));
    // The event scan keeps one 32-bit hit mask per kind and thread run.
    if (run > 32) throw RuntimeFailure("FFT band bank: event run longer than 32 positions");
    return FftBankGeometry{p.bank->max_half, p.fft_valid, run, p.total_blocks, p.d_blk_off};
  }

  ContourView contour_view(const Plan& p) const {
    ContourView cv{};
    cv.batch = batch_view(p);
    cv.pruned = ptr<double>(p.at.pruned); cv.pruned_scores = ptr<double>(p.at.pruned_scores);
    cv.best = ptr<double>(p.at.best); cv.count = ptr<int>(p.at.count);
    cv.scratch_off = p.d_scratch_off; cv.scratch = ptr<double>(p.at.scratch);
    cv.smoothed = ptr<double>(p.at.smoothed); cv.period = p.s.period; cv.out_off = p.d_out_off;
    cv.f0_out = ptr<double>(p.at.f0); cv.t_out = ptr<double>(p.at.times);
    cv.column_multiple = 7;   // OverlapF0Candidates' seven groups
    cv.fixed_out = nullptr;
    int64_t longest = 0;
    for (int c = 0; c < p.clips; ++c) longest = std::max(longest, p.frame_off[c + 1] - p.frame_off[c]);
    cv.extend_blocks = p.extend_blocks > 0 ? p.extend_blocks : contour_extend_blocks(longest);
    cv.finish_threads = p.contour_threads;
    return cv;
  }

  // Decimation (or copy) of the clips at `x` into the arena's y, then DC
  // removal.
  void enqueue_waveform(Plan& p, const double* x, cudaStream_t s) {
    double* y = ptr<double>(p.at.y);
    if (p.ratio > 1)
      check(launch_decimate(decimate_view(p), x, ptr<double>(p.at.u), ptr<double>(p.at.states), p.total_seg, y, s),
            "decimate");
    else
      check(launch_copy(x, p.x_off[p.clips], y, s), "copy");
    check(launch_remove_mean(batch_view(p), dc_view(p), y, ptr<double>(p.at.bins), s), "remove_mean");
  }

  // Enqueues every stage on `s`. With `marks_on`, records stage events.
  void enqueue(Plan& p, cudaStream_t s, bool marks_on) {
    const int B = p.clips;
    const int64_t F = p.frame_off[B];
    const BatchView bv = batch_view(p);
    auto mark = [&](int i) { if (marks_on) check(cudaEventRecord(marks[i], s), "cudaEventRecord"); };
    double* x = ptr<double>(p.at.x);
    double* y = ptr<double>(p.at.y);
    mark(0);
    check(cudaMemsetAsync(ptr<int>(p.at.flag), 0, 16, s), "memset");
    check(launch_check_finite(x, p.x_off[B], ptr<int>(p.at.flag), sms, s), "check_finite");
    enqueue_waveform(p, x, s);
    mark(1);
    const BankView kv = bank_view(p);
    check(cudaMemsetAsync(ptr<int>(p.at.queue), 0, 16, s), "memset");
    if (p.use_fft) {
      check(launch_fft_bank(kv, fft_geometry(p), y, ptr<double>(p.at.bins), twiddles, p.filters,
                            ptr<double2>(p.at.spectra), ptr<int>(p.at.queue), ptr<double>(p.at.slots), p.bank_ctas,
                            ptr<double>(p.at.raw), s),
            "band_bank_fft");
    } else {
      check(launch_band_bank(kv, y, ptr<double>(p.at.bins), ptr<int>(p.at.queue), ptr<double>(p.at.slots),
                             p.bank_ctas, ptr<double>(p.at.raw), s),
            "band_bank");
    }
    mark(2);
    check(cudaMemsetAsync(ptr<int>(p.at.count), 0, 4 * B, s), "memset");
    check(launch_candidates(bv, ptr<double>(p.at.raw), F, ptr<double>(p.at.cand), ptr<int>(p.at.count), s),
          "candidates");
    mark(3);
    RefineBuffers rb{};
    rb.class_count = ptr<int>(p.at.classes);
    rb.class_cursor = rb.class_count + kRefineClasses;
    rb.total = rb.class_cursor + kRefineClasses;
    rb.jobs = ptr<RefineJob>(p.at.jobs);
    rb.keys = ptr<ulonglong2>(p.at.keys);
    rb.leaders = ptr<unsigned long long>(p.at.leaders);
    rb.item_off = ptr<int64_t>(p.at.item_off);
    rb.twiddles = twiddles;
    check(launch_refine(bv, rb, y, ptr<double>(p.at.cand), ptr<int>(p.at.count), F,
                        ptr<double>(p.at.refined), ptr<double>(p.at.scores), sms, p.refine_shape, s),
          "refine");
    mark(4);
    check(launch_prune(bv, ptr<double>(p.at.refined), ptr<double>(p.at.scores), ptr<int>(p.at.count), F,
                       ptr<double>(p.at.pruned), ptr<double>(p.at.pruned_scores), ptr<double>(p.at.best), s),
          "prune");
    mark(5);
    check(launch_contour(contour_view(p), s), "contour");
    mark(6);
  }

  // The tape of the F0 gradient for the run just enqueued on `s` (it reads
  // that run's candidates and contour scratch).
  void enqueue_tape(Plan& p, double* tape, cudaStream_t s) {
    check(launch_tape(contour_view(p), ptr<double>(p.at.cand), p.frame_off[p.clips], tape, s), "tape");
  }

  // Backward pass of the per-band-candidate gradient: dL/dx from
  // dL/draw[band][frame]. Recomputes y, reruns the FFT band bank with its
  // dump, then the band-bank adjoint, the transpose of the filters, and the
  // DC-removal and decimation adjoints.
  void enqueue_raw_backward(Plan& p, const double* x, const double* grad_raw, double* grad_x, cudaStream_t s) {
    if (!p.use_fft)
      throw InvalidArgument("the per-band candidate gradient needs the FFT band bank (f0_floor is too low)");
    const int B = p.clips;
    const int64_t F = p.frame_off[B], y_total = p.y_off[B];
    const FftBankGeometry geo = fft_geometry(p);
    const int ctas = p.bank_ctas;
    const size_t dump_n = size_t(p.bands) * size_t(p.total_blocks) * size_t(p.fft_valid + 2);
    const size_t gradf_n = size_t(p.bands) * size_t(y_total);
    const size_t slot_n = size_t(ctas) * 4 * size_t(p.slot_capacity);
    const size_t need = align_up(8 * dump_n) + align_up(8 * gradf_n) + 3 * align_up(8 * slot_n);
    raw_buf.reserve(need, last, s, false, "cudaMalloc(raw gradient)");
    char* m = static_cast<char*>(raw_buf.ptr);
    double* dump = reinterpret_cast<double*>(m);
    double* grad_f = reinterpret_cast<double*>(m + align_up(8 * dump_n));
    char* slots = m + align_up(8 * dump_n) + align_up(8 * gradf_n);
    enqueue_waveform(p, x, s);
    BankView kv = bank_view(p);
    kv.dump = dump;
    check(cudaMemsetAsync(ptr<int>(p.at.queue), 0, 16, s), "memset");
    check(launch_fft_bank(kv, geo, ptr<double>(p.at.y), ptr<double>(p.at.bins), twiddles, p.filters,
                          ptr<double2>(p.at.spectra), ptr<int>(p.at.queue), ptr<double>(p.at.slots), ctas,
                          ptr<double>(p.at.raw), s),
          "band_bank_fft");
    check(cudaMemsetAsync(grad_f, 0, 8 * gradf_n, s), "memset");
    check(cudaMemsetAsync(ptr<int>(p.at.queue), 0, 16, s), "memset");
    RawAdjointView rv{};
    rv.batch = batch_view(p);
    rv.geo = geo;
    rv.items = p.d_items; rv.item_count = static_cast<int>(p.items.size());
    rv.centre = p.d_centre;
    rv.dump = dump;
    rv.grad_raw = grad_raw;
    rv.total_frames = F;
    rv.slot_capacity = p.slot_capacity;
    rv.edges = reinterpret_cast<double*>(slots);
    rv.where = reinterpret_cast<long long*>(slots + align_up(8 * slot_n));
    rv.grad_edges = reinterpret_cast<double*>(slots + 2 * align_up(8 * slot_n));
    rv.queue = ptr<int>(p.at.queue);
    rv.grad_f = grad_f;
    rv.y_total = y_total;
    check(launch_raw_adjoint(rv, ctas, s), "raw_adjoint");
    double* grad_y = ptr<double>(p.at.grad_y);
    check(launch_band_correlate(rv.batch, grad_f, y_total, p.d_half, p.d_tap_off, p.d_taps, grad_y, s),
          "band_correlate");
    check(launch_remove_mean_adjoint(rv.batch, dc_view(p), grad_y, s), "remove_mean_adjoint");
    if (p.ratio > 1)
      check(launch_decimate_adjoint(decimate_view(p), grad_y, ptr<double>(p.at.u), ptr<double>(p.at.states),
                                    p.total_seg, grad_x, s),
            "decimate_adjoint");
    else
      check(launch_copy(grad_y, p.x_off[B], grad_x, s), "copy");
  }

  // Backward pass of the F0 gradient: dL/dx for the clips at `x` from dL/df0
  // and the forward pass's tape. The waveform y is recomputed from x; the
  // adjoints run in reverse stage order. The contour's adjoint reads only the
  // tape and dL/df0, so it runs on the workspace's stream, forked from and
  // joined back into `s`, while `s` recomputes the waveform.
  void enqueue_backward(Plan& p, const double* x, const double* tape, const double* grad_f0, double* grad_x,
                        cudaStream_t s) {
    const int B = p.clips;
    const int64_t F = p.frame_off[B];
    const BatchView bv = batch_view(p);
    GradView gv{};
    gv.batch = bv;
    gv.tape = tape;
    gv.scratch_off = p.d_scratch_off; gv.scratch = ptr<double>(p.at.scratch);
    gv.period = p.s.period; gv.out_off = p.d_out_off;
    gv.grad_f0 = grad_f0;
    gv.grad_fixed = ptr<double>(p.at.grad_fixed);
    check(cudaEventRecord(fork, s), "cudaEventRecord");
    check(cudaStreamWaitEvent(stream, fork, 0), "cudaStreamWaitEvent");
    check(launch_contour_adjoint(gv, stream), "contour_adjoint");
    check(cudaEventRecord(join, stream), "cudaEventRecord");
    enqueue_waveform(p, x, s);
    double* grad_y = ptr<double>(p.at.grad_y);
    check(cudaMemsetAsync(grad_y, 0, 8 * p.y_off[B], s), "memset");
    check(cudaStreamWaitEvent(s, join, 0), "cudaStreamWaitEvent");
    check(launch_refine_adjoint(bv, ptr<double>(p.at.y), tape, gv.grad_fixed, F, twiddles, grad_y, sms, s),
          "refine_adjoint");
    check(launch_remove_mean_adjoint(bv, dc_view(p), grad_y, s), "remove_mean_adjoint");
    if (p.ratio > 1)
      check(launch_decimate_adjoint(decimate_view(p), grad_y, ptr<double>(p.at.u), ptr<double>(p.at.states),
                                    p.total_seg, grad_x, s),
            "decimate_adjoint");
    else
      check(launch_copy(grad_y, p.x_off[B], grad_x, s), "copy");
  }

  // Autotuner: picks the refinement launch shape and the contour's section-
  // extension blocks per clip for the plan's key the first time a plan with
  // that key runs. The key is fs, the f0 range, and the length buckets
  // (floor of log2) of the batch's samples and of its longest clip's frames.
  // It runs the pipeline once to produce the stages' inputs, then times the
  // refinement alone under every candidate shape and the contour under every
  // candidate block count (each launched twice, the second timed, so that
  // lazy module loading is not timed) and keeps the fastest. Every candidate
  // gives bit-identical results, so tuning never changes an output.
  // HARVEST_B200_AUTOTUNE=0 skips it and uses the defaults.
  void autotune(Plan& p, cudaStream_t s) {
    p.tuned = true;
    auto log2_bucket = [](int64_t v) {
      int b = 0;
      while ((int64_t(2) << b) <= v) ++b;
      return b;
    };
    int64_t longest = 0;
    for (int c = 0; c < p.clips; ++c) longest = std::max(longest, p.frame_off[c + 1] - p.frame_off[c]);
    const auto key = std::make_tuple(p.s.fs, p.s.floor, p.s.ceil, log2_bucket(p.x_off[p.clips]), log2_bucket(longest));
    g_tuning[2] = 0;
    // HARVEST_B200_CONTOUR_BLOCKS=n forces the contour's extension blocks.
    if (const char* forced = std::getenv("HARVEST_B200_CONTOUR_BLOCKS")) {
      const int e = std::atoi(forced);
      if (e >= 1 && e <= 64) p.extend_blocks = e;
    }
    // HARVEST_B200_REFINE_SHAPE=min_blocks,blocks_per_sm forces a shape.
    if (const char* forced = std::getenv("HARVEST_B200_REFINE_SHAPE")) {
      int a = 0, b = 0;
      if (std::sscanf(forced, "%d,%d", &a, &b) == 2 && (a == 1 || a == 4 || a == 5) && b >= 1 && b <= 1024) {
        p.refine_shape = RefineShape{a, b};
        return;
      }
    }
    auto it = tuned_shapes.find(key);
    if (it != tuned_shapes.end()) {
      p.refine_shape = it->second.refine;
      if (!p.extend_blocks) p.extend_blocks = it->second.extend_blocks;
      return;
    }
    const char* env = std::getenv("HARVEST_B200_AUTOTUNE");
    if (env && !std::strcmp(env, "0")) {
      p.refine_shape = RefineShape{};
      return;
    }
    enqueue(p, s, false);
    const BatchView bv = batch_view(p);
    RefineBuffers rb{};
    rb.class_count = ptr<int>(p.at.classes);
    rb.class_cursor = rb.class_count + kRefineClasses;
    rb.total = rb.class_cursor + kRefineClasses;
    rb.jobs = ptr<RefineJob>(p.at.jobs);
    rb.keys = ptr<ulonglong2>(p.at.keys);
    rb.leaders = ptr<unsigned long long>(p.at.leaders);
    rb.item_off = ptr<int64_t>(p.at.item_off);
    rb.twiddles = twiddles;
    const int64_t F = p.frame_off[p.clips];
    RefineShape best{};
    float best_ms = 0.0f;
    for (int min_blocks : {1, 4, 5})
      for (int per_sm : {16, 32, 64}) {
        RefineShape shape{min_blocks, per_sm};
        for (int rep = 0; rep < 2; ++rep) {
          check(cudaEventRecord(marks[0], s), "cudaEventRecord");
          check(launch_refine(bv, rb, ptr<double>(p.at.y), ptr<double>(p.at.cand), ptr<int>(p.at.count), F,
                              ptr<double>(p.at.refined), ptr<double>(p.at.scores), sms, shape, s),
                "refine");
          check(cudaEventRecord(marks[1], s), "cudaEventRecord");
        }
        check(cudaEventSynchronize(marks[1]), "cudaEventSynchronize");
        float ms = 0.0f;
        check(cudaEventElapsedTime(&ms, marks[0], marks[1]), "cudaEventElapsedTime");
        if (best_ms == 0.0f || ms < best_ms) { best_ms = ms; best = shape; }
      }
    // The contour, with the refinement's own outputs (the same bits under
    // every shape) still in place.
    int best_blocks = p.extend_blocks;
    if (!best_blocks) {
      best_ms = 0.0f;
      for (int blocks : {1, 2, 4, 8, 16, 32}) {
        p.extend_blocks = blocks;
        const ContourView cv = contour_view(p);
        for (int rep = 0; rep < 2; ++rep) {
          check(cudaEventRecord(marks[0], s), "cudaEventRecord");
          check(launch_contour(cv, s), "contour");
          check(cudaEventRecord(marks[1], s), "cudaEventRecord");
        }
        check(cudaEventSynchronize(marks[1]), "cudaEventSynchronize");
        float ms = 0.0f;
        check(cudaEventElapsedTime(&ms, marks[0], marks[1]), "cudaEventElapsedTime");
        if (best_ms == 0.0f || ms < best_ms) { best_ms = ms; best_blocks = blocks; }
      }
    }
    tuned_shapes[key] = Tuning{best, best_blocks};
    p.refine_shape = best;
    p.extend_blocks = best_blocks;
    g_tuning[2] = 1;
  }

  // Runs the compute of `p` on stream `s`, through the plan's graph when
  // allowed. Inputs are in the arena's x region; outputs land in f0/times.
  void run(Plan& p, cudaStream_t s, bool use_graph, bool marks_on) {
    if (!p.tuned) autotune(p, s);
    else g_tuning[2] = 0;
    g_tuning[0] = p.refine_shape.min_blocks;
    g_tuning[1] = p.refine_shape.blocks_per_sm;
    if (!use_graph || marks_on) {
      enqueue(p, s, marks_on);
      return;
    }
    if (!p.graph || p.graph_arena != arena.ptr) {
      if (p.graph) { cudaGraphExecDestroy(p.graph); p.graph = nullptr; }
      cudaGraph_t g = nullptr;
      check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
      try {
        enqueue(p, stream, false);
      } catch (...) {
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      check(cudaStreamEndCapture(stream, &g), "cudaStreamEndCapture");
      cudaError_t e = cudaGraphInstantiate(&p.graph, g, 0);
      cudaGraphDestroy(g);
      check(e, "cudaGraphInstantiate");
      p.graph_arena = arena.ptr;
    }
    check(cudaGraphLaunch(p.graph, s), "cudaGraphLaunch");
  }
};

using WorkspaceCache = DeviceCache<Workspace>;

WorkspaceCache& cache() {
  // Never destroyed: leases may end during static teardown.
  static WorkspaceCache* c = new WorkspaceCache([](int device) { return std::make_unique<Workspace>(device); });
  return *c;
}

const char* kStageNames[HV_STAGE_COUNT] = {"decimate", "band_bank", "candidates", "refine", "prune", "contour"};

// Copies the stage intervals of the workspace's last recorded run.
void collect_stage_ms(Workspace& ws) {
  for (int i = 0; i < HV_STAGE_COUNT; ++i) {
    float ms = 0;
    check(cudaEventElapsedTime(&ms, ws.marks[i], ws.marks[i + 1]), "cudaEventElapsedTime");
    g_stage_ms[i] = ms;
  }
}

// Shared body of the host-pointer entry points; with `pcm`, the input is
// PCM16 (x is ignored) and is converted on the device.
void run_host(const double* x, const int64_t* offsets, int clips, const Settings& s, int device,
              double* f0, double* times, bool use_graph, bool record, const int16_t* pcm = nullptr) {
  check_device(device);
  WorkspaceCache::Lease lease(cache(), device);
  Workspace& ws = lease.get();
  ContextGuard guard(ws.ctx.get());
  Plan& p = ws.prepare(s, offsets, clips, ws.stream);
  const int64_t total_x = p.x_off[clips], total_out = p.out_off[clips];
  if (pcm) {
    check(cudaMemcpyAsync(ws.ptr<int16_t>(p.at.pcm), pcm + offsets[0], 2 * total_x, cudaMemcpyHostToDevice,
                          ws.stream),
          "cudaMemcpy(pcm)");
    check(launch_pcm16(ws.ptr<int16_t>(p.at.pcm), total_x, ws.ptr<double>(p.at.x), ws.sms, ws.stream), "pcm16");
  } else {
    check(cudaMemcpyAsync(ws.ptr<double>(p.at.x), x + offsets[0], 8 * total_x, cudaMemcpyHostToDevice,
                          ws.stream),
          "cudaMemcpy(x)");
  }
  ws.run(p, ws.stream, use_graph, record);
  // Samples are checked for finiteness on the device; nothing is copied back
  // for input the reference would have rejected.
  check(cudaMemcpyAsync(ws.host_flag, ws.ptr<int>(p.at.flag), sizeof(int), cudaMemcpyDeviceToHost, ws.stream),
        "cudaMemcpy(flag)");
  check(cudaStreamSynchronize(ws.stream), "harvest");
  if (*ws.host_flag) {
    check(cudaEventRecord(ws.last, ws.stream), "cudaEventRecord");
    throw InvalidArgument("x must contain only finite samples");
  }
  check(cudaMemcpyAsync(f0, ws.ptr<double>(p.at.f0), 8 * total_out, cudaMemcpyDeviceToHost, ws.stream),
        "cudaMemcpy(f0)");
  if (times)
    check(cudaMemcpyAsync(times, ws.ptr<double>(p.at.times), 8 * total_out, cudaMemcpyDeviceToHost, ws.stream),
          "cudaMemcpy(times)");
  check(cudaEventRecord(ws.last, ws.stream), "cudaEventRecord");
  check(cudaStreamSynchronize(ws.stream), "harvest");
  if (record) collect_stage_ms(ws);
}

// Settings and offsets of a batch, clip by clip.
void validate_batch(const int64_t* offsets, int clips, int fs, double f0_floor, double f0_ceil,
                    double frame_period) {
  if (clips <= 0 || !offsets) throw InvalidArgument("a batch needs at least one clip and its offsets");
  for (int c = 0; c < clips; ++c) {
    if (offsets[c + 1] < offsets[c]) throw InvalidArgument("offsets must be nondecreasing");
    validate_settings(offsets[c + 1] - offsets[c], fs, f0_floor, f0_ceil, frame_period);
  }
}

// ---------------------------------------------- allocation-free decimation --
// Scratch of hv_decimate_noalloc: a fixed array in the library's device
// image, present on every GPU that loads the library for the life of the
// process. It holds the forward low-pass pass (n + 2 lag + 18 doubles), the
// segment states (6 per 256 samples), a 16-word tail: the offset tables
// (words 0-7), the FFT size (word 8), the three edge bins (words 10-12)
// that the DC removal writes and its chunk table (words 14-15), and the DC
// removal's 4 doubles per chunk.
constexpr int max_decimation_lag() {
  int m = 0;
  for (int r = 2; r <= 12; ++r) m = decimation_lag(r) > m ? decimation_lag(r) : m;
  return m;
}
constexpr int kNoAllocMaxLag = 144;
static_assert(max_decimation_lag() == kNoAllocMaxLag, "largest decimation lag over ratios 2-12");
constexpr int64_t kNoAllocMaxSamples = int64_t(1) << 20;
constexpr int64_t kNoAllocPadded = kNoAllocMaxSamples + 2 * kNoAllocMaxLag + 18;
constexpr int64_t kNoAllocSegments = (kNoAllocPadded + kSegment - 1) / kSegment;
constexpr int64_t kNoAllocMeta = 16;
constexpr int64_t kNoAllocDcChunks = (kNoAllocMaxSamples + kDcChunk - 1) / kDcChunk;   // y has at most n samples
constexpr int64_t kNoAllocDoubles = kNoAllocPadded + 6 * kNoAllocSegments + kNoAllocMeta + 4 * kNoAllocDcChunks;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// Writes the one-clip offset tables into the scratch (no host copies).
__global__ void noalloc_tables(int64_t* meta, int64_t n, int64_t y_len, int64_t padded, int64_t segments,
                               int nfft, int64_t dc_chunks) {
  meta[0] = 0; meta[1] = n;          // x_off
  meta[2] = 0; meta[3] = y_len;      // y_off
  meta[4] = 0; meta[5] = padded;     // t_off
  meta[6] = 0; meta[7] = segments;   // seg_off
  reinterpret_cast<int*>(meta + 8)[0] = nfft;
  meta[14] = 0; meta[15] = dc_chunks;   // the DC removal's chunk table
}

// Per device: the retained primary context and the scratch's device address,
// set up once by the first call on that device (with that device's context
// current), which also loads every kernel the entry point launches so that
// later calls do not load module code (which may allocate). A failed set-up
// is not remembered: the next call tries again.
struct NoAllocDevice {
  std::once_flag once;
  std::unique_ptr<PrimaryContext> ctx;
  double* scratch = nullptr;
};
NoAllocDevice& noalloc_device(int device) {
  static std::mutex mutex;
  // Never destroyed: releasing primary contexts during static teardown may
  // run after the CUDA driver has shut down.
  static auto* devices = new std::map<int, std::unique_ptr<NoAllocDevice>>();
  std::lock_guard<std::mutex> lock(mutex);
  auto& slot = (*devices)[device];
  if (!slot) slot = std::make_unique<NoAllocDevice>();
  return *slot;
}

void noalloc_setup(NoAllocDevice& dev, int device) {
  auto ctx = std::make_unique<PrimaryContext>(device);
  ContextGuard g(ctx->get());
  void* address = nullptr;
  check(cudaGetSymbolAddress(&address, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)");
  if (!address) throw RuntimeFailure("device scratch unavailable");
  cudaFuncAttributes attr;
  check(cudaFuncGetAttributes(&attr, reinterpret_cast<const void*>(noalloc_tables)), "load noalloc_tables");
  check(preload_decimation_kernels(), "load decimation kernels");
  dev.scratch = static_cast<double*>(address);
  dev.ctx = std::move(ctx);
}

}  // namespace
}  // namespace hv

using namespace hv;

extern "C" {

const char* hv_last_error(void) { return g_error.c_str(); }

int hv_cuda_available(int device) {
  if (device < 0) return 0;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) { cudaGetLastError(); return 0; }
  if (device >= count) return 0;
  int major = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return major >= 10 ? 1 : 0;
}

int64_t hv_output_length(int64_t n, int fs, double frame_period) {
  if (n <= 0 || fs <= 0 || !(frame_period > 0) || !std::isfinite(frame_period)) return -1;
  double v = 1000.0 * n / fs / frame_period;
  if (!(v < INT_MAX)) return -1;
  return samples_for(fs, n, frame_period);
}

int hv_validate(const double* x, int64_t n, int fs, double f0_floor, double f0_ceil, double frame_period) {
  return guarded([&] {
    validate_settings(n, fs, f0_floor, f0_ceil, frame_period);
    if (!x) throw InvalidArgument("x is null");
    validate_samples(x, n);
  });
}

int hv_harvest(const double* x, int64_t n, int fs, double f0_floor, double f0_ceil, double frame_period,
               int device, double* f0, double* times, int64_t out_len) {
  return guarded([&] {
    validate_settings(n, fs, f0_floor, f0_ceil, frame_period);
    if (!x || !f0 || !times) throw InvalidArgument("null buffer");
    if (out_len != samples_for(fs, n, frame_period)) throw InvalidArgument("output length mismatch");
    int64_t offsets[2] = {0, n};
    run_host(x, offsets, 1, Settings{fs, f0_floor, f0_ceil, frame_period}, device, f0, times, false, false);
  });
}

int hv_profile(const double* x, int64_t n, int fs, double f0_floor, double f0_ceil, double frame_period,
               int device, double* f0, double* times, int64_t out_len, double* stage_ms) {
  return guarded([&] {
    validate_settings(n, fs, f0_floor, f0_ceil, frame_period);
    if (!x || !f0 || !times || !stage_ms) throw InvalidArgument("null buffer");
    if (out_len != samples_for(fs, n, frame_period)) throw InvalidArgument("output length mismatch");
    int64_t offsets[2] = {0, n};
    run_host(x, offsets, 1, Settings{fs, f0_floor, f0_ceil, frame_period}, device, f0, times, false, true);
    std::memcpy(stage_ms, g_stage_ms, sizeof g_stage_ms);
  });
}

int hv_last_stage_ms(double* stage_ms) {
  return guarded([&] {
    if (!stage_ms) throw InvalidArgument("null buffer");
    std::memcpy(stage_ms, g_stage_ms, sizeof g_stage_ms);
  });
}

int hv_last_tuning(int* shape) {
  return guarded([&] {
    if (!shape) throw InvalidArgument("null buffer");
    std::memcpy(shape, g_tuning, sizeof g_tuning);
  });
}

const char* hv_stage_name(int stage) {
  return stage >= 0 && stage < HV_STAGE_COUNT ? kStageNames[stage] : "";
}

int hv_harvest_batch(const double* x, const int64_t* offsets, int clips, int fs, double f0_floor,
                     double f0_ceil, double frame_period, int device, double* f0, double* times,
                     unsigned flags, void* stream) {
  return guarded([&] {
    validate_batch(offsets, clips, fs, f0_floor, f0_ceil, frame_period);
    if (!x || !f0) throw InvalidArgument("null buffer");
    Settings s{fs, f0_floor, f0_ceil, frame_period};
    const bool record = (flags & HV_RECORD_STAGES) != 0;
    const bool use_graph = !(flags & HV_NO_GRAPH) && !record;
    if (!(flags & HV_DEVICE_POINTERS)) {
      run_host(x, offsets, clips, s, device, f0, times, use_graph, record);
      return;
    }
    check_device(device);
    WorkspaceCache::Lease lease(cache(), device);
    Workspace& ws = lease.get();
    ContextGuard guard(ws.ctx.get());
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream)
                             : ((flags & HV_NULL_IS_LEGACY_STREAM) ? cudaStreamLegacy : ws.stream);
    Plan& p = ws.prepare(s, offsets, clips, st);
    const int64_t total_x = p.x_off[clips], total_out = p.out_off[clips];
    check(cudaMemcpyAsync(ws.ptr<double>(p.at.x), x + offsets[0], 8 * total_x, cudaMemcpyDeviceToDevice, st),
          "cudaMemcpy(x)");
    ws.run(p, st, use_graph, record);
    check(cudaMemcpyAsync(f0, ws.ptr<double>(p.at.f0), 8 * total_out, cudaMemcpyDeviceToDevice, st),
          "cudaMemcpy(f0)");
    if (times)
      check(cudaMemcpyAsync(times, ws.ptr<double>(p.at.times), 8 * total_out, cudaMemcpyDeviceToDevice, st),
            "cudaMemcpy(times)");
    // The workspace is reused by the next call on this device, on whatever
    // stream; that call waits for this event first.
    check(cudaEventRecord(ws.last, st), "cudaEventRecord");
    if (record) {
      check(cudaStreamSynchronize(st), "harvest_batch");
      collect_stage_ms(ws);
    }
  });
}

int hv_harvest_batch_pcm16(const int16_t* x, const int64_t* offsets, int clips, int fs, double f0_floor,
                           double f0_ceil, double frame_period, int device, double* f0, double* times,
                           unsigned flags, void* stream) {
  return guarded([&] {
    validate_batch(offsets, clips, fs, f0_floor, f0_ceil, frame_period);
    if (!x || !f0) throw InvalidArgument("null buffer");
    Settings s{fs, f0_floor, f0_ceil, frame_period};
    const bool use_graph = !(flags & HV_NO_GRAPH);
    if (!(flags & HV_DEVICE_POINTERS)) {
      run_host(nullptr, offsets, clips, s, device, f0, times, use_graph, false, x);
      return;
    }
    check_device(device);
    WorkspaceCache::Lease lease(cache(), device);
    Workspace& ws = lease.get();
    ContextGuard guard(ws.ctx.get());
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream)
                             : ((flags & HV_NULL_IS_LEGACY_STREAM) ? cudaStreamLegacy : ws.stream);
    Plan& p = ws.prepare(s, offsets, clips, st);
    const int64_t total_x = p.x_off[clips], total_out = p.out_off[clips];
    check(launch_pcm16(x + offsets[0], total_x, ws.ptr<double>(p.at.x), ws.sms, st), "pcm16");
    ws.run(p, st, use_graph, false);
    check(cudaMemcpyAsync(f0, ws.ptr<double>(p.at.f0), 8 * total_out, cudaMemcpyDeviceToDevice, st),
          "cudaMemcpy(f0)");
    if (times)
      check(cudaMemcpyAsync(times, ws.ptr<double>(p.at.times), 8 * total_out, cudaMemcpyDeviceToDevice, st),
            "cudaMemcpy(times)");
    check(cudaEventRecord(ws.last, st), "cudaEventRecord");
  });
}

int hv_compare_batch(const double* reference, const double* f0, const int64_t* offsets, int clips, int device,
                     double* stats, unsigned flags, void* stream) {
  return guarded([&] {
    if (clips <= 0 || !offsets) throw InvalidArgument("a batch needs at least one clip and its offsets");
    if (!reference || !f0 || !stats) throw InvalidArgument("null buffer");
    if (offsets[0] < 0) throw InvalidArgument("offsets must be nonnegative");
    for (int c = 0; c < clips; ++c)
      if (offsets[c + 1] < offsets[c]) throw InvalidArgument("offsets must be nondecreasing");
    const int64_t base = offsets[0], total = offsets[clips] - offsets[0];
    const bool on_device = (flags & HV_DEVICE_POINTERS) != 0;
    if (!on_device)
      for (int64_t i = base; i < base + total; ++i)
        if (!std::isfinite(reference[i]) || !std::isfinite(f0[i]) || reference[i] < 0 || f0[i] < 0)
          throw InvalidArgument("F0 tracks must contain only finite, nonnegative values");
    check_device(device);
    WorkspaceCache::Lease lease(cache(), device);
    Workspace& ws = lease.get();
    ContextGuard guard(ws.ctx.get());
    cudaStream_t st = ws.stream;
    if (on_device && stream) st = static_cast<cudaStream_t>(stream);
    else if (on_device && (flags & HV_NULL_IS_LEGACY_STREAM)) st = cudaStreamLegacy;
    // Workspace buffer: [relative offsets | reference | f0 | stats]; the
    // tracks and stats only for host inputs.
    const size_t off_bytes = align_up(8 * size_t(clips + 1));
    const size_t track_bytes = on_device ? 0 : align_up(8 * size_t(total));
    const size_t stat_bytes = on_device ? 0 : align_up(8 * 7 * size_t(clips));
    const size_t need = off_bytes + 2 * track_bytes + stat_bytes;
    ws.metric_buf.reserve(need, ws.last, st, false, "cudaMalloc(metrics)");
    check(cudaStreamWaitEvent(st, ws.last, 0), "cudaStreamWaitEvent");
    char* m = static_cast<char*>(ws.metric_buf.ptr);
    std::vector<int64_t> rel(clips + 1);
    for (int c = 0; c <= clips; ++c) rel[c] = offsets[c] - base;
    int64_t* d_off = reinterpret_cast<int64_t*>(m);
    check(cudaMemcpyAsync(d_off, rel.data(), 8 * rel.size(), cudaMemcpyHostToDevice, st), "cudaMemcpy(offsets)");
    if (on_device) {
      check(launch_compare(reference + base, f0 + base, d_off, clips, stats, st), "compare");
    } else {
      double* d_ref = reinterpret_cast<double*>(m + off_bytes);
      double* d_f0 = reinterpret_cast<double*>(m + off_bytes + track_bytes);
      double* d_stats = reinterpret_cast<double*>(m + off_bytes + 2 * track_bytes);
      check(cudaMemcpyAsync(d_ref, reference + base, 8 * total, cudaMemcpyHostToDevice, st), "cudaMemcpy(reference)");
      check(cudaMemcpyAsync(d_f0, f0 + base, 8 * total, cudaMemcpyHostToDevice, st), "cudaMemcpy(f0)");
      check(launch_compare(d_ref, d_f0, d_off, clips, d_stats, st), "compare");
      check(cudaMemcpyAsync(stats, d_stats, 8 * 7 * size_t(clips), cudaMemcpyDeviceToHost, st), "cudaMemcpy(stats)");
      check(cudaStreamSynchronize(st), "compare");
    }
    check(cudaEventRecord(ws.last, st), "cudaEventRecord");
  });
}

int hv_harvest_grad_forward(const double* x, const int64_t* offsets, int clips, int fs, double f0_floor,
                            double f0_ceil, double frame_period, int device, double* f0, double* times,
                            double* tape, void* stream) {
  return guarded([&] {
    validate_batch(offsets, clips, fs, f0_floor, f0_ceil, frame_period);
    if (!x || !f0 || !tape) throw InvalidArgument("null buffer");
    check_device(device);
    WorkspaceCache::Lease lease(cache(), device);
    Workspace& ws = lease.get();
    ContextGuard guard(ws.ctx.get());
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
    Plan& p = ws.prepare(Settings{fs, f0_floor, f0_ceil, frame_period}, offsets, clips, st);
    const int64_t total_x = p.x_off[clips], total_out = p.out_off[clips];
    check(cudaMemcpyAsync(ws.ptr<double>(p.at.x), x + offsets[0], 8 * total_x, cudaMemcpyDeviceToDevice, st),
          "cudaMemcpy(x)");
    ws.run(p, st, true, false);
    check(cudaMemcpyAsync(f0, ws.ptr<double>(p.at.f0), 8 * total_out, cudaMemcpyDeviceToDevice, st),
          "cudaMemcpy(f0)");
    if (times)
      check(cudaMemcpyAsync(times, ws.ptr<double>(p.at.times), 8 * total_out, cudaMemcpyDeviceToDevice, st),
            "cudaMemcpy(times)");
    ws.enqueue_tape(p, tape, st);
    check(cudaEventRecord(ws.last, st), "cudaEventRecord");
  });
}

int hv_harvest_grad_backward(const double* x, const int64_t* offsets, int clips, int fs, double f0_floor,
                             double f0_ceil, double frame_period, int device, const double* tape,
                             const double* grad_f0, double* grad_x, void* stream) {
  return guarded([&] {
    validate_batch(offsets, clips, fs, f0_floor, f0_ceil, frame_period);
    if (!x || !tape || !grad_f0 || !grad_x) throw InvalidArgument("null buffer");
    check_device(device);
    WorkspaceCache::Lease lease(cache(), device);
    Workspace& ws = lease.get();
    ContextGuard guard(ws.ctx.get());
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
    Plan& p = ws.prepare(Settings{fs, f0_floor, f0_ceil, frame_period}, offsets, clips, st);
    ws.enqueue_backward(p, x + offsets[0], tape, grad_f0, grad_x + offsets[0], st);
    check(cudaEventRecord(ws.last, st), "cudaEventRecord");
  });
}

int hv_raw_candidates(const double* x, const int64_t* offsets, int clips, int fs, double f0_floor,
                      double f0_ceil, int device, double* raw, void* stream) {
  return guarded([&] {
    validate_batch(offsets, clips, fs, f0_floor, f0_ceil, 5.0);
    if (!x || !raw) throw InvalidArgument("null buffer");
    check_device(device);
    WorkspaceCache::Lease lease(cache(), device);
    Workspace& ws = lease.get();
    ContextGuard guard(ws.ctx.get());
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
    Plan& p = ws.prepare(Settings{fs, f0_floor, f0_ceil, 5.0}, offsets, clips, st);
    check(cudaMemcpyAsync(ws.ptr<double>(p.at.x), x + offsets[0], 8 * p.x_off[clips], cudaMemcpyDeviceToDevice, st),
          "cudaMemcpy(x)");
    ws.run(p, st, true, false);
    check(cudaMemcpyAsync(raw, ws.ptr<double>(p.at.raw), 8 * size_t(p.bands) * size_t(p.frame_off[clips]),
                          cudaMemcpyDeviceToDevice, st),
          "cudaMemcpy(raw)");
    check(cudaEventRecord(ws.last, st), "cudaEventRecord");
  });
}

int hv_raw_candidates_backward(const double* x, const int64_t* offsets, int clips, int fs, double f0_floor,
                               double f0_ceil, int device, const double* grad_raw, double* grad_x, void* stream) {
  return guarded([&] {
    validate_batch(offsets, clips, fs, f0_floor, f0_ceil, 5.0);
    if (!x || !grad_raw || !grad_x) throw InvalidArgument("null buffer");
    check_device(device);
    WorkspaceCache::Lease lease(cache(), device);
    Workspace& ws = lease.get();
    ContextGuard guard(ws.ctx.get());
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
    Plan& p = ws.prepare(Settings{fs, f0_floor, f0_ceil, 5.0}, offsets, clips, st);
    ws.enqueue_raw_backward(p, x + offsets[0], grad_raw, grad_x + offsets[0], st);
    check(cudaEventRecord(ws.last, st), "cudaEventRecord");
  });
}

int64_t hv_band_count(double f0_floor, double f0_ceil) {
  if (!(f0_floor > 0) || !(f0_ceil > f0_floor) || !std::isfinite(f0_ceil)) return -1;
  return band_count(f0_floor, f0_ceil);
}

int hv_harvest_stages(const double* x, int64_t n, int fs, double f0_floor, double f0_ceil, int device,
                      double* y, double* raw, int* count, double* cand, double* refined, double* scores,
                      double* pruned, double* pruned_scores, double* best, double* smoothed) {
  return guarded([&] {
    validate_settings(n, fs, f0_floor, f0_ceil, 5.0);
    if (!x) throw InvalidArgument("null buffer");
    validate_samples(x, n);
    check_device(device);
    WorkspaceCache::Lease lease(cache(), device);
    Workspace& ws = lease.get();
    ContextGuard guard(ws.ctx.get());
    int64_t offsets[2] = {0, n};
    Plan& p = ws.prepare(Settings{fs, f0_floor, f0_ceil, 5.0}, offsets, 1, ws.stream);
    check(cudaMemcpyAsync(ws.ptr<double>(p.at.x), x, 8 * n, cudaMemcpyHostToDevice, ws.stream), "cudaMemcpy(x)");
    // Refinement and pruning leave the columns past 7 count untouched; the
    // dump shows them as zeros.
    const int64_t F = p.frame_off[1];
    for (size_t at : {p.at.refined, p.at.scores, p.at.pruned, p.at.pruned_scores})
      check(cudaMemsetAsync(ws.ptr<double>(at), 0, 8 * size_t(p.capacity) * F, ws.stream), "memset");
    ws.run(p, ws.stream, false, false);
    auto out = [&](void* dst, size_t at, size_t bytes) {
      if (dst) check(cudaMemcpyAsync(dst, ws.ptr<char>(at), bytes, cudaMemcpyDeviceToHost, ws.stream), "cudaMemcpy");
    };
    out(y, p.at.y, 8 * p.y_off[1]);
    out(raw, p.at.raw, 8 * size_t(p.bands) * F);
    out(count, p.at.count, 4);
    out(cand, p.at.cand, 8 * size_t(p.per_group) * F);
    out(refined, p.at.refined, 8 * size_t(p.capacity) * F);
    out(scores, p.at.scores, 8 * size_t(p.capacity) * F);
    out(pruned, p.at.pruned, 8 * size_t(p.capacity) * F);
    out(pruned_scores, p.at.pruned_scores, 8 * size_t(p.capacity) * F);
    out(best, p.at.best, 8 * F);
    out(smoothed, p.at.smoothed, 8 * F);
    check(cudaEventRecord(ws.last, ws.stream), "cudaEventRecord");
    check(cudaStreamSynchronize(ws.stream), "harvest_stages");
  });
}

int hv_decimate_noalloc(const double* x, int64_t n, int fs, int device, double* y, void* stream) {
  return guarded([&] {
    if (fs < 8000 || fs > 192000) throw InvalidArgument("fs must be between 8000 and 192000 Hz");
    const int ratio = ratio_for(fs);
    if (n < int64_t(2) * ratio)
      throw InvalidArgument("x is too short: require at least two samples after internal decimation");
    if (n > kNoAllocMaxSamples)
      throw InvalidArgument("hv_decimate_noalloc accepts at most " + std::to_string(kNoAllocMaxSamples) +
                            " samples per call (its device scratch is fixed); use hv_harvest_batch for longer input");
    if (!x || !y) throw InvalidArgument("null buffer");
    check_device(device);
    NoAllocDevice& dev = noalloc_device(device);
    // An exception leaves the once_flag unset, so a failed set-up is retried.
    std::call_once(dev.once, [&] { noalloc_setup(dev, device); });
    ContextGuard guard(dev.ctx->get());
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t y_len = (n + ratio - 1) / ratio;
    const int lag = decimation_lag(ratio);
    const int64_t padded = ratio > 1 ? n + 2 * lag + 18 : 0;
    const int64_t segments = ratio > 1 ? (padded + kSegment - 1) / kSegment : 0;
    double* u = dev.scratch;
    double* states = u + kNoAllocPadded;
    int64_t* meta = reinterpret_cast<int64_t*>(states + 6 * kNoAllocSegments);
    double* bins = reinterpret_cast<double*>(meta + 10);
    const DcChunks dc{meta + 14, dc_chunk_count(y_len), reinterpret_cast<double*>(meta + kNoAllocMeta)};
    noalloc_tables<<<1, 1, 0, s>>>(meta, n, y_len, padded, segments, static_cast<int>(2 * y_len), dc.total);
    check(cudaGetLastError(), "noalloc_tables");
    // The DC removal reads only clips, y_off and nfft of its batch view.
    BatchView bv{};
    bv.clips = 1; bv.ratio = ratio; bv.fs_r = double(fs) / ratio;
    bv.x_off = meta; bv.y_off = meta + 2;
    bv.nfft = reinterpret_cast<const int*>(meta + 8);
    if (ratio > 1) {
      DecimateView dv{};
      dv.clips = 1; dv.ratio = ratio; dv.lag = lag; dv.seg_len = kSegment;
      std::memcpy(dv.a, kLowA[ratio], sizeof dv.a);
      std::memcpy(dv.b, kLowB[ratio], sizeof dv.b);
      const double* a = kLowA[ratio];
      double A[9] = {a[0], a[1], a[2], 1, 0, 0, 0, 1, 0};
      double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
      for (int e = kSegment; e; e >>= 1) {
        if (e & 1) mat3_mul(R, A, R);
        mat3_mul(A, A, A);
      }
      std::memcpy(dv.trans, R, sizeof R);
      dv.x_off = meta; dv.y_off = meta + 2; dv.t_off = meta + 4; dv.seg_off = meta + 6;
      check(launch_decimate(dv, x, u, states, segments, y, s), "decimate");
    } else {
      check(launch_copy(x, n, y, s), "copy");
    }
    check(launch_remove_mean(bv, dc, y, bins, s), "remove_mean");
  });
}

int hv_contour_batch(const double* f0_candidates, const double* scores, const double* base,
                     const int64_t* frame_offsets, int clips, int columns, int stride, int device, double* fixed,
                     double* smoothed, unsigned flags, void* stream) {
  return guarded([&] {
    if (clips <= 0 || !frame_offsets) throw InvalidArgument("a batch needs at least one clip and its offsets");
    if (!f0_candidates || !scores || !smoothed) throw InvalidArgument("null buffer");
    if (stride < 1 || columns < 0 || columns > stride || columns > kRefineColumns)
      throw InvalidArgument("require 0 <= columns <= stride, 1 <= stride and columns <= 1024");
    if (frame_offsets[0] != 0) throw InvalidArgument("frame offsets must start at 0");
    for (int c = 0; c < clips; ++c)
      if (frame_offsets[c + 1] - frame_offsets[c] < 1 || frame_offsets[c + 1] - frame_offsets[c] >= (1 << 30))
        throw InvalidArgument("every clip needs between 1 and 2^30 - 1 frames");
    const int64_t F = frame_offsets[clips];
    if (F >= (int64_t(1) << 31)) throw InvalidArgument("more than 2^31 frames");
    const bool on_device = (flags & HV_DEVICE_POINTERS) != 0;
    check_device(device);
    WorkspaceCache::Lease lease(cache(), device);
    Workspace& ws = lease.get();
    ContextGuard guard(ws.ctx.get());
    cudaStream_t st = ws.stream;
    if (on_device && stream) st = static_cast<cudaStream_t>(stream);
    else if (on_device && (flags & HV_NULL_IS_LEGACY_STREAM)) st = cudaStreamLegacy;
    // Host tables: scratch offsets per clip, columns per clip.
    std::vector<int64_t> scratch_off(clips + 1, 0);
    const int finish_threads = clips < ws.sms ? 512 : 256;
    for (int c = 0; c < clips; ++c)
      scratch_off[c + 1] =
          scratch_off[c] + contour_scratch(frame_offsets[c + 1] - frame_offsets[c], finish_threads);
    std::vector<int> cols(clips, columns);
    // Workspace buffer: [frame offsets | scratch offsets | columns | base |
    // scratch | (host inputs: candidates, scores) | (host outputs: fixed,
    // smoothed)].
    const size_t o_f = 0, o_s = align_up(8 * size_t(clips + 1)), o_c = o_s + align_up(8 * size_t(clips + 1));
    const size_t o_b = o_c + align_up(4 * size_t(clips));
    const size_t o_sc = o_b + align_up(8 * size_t(F));
    const size_t matrix = on_device ? 0 : align_up(8 * size_t(F) * size_t(stride));
    const size_t o_in = o_sc + align_up(8 * size_t(scratch_off[clips]));
    const size_t o_out = o_in + 2 * matrix;
    const size_t need = o_out + (on_device ? 0 : 2 * align_up(8 * size_t(F)));
    ws.contour_buf.reserve(need, ws.last, st, false, "cudaMalloc(contour)");
    check(cudaStreamWaitEvent(st, ws.last, 0), "cudaStreamWaitEvent");
    char* m = static_cast<char*>(ws.contour_buf.ptr);
    int64_t* d_off = reinterpret_cast<int64_t*>(m + o_f);
    int64_t* d_soff = reinterpret_cast<int64_t*>(m + o_s);
    int* d_cols = reinterpret_cast<int*>(m + o_c);
    double* d_base = reinterpret_cast<double*>(m + o_b);
    const double* d_cand = f0_candidates;
    const double* d_scores = scores;
    double* d_fixed = fixed;
    double* d_smoothed = smoothed;
    check(cudaMemcpyAsync(d_off, frame_offsets, 8 * size_t(clips + 1), cudaMemcpyHostToDevice, st), "cudaMemcpy");
    check(cudaMemcpyAsync(d_soff, scratch_off.data(), 8 * size_t(clips + 1), cudaMemcpyHostToDevice, st),
          "cudaMemcpy");
    check(cudaMemcpyAsync(d_cols, cols.data(), 4 * size_t(clips), cudaMemcpyHostToDevice, st), "cudaMemcpy");
    if (!on_device) {
      double* c_in = reinterpret_cast<double*>(m + o_in);
      double* s_in = reinterpret_cast<double*>(m + o_in + matrix);
      check(cudaMemcpyAsync(c_in, f0_candidates, 8 * size_t(F) * stride, cudaMemcpyHostToDevice, st), "cudaMemcpy");
      check(cudaMemcpyAsync(s_in, scores, 8 * size_t(F) * stride, cudaMemcpyHostToDevice, st), "cudaMemcpy");
      d_cand = c_in;
      d_scores = s_in;
      d_fixed = reinterpret_cast<double*>(m + o_out);
      d_smoothed = reinterpret_cast<double*>(m + o_out + align_up(8 * size_t(F)));
    }
    if (base)
      check(cudaMemcpyAsync(d_base, base, 8 * size_t(F), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            st),
            "cudaMemcpy(base)");
    else
      check(launch_search_base(d_cand, d_scores, F, stride, d_off, clips, d_cols, d_base, st), "search_base");
    ContourView cv{};
    cv.batch.clips = clips;
    cv.batch.capacity = stride;
    cv.batch.frame_off = d_off;
    cv.pruned = d_cand;
    cv.pruned_scores = d_scores;
    cv.best = d_base;
    cv.count = d_cols;
    cv.column_multiple = 1;
    cv.scratch_off = d_soff;
    cv.scratch = reinterpret_cast<double*>(m + o_sc);
    cv.smoothed = d_smoothed;
    cv.fixed_out = d_fixed;
    cv.f0_out = nullptr;
    int64_t longest = 0;
    for (int c = 0; c < clips; ++c) longest = std::max(longest, frame_offsets[c + 1] - frame_offsets[c]);
    cv.extend_blocks = contour_extend_blocks(longest);
    cv.finish_threads = finish_threads;
    check(launch_contour(cv, st), "contour");
    if (!on_device) {
      if (fixed)
        check(cudaMemcpyAsync(fixed, d_fixed, 8 * size_t(F), cudaMemcpyDeviceToHost, st), "cudaMemcpy(fixed)");
      check(cudaMemcpyAsync(smoothed, d_smoothed, 8 * size_t(F), cudaMemcpyDeviceToHost, st), "cudaMemcpy(smoothed)");
    }
    check(cudaEventRecord(ws.last, st), "cudaEventRecord");
    if (!on_device) check(cudaStreamSynchronize(st), "contour");
  });
}

int hv_clear_cache(void) {
  return guarded([&] { cache().clear(); });
}

}  // extern "C"
