/*
 * harvest_b200.h — C ABI of the B200 Harvest F0 engine (libharvest_b200.so).
 *
 * Plain pointers and sizes only; no exceptions cross this boundary. Every
 * entry point returns a status code; on failure a message for the calling
 * thread is available from hv_last_error(). The Python package maps
 * HV_INVALID_ARGUMENT to ValueError and HV_RUNTIME_ERROR to RuntimeError,
 * which is how the reference's nanobind layer reports the same failures
 * (reference src/bindings.cpp:18-39, src/cuda_device.h:8-40).
 *
 * Threading: calls may come from any thread. Calls on one device take turns
 * on that device's cached workspace; calls on different devices run in
 * parallel (reference src/workspace_cache.h:10-12). The caller's current
 * CUDA context is restored before every call returns (reference
 * src/cuda_device.h:90-108).
 */
#ifndef HARVEST_B200_H_
#define HARVEST_B200_H_

#include <stdint.h>

#if defined(__GNUC__)
#define HV_API __attribute__((visibility("default")))
#else
#define HV_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define HV_OK 0
#define HV_INVALID_ARGUMENT 1 /* bad sizes, rates, ranges, samples or device index */
#define HV_RUNTIME_ERROR 2    /* no usable GPU, CUDA failure, out of memory */

/* Flags for hv_harvest_batch. */
#define HV_DEVICE_POINTERS 1u /* x, f0 and times are device pointers on `device` */
#define HV_NO_GRAPH 2u        /* launch stage by stage instead of replaying a CUDA graph */
#define HV_RECORD_STAGES 4u   /* launch stage by stage with CUDA events between stages; the
                                 call waits for the GPU and hv_last_stage_ms() returns the
                                 per-stage device milliseconds of this call */
#define HV_NULL_IS_LEGACY_STREAM 8u /* with HV_DEVICE_POINTERS: a NULL `stream` is the legacy
                                 default stream (PyTorch's default stream), not the
                                 engine's own */

/* Message describing the last failure on the calling thread ("" if none). */
HV_API const char* hv_last_error(void);

/* 1 if `device` is a visible GPU this library can run on, else 0. Never
 * fails (reference bindings.cpp:66-67, cuda_available). */
HV_API int hv_cuda_available(int device);

/* Number of output frames for n samples at fs and frame_period (ms), as
 * GetSamplesForHarvest (reference third_party/world/src/harvest.cpp:1219);
 * -1 if the arguments are invalid. */
HV_API int64_t hv_output_length(int64_t n, int fs, double frame_period);

/* Checks one clip's arguments and samples exactly as the reference's
 * validate() (reference src/bindings.cpp:18-39). */
HV_API int hv_validate(const double* x, int64_t n, int fs, double f0_floor, double f0_ceil,
                double frame_period);

/* Harvest on one clip of host memory; replaces the reference's
 * _core.harvest (reference src/bindings.cpp:68-80) and analyze()
 * (reference src/engine.cpp:240-333). f0 and times receive
 * hv_output_length(n, fs, frame_period) values (out_len must equal it). */
HV_API int hv_harvest(const double* x, int64_t n, int fs, double f0_floor, double f0_ceil,
               double frame_period, int device, double* f0, double* times, int64_t out_len);

/* Harvest on `clips` clips packed back to back: clip c is
 * x[offsets[c] .. offsets[c+1]). offsets (clips + 1 entries) is host memory.
 * Outputs are packed the same way with per-clip lengths
 * hv_output_length(offsets[c+1] - offsets[c], fs, frame_period). With
 * HV_DEVICE_POINTERS, x/f0/times are device memory and the work is ordered
 * on `stream` (a cudaStream_t, NULL for the engine's own stream); the call
 * returns once the work is enqueued, and non-finite samples cannot be
 * reported (they yield unspecified F0 values, never a fault). Without it,
 * the call is synchronous and rejects non-finite samples with
 * HV_INVALID_ARGUMENT, checked on the device before any output is copied.
 * No counterpart in the reference, which processes one clip per call. */
HV_API int hv_harvest_batch(const double* x, const int64_t* offsets, int clips, int fs,
                     double f0_floor, double f0_ceil, double frame_period, int device,
                     double* f0, double* times, unsigned flags, void* stream);

/* hv_harvest_batch on 16-bit PCM input: each sample is read as
 * sample / 32768, the conversion the reference's benchmark applies to mono
 * PCM16 WAV files (reference benchmarks/benchmark.py:80-84), so results equal
 * hv_harvest_batch on the converted samples bit for bit. The conversion runs
 * on the device, so a host batch crosses PCIe at 2 bytes per sample instead
 * of 8. Flags as hv_harvest_batch (HV_RECORD_STAGES excepted). No counterpart
 * in the reference's API. */
HV_API int hv_harvest_batch_pcm16(const int16_t* x, const int64_t* offsets, int clips, int fs,
                                  double f0_floor, double f0_ceil, double frame_period, int device,
                                  double* f0, double* times, unsigned flags, void* stream);

/* Like hv_harvest, also reporting per-stage device milliseconds into
 * stage_ms[HV_STAGE_COUNT] (reference _profile, src/bindings.cpp:90-104). */
#define HV_STAGE_COUNT 6
HV_API const char* hv_stage_name(int stage);
/* Per-stage device milliseconds of the calling thread's last call made with
 * HV_RECORD_STAGES (or hv_profile) into stage_ms[HV_STAGE_COUNT]. */
HV_API int hv_last_stage_ms(double* stage_ms);
HV_API int hv_profile(const double* x, int64_t n, int fs, double f0_floor, double f0_ceil,
               double frame_period, int device, double* f0, double* times, int64_t out_len,
               double* stage_ms);

/* Refinement launch shape of the calling thread's last Harvest call (no
 * reference counterpart). The engine autotunes it, with the contour's
 * extension blocks, once per (fs, f0_floor, f0_ceil, log2 of the batch's
 * total samples, log2 of its longest clip's frames) on each device, the first time
 * a batch with that key runs, by timing every candidate shape on that
 * batch; all shapes give bit-identical results. shape[0]: minimum resident
 * 128-thread blocks per SM of the kernel instance (1, 4 or 5), shape[1]:
 * grid blocks per SM (16, 32 or 64), shape[2]: 1 if that call ran the
 * tuning, else 0. HARVEST_B200_AUTOTUNE=0 in the environment turns tuning
 * off (shape 4, 32). */
HV_API int hv_last_tuning(int* shape);

/* Accuracy of one F0 track against another for every clip of a batch,
 * computed on the device: the statistics of the reference's benchmark
 * comparison (reference benchmarks/benchmark.py:20-37). reference and f0 are
 * packed alike, clip c spanning [offsets[c], offsets[c+1]) (offsets: host,
 * clips + 1 entries). stats receives 7 doubles per clip: frames,
 * reference-voiced frames, jointly voiced frames, voiced/unvoiced
 * disagreement (fraction of frames), 99th-percentile and maximum
 * |1200 log2(f0 / reference)| cents over jointly voiced frames (numpy's
 * linear quantile; NaN without such frames), and the count above 600 cents.
 * With HV_DEVICE_POINTERS the tracks and stats are device memory and the call
 * is ordered on `stream` (HV_NULL_IS_LEGACY_STREAM as for hv_harvest_batch);
 * otherwise host memory, validated as finite and nonnegative, and the call
 * returns with the stats. No counterpart in the reference's API. */
HV_API int hv_compare_batch(const double* reference, const double* f0, const int64_t* offsets, int clips,
                            int device, double* stats, unsigned flags, void* stream);

/* F0 gradient (no reference counterpart; the reference has no derivative).
 * Harvest is piecewise smooth in x: with every discrete choice of a forward
 * pass held fixed (candidates kept, voicing, FixF0Contour's choices, the
 * section boundaries), the output F0 is a smooth function of the waveform
 * through the refined candidates' spectra, FixStep4's gap fills, the
 * smoothing filter and the resampling.
 *
 * hv_harvest_grad_forward is hv_harvest_batch on device pointers that also
 * writes `tape` (device memory, 2 doubles per 1 ms analysis frame, i.e.
 * hv_output_length(n, fs, 1.0) frames per clip, clips in order): the
 * FixF0Contour step-3 F0 and the initial candidate F0 it was refined from.
 * hv_harvest_grad_backward takes the same x, offsets and settings, that tape
 * and dL/df0 (device, laid out like f0) and writes dL/dx (device, laid out
 * like x); it recomputes the decimated waveform and the spectra rather than
 * storing them. Both order their work on `stream`; NULL is the legacy
 * default stream (PyTorch's default stream), not the engine's own stream.
 * Contributions of overlapping refinement windows are added with atomics,
 * so dL/dx is reproducible to rounding, not bit for bit. */
HV_API int hv_harvest_grad_forward(const double* x, const int64_t* offsets, int clips, int fs,
                                   double f0_floor, double f0_ceil, double frame_period, int device,
                                   double* f0, double* times, double* tape, void* stream);
HV_API int hv_harvest_grad_backward(const double* x, const int64_t* offsets, int clips, int fs,
                                    double f0_floor, double f0_ceil, double frame_period, int device,
                                    const double* tape, const double* grad_f0, double* grad_x,
                                    void* stream);

/* Per-band candidates with a gradient (no reference counterpart). The
 * band-pass bank's candidates (GetF0CandidateContour, reference
 * third_party/world/src/harvest.cpp:240-293) of clips packed as for
 * hv_harvest_batch, on device pointers: raw receives
 * hv_band_count(f0_floor, f0_ceil) rows of sum_c hv_output_length(n_c, fs,
 * 1.0) doubles (row b holds band b's candidate at every 1 ms frame of every
 * clip, clips in order; 0 where the band has none).
 * hv_raw_candidates_backward takes dL/draw in that layout and writes dL/dx
 * (laid out like x): the fine zero-crossing and extremum positions, and so
 * the candidates, are smooth in x while the events themselves, each frame's
 * interpolation segments and the range checks are held fixed. It
 * recomputes the waveform and reruns the band bank, and needs the FFT band
 * bank (HV_INVALID_ARGUMENT for floors so low that the direct FIR is used).
 * WORLD's final-bin term is held fixed in the derivative. Streams as
 * hv_harvest_grad_forward. */
HV_API int64_t hv_band_count(double f0_floor, double f0_ceil);
HV_API int hv_raw_candidates(const double* x, const int64_t* offsets, int clips, int fs, double f0_floor,
                             double f0_ceil, int device, double* raw, void* stream);
HV_API int hv_raw_candidates_backward(const double* x, const int64_t* offsets, int clips, int fs,
                                      double f0_floor, double f0_ceil, int device, const double* grad_raw,
                                      double* grad_x, void* stream);

/* Diagnostic: runs hv_harvest on one clip and copies the intermediate stage
 * buffers to host memory, for stage-by-stage parity tests. Any pointer may
 * be NULL. Shapes (row-major, frames = analysis frames on the 1 ms grid,
 * cap = 7 * round(bands / 10)): y[y_len] decimated and DC-free waveform;
 * raw[bands * frames] per-band candidates; count[1] candidates per frame;
 * cand[frames * cap/7] candidates before overlap; refined, scores, pruned,
 * pruned_scores[frames * cap]; best[frames]; smoothed[frames]. Mirrors the
 * reference's stage split of src/engine.cpp:292-326. */
HV_API int hv_harvest_stages(const double* x, int64_t n, int fs, double f0_floor, double f0_ceil,
                             int device, double* y, double* raw, int* count, double* cand,
                             double* refined, double* scores, double* pruned,
                             double* pruned_scores, double* best, double* smoothed);

/* Contour stage on caller-given candidates: FixF0Contour and
 * SmoothF0Contour of WORLD (reference third_party/world/src/harvest.cpp:
 * 693-1113; the reference's own host adapters are src/engine.cpp:55-214),
 * run by the engine's contour kernel exactly as hv_harvest runs them after
 * pruning. f0_candidates and scores are [F][stride] row-major (F =
 * frame_offsets[clips]); clip c owns rows frame_offsets[c] ..
 * frame_offsets[c + 1] - 1 (at least one row each) and its first `columns`
 * columns are its candidates (WORLD's number_of_candidates). With base NULL
 * the base contour is SearchF0Base's (highest score per frame, first on
 * ties); otherwise FixStep1-4 start from base[F]. fixed[F] (may be NULL)
 * receives FixF0Contour's result and smoothed[F] SmoothF0Contour's. Host
 * pointers by default (the call waits); with HV_DEVICE_POINTERS every array
 * is a device pointer and the work is enqueued on `stream` as for
 * hv_harvest_batch. No counterpart of its own in the reference's ABI: it
 * exposes the stage its tests/cpp/test_contour.cpp checks. */
HV_API int hv_contour_batch(const double* f0_candidates, const double* scores, const double* base,
                            const int64_t* frame_offsets, int clips, int columns, int stride, int device,
                            double* fixed, double* smoothed, unsigned flags, void* stream);

/* Allocation-free decimation: the decimation and DC-removal stage of
 * hv_harvest on one clip, for callers that cannot allocate device memory
 * at the point of the call: real-time audio callbacks that must not block
 * inside the driver's allocator, processes whose GPU memory is wholly held
 * by a caching allocator or a fixed budget, and deployments that forbid
 * device allocation after start-up. It has no counterpart in the
 * reference, whose decimation always allocates a workspace.
 *
 * x (n samples) and y (ceil(n / r) samples, r = clamp(round(fs / 8000),
 * 1, 12)) are device pointers on `device`; the work is enqueued on `stream`
 * (a cudaStream_t of that device's primary context, NULL for its default
 * stream) and the call returns without waiting. y receives exactly what
 * hv_harvest_stages returns as y.
 *
 * The scratch is one fixed array in the library's device image (about
 * 8.6 MB, held on every GPU that loads the library until the process
 * exits), so n may not exceed 1048576 samples; longer input is rejected
 * with HV_INVALID_ARGUMENT. No cudaMalloc, cudaFree or other allocating
 * routine is called. The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) and retains the primary context;
 * make that first call before any stream capture. Every call on a device
 * shares the array and leaves its contents behind: each call writes every
 * scratch word it reads, so nothing needs clearing, but calls whose work
 * overlaps on the GPU (different streams without ordering) race on it. */
HV_API int hv_decimate_noalloc(const double* x, int64_t n, int fs, int device, double* y, void* stream);

/* Releases cached device and host working memory on every device.
 * Workspaces in use finish their call first (reference bindings.cpp:60-65,
 * src/workspace_cache.h:61-70). */
HV_API int hv_clear_cache(void);

#ifdef __cplusplus
}
#endif

#endif /* HARVEST_B200_H_ */
