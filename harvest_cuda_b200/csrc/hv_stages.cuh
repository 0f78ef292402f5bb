// Stage interfaces: the views each kernel family receives and the host-side
// launchers the engine calls. Included by the kernels and by engine.cu.
#pragma once
#include "hv_device.cuh"

namespace hv {

// Candidate in column `col` of frame `gf` after overlap: column g*K + j of
// frame f holds candidate j of frame f (g = 0), f - g (g = 1..3) or
// f + g - 3 (g = 4..6); other columns are zero.
__device__ __forceinline__ double overlapped_candidate(const BatchView& v, const double* cand,
                                                       const int* count, int64_t gf, int col) {
  int c = owner(v.frame_off, v.clips, gf);
  int64_t row0 = v.frame_off[c];
  int frames = static_cast<int>(v.frame_off[c + 1] - row0);
  int f = static_cast<int>(gf - row0);
  int k = count[c];
  if (col >= 7 * k) return 0.0;
  int g = col / k, j = col - g * k;
  int src = g == 0 ? f : (g <= 3 ? f - g : f + (g - 3));
  if (src < 0 || src >= frames) return 0.0;
  return cand[(row0 + src) * v.per_group + j];
}

struct DecimateView {
  int clips;
  int ratio;
  int lag;
  int seg_len;                 // S
  double a[3], b[2];           // FilterForDecimate coefficients for `ratio`
  double trans[9];             // A^S, row-major
  const int64_t* x_off;        // [clips + 1]
  const int64_t* y_off;        // [clips + 1]
  const int64_t* t_off;        // [clips + 1] padded-sequence offsets (T_c = n + 2 lag + 18)
  const int64_t* seg_off;      // [clips + 1] segment offsets
};

struct BankView {
  BatchView batch;
  const double* centre;      // [bands] band centre frequency
  const int* half;           // [bands] filter half length
  const int64_t* tap_off;    // [bands + 1] reversed taps, padded to kFirR
  const double* taps_rev;    // reversed taps, zero padded
  const int2* items;         // (clip, band), longest first
  int item_count;
  int max_pad_taps;          // max padded tap count over bands
  int64_t total_frames;
  int64_t slot_capacity;     // events per kind per CTA slot
  // Optional (FFT bank only; null otherwise): every block's filtered samples
  // as its event scan reads them, lookahead included, at
  // dump[(band * total_blocks + block) * (valid + 2) + q], for the adjoint of
  // the per-band candidates.
  double* dump;
};

struct ContourView {
  BatchView batch;
  const double* pruned;         // [frames][capacity]
  const double* pruned_scores;  // [frames][capacity]
  const double* best;           // [frames] SearchF0Base
  const int* count;             // [clips]
  const int64_t* scratch_off;   // [clips + 1] in doubles
  double* scratch;
  double* smoothed;             // [frames] 1 ms contour
  double period;                // frame_period in ms
  const int64_t* out_off;       // [clips + 1]
  double* f0_out;               // resampled output; skipped when null
  double* t_out;
  int column_multiple;          // candidate columns of clip c: column_multiple * count[c]
  double* fixed_out;            // [frames] FixF0Contour's result, when not null
  int extend_blocks;            // blocks per clip of the section-extension kernel
  int finish_threads;           // block size of contour_finish (256 or 512); sizes the scratch
};

// Blocks per clip of the contour's section-extension kernel for a batch
// whose longest clip has `max_frames` analysis frames.
inline int contour_extend_blocks(int64_t max_frames) {
  const int64_t b = (max_frames + 1023) / 1024;
  return static_cast<int>(b < 1 ? 1 : (b > 32 ? 32 : b));
}

// The F0 gradient holds every discrete choice of the forward pass fixed.
// Its tape has two doubles per 1 ms frame: the FixF0Contour step-3 value and,
// where that value is nonzero, the initial candidate F0 whose refinement it
// is (0 elsewhere).
struct GradView {
  BatchView batch;
  const double* tape;           // [frames][2]
  const int64_t* scratch_off;   // [clips + 1] in doubles, as ContourView
  double* scratch;
  double period;                // frame_period in ms
  const int64_t* out_off;       // [clips + 1]
  const double* grad_f0;        // [outputs] dL/df0
  double* grad_fixed;           // [frames] dL/d(step-3 value)
};

cudaError_t launch_decimate(const DecimateView& v, const double* x, double* u, double* states,
                            int64_t segments, double* y, cudaStream_t stream);
cudaError_t launch_copy(const double* x, int64_t total, double* y, cudaStream_t stream);
cudaError_t preload_decimation_kernels();
cudaError_t launch_compare(const double* ref, const double* f0, const int64_t* off, int clips, double* stats,
                           cudaStream_t stream);
cudaError_t launch_pcm16(const int16_t* in, int64_t total, double* out, int sms, cudaStream_t stream);
cudaError_t launch_check_finite(const double* x, int64_t total, int* flag, int sms, cudaStream_t stream);
// The DC removal's chunks: clip c's waveform is cut into chunks of kDcChunk
// samples, numbered chunk_off[c] .. chunk_off[c + 1] - 1 over the batch (a
// clip of no samples still has one), and parts holds 4 doubles per chunk.
constexpr int kDcChunk = 8192;
inline int64_t dc_chunk_count(int64_t samples) { return samples > 0 ? (samples + kDcChunk - 1) / kDcChunk : 1; }
struct DcChunks {
  const int64_t* chunk_off;   // [clips + 1]
  int64_t total;              // chunk_off[clips]
  double* parts;              // [total][4]
};
cudaError_t launch_remove_mean(const BatchView& v, const DcChunks& d, double* y, double* bins, cudaStream_t stream);

size_t band_bank_smem_bytes(int max_pad_taps);
int band_bank_tap_multiple();
int band_bank_threads();
int band_bank_ctas_per_sm(int max_pad_taps);
cudaError_t launch_band_bank(const BankView& v, const double* y, const double* edge_bins,
                             int* queue, double* slots, int ctas, double* raw,
                             cudaStream_t stream);

// Overlap-save geometry of the FFT band bank: real blocks of 8192 samples,
// `valid` = 8192 - 2 - 2 max_half new outputs per block.
struct FftBankGeometry {
  int max_half;
  int valid;
  int run;                 // event-scan positions per thread: even, run * 256 >= valid + 2
  int64_t total_blocks;
  const int64_t* blk_off;  // [clips + 1] block offsets
};
// Adjoint of the band bank for the per-band candidates (bank_adjoint.cu).
struct RawAdjointView {
  BatchView batch;
  FftBankGeometry geo;
  const int2* items;           // (clip, band), as the band bank's
  int item_count;
  const double* centre;        // [bands]
  const double* dump;          // band bank dump (BankView::dump)
  const double* grad_raw;      // [bands][total_frames] dL/draw
  int64_t total_frames;
  int64_t slot_capacity;       // events per kind per CTA
  double* edges;               // per CTA [4][slot_capacity]: fine edges
  long long* where;            // per CTA [4][slot_capacity]: block * (valid + 2) + q of each event
  double* grad_edges;          // per CTA [4][slot_capacity]: dL/de
  int* queue;
  double* grad_f;              // [bands][y_total] dL/df_b, zeroed
  int64_t y_total;
};
cudaError_t launch_raw_adjoint(const RawAdjointView& v, int ctas, cudaStream_t stream);
cudaError_t launch_band_correlate(const BatchView& v, const double* grad_f, int64_t y_total, const int* half,
                                  const int64_t* tap_off, const double* taps_rev, double* grad_y,
                                  cudaStream_t stream);

// Entries of the workspace twiddle table e^{-2 pi i t / kTwiddleN} (the FFT
// band bank's real block length).
constexpr int kTwiddleN = 8192;
size_t fft_bank_smem_bytes();
int fft_bank_block_length();
int fft_bank_ctas_per_sm();
cudaError_t launch_twiddles(double2* tw, cudaStream_t stream);
cudaError_t launch_filter_spectra(const int* half, const int64_t* tap_off, const double* taps_rev, int bands,
                                  int max_half, const double2* tw, double* amps, cudaStream_t stream);
cudaError_t launch_fft_bank(const BankView& v, const FftBankGeometry& g, const double* y, const double* edge_bins,
                            const double2* tw, const double* amps, double2* spectra, int* queue,
                            double* slots, int ctas, double* raw, cudaStream_t stream);

cudaError_t launch_candidates(const BatchView& v, const double* raw, int64_t total_frames,
                              double* cand, int* count, cudaStream_t stream);
constexpr int kRefineClasses = 72;   // quarter-octave window-length classes
constexpr int kRefineColumns = 1024; // job key = frame * kRefineColumns + column
// Bits 41-47 of a job key: the overlap groups whose cells share the job's
// spectra (frame * kRefineColumns + column stays below 2^41).
constexpr int kJobSiblingShift = 41;
struct RefineJob {
  double f0c;
  long long key;
};
struct RefineBuffers {
  int* class_count;    // [kRefineClasses]
  int* class_cursor;   // [kRefineClasses]
  int* total;          // [1]
  RefineJob* jobs;     // [frames * capacity]
  ulonglong2* keys;    // [frames * per_group] refinement key of every official candidate
  unsigned long long* leaders;  // [frames * per_group][2] job classes and sibling masks of the 7 overlap cells
  int64_t* item_off;   // [clips + 1] bucket items (frame, official candidate) per clip, prefix
  const double2* twiddles;  // [kTwiddleN] e^{-2 pi i t / kTwiddleN}
};
// Launch shape of the refinement jobs: minimum resident 128-thread blocks per
// SM the kernel instance is compiled for (1, 4 or 5; fewer registers per
// thread for more blocks) and grid blocks per SM. Every shape computes the
// same values bit for bit.
struct RefineShape {
  int min_blocks = 4;
  int blocks_per_sm = 32;
};

cudaError_t launch_refine(const BatchView& v, const RefineBuffers& b, const double* y,
                          const double* cand, const int* count, int64_t total_frames, double* refined,
                          double* scores, int sms, RefineShape shape, cudaStream_t stream);
cudaError_t launch_prune(const BatchView& v, const double* refined, const double* scores,
                         const int* count, int64_t total_frames, double* pruned,
                         double* pruned_scores, double* best, cudaStream_t stream);

int64_t contour_scratch(int64_t frames, int finish_threads);
cudaError_t launch_tape(const ContourView& v, const double* cand, int64_t total_frames, double* tape,
                        cudaStream_t stream);
cudaError_t launch_contour_adjoint(const GradView& v, cudaStream_t stream);
cudaError_t launch_refine_adjoint(const BatchView& v, const double* y, const double* tape,
                                  const double* grad_fixed, int64_t total_frames, const double2* tw,
                                  double* grad_y, int sms, cudaStream_t stream);
cudaError_t launch_remove_mean_adjoint(const BatchView& v, const DcChunks& d, double* grad_y, cudaStream_t stream);
cudaError_t launch_decimate_adjoint(const DecimateView& v, const double* grad_y, double* u, double* states,
                                    int64_t segments, double* grad_x, cudaStream_t stream);
cudaError_t launch_contour(const ContourView& v, cudaStream_t stream);
cudaError_t launch_search_base(const double* cand, const double* scores, int64_t total_frames, int stride,
                               const int64_t* frame_off, int clips, const int* columns, double* base,
                               cudaStream_t stream);

}  // namespace hv
