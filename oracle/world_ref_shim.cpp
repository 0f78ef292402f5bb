// TEST INFRASTRUCTURE ONLY — never linked into or called by the product.
//
// C-ABI shim over the reference's bundled WORLD Harvest (pyworld 0.3.5
// sources, third_party/world/src/*.cpp). The Makefile in this directory
// compiles those sources where they lie in the reference tree together with
// this file into oracle/_ref/libworld_ref.so. Including harvest.cpp gives this
// translation unit the file-static stage routines, the same technique the
// reference uses in src/engine.cpp:11-13, so every stage can be dumped.
//
// Exported symbols match oracle/harvest_oracle.c so tests can swap the two.
#include "harvest.cpp"  // third_party/world/src/harvest.cpp (via -I)

#include <cstring>
#include <vector>

namespace {
struct Params {
  int ratio, y_len, fft_size, bands, frames, capacity;
  double fs_r;
};

// Parameter derivation of HarvestGeneralBody (harvest.cpp:1149-1181) and
// Harvest (harvest.cpp:1226-1228).
Params derive(int n, int fs, double f0_floor, double f0_ceil) {
  Params p;
  double adjusted_floor = f0_floor * 0.9, adjusted_ceil = f0_ceil * 1.1;
  p.bands = 1 + static_cast<int>(log(adjusted_ceil / adjusted_floor) /
                                 world::kLog2 * 40.0);
  int speed = matlab_round(fs / 8000.0);
  p.ratio = MyMaxInt(MyMinInt(speed, 12), 1);
  p.y_len = static_cast<int>(ceil(static_cast<double>(n) / p.ratio));
  p.fs_r = static_cast<double>(fs) / p.ratio;
  double b0 = adjusted_floor * pow(2.0, 1.0 / 40.0);
  p.fft_size = GetSuitableFFTSize(p.y_len + 5 + 2 * static_cast<int>(2.0 * p.fs_r / b0));
  p.frames = GetSamplesForHarvest(fs, n, 1);
  p.capacity = matlab_round(p.bands / 10.0) * 7;
  return p;
}
}  // namespace

extern "C" {

int oracle_params(int n, int fs, double f0_floor, double f0_ceil, int* out) {
  Params p = derive(n, fs, f0_floor, f0_ceil);
  out[0] = p.ratio; out[1] = p.y_len; out[2] = p.fft_size;
  out[3] = p.bands; out[4] = p.frames; out[5] = p.capacity;
  return 0;
}

int oracle_output_length(int n, int fs, double period) {
  return GetSamplesForHarvest(fs, n, period);
}

// Whole pipeline: WORLD's public entry point (harvest.cpp:1223-1255).
void oracle_harvest(const double* x, int n, int fs, double f0_floor, double f0_ceil,
                    double period, double* times, double* f0) {
  HarvestOption option{f0_floor, f0_ceil, period};
  Harvest(x, n, fs, &option, times, f0);
}

// Stage dump on the 1 ms grid, in the order of HarvestGeneralBody
// (harvest.cpp:1145-1215). Array shapes (row-major):
//   y[y_len], raw[bands*frames], cand/refined/scores/pruned/pruned_scores
//   [frames*capacity], base/fixed/smoothed[frames]; *count = candidates per
//   frame before overlap (the returned number of columns is 7 * *count).
void oracle_stages(const double* x, int n, int fs, double f0_floor, double f0_ceil,
                   double* y_out, double* raw_out, int* count_out,
                   double* cand_out, double* refined_out, double* scores_out,
                   double* pruned_out, double* pruned_scores_out,
                   double* base_out, double* fixed_out, double* smoothed_out) {
  Params p = derive(n, fs, f0_floor, f0_ceil);
  std::vector<double> boundaries(p.bands);
  double adjusted_floor = f0_floor * 0.9;
  for (int i = 0; i < p.bands; ++i)
    boundaries[i] = adjusted_floor * pow(2.0, (i + 1) / 40.0);

  std::vector<double> y(p.fft_size);
  std::vector<fft_complex> spectrum(p.fft_size);
  GetWaveformAndSpectrum(x, n, p.y_len, p.fs_r, p.fft_size, p.ratio, y.data(),
                         spectrum.data());
  std::memcpy(y_out, y.data(), sizeof(double) * p.y_len);

  std::vector<double> times(p.frames);
  for (int i = 0; i < p.frames; ++i) times[i] = i * 1 / 1000.0;

  std::vector<double> raw_storage(size_t(p.bands) * p.frames);
  std::vector<double*> raw(p.bands);
  for (int b = 0; b < p.bands; ++b) raw[b] = raw_storage.data() + size_t(b) * p.frames;
  GetRawF0Candidates(boundaries.data(), p.bands, p.fs_r, p.y_len, times.data(),
                     p.frames, spectrum.data(), p.fft_size, f0_floor, f0_ceil, raw.data());
  std::memcpy(raw_out, raw_storage.data(), sizeof(double) * raw_storage.size());

  std::vector<double> cand_storage(size_t(p.frames) * p.capacity, 0.0);
  std::vector<double> score_storage(size_t(p.frames) * p.capacity, 0.0);
  std::vector<double*> cand(p.frames), score(p.frames);
  for (int i = 0; i < p.frames; ++i) {
    cand[i] = cand_storage.data() + size_t(i) * p.capacity;
    score[i] = score_storage.data() + size_t(i) * p.capacity;
  }
  int count = DetectOfficialF0Candidates(raw.data(), p.bands, p.frames, p.capacity,
                                         cand.data());
  OverlapF0Candidates(p.frames, count, cand.data());
  *count_out = count;
  std::memcpy(cand_out, cand_storage.data(), sizeof(double) * cand_storage.size());

  int columns = count * 7;
  RefineF0Candidates(y.data(), p.y_len, p.fs_r, times.data(), p.frames, columns,
                     f0_floor, f0_ceil, cand.data(), score.data());
  std::memcpy(refined_out, cand_storage.data(), sizeof(double) * cand_storage.size());
  std::memcpy(scores_out, score_storage.data(), sizeof(double) * score_storage.size());

  RemoveUnreliableCandidates(p.frames, columns, cand.data(), score.data());
  std::memcpy(pruned_out, cand_storage.data(), sizeof(double) * cand_storage.size());
  std::memcpy(pruned_scores_out, score_storage.data(),
              sizeof(double) * score_storage.size());

  SearchF0Base(cand.data(), score.data(), p.frames, columns, base_out);
  FixF0Contour(cand.data(), score.data(), p.frames, columns, fixed_out);
  for (int i = 0; i < p.frames; ++i) smoothed_out[i] = 0.0;
  SmoothF0Contour(fixed_out, p.frames, smoothed_out);
}

// FixF0Contour alone (harvest.cpp:1027-1044) on caller-provided candidates,
// for contour-stage unit tests with synthetic candidate tracks.
void oracle_fix_contour(const double* cand, const double* scores, int frames,
                        int columns, int stride, double* fixed_out) {
  std::vector<const double*> c(frames), s(frames);
  for (int i = 0; i < frames; ++i) {
    c[i] = cand + size_t(i) * stride;
    s[i] = scores + size_t(i) * stride;
  }
  FixF0Contour(c.data(), s.data(), frames, columns, fixed_out);
}

// FixStep1-4 of FixF0Contour (harvest.cpp:1027-1044) from a caller-given
// base contour in place of SearchF0Base's.
void oracle_fix_contour_base(const double* base, const double* cand, const double* scores, int frames,
                             int columns, int stride, double* fixed_out) {
  std::vector<const double*> c(frames), s(frames);
  for (int i = 0; i < frames; ++i) {
    c[i] = cand + size_t(i) * stride;
    s[i] = scores + size_t(i) * stride;
  }
  std::vector<double> a(frames + 1), b(frames + 1);
  FixStep1(base, frames, 0.008, b.data());
  FixStep2(b.data(), frames, 6, a.data());
  FixStep3(a.data(), frames, columns, c.data(), 0.18, s.data(), b.data());
  FixStep4(b.data(), frames, 9, fixed_out);
}

// SmoothF0Contour alone (harvest.cpp:1079-1113).
void oracle_smooth_contour(const double* f0, int frames, double* out) {
  for (int i = 0; i < frames; ++i) out[i] = 0.0;
  SmoothF0Contour(f0, frames, out);
}

}  // extern "C"
