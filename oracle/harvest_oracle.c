/*
 * harvest_oracle.c — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of WORLD's Harvest F0 estimator as bundled with the
 * reference (third_party/world/src/harvest.cpp, matlabfunctions.cpp,
 * common.cpp; pyworld 0.3.5 sources). It is the checker that the CUDA engine
 * is compared against in tests/, in __graft_entry__.smoke() and in the CPU
 * baseline leg of bench.py. The product never loads it.
 *
 * Every stage function names the reference lines it restates. The quirks of
 * the reference are part of the algorithm and are restated deliberately:
 * the overwritten final spectrum bins, the unnormalised inverse FFT, the
 * half+1 delay, histc's end clamping, GetBoundaryList's i - count%2, the
 * carried mean of ExtendSub, MakeSortedOrder's partial sort and MergeF0's
 * reuse of boundary pair 0.
 *
 * The one deliberate difference: the FFT is a textbook radix-2 transform
 * written here (WORLD uses Ooura's rdft, fft.cpp). Its results therefore
 * differ from WORLD's in the last bits; tests pin this file against the
 * reference library built from the reference sources (oracle/_ref).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.1415926535897932384    /* world::kPi, constantnumbers.h:18 */
#define ORC_LN2 0.69314718055994529     /* world::kLog2, constantnumbers.h:24 */
#define ORC_GUARD 0.000000000001        /* kMySafeGuardMinimum, :19 */

typedef struct { double re, im; } cplx;

/* matlab_round (matlabfunctions.cpp:206-208): half away from zero. */
static int round_away(double v) { return v > 0 ? (int)(v + 0.5) : (int)(v - 0.5); }
static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

/* GetSuitableFFTSize (common.cpp:51-54). */
static int suitable_fft_size(int samples) {
  return (int)pow(2.0, (int)(log((double)samples) / ORC_LN2) + 1.0);
}

/* GetSamplesForHarvest (harvest.cpp:1219-1221). */
static int frames_for(int fs, int n, double period) {
  return (int)(1000.0 * n / fs / period) + 1;
}

typedef struct {
  int ratio, y_len, fft_size, bands, frames, capacity;
  double fs_r;
} orc_params;

/* Parameter derivation, HarvestGeneralBody (harvest.cpp:1149-1181) with the
 * ratio from Harvest (harvest.cpp:1226-1228). */
static orc_params derive(int n, int fs, double f0_floor, double f0_ceil) {
  orc_params p;
  double lo = f0_floor * 0.9, hi = f0_ceil * 1.1;
  p.bands = 1 + (int)(log(hi / lo) / ORC_LN2 * 40.0);
  p.ratio = imax(imin(round_away(fs / 8000.0), 12), 1);
  p.y_len = (int)ceil((double)n / p.ratio);
  p.fs_r = (double)fs / p.ratio;
  double first = lo * pow(2.0, 1 / 40.0);
  p.fft_size = suitable_fft_size(p.y_len + 5 + 2 * (int)(2.0 * p.fs_r / first));
  p.frames = frames_for(fs, n, 1.0);
  p.capacity = round_away(p.bands / 10.0) * 7;
  return p;
}

/* ------------------------------------------------------------------------ */
/* FFT written for this checker (not Ooura's): iterative radix-2, in place.
 * sign = -1 computes sum a[j] e^{-2 pi i jk/n}; sign = +1 the unnormalised
 * inverse. Conventions match WORLD's wrappers (fft.cpp:26-72): forward r2c
 * with the e^{-i} kernel, c2r unnormalised and ignoring the imaginary parts
 * of bins 0 and n/2. */
static void fft_c2c(cplx* a, int n, int sign) {
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j |= bit;
    if (i < j) { cplx t = a[i]; a[i] = a[j]; a[j] = t; }
  }
  for (int len = 2; len <= n; len <<= 1) {
    int half = len >> 1;
    for (int k = 0; k < half; ++k) {
      double angle = 2.0 * ORC_PI * k / len;
      double wr = cos(angle), wi = sign * sin(angle);
      for (int i = k; i < n; i += len) {
        cplx u = a[i], v = a[i + half];
        double tr = v.re * wr - v.im * wi, ti = v.re * wi + v.im * wr;
        a[i].re = u.re + tr; a[i].im = u.im + ti;
        a[i + half].re = u.re - tr; a[i + half].im = u.im - ti;
      }
    }
  }
}

static void rfft(const double* x, int n, cplx* out /* n/2+1 */, cplx* work /* n */) {
  for (int i = 0; i < n; ++i) { work[i].re = x[i]; work[i].im = 0.0; }
  fft_c2c(work, n, -1);
  for (int k = 0; k <= n / 2; ++k) out[k] = work[k];
  out[0].im = 0.0;
  out[n / 2].im = 0.0;
}

static void irfft_unnormalised(const cplx* in /* n/2+1 */, int n, double* out, cplx* work) {
  work[0].re = in[0].re; work[0].im = 0.0;
  work[n / 2].re = in[n / 2].re; work[n / 2].im = 0.0;
  for (int k = 1; k < n / 2; ++k) {
    work[k] = in[k];
    work[n - k].re = in[k].re; work[n - k].im = -in[k].im;
  }
  fft_c2c(work, n, +1);
  for (int i = 0; i < n; ++i) out[i] = work[i].re;
}

/* ------------------------------------------------------------------------ */
/* a2: decimation. Coefficients of the order-3 low-pass per ratio, the table of
 * FilterForDecimate (matlabfunctions.cpp:27-113); rows 0 and 1 unused. */
static const double kLowpassA[13][3] = {
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
  {2.4981398605924205, -2.1368928194784025, 0.62187513816221485},
};
static const double kLowpassB[13][2] = {
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
  {0.0021097275904709001, 0.0063291827714127002},
};

/* One causal pass (matlabfunctions.cpp:115-124), direct form II, written so
 * the evaluation order of each output matches the reference expression. */
static void lowpass_pass(const double* in, int len, int r, double* out) {
  const double* a = kLowpassA[r];
  const double* b = kLowpassB[r];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int i = 0; i < len; ++i) {
    double w = in[i] + a[0] * s0 + a[1] * s1 + a[2] * s2;
    out[i] = b[0] * w + b[1] * s0 + b[1] * s1 + b[0] * s2;
    s2 = s1; s1 = s0; s0 = w;
  }
}

/* GetWaveformAndSpectrumSub (harvest.cpp:43-66) + decimate
 * (matlabfunctions.cpp:178-204): edge-hold padding by `lag`, 9-sample odd
 * reflection, forward-backward low-pass, every r-th sample. */
static void decimate_for_f0(const double* x, int n, int r, int y_len, double* y) {
  if (r == 1) { memcpy(y, x, sizeof(double) * (size_t)n); return; }
  int lag = (int)(ceil(140.0 / r) * r);
  int m = n + 2 * lag;
  int total = m + 18;
  double* ext = malloc(sizeof(double) * (size_t)m);
  double* a = malloc(sizeof(double) * (size_t)total);
  double* b = malloc(sizeof(double) * (size_t)total);
  for (int i = 0; i < m; ++i) ext[i] = x[imin(imax(i - lag, 0), n - 1)];
  for (int i = 0; i < 9; ++i) a[i] = 2 * ext[0] - ext[9 - i];
  for (int i = 0; i < m; ++i) a[9 + i] = ext[i];
  for (int i = 0; i < 9; ++i) a[9 + m + i] = 2 * ext[m - 1] - ext[m - 2 - i];
  lowpass_pass(a, total, r, b);
  for (int i = 0; i < total; ++i) a[i] = b[total - 1 - i];
  lowpass_pass(a, total, r, b);
  for (int i = 0; i < total; ++i) a[i] = b[total - 1 - i];
  int nout = (m - 1) / r + 1;
  int nbeg = r - r * nout + m;
  int skip = lag / r;
  for (int i = 0; i < y_len; ++i) y[i] = a[nbeg + (skip + i) * r + 8];
  free(ext); free(a); free(b);
}

/* a3: DC removal, sequential sum (harvest.cpp:82-86). */
static void remove_mean(double* y, int len) {
  double mean = 0.0;
  for (int i = 0; i < len; ++i) mean += y[i];
  mean /= len;
  for (int i = 0; i < len; ++i) y[i] -= mean;
}

/* ------------------------------------------------------------------------ */
/* a5-a7: one band of the filter bank, GetFilteredSignal (harvest.cpp:99-148)
 * with NuttallWindow (common.cpp:113-121). `spec` is rfft(y zero-padded). */
static void band_filter(double centre, int n, double fs, const cplx* spec, int y_len,
                        double* filtered /* n */, double* taps /* n */, cplx* full /* n */,
                        cplx* work /* n */) {
  int half = round_away(fs / centre * 2.0);
  int len = half * 2 + 1;
  for (int i = 0; i < len; ++i) {
    double t = i / (len - 1.0);
    taps[i] = 0.355768 - 0.487396 * cos(2.0 * ORC_PI * t) +
              0.144232 * cos(4.0 * ORC_PI * t) - 0.012604 * cos(6.0 * ORC_PI * t);
  }
  for (int i = -half; i <= half; ++i) taps[i + half] *= cos(2 * ORC_PI * centre * i / fs);
  for (int i = len; i < n; ++i) taps[i] = 0.0;
  rfft(taps, n, full, work);
  /* Spectrum product. The reference mirrors each product into bin n-i-1 while
   * it walks upwards, so bin n/2 is overwritten with product n/2-1 before it
   * is multiplied, and bin n/2-1 receives that result (harvest.cpp:116-133). */
  for (int k = n / 2 + 1; k < n; ++k) full[k].re = full[k].im = 0.0;
  for (int i = 0; i <= n / 2; ++i) {
    double re = spec[i].re * full[i].re - spec[i].im * full[i].im;
    double im = spec[i].re * full[i].im + spec[i].im * full[i].re;
    full[i].re = re; full[i].im = im;
    if (i >= 1) full[n - i - 1] = full[i];
  }
  irfft_unnormalised(full, n, filtered, work);
  int bias = half + 1;
  for (int i = 0; i < y_len; ++i) filtered[i] = filtered[i + bias];
}

/* a8: negative-going zero crossings of s[0..len) and their intervals,
 * ZeroCrossingEngine (harvest.cpp:162-197). Returns the interval count. */
static int crossing_intervals(const double* s, int len, double fs, double* where,
                              double* value, double* fine /* len */) {
  int count = 0;
  for (int i = 0; i + 1 < len; ++i) {
    if (0.0 < s[i] && s[i + 1] <= 0.0) {
      int e = i + 1;
      fine[count++] = e - s[e - 1] / (s[e] - s[e - 1]);
    }
  }
  if (count < 2) return 0;
  for (int i = 0; i + 1 < count; ++i) {
    value[i] = fs / (fine[i + 1] - fine[i]);
    where[i] = (fine[i] + fine[i + 1]) / 2.0 / fs;
  }
  return count - 1;
}

/* a9: interp1 with histc's end clamping (matlabfunctions.cpp:136-176): the
 * segment index is the count of knots <= t, clamped to [1, count-1]. */
static void interp_clamped(const double* xk, const double* yk, int count, const double* t,
                           int frames, double* out) {
  int k = 0; /* number of knots <= t, monotone in t */
  for (int f = 0; f < frames; ++f) {
    while (k < count && xk[k] <= t[f]) ++k;
    int seg = imin(imax(k, 1), count - 1);
    double s = (t[f] - xk[seg - 1]) / (xk[seg] - xk[seg - 1]);
    out[f] = yk[seg - 1] + s * (yk[seg] - yk[seg - 1]);
  }
}

/* a8-a9 for one band: GetFourZeroCrossingIntervals (harvest.cpp:206-238),
 * GetF0CandidateContour(Sub) (harvest.cpp:240-293). Mutates `f`. */
static void band_candidates(double* f, int y_len, double fs, double centre, double f0_floor,
                            double f0_ceil, const double* t, int frames, double* out,
                            double* buf /* 9 * y_len */) {
  double* where[4]; double* value[4]; int count[4];
  double* fine = buf + 8 * (size_t)y_len;
  for (int k = 0; k < 4; ++k) {
    where[k] = buf + (size_t)(2 * k) * y_len;
    value[k] = buf + (size_t)(2 * k + 1) * y_len;
  }
  count[0] = crossing_intervals(f, y_len, fs, where[0], value[0], fine);
  for (int i = 0; i < y_len; ++i) f[i] = -f[i];
  count[1] = crossing_intervals(f, y_len, fs, where[1], value[1], fine);
  for (int i = 0; i + 1 < y_len; ++i) f[i] = f[i] - f[i + 1];
  count[2] = crossing_intervals(f, y_len - 1, fs, where[2], value[2], fine);
  for (int i = 0; i + 1 < y_len; ++i) f[i] = -f[i];
  count[3] = crossing_intervals(f, y_len - 1, fs, where[3], value[3], fine);
  if (count[0] <= 2 || count[1] <= 2 || count[2] <= 2 || count[3] <= 2) {
    for (int i = 0; i < frames; ++i) out[i] = 0.0;
    return;
  }
  double* tmp = malloc(sizeof(double) * 4 * (size_t)frames);
  for (int k = 0; k < 4; ++k)
    interp_clamped(where[k], value[k], count[k], t, frames, tmp + (size_t)k * frames);
  double upper = centre * 1.1, lower = centre * 0.9;
  for (int i = 0; i < frames; ++i) {
    double v = (tmp[i] + tmp[frames + i] + tmp[2 * frames + i] + tmp[3 * frames + i]) / 4.0;
    if (v > upper || v < lower || v > f0_ceil || v < f0_floor) v = 0.0;
    out[i] = v;
  }
  free(tmp);
}

/* a10: DetectOfficialF0Candidates(Sub1/Sub2) (harvest.cpp:348-412). Writes
 * [frames][capacity] with zero fill; returns the maximum count per frame. */
static int official_candidates(const double* raw, int bands, int frames, int capacity,
                               double* cand) {
  int best = 0;
  for (int f = 0; f < frames; ++f) {
    double* row = cand + (size_t)f * capacity;
    int n = 0, start = -1;
    for (int b = 1; b < bands; ++b) {
      int now = b == bands - 1 ? 0 : raw[(size_t)b * frames + f] > 0;
      int before = b - 1 == 0 ? 0 : raw[(size_t)(b - 1) * frames + f] > 0;
      if (now - before == 1) start = b;
      if (now - before == -1) {
        int end = b;
        if (end - start >= 10) {
          double sum = 0.0;
          for (int j = start; j < end; ++j) sum += raw[(size_t)j * frames + f];
          sum /= (end - start);
          row[n++] = sum;
        }
      }
    }
    for (int j = n; j < capacity; ++j) row[j] = 0.0;
    if (n > best) best = n;
  }
  return best;
}

/* a11: OverlapF0Candidates (harvest.cpp:417-429). */
static void overlap_candidates(int frames, int count, int capacity, double* cand) {
  for (int i = 1; i <= 3; ++i)
    for (int j = 0; j < count; ++j) {
      for (int k = i; k < frames; ++k)
        cand[(size_t)k * capacity + j + count * i] = cand[(size_t)(k - i) * capacity + j];
      for (int k = 0; k < frames - i; ++k)
        cand[(size_t)k * capacity + j + count * (i + 3)] = cand[(size_t)(k + i) * capacity + j];
    }
}

/* a12: GetRefinedF0 / GetMeanF0 / GetBaseIndex / GetMainWindow /
 * GetDiffWindow / GetSpectra / FixF0 (harvest.cpp:434-617). */
static void refine_one(const double* y, int y_len, double fs, double t, double f0c,
                       double f0_floor, double f0_ceil, double* f0_out, double* score_out) {
  if (f0c <= 0.0) { *f0_out = 0.0; *score_out = 0.0; return; }
  int half = (int)(1.5 * fs / f0c + 1.0);
  int len = half * 2 + 1;
  double span = (2.0 * half + 1.0) / fs;
  int n = (int)pow(2.0, 2.0 + (int)(log(half * 2.0 + 1.0) / ORC_LN2));
  int base = round_away((t + (-half) / fs) * fs + 0.001);
  double* w = malloc(sizeof(double) * (size_t)len);
  double* dw = malloc(sizeof(double) * (size_t)len);
  double* buf = malloc(sizeof(double) * (size_t)n);
  cplx* work = malloc(sizeof(cplx) * (size_t)n);
  cplx* main_s = malloc(sizeof(cplx) * (size_t)(n / 2 + 1));
  cplx* diff_s = malloc(sizeof(cplx) * (size_t)(n / 2 + 1));
  for (int i = 0; i < len; ++i) {
    double tmp = (base + i - 1.0) / fs - t;
    w[i] = 0.42 + 0.5 * cos(2.0 * ORC_PI * tmp / span) + 0.08 * cos(4.0 * ORC_PI * tmp / span);
  }
  dw[0] = -w[1] / 2.0;
  for (int i = 1; i < len - 1; ++i) dw[i] = -(w[i + 1] - w[i - 1]) / 2.0;
  dw[len - 1] = w[len - 2] / 2.0;
  for (int pass = 0; pass < 2; ++pass) {
    const double* win = pass ? dw : w;
    for (int i = 0; i < len; ++i) buf[i] = y[imax(0, imin(y_len - 1, base + i - 1))] * win[i];
    for (int i = len; i < n; ++i) buf[i] = 0.0;
    rfft(buf, n, pass ? diff_s : main_s, work);
  }
  int harmonics = imin((int)(fs / 2.0 / f0c), 6);
  double num = 0.0, den = 0.0, err = 0.0;
  for (int h = 0; h < harmonics; ++h) {
    int k = round_away(f0c * n / fs * (h + 1));
    double power = main_s[k].re * main_s[k].re + main_s[k].im * main_s[k].im;
    double cross = main_s[k].re * diff_s[k].im - main_s[k].im * diff_s[k].re;
    double inst = power == 0.0 ? 0.0 : (double)k * fs / n + cross / power * fs / 2.0 / ORC_PI;
    double amp = sqrt(power);
    num += amp * inst;
    den += amp * (h + 1.0);
    err += fabs((inst / (h + 1.0) - f0c) / f0c);
  }
  double refined = num / (den + ORC_GUARD);
  double score = 1.0 / (err / harmonics + ORC_GUARD);
  if (refined < f0_floor || refined > f0_ceil || score < 2.5) refined = score = 0.0;
  *f0_out = refined; *score_out = score;
  free(w); free(dw); free(buf); free(work); free(main_s); free(diff_s);
}

/* a13: SelectBestF0 (harvest.cpp:636-650). */
static double select_best(double ref, const double* cand, int count, double allowed,
                          double* best_error) {
  double best = 0.0;
  *best_error = allowed;
  for (int i = 0; i < count; ++i) {
    double e = fabs(ref - cand[i]) / ref;
    if (e > *best_error) continue;
    best = cand[i];
    *best_error = e;
  }
  return best;
}

/* a13: RemoveUnreliableCandidates(Sub) (harvest.cpp:652-688). */
static void prune(int frames, int columns, int stride, double* cand, double* score) {
  double* orig = malloc(sizeof(double) * (size_t)frames * (size_t)(columns ? columns : 1));
  for (int f = 0; f < frames; ++f)
    for (int j = 0; j < columns; ++j) orig[(size_t)f * columns + j] = cand[(size_t)f * stride + j];
  for (int f = 1; f < frames - 1; ++f)
    for (int j = 0; j < columns; ++j) {
      double ref = cand[(size_t)f * stride + j];
      if (ref == 0) continue;
      double e1, e2;
      select_best(ref, orig + (size_t)(f + 1) * columns, columns, 1.0, &e1);
      select_best(ref, orig + (size_t)(f - 1) * columns, columns, 1.0, &e2);
      double e = e1 < e2 ? e1 : e2;
      if (e <= 0.05) continue;
      cand[(size_t)f * stride + j] = 0;
      score[(size_t)f * stride + j] = 0;
    }
  free(orig);
}

/* SearchF0Base (harvest.cpp:693-705). */
static void best_per_frame(const double* cand, const double* score, int frames, int columns,
                           int stride, double* out) {
  for (int f = 0; f < frames; ++f) {
    double top = 0.0;
    out[f] = 0.0;
    for (int j = 0; j < columns; ++j)
      if (score[(size_t)f * stride + j] > top) {
        out[f] = cand[(size_t)f * stride + j];
        top = score[(size_t)f * stride + j];
      }
  }
}

/* ------------------------------------------------------------------------ */
/* a14: FixF0Contour and its steps (harvest.cpp:710-1044). */

/* GetBoundaryList (harvest.cpp:727-743): rising edges at the first voiced
 * frame, falling edges at the last voiced frame; both ends forced unvoiced. */
static int boundary_list(const double* f0, int len, int* out) {
  int count = 0, prev = 0;
  for (int i = 1; i < len; ++i) {
    int v = (i == len - 1) ? 0 : f0[i] > 0;
    if (v != prev) { out[count] = i - count % 2; ++count; }
    prev = v;
  }
  return count;
}

static void fix_step1(const double* base, int frames, double allowed, double* out) {
  for (int i = 0; i < frames; ++i) out[i] = 0.0;
  for (int i = 2; i < frames; ++i) {
    if (base[i] == 0.0) continue;
    double ref = base[i - 1] * 2 - base[i - 2];
    out[i] = fabs((base[i] - ref) / ref) > allowed &&
             fabs((base[i] - base[i - 1])) / base[i - 1] > allowed ? 0.0 : base[i];
  }
}

static void fix_step2(const double* in, int frames, int minimum, double* out, int* bl) {
  memcpy(out, in, sizeof(double) * (size_t)frames);
  int nb = boundary_list(in, frames, bl);
  for (int i = 0; i < nb / 2; ++i) {
    if (bl[2 * i + 1] - bl[2 * i] >= minimum) continue;
    for (int j = bl[2 * i]; j <= bl[2 * i + 1]; ++j) out[j] = 0.0;
  }
}

/* ExtendF0 (harvest.cpp:791-820). */
static int extend_one(int frames, int origin, int last, int shift, const double* cand,
                      int columns, int stride, double allowed, double* ext) {
  (void)frames;
  double cur = ext[origin];
  int reached = origin, misses = 0;
  int distance = abs(last - origin);
  for (int i = 0; i <= distance; ++i) {
    int idx = origin + shift * i + shift;
    double dummy;
    ext[idx] = select_best(cur, cand + (size_t)idx * stride, columns, allowed, &dummy);
    if (ext[idx] == 0.0) {
      ++misses;
    } else {
      cur = ext[idx];
      misses = 0;
      reached = idx;
    }
    if (misses == 4) break;
  }
  return reached;
}

/* SearchScore (harvest.cpp:901-907). */
static double search_score(double f0, const double* cand, const double* score, int columns) {
  double s = 0.0;
  for (int i = 0; i < columns; ++i)
    if (f0 == cand[i] && s < score[i]) s = score[i];
  return s;
}

/* FixStep3: GetMultiChannelF0, Extend, ExtendSub, MakeSortedOrder, MergeF0,
 * MergeF0Sub (harvest.cpp:767-995). Sections are kept as full-length rows,
 * like the reference, and swapped by index. */
static void fix_step3(const double* in, int frames, int columns, int stride, const double* cand,
                      double allowed, const double* score, double* out, int* bl) {
  memcpy(out, in, sizeof(double) * (size_t)frames);
  int nb = boundary_list(in, frames, bl);
  int sections = nb / 2;
  if (sections == 0) return;
  double** ch = malloc(sizeof(double*) * (size_t)sections);
  for (int i = 0; i < sections; ++i) {
    ch[i] = calloc((size_t)frames, sizeof(double));
    for (int j = bl[2 * i]; j <= bl[2 * i + 1]; ++j) ch[i][j] = in[j];
  }
  /* Extend (harvest.cpp:861-878): forward from the end, then backward. */
  for (int i = 0; i < sections; ++i) {
    int end = bl[2 * i + 1], start = bl[2 * i];
    bl[2 * i + 1] = extend_one(frames, end, imin(frames - 2, end + 100), 1, cand, columns,
                               stride, allowed, ch[i]);
    bl[2 * i] = extend_one(frames, start, imax(1, start - 100), -1, cand, columns, stride,
                           allowed, ch[i]);
  }
  /* ExtendSub (harvest.cpp:840-856): the running mean is never reset. */
  int kept = 0;
  double mean = 0.0;
  for (int i = 0; i < sections; ++i) {
    int st = bl[2 * i], ed = bl[2 * i + 1];
    for (int j = st; j < ed; ++j) mean += ch[i][j];
    mean /= ed - st;
    if (2200.0 / mean < ed - st) {
      double* tp = ch[kept]; ch[kept] = ch[i]; ch[i] = tp;
      int t0 = bl[2 * kept], t1 = bl[2 * kept + 1];
      bl[2 * kept] = bl[2 * i]; bl[2 * kept + 1] = bl[2 * i + 1];
      bl[2 * i] = t0; bl[2 * i + 1] = t1;
      ++kept;
    }
  }
  if (kept != 0) {
    /* MakeSortedOrder (harvest.cpp:883-896), restated as written: the inner
     * loop swaps entries i and j and stops at the first non-inversion. */
    int* order = malloc(sizeof(int) * (size_t)kept);
    for (int i = 0; i < kept; ++i) order[i] = i;
    for (int i = 1; i < kept; ++i)
      for (int j = i - 1; j >= 0; --j) {
        if (bl[order[j] * 2] > bl[order[i] * 2]) {
          int t = order[i]; order[i] = order[j]; order[j] = t;
        } else {
          break;
        }
      }
    /* MergeF0 (harvest.cpp:937-963); pair 0 of the list is reused as the
     * running merged extent. */
    for (int i = 0; i < frames; ++i) out[i] = ch[0][i];
    for (int i = 1; i < kept; ++i) {
      int o = order[i];
      int st2 = bl[2 * o], ed2 = bl[2 * o + 1];
      if (st2 - bl[1] > 0) {
        for (int j = st2; j <= ed2; ++j) out[j] = ch[o][j];
        bl[0] = st2;
        bl[1] = ed2;
      } else {
        int st1 = bl[0], ed1 = bl[1];
        if (st1 <= st2 && ed1 >= ed2) {
          bl[1] = ed1;
          continue;
        }
        double s1 = 0.0, s2 = 0.0;
        for (int j = st2; j <= ed1; ++j) {
          s1 += search_score(out[j], cand + (size_t)j * stride, score + (size_t)j * stride, columns);
          s2 += search_score(ch[o][j], cand + (size_t)j * stride, score + (size_t)j * stride, columns);
        }
        int from = s1 > s2 ? ed1 : st2;
        for (int j = from; j <= ed2; ++j) out[j] = ch[o][j];
        bl[1] = ed2;
      }
    }
    free(order);
  }
  for (int i = 0; i < sections; ++i) free(ch[i]);
  free(ch);
}

/* FixStep4 (harvest.cpp:1000-1022): linear fill of short gaps, from
 * f0[end]+1 to f0[start]-1 as the reference writes it. */
static void fix_step4(const double* in, int frames, int threshold, double* out, int* bl) {
  memcpy(out, in, sizeof(double) * (size_t)frames);
  int nb = boundary_list(in, frames, bl);
  for (int i = 0; i < nb / 2 - 1; ++i) {
    int distance = bl[2 * (i + 1)] - bl[2 * i + 1] - 1;
    if (distance >= threshold) continue;
    double v0 = in[bl[2 * i + 1]] + 1;
    double v1 = in[bl[2 * (i + 1)]] - 1;
    double slope = (v1 - v0) / (distance + 1.0);
    int c = 1;
    for (int j = bl[2 * i + 1] + 1; j <= bl[2 * (i + 1)] - 1; ++j) out[j] = v0 + slope * c++;
  }
}

static void fix_contour(const double* cand, const double* score, int frames, int columns,
                        int stride, double* out) {
  double* a = malloc(sizeof(double) * (size_t)frames);
  double* b = malloc(sizeof(double) * (size_t)frames);
  int* bl = malloc(sizeof(int) * (size_t)(frames + 1));
  best_per_frame(cand, score, frames, columns, stride, a);
  fix_step1(a, frames, 0.008, b);
  fix_step2(b, frames, 6, a, bl);
  fix_step3(a, frames, columns, stride, cand, 0.18, score, b, bl);
  fix_step4(b, frames, 9, out, bl);
  free(a); free(b); free(bl);
}

/* a15: SmoothF0Contour + FilteringF0 (harvest.cpp:1049-1113). */
static void smooth_contour(const double* f0, int frames, double* out) {
  static const double b[2] = {0.0078202080334971724, 0.015640416066994345};
  static const double a[2] = {1.7347257688092754, -0.76600660094326412};
  const int lag = 300;
  int len = frames + 2 * lag;
  double* padded = calloc((size_t)len, sizeof(double));
  double* chan = malloc(sizeof(double) * (size_t)len);
  double* rev = malloc(sizeof(double) * (size_t)len);
  double* res = malloc(sizeof(double) * (size_t)len);
  int* bl = malloc(sizeof(int) * (size_t)(len + 1));
  for (int i = 0; i < frames; ++i) padded[lag + i] = f0[i];
  int nb = boundary_list(padded, len, bl);
  for (int s = 0; s < nb / 2; ++s) {
    int st = bl[2 * s], ed = bl[2 * s + 1];
    for (int i = 0; i < len; ++i) chan[i] = (i < st) ? padded[st] : (i > ed ? padded[ed] : padded[i]);
    double w0 = 0.0, w1 = 0.0;
    for (int i = 0; i < len; ++i) {
      double wt = chan[i] + a[0] * w0 + a[1] * w1;
      rev[len - i - 1] = b[0] * wt + b[1] * w0 + b[0] * w1;
      w1 = w0; w0 = wt;
    }
    w0 = w1 = 0.0;
    for (int i = 0; i < len; ++i) {
      double wt = rev[i] + a[0] * w0 + a[1] * w1;
      res[len - i - 1] = b[0] * wt + b[1] * w0 + b[0] * w1;
      w1 = w0; w0 = wt;
    }
    for (int j = st; j <= ed; ++j) out[j - lag] = res[j];
  }
  free(padded); free(chan); free(rev); free(res); free(bl);
}

/* ------------------------------------------------------------------------ */
/* Exported checker API (same symbols as world_ref_shim.cpp). */

int oracle_params(int n, int fs, double f0_floor, double f0_ceil, int* out) {
  orc_params p = derive(n, fs, f0_floor, f0_ceil);
  out[0] = p.ratio; out[1] = p.y_len; out[2] = p.fft_size;
  out[3] = p.bands; out[4] = p.frames; out[5] = p.capacity;
  return 0;
}

int oracle_output_length(int n, int fs, double period) { return frames_for(fs, n, period); }

typedef struct {
  double *y, *raw, *cand, *refined, *scores, *pruned, *pruned_scores, *base, *fixed, *smoothed;
  int count;
} orc_stage_out;

static void run_stages(const double* x, int n, int fs, double f0_floor, double f0_ceil,
                       orc_stage_out* o) {
  orc_params p = derive(n, fs, f0_floor, f0_ceil);
  int nfft = p.fft_size;
  double* y = calloc((size_t)nfft, sizeof(double));
  decimate_for_f0(x, n, p.ratio, p.y_len, y);
  remove_mean(y, p.y_len);
  if (o->y) memcpy(o->y, y, sizeof(double) * (size_t)p.y_len);

  cplx* work = malloc(sizeof(cplx) * (size_t)nfft);
  cplx* spec = malloc(sizeof(cplx) * (size_t)(nfft / 2 + 1));
  rfft(y, nfft, spec, work);

  double* t = malloc(sizeof(double) * (size_t)p.frames);
  for (int i = 0; i < p.frames; ++i) t[i] = i * 1 / 1000.0;
  double* raw = malloc(sizeof(double) * (size_t)p.bands * (size_t)p.frames);
  double* filtered = malloc(sizeof(double) * (size_t)nfft);
  double* taps = malloc(sizeof(double) * (size_t)nfft);
  cplx* full = malloc(sizeof(cplx) * (size_t)nfft);
  double* evbuf = malloc(sizeof(double) * 9 * (size_t)p.y_len);
  double lo = f0_floor * 0.9;
  for (int b = 0; b < p.bands; ++b) {
    double centre = lo * pow(2.0, (b + 1) / 40.0);
    band_filter(centre, nfft, p.fs_r, spec, p.y_len, filtered, taps, full, work);
    band_candidates(filtered, p.y_len, p.fs_r, centre, f0_floor, f0_ceil, t, p.frames,
                    raw + (size_t)b * p.frames, evbuf);
  }
  if (o->raw) memcpy(o->raw, raw, sizeof(double) * (size_t)p.bands * (size_t)p.frames);

  size_t cells = (size_t)p.frames * (size_t)p.capacity;
  double* cand = calloc(cells ? cells : 1, sizeof(double));
  double* score = calloc(cells ? cells : 1, sizeof(double));
  int count = official_candidates(raw, p.bands, p.frames, p.capacity, cand);
  overlap_candidates(p.frames, count, p.capacity, cand);
  o->count = count;
  if (o->cand) memcpy(o->cand, cand, sizeof(double) * cells);
  int columns = count * 7;
  for (int f = 0; f < p.frames; ++f)
    for (int j = 0; j < columns; ++j) {
      size_t at = (size_t)f * p.capacity + j;
      refine_one(y, p.y_len, p.fs_r, t[f], cand[at], f0_floor, f0_ceil, &cand[at], &score[at]);
    }
  if (o->refined) memcpy(o->refined, cand, sizeof(double) * cells);
  if (o->scores) memcpy(o->scores, score, sizeof(double) * cells);
  prune(p.frames, columns, p.capacity, cand, score);
  if (o->pruned) memcpy(o->pruned, cand, sizeof(double) * cells);
  if (o->pruned_scores) memcpy(o->pruned_scores, score, sizeof(double) * cells);
  double* base = malloc(sizeof(double) * (size_t)p.frames);
  double* fixed = malloc(sizeof(double) * (size_t)p.frames);
  double* smoothed = calloc((size_t)p.frames, sizeof(double));
  best_per_frame(cand, score, p.frames, columns, p.capacity, base);
  fix_contour(cand, score, p.frames, columns, p.capacity, fixed);
  smooth_contour(fixed, p.frames, smoothed);
  if (o->base) memcpy(o->base, base, sizeof(double) * (size_t)p.frames);
  if (o->fixed) memcpy(o->fixed, fixed, sizeof(double) * (size_t)p.frames);
  if (o->smoothed) memcpy(o->smoothed, smoothed, sizeof(double) * (size_t)p.frames);

  free(y); free(work); free(spec); free(t); free(raw); free(filtered); free(taps); free(full);
  free(evbuf); free(cand); free(score); free(base); free(fixed); free(smoothed);
}

void oracle_stages(const double* x, int n, int fs, double f0_floor, double f0_ceil,
                   double* y_out, double* raw_out, int* count_out, double* cand_out,
                   double* refined_out, double* scores_out, double* pruned_out,
                   double* pruned_scores_out, double* base_out, double* fixed_out,
                   double* smoothed_out) {
  orc_stage_out o = {y_out, raw_out, cand_out, refined_out, scores_out, pruned_out,
                     pruned_scores_out, base_out, fixed_out, smoothed_out, 0};
  run_stages(x, n, fs, f0_floor, f0_ceil, &o);
  *count_out = o.count;
}

/* Harvest (harvest.cpp:1223-1255): 1 ms analysis, then nearest-frame
 * resampling onto frame_period (a16). */
void oracle_harvest(const double* x, int n, int fs, double f0_floor, double f0_ceil,
                    double period, double* times, double* f0) {
  orc_params p = derive(n, fs, f0_floor, f0_ceil);
  double* smoothed = calloc((size_t)p.frames, sizeof(double));
  orc_stage_out o = {0};
  o.smoothed = smoothed;
  run_stages(x, n, fs, f0_floor, f0_ceil, &o);
  if (period == 1.0) {
    for (int i = 0; i < p.frames; ++i) { times[i] = i * 1 / 1000.0; f0[i] = smoothed[i]; }
  } else {
    int out_len = frames_for(fs, n, period);
    for (int i = 0; i < out_len; ++i) {
      times[i] = i * period / 1000.0;
      f0[i] = smoothed[imin(p.frames - 1, round_away(times[i] * 1000.0))];
    }
  }
  free(smoothed);
}

void oracle_fix_contour(const double* cand, const double* scores, int frames, int columns,
                        int stride, double* fixed_out) {
  fix_contour(cand, scores, frames, columns, stride, fixed_out);
}

/* FixStep1-4 of FixF0Contour (harvest.cpp:1027-1044) from a caller-given
 * base contour in place of SearchF0Base's. */
void oracle_fix_contour_base(const double* base, const double* cand, const double* scores, int frames,
                             int columns, int stride, double* fixed_out) {
  double* a = malloc(sizeof(double) * (size_t)(frames > 0 ? frames : 1));
  double* b = malloc(sizeof(double) * (size_t)(frames > 0 ? frames : 1));
  int* bl = malloc(sizeof(int) * (size_t)(frames + 1));
  fix_step1(base, frames, 0.008, b);
  fix_step2(b, frames, 6, a, bl);
  fix_step3(a, frames, columns, stride, cand, 0.18, scores, b, bl);
  fix_step4(b, frames, 9, fixed_out, bl);
  free(a); free(b); free(bl);
}

void oracle_smooth_contour(const double* f0, int frames, double* out) {
  for (int i = 0; i < frames; ++i) out[i] = 0.0;
  smooth_contour(f0, frames, out);
}
