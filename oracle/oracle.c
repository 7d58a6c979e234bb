/*
 * oracle.c -- CPU restatement of Heimdall's per-gulp search chain.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Compiled with -ffp-contract=off
 * so every float expression rounds exactly as written; types and operation
 * order follow the cited reference lines so results can be compared bit for
 * bit.  Where the reference reads memory it never wrote (one element past a
 * series) the restatement defines that value as 0 and the product does the
 * same.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Selection networks.  Pipeline/median_filter.cu:21-75 chooses the middle  */
/* element(s) with hand-written comparison trees; any exact selection gives */
/* the same value for non-NaN input, so these use small compare-exchange    */
/* networks instead.                                                        */
/* ------------------------------------------------------------------------ */
#define OR_CSWAP(x, y) do { if ((y) < (x)) { float t_ = (x); (x) = (y); (y) = t_; } } while (0)

float or_median3(float a, float b, float c) {
  OR_CSWAP(a, b);
  OR_CSWAP(b, c);
  OR_CSWAP(a, b);
  return b;
}

/* Mean of the two middle values (median_filter.cu:28-38: 0.5f*(x+y)). */
float or_median4(float a, float b, float c, float d) {
  OR_CSWAP(a, b);
  OR_CSWAP(c, d);
  OR_CSWAP(a, c);
  OR_CSWAP(b, d);
  /* now a is the minimum and d the maximum; b, c are the middle pair */
  return 0.5f * (b + c);
}

/* Median of five with six comparisons: the smaller of two sorted-pair minima
 * has three elements above it and can be dropped, twice. */
float or_median5(float a, float b, float c, float d, float e) {
  float t;
  OR_CSWAP(a, b);
  OR_CSWAP(c, d);
  if (c < a) { t = a; a = c; c = t; t = b; b = d; d = t; }
  /* a is below b, c, d: drop it, bring in e */
  a = e;
  OR_CSWAP(a, b);
  if (c < a) { t = a; a = c; c = t; t = b; b = d; d = t; }
  /* a is the second smallest of the five; the median is min(b, c) */
  return (c < b) ? c : b;
}

/* ------------------------------------------------------------------------ */
/* dedisp restatement                                                        */
/* ------------------------------------------------------------------------ */

/* DM trial spacing (pipeline.cu:178-182 -> dedisp; golden vector
 * Share/dm2000.list).  Smearing model, times in microseconds:
 *   W(p)^2 = dt^2 + ti^2 + (a p)^2,   a = 8.3 df / f^3  (df MHz, f GHz at the
 *   band centre) is the intra-channel dispersion smearing per unit DM.
 * Searching trial p for a pulse at DM x adds b (x - p) with b = a*nchans/4.
 * The next trial x solves  dt^2+ti^2 + (a x)^2 + b^2 (x-p)^2 = tol^2 W(p)^2,
 *   x = (b^2 p + sqrt(-a^2 b^2 p^2 + (a^2+b^2)(c + tol^2 a^2 p^2))) / (a^2+b^2)
 * with c = (dt^2 + ti^2)(tol^2 - 1).  Trials are stored as float and the
 * stored value seeds the next step; generation stops at the first trial at or
 * beyond dm_end. */
size_t or_generate_dm_list(float dm_start, float dm_end, double dt, double ti,
                           double f0, double df, size_t nchans, double tol,
                           float* out, size_t cap) {
  double dt_us = dt * 1e6;
  double f = (f0 + ((double)(nchans / 2) - 0.5) * df) * 1e-3;
  double tol2 = tol * tol;
  double a = 8.3 * df / (f * f * f);
  double a2 = a * a;
  double b2 = a2 * ((double)(nchans * nchans) / 16.0);
  double c = (dt_us * dt_us + ti * ti) * (tol2 - 1.0);
  size_t n = 0;
  float last = dm_start;
  if (cap > 0) out[0] = last;
  n = 1;
  while (last < dm_end) {
    double p = (double)last;
    double k = c + tol2 * a2 * p * p;
    double x = (b2 * p + sqrt(-a2 * b2 * p * p + (a2 + b2) * k)) / (a2 + b2);
    last = (float)x;
    if (n < cap) out[n] = last;
    n++;
  }
  return n;
}

/* Per-channel delay coefficient in samples per unit DM (include/dedisp.h). */
void or_delay_table(size_t nchans, float dt, float f0, float df, float* table) {
  const float K = 4148.808f;
  float b = 1.0f / f0;
  for (size_t c = 0; c < nchans; c++) {
    float fc = f0 + (float)c * df;
    float a = 1.0f / fc;
    table[c] = K * (a * a - b * b) / dt;
  }
}

size_t or_delay(float dm, float table_c) {
  float v = dm * table_c + 0.5f;
  if (!(v > 0.0f)) return 0;
  return (size_t)v;
}

size_t or_max_delay(const float* dm_list, size_t dm_count, const float* table,
                    size_t nchans) {
  size_t m = 0;
  for (size_t d = 0; d < dm_count; d++)
    for (size_t c = 0; c < nchans; c++) {
      size_t v = or_delay(dm_list[d], table[c]);
      if (v > m) m = v;
    }
  return m;
}

/* Adaptive time resolution (dedisp_enable_adaptive_dt, pipeline.cu:187-196;
 * the external dedisp library is not in the tree, so this is a restatement of
 * the published method, Barsdell et al. 2012, MNRAS 422, 379: a trial is
 * searched at a coarser sampling time while the coarsening adds little to its
 * total smearing).  Choices made here: the smearing of trial DM at sampling
 * time T is the generator's model above, W(DM, T)^2 = T^2 + ti^2 + (a DM)^2
 * (microseconds, the same a and band centre); factors start at 1 for the
 * first trial and never decrease; trial d takes twice the previous factor s
 * when W(DM_d, 2 s dt) / W(DM_d, s dt) < tol, else keeps s; double
 * precision throughout. */
void or_scrunch_factors(const float* dm_list, size_t dm_count, double dt, double ti,
                        double f0, double df, size_t nchans, double tol, size_t* out) {
  double dt_us = dt * 1e6;
  double f = (f0 + ((double)(nchans / 2) - 0.5) * df) * 1e-3;
  double a = 8.3 * df / (f * f * f);
  size_t s = 1;
  for (size_t d = 0; d < dm_count; d++) {
    if (d > 0) {
      double sm = a * (double)dm_list[d];
      double t1 = (double)s * dt_us, t2 = 2.0 * (double)s * dt_us;
      double w1 = sqrt(t1 * t1 + ti * ti + sm * sm);
      double w2 = sqrt(t2 * t2 + ti * ti + sm * sm);
      if (w2 / w1 < tol) s *= 2;
    }
    out[d] = s;
  }
}

/* out[d][t] = (float) sum_c killmask[c] * in[t + delay(d,c)][c] for
 * t < nsamps - max_delay; exact integer sums (8-bit input).
 * With scrunch factors (NULL: all 1), trial d with factor s is computed at
 * sampling time s dt from the scrunched input
 *   in_s[c][u] = (sum_{j<s} in[s u + j][c] + s/2) / s   (a byte: the mean,
 *                                                        rounded half up)
 * as out[d][u] = sum_c killmask[c] * in_s[c][u + delay(d,c) / s] for
 * u < (nsamps - max_delay) / s (integer divisions; every index stays below
 * nsamps / s). */
void or_dedisperse_scrunched(const uint8_t* in, size_t nsamps, size_t in_stride,
                             size_t nchans, const int* killmask, const float* dm_list,
                             size_t dm_count, const float* table, const size_t* scrunch,
                             float* out, size_t out_stride, int nthreads) {
  size_t max_delay = or_max_delay(dm_list, dm_count, table, nchans);
  size_t nout = nsamps - max_delay;
  /* channel-major copies (one per scrunch factor) so the inner loop runs
   * along time */
  uint8_t* ft[32] = {0};
  size_t flen[32] = {0};
  for (size_t d = 0; d < dm_count; d++) {
    size_t s = scrunch ? scrunch[d] : 1;
    int k = 0;
    while (((size_t)1 << k) < s) k++;
    if (k >= 32 || ft[k]) continue;
    size_t ns = nsamps / s;
    flen[k] = ns;
    ft[k] = (uint8_t*)malloc(nchans * ns + 1);
    for (size_t u = 0; u < ns; u++)
      for (size_t c = 0; c < nchans; c++) {
        unsigned sum = 0;
        for (size_t j = 0; j < s; j++) sum += in[(s * u + j) * in_stride + c];
        ft[k][c * ns + u] = (uint8_t)((sum + (unsigned)(s / 2)) / (unsigned)s);
      }
  }
  const size_t TB = 4096;
  size_t ntb = (nout + TB - 1) / TB;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (long long job = 0; job < (long long)(dm_count * ntb); job++) {
    size_t d = (size_t)job / ntb, tb = (size_t)job % ntb;
    size_t s = scrunch ? scrunch[d] : 1;
    int k = 0;
    while (((size_t)1 << k) < s) k++;
    size_t nout_s = nout / s, ns = flen[k];
    size_t t0 = tb * TB, t1 = t0 + TB < nout_s ? t0 + TB : nout_s;
    if (t0 >= t1) continue;
    int32_t acc[4096];
    memset(acc, 0, sizeof(acc));
    for (size_t c = 0; c < nchans; c++) {
      if (!killmask[c]) continue;
      const uint8_t* row = ft[k] + c * ns + or_delay(dm_list[d], table[c]) / s;
      for (size_t t = t0; t < t1; t++) acc[t - t0] += row[t];
    }
    for (size_t t = t0; t < t1; t++) out[d * out_stride + t] = (float)acc[t - t0];
  }
  for (int k = 0; k < 32; k++) free(ft[k]);
}

void or_dedisperse(const uint8_t* in, size_t nsamps, size_t in_stride,
                   size_t nchans, const int* killmask, const float* dm_list,
                   size_t dm_count, const float* table, float* out,
                   size_t out_stride, int nthreads) {
  or_dedisperse_scrunched(in, nsamps, in_stride, nchans, killmask, dm_list, dm_count, table,
                          NULL, out, out_stride, nthreads);
}

/* ------------------------------------------------------------------------ */
/* Stage restatements                                                        */
/* ------------------------------------------------------------------------ */

static unsigned f2u(float x) { return (x != x) ? 0u : (unsigned)x; }

/* Pipeline/median_filter.cu:451-479 */
void or_linear_stretch(const float* in, size_t in_count, float* out, size_t out_count) {
  float step = (float)(in_count - 1) / (float)(out_count - 1);
  for (unsigned i = 0; i < (unsigned)out_count; i++) {
    float x = (float)i * step;
    unsigned j = f2u(x);
    float fr = x - (float)j;
    out[i] = in[j] + (((double)fr > 1e-5) ? fr * (in[j + 1] - in[j]) : 0.f);
  }
}

/* Pipeline/median_filter.cu:481-519 */
void or_linear_stretch_beam(const float* in, size_t in_count_beam, float* out,
                            size_t out_count_beam, size_t nbeam) {
  float step = (float)(in_count_beam - 1) / (float)out_count_beam;
  size_t out_count = out_count_beam * nbeam;
  for (unsigned i = 0; i < (unsigned)out_count; i++) {
    size_t beam = i / out_count_beam;
    float x = (float)i * step;
    unsigned k = f2u(x + (float)beam);
    float o = (x - (float)k) + (float)beam;
    out[i] = in[k] + (((double)o > 1e-5) ? o * (in[k + 1] - in[k]) : 0.f);
  }
}

/* Pipeline/median_filter.cu:288-322 */
void or_median_scrunch5(const float* in, size_t count, float* out) {
  if (count == 1) out[0] = in[0];
  else if (count == 2) out[0] = 0.5f * (in[0] + in[1]);
  else if (count == 3) out[0] = or_median3(in[0], in[1], in[2]);
  else if (count == 4) out[0] = or_median4(in[0], in[1], in[2], in[3]);
  else {
    size_t oc = count / 5;
    for (size_t i = 0; i < oc; i++)
      out[i] = or_median5(in[5 * i], in[5 * i + 1], in[5 * i + 2], in[5 * i + 3], in[5 * i + 4]);
  }
}

/* Pipeline/median_filter.cu:194-235,365-395 */
void or_median_scrunch5_beam(const float* in, size_t beam_stride, size_t nbeam, float* out) {
  if (beam_stride > 4) {
    size_t oc = beam_stride / 5, total = nbeam * oc;
    for (size_t o = 0; o < total; o++) {
      size_t beam = o / oc, i = (o % oc) * 5, off = beam * beam_stride + i;
      out[o] = or_median5(in[off], in[off + 1], in[off + 2], in[off + 3], in[off + 4]);
    }
  } else {
    for (size_t o = 0; o < nbeam; o++) {
      size_t off = o * beam_stride;
      if (beam_stride == 1) out[o] = in[off];
      else if (beam_stride == 2) out[o] = 0.5f * (in[off] + in[off + 1]);
      else if (beam_stride == 3) out[o] = or_median3(in[off], in[off + 1], in[off + 2]);
      else out[o] = or_median4(in[off], in[off + 1], in[off + 2], in[off + 3]);
    }
  }
}

/* Scrunch plan of Pipeline/remove_baseline.cu:36-46. */
void or_baseline_plan(size_t beam_stride, size_t smooth_radius,
                      size_t* sample_count, size_t* nscrunches, size_t* count_round) {
  float oversample = 2;
  float q = oversample * (float)beam_stride / (float)(2 * smooth_radius);
  size_t sc = (size_t)((double)q + 0.5);
  *sample_count = sc;
  if (sc == 0) { *nscrunches = 0; *count_round = 0; return; }
  size_t ns = (size_t)(log((double)(beam_stride / sc)) / log(5.));
  *nscrunches = ns;
  *count_round = (size_t)(pow(5., (double)ns) * (double)sc);
}

/* Pipeline/remove_baseline.cu:21-102 (the OPTIMIZED branch).  `data` holds
 * data_len valid floats followed by one readable zero. */
int or_remove_baseline(float* data, size_t data_len, size_t beam_stride,
                       size_t beam_count, size_t smooth_radius, size_t nbeams) {
  size_t sample_count, nscr, count_round;
  (void)data_len;
  or_baseline_plan(beam_stride, smooth_radius, &sample_count, &nscr, &count_round);
  if (sample_count == 0) return 0;
  size_t dm_delay = beam_stride - beam_count;
  size_t nbm = nbeams - 1;
  size_t nsamps = beam_stride * nbeams - dm_delay;
  float* buf1 = (float*)calloc(nbeams * count_round + 8, sizeof(float));
  float* buf2 = (float*)calloc(nbeams * (count_round / 5) + 8, sizeof(float));
  float* base = (float*)calloc(beam_stride * nbeams + 8, sizeof(float));
  or_linear_stretch_beam(data, beam_stride, buf1, count_round, nbm);
  or_linear_stretch(data + nbm * beam_stride, beam_count, buf1 + nbm * count_round, count_round);
  float* p1 = buf1; float* p2 = buf2;
  for (size_t size = count_round; size > sample_count; size /= 5) {
    or_median_scrunch5_beam(p1, size, nbeams, p2);
    float* t = p1; p1 = p2; p2 = t;
  }
  or_linear_stretch_beam(p1, sample_count, base, beam_stride, nbm);
  or_linear_stretch(p1 + nbm * sample_count, sample_count, base + nbm * beam_stride, beam_count);
  for (size_t i = 0; i < nsamps; i++) data[i] = data[i] - base[i];
  free(buf1); free(buf2); free(base);
  return 0;
}

/* Pipeline/get_rms.cu:384-418 (delta is held as a float). */
static void or_reblock_abs_beam(const float* in, size_t in_stride, size_t in_length,
                                float* out, size_t nbeam) {
  size_t oc = in_length * nbeam;
  float delta = (float)(in_stride - in_length);
  for (unsigned o = 0; o < (unsigned)oc; o++) {
    size_t beam = o / in_length;
    size_t i = (size_t)((float)beam * delta + (float)o);
    out[o] = fabsf(in[i]);
  }
}

/* Pipeline/get_rms.cu:236-270 */
void or_rms_beams(const float* data, float* rms, size_t beam_stride,
                  size_t beam_count, size_t nbeams) {
  size_t count = nbeams * beam_count;
  float* b1 = (float*)calloc(count + 8, sizeof(float));
  float* b2 = (float*)calloc(count / 5 + 8, sizeof(float));
  or_reblock_abs_beam(data, beam_stride, beam_count, b1, nbeams);
  for (size_t size = beam_count; size > 1; size /= 5) {
    or_median_scrunch5_beam(b1, size, nbeams, b2);
    float* t = b1; b1 = b2; b2 = t;
  }
  for (size_t b = 0; b < nbeams; b++) rms[b] = b1[b] * (float)1.4862;
  free(b1); free(b2);
}

/* Pipeline/get_rms.cu:274-301 */
float or_rms_block(const float* data, size_t beam_stride, size_t beam_count, size_t nbeams) {
  size_t count = nbeams * beam_count;
  float* b1 = (float*)calloc(count + 8, sizeof(float));
  float* b2 = (float*)calloc(count / 5 + 8, sizeof(float));
  or_reblock_abs_beam(data, beam_stride, beam_count, b1, nbeams);
  for (size_t size = count; size > 1; size /= 5) {
    or_median_scrunch5(b1, size, b2);
    float* t = b1; b1 = b2; b2 = t;
  }
  float m = b1[0];
  free(b1); free(b2);
  return (float)((double)m * 1.4862);
}

/* Pipeline/get_rms.cu:344-356,372-382 */
void or_normalise_beams(float* data, const float* rms, size_t beam_stride, size_t count) {
  for (unsigned i = 0; i < (unsigned)count; i++) data[i] = data[i] / rms[i / beam_stride];
}

/* Pipeline/get_rms.cu:359-370 */
void or_normalise_scalar(float* data, float rms, size_t count) {
  float r = 1.0f / rms;
  for (size_t i = 0; i < count; i++) data[i] = data[i] * r;
}

/* Pipeline/matched_filter.cu:21-32 on Thrust's sequential scan: out[0] = 0,
 * out[k+1] = out[k] + in[k]; n_in inputs give n_in outputs. */
void or_exclusive_scan(const float* in, size_t n_in, float* out) {
  float sum = 0.0f;
  for (size_t k = 0; k < n_in; k++) { float tmp = in[k]; out[k] = sum; sum = sum + tmp; }
}

/* Pipeline/matched_filter.cu:37-67 with strided_range (hd/strided_range.h:111-151) */
void or_matched_filter(const float* scanned, size_t scanned_size, size_t max_width,
                       float* out, size_t width, size_t tscrunch) {
  size_t offset = max_width / 2;
  size_t ahead = (width - 1) / 2 + 1;
  size_t behind = width / 2;
  size_t out_count = scanned_size - max_width;
  size_t n = (out_count + tscrunch - 1) / tscrunch;
  for (size_t k = 0; k < n; k++)
    out[k] = scanned[offset + ahead + k * tscrunch] - scanned[offset - behind + k * tscrunch];
}

/* ------------------------------------------------------------------------ */
/* Giants                                                                    */
/* ------------------------------------------------------------------------ */
void or_giants_init(or_giants* g) { memset(g, 0, sizeof(*g)); }

void or_giants_free(or_giants* g) {
  free(g->peaks); free(g->inds); free(g->begins); free(g->ends);
  free(g->filter_inds); free(g->dm_inds); free(g->members);
  memset(g, 0, sizeof(*g));
}

static void or_giants_reserve(or_giants* g, size_t n) {
  if (n <= g->cap) return;
  size_t cap = g->cap ? g->cap : 64;
  while (cap < n) cap *= 2;
  g->peaks = (float*)realloc(g->peaks, cap * sizeof(float));
  g->inds = (size_t*)realloc(g->inds, cap * sizeof(size_t));
  g->begins = (size_t*)realloc(g->begins, cap * sizeof(size_t));
  g->ends = (size_t*)realloc(g->ends, cap * sizeof(size_t));
  g->filter_inds = (size_t*)realloc(g->filter_inds, cap * sizeof(size_t));
  g->dm_inds = (size_t*)realloc(g->dm_inds, cap * sizeof(size_t));
  g->members = (size_t*)realloc(g->members, cap * sizeof(size_t));
  g->cap = cap;
}

/* Pipeline/find_giants.cu:101-316: samples with (i % beam_stride) < beam_count
 * and value > thresh, grouped into segments broken where the index gap
 * exceeds merge_dist; per segment the first maximum (peak, index), the first
 * index (begin) and the last index + 1 (end). */
size_t or_find_giants(const float* data, size_t count, float thresh, size_t merge_dist,
                      size_t beam_stride, size_t beam_count, or_giants* out) {
  size_t added = 0;
  int open = 0;
  size_t last = 0;
  for (unsigned i = 0; i < (unsigned)count; i++) {
    size_t samp = (size_t)i % beam_stride;
    float v = data[i];
    if (!(samp < beam_count && v > thresh)) continue;
    if (!open || i > last + merge_dist) {
      or_giants_reserve(out, out->count + 1);
      size_t k = out->count++;
      out->peaks[k] = v; out->inds[k] = i; out->begins[k] = i; out->ends[k] = i + 1;
      out->filter_inds[k] = 0; out->dm_inds[k] = 0; out->members[k] = 1;
      open = 1; added++;
    } else {
      size_t k = out->count - 1;
      if (!(out->peaks[k] >= v)) { out->peaks[k] = v; out->inds[k] = i; }
      out->ends[k] = (size_t)i + 1;
    }
    last = i;
  }
  return added;
}

/* ------------------------------------------------------------------------ */
/* Clustering: Pipeline/label_candidate_clusters.cu:141-197,203-394 with      */
/* are_coincident_beam (hd/are_coincident.cuh:47-68).  The reference runs the */
/* neighbour sweep as a racy parallel for_each; this restatement fixes the    */
/* sequential order (the reference's own result with one thread).            */
/* ------------------------------------------------------------------------ */
static int or_coincident(size_t si, size_t sj, size_t bi, size_t bj, size_t fi, size_t fj,
                         size_t di, size_t dj, size_t time_tol, size_t filter_tol,
                         size_t dm_tol) {
  int wi = 1 << (int)fi, wj = 1 << (int)fj;
  size_t tt = time_tol * (size_t)(wi > wj ? wi : wj);
  return bi == bj && (size_t)abs((int)sj - (int)si) <= tt &&
         (size_t)abs((int)fj - (int)fi) <= filter_tol &&
         (size_t)abs((int)dj - (int)di) <= dm_tol;
}

size_t or_label_clusters(size_t count, const or_giants* g, size_t time_tol,
                         size_t filter_tol, size_t dm_tol, size_t nsamps_beam,
                         size_t* labels) {
  for (size_t i = 0; i < count; i++) labels[i] = i;
  int sorted = 1;
  for (size_t i = 1; i < count; i++) if (g->dm_inds[i] < g->dm_inds[i - 1]) { sorted = 0; break; }
  size_t lo = 0;
  for (size_t i = 0; i < count; i++) {
    size_t si = g->inds[i], bi = si / nsamps_beam, fi = g->filter_inds[i], di = g->dm_inds[i];
    size_t j0 = 0, j1 = count;
    if (sorted) {
      /* giants are in DM order: restrict j to |dm_j - dm_i| <= dm_tol */
      while (lo < count && g->dm_inds[lo] + dm_tol < di) lo++;
      j0 = lo;
      j1 = i;
      while (j1 < count && g->dm_inds[j1] <= di + dm_tol) j1++;
    }
    for (size_t j = j0; j < j1; j++) {
      if (j == i) continue;
      size_t sj = g->inds[j];
      if (or_coincident(si, sj, bi, sj / nsamps_beam, fi, g->filter_inds[j], di,
                        g->dm_inds[j], time_tol, filter_tol, dm_tol)) {
        int a = (int)labels[i], b = (int)labels[j];
        labels[i] = (size_t)(a < b ? a : b);
      }
    }
  }
  for (size_t i = 0; i < count; i++) {
    size_t cur = i;
    while (labels[cur] != cur) cur = labels[cur];
    labels[i] = cur;
  }
  size_t roots = 0;
  for (size_t i = 0; i < count; i++) roots += (labels[i] == i);
  return roots;
}

/* Pipeline/merge_candidates.cu:21-134: stable sort by label, then per label
 * keep the first member with the largest peak and sum the member counts. */
void or_merge(size_t count, const size_t* labels, const or_giants* g,
              size_t label_count, or_giants* groups) {
  or_giants_reserve(groups, label_count + 1);
  groups->count = 0;
  /* labels are root indices; groups come out in ascending label order, and
   * members of a group in ascending giant index order */
  size_t* slot = (size_t*)malloc((count + 1) * sizeof(size_t));
  for (size_t i = 0; i < count; i++) slot[i] = (size_t)-1;
  for (size_t i = 0; i < count; i++)
    if (labels[i] == i) slot[i] = groups->count++;
  for (size_t k = 0; k < groups->count; k++) groups->members[k] = 0;
  char* seen = (char*)calloc(groups->count + 1, 1);
  for (size_t i = 0; i < count; i++) {
    size_t k = slot[labels[i]];
    if (!seen[k]) {
      seen[k] = 1;
      groups->peaks[k] = g->peaks[i]; groups->inds[k] = g->inds[i];
      groups->begins[k] = g->begins[i]; groups->ends[k] = g->ends[i];
      groups->filter_inds[k] = g->filter_inds[i]; groups->dm_inds[k] = g->dm_inds[i];
      groups->members[k] = g->members[i];
    } else {
      size_t m = groups->members[k] + g->members[i];
      if (!(groups->peaks[k] >= g->peaks[i])) {
        groups->peaks[k] = g->peaks[i]; groups->inds[k] = g->inds[i];
        groups->begins[k] = g->begins[i]; groups->ends[k] = g->ends[i];
        groups->filter_inds[k] = g->filter_inds[i]; groups->dm_inds[k] = g->dm_inds[i];
      }
      groups->members[k] = m;
    }
  }
  free(seen); free(slot);
}

/* ------------------------------------------------------------------------ */
/* RFI cleaning: Pipeline/clean_filterbank_rfi.cu                           */
/* ------------------------------------------------------------------------ */

/* Robert Jenkins' 32-bit integer mix (clean_filterbank_rfi.cu:33-43). */
uint32_t or_hash(uint32_t a) {
  a = (a + 0x7ed55d16u) + (a << 12);
  a = (a ^ 0xc761c23cu) ^ (a >> 19);
  a = (a + 0x165667b1u) + (a << 5);
  a = (a + 0xd3a2646cu) ^ (a << 9);
  a = (a + 0xfd7046c5u) + (a << 3);
  a = (a ^ 0xb55a4f09u) ^ (a >> 16);
  return a;
}

/* Park-Miller minimal-standard generator (multiplier 48271, modulus 2^31-1,
 * outputs 1..2^31-2), the engine behind thrust::default_random_engine, and
 * Thrust's integer distribution: a double in [lo, hi+1) from
 * (x - 1) / (2^31 - 2), truncated (thrust/random/detail/
 * uniform_int_distribution.inl, uniform_real_distribution.inl). */
static uint32_t or_minstd_next(uint32_t* s) {
  *s = (uint32_t)(((uint64_t)48271u * (uint64_t)(*s)) % 2147483647ull);
  return *s;
}

uint32_t or_uniform_uint(uint32_t* state, uint32_t lo, uint32_t hi) {
  double a = (double)lo;
  double b = (double)hi + 1.0;
  double u = (double)(or_minstd_next(state) - 1u);
  u = u / (1.0 + (double)(2147483646u - 1u));
  double r = u * (b - a) + a;
  return (uint32_t)r;
}

static uint32_t or_minstd_seed(uint32_t s) {
  uint32_t m = s % 2147483647u;
  return m == 0 ? 1u : m;
}

/* zap_filterbank_rfi (clean_filterbank_rfi.cu:55-113,197-234) */
static void or_zap(const int* mask, const uint8_t* in, size_t nsamps, size_t nbits,
                   size_t nchans, size_t max_resample_dist, uint8_t* out) {
  unsigned stride = (unsigned)(nchans * nbits / 8 / 4);
  unsigned ns = (unsigned)nsamps, r = (unsigned)max_resample_dist;
  uint32_t bitmask = (1u << nbits) - 1u;
  const uint32_t* win = (const uint32_t*)in;
  uint32_t* wout = (uint32_t*)out;
  unsigned total = ns * stride;
  for (unsigned i = 0; i < total; i++) {
    unsigned t = i / stride, c = i % stride;
    uint32_t result;
    if (mask[t]) {
      uint32_t st = or_minstd_seed(or_hash(i));
      result = 0;
      for (unsigned k = 0; k < 32; k += (unsigned)nbits) {
        unsigned min_t = t > r ? t - r : 0;
        unsigned max_t = t < ns - 1 - r ? t + r : ns - 1;
        unsigned nt = or_uniform_uint(&st, min_t, max_t);
        int attempts = 0;
        while (mask[nt] && ++attempts < 11) nt = or_uniform_uint(&st, min_t, max_t);
        uint32_t val = (win[nt * stride + c] >> k) & bitmask;
        result |= val << k;
      }
    } else {
      result = win[i];
    }
    wout[i] = result;
  }
}

/* ---- narrow-band RFI (the branch clean_filterbank_rfi.cu:303 disables) --- */

/* Pipeline/median_filter.cu:99-124 (median_filter5_kernel): a 5-wide
 * running median with the window shrunk to 3 or 4 at the ends. */
static void or_median_filter5(const float* in, size_t count, float* out) {
  for (size_t i = 0; i < count; i++) {
    if (i > 1 && i < count - 2)
      out[i] = or_median5(in[i - 2], in[i - 1], in[i], in[i + 1], in[i + 2]);
    else if (i == 0)
      out[i] = or_median3(in[i], in[i + 1], in[i + 2]);
    else if (i == 1)
      out[i] = or_median4(in[i - 1], in[i], in[i + 1], in[i + 2]);
    else if (i == count - 1)
      out[i] = or_median3(in[i], in[i - 1], in[i - 2]);
    else
      out[i] = or_median4(in[i + 1], in[i], in[i - 1], in[i - 2]);
  }
}

/* Pipeline/median_filter.cu:422-432 (thrust::adjacent_difference with the
 * mean of neighbours): out[0] = in[0], out[i] = 0.5 (in[i] + in[i-1]). */
static void or_mean_filter2(const float* in, size_t count, float* out) {
  if (count == 0) return;
  out[0] = in[0];
  for (size_t i = 1; i < count; i++) out[i] = 0.5f * (in[i] + in[i - 1]);
}

/* Pipeline/median_filter.cu:345-361: median5 of corresponding elements of
 * five consecutive arrays of `size` values. */
static void or_median_scrunch5_array(const float* in, size_t size, size_t count, float* out) {
  size_t oc = count / 5;
  for (size_t a = 0; a < oc; a++)
    for (size_t j = 0; j < size; j++)
      out[a * size + j] = or_median5(in[(5 * a) * size + j], in[(5 * a + 1) * size + j],
                                     in[(5 * a + 2) * size + j], in[(5 * a + 3) * size + j],
                                     in[(5 * a + 4) * size + j]);
}

/* measure_bandpass.cu:141-163 / 223-245: scrunch by 5, 5-wide median, mean of
 * neighbours, stretch back to nchans/5*5 and extrapolate the rest linearly
 * (v in place; tmp holds nchans/5 values). */
static void or_smooth_band(float* v, size_t nchans, float* tmp) {
  size_t n5 = nchans / 5;
  or_median_scrunch5(v, nchans, tmp);
  or_median_filter5(tmp, n5, v);
  or_mean_filter2(v, n5, tmp);
  /* for some channel counts (1140, 2220, ...) float rounding puts the last
   * stretched sample just past the last input with a fraction above 1e-5,
   * so the stretch reads one element past the nchans/5 values (the
   * reference reads past its vector there); that element is defined as 0 */
  tmp[n5] = 0.f;
  or_linear_stretch(tmp, n5, v, n5 * 5);
  for (size_t i = n5 * 5; i < nchans; i++) v[i] = 2 * v[i - 1] - v[i - 2];
}

static int or_cmp_float(const void* a, const void* b) {
  float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}

/* Pipeline/measure_bandpass.cu:45-275: 3125 spectra drawn with
 * thrust::default_random_engine(123456) and uniform_int(0, nsamps-1), their
 * recursive median per channel (5 levels of median-of-5), smoothed: the
 * bandpass; the recursive median of |spectrum - bandpass| times 1.4826,
 * smoothed: the band's deviation, whose median over channels is *rms. */
void or_measure_bandpass(const uint8_t* fb, size_t nsamps, size_t nchans, float* bp,
                         float* rms) {
  const size_t N = 3125;
  float* s1 = (float*)malloc(N * nchans * sizeof(float));
  float* s2 = (float*)malloc(N / 5 * nchans * sizeof(float));
  float* s3 = (float*)malloc(N / 25 * nchans * sizeof(float));
  float* s4 = (float*)malloc(N / 125 * nchans * sizeof(float));
  float* s5 = (float*)malloc(N / 625 * nchans * sizeof(float));
  float* tmp = (float*)malloc((nchans / 5 + 1) * sizeof(float));
  float* mad = (float*)malloc(nchans * sizeof(float));
  uint32_t st = or_minstd_seed(123456u);
  for (size_t i = 0; i < N; i++) {
    uint32_t t = or_uniform_uint(&st, 0u, (uint32_t)(nsamps - 1));
    for (size_t c = 0; c < nchans; c++) s1[i * nchans + c] = (float)fb[(size_t)t * nchans + c];
  }
  or_median_scrunch5_array(s1, nchans, N, s2);
  or_median_scrunch5_array(s2, nchans, N / 5, s3);
  or_median_scrunch5_array(s3, nchans, N / 25, s4);
  or_median_scrunch5_array(s4, nchans, N / 125, s5);
  or_median_scrunch5_array(s5, nchans, N / 625, bp);
  or_smooth_band(bp, nchans, tmp);
  for (size_t i = 0; i < N; i++)
    for (size_t c = 0; c < nchans; c++)
      s1[i * nchans + c] = fabsf(s1[i * nchans + c] - bp[c]);
  or_median_scrunch5_array(s1, nchans, N, s2);
  or_median_scrunch5_array(s2, nchans, N / 5, s3);
  or_median_scrunch5_array(s3, nchans, N / 25, s4);
  or_median_scrunch5_array(s4, nchans, N / 125, s5);
  or_median_scrunch5_array(s5, nchans, N / 625, mad);
  for (size_t c = 0; c < nchans; c++) mad[c] = mad[c] * 1.4826f;
  or_smooth_band(mad, nchans, tmp);
  memcpy(s2, mad, nchans * sizeof(float));
  qsort(s2, nchans, sizeof(float), or_cmp_float);
  *rms = s2[nchans / 2];
  free(s1); free(s2); free(s3); free(s4); free(s5); free(tmp); free(mad);
}

/* zap_narrow_rfi_functor (clean_filterbank_rfi.cu:114-193) over words
 * [w0, w1) in index order, in place: a byte whose |value - bandpass| is
 * above thresh is replaced by the byte of a channel drawn within
 * max_dist (up to 10 redraws while the drawn one is bad too).  As in the
 * reference, the bandpass entry and the draw range use channel w + k (w the
 * word's index in its spectrum, k the byte), and draws read the spectrum as
 * already zapped by earlier words. */
static void or_zap_narrow(uint8_t* data, size_t w0, size_t w1, const float* bp, float thresh,
                          unsigned stride, unsigned nchans, unsigned max_dist) {
  uint32_t* d = (uint32_t*)data;
  for (size_t i = w0; i < w1; i++) {
    unsigned t = (unsigned)(i / stride), w = (unsigned)(i % stride);
    uint32_t word = d[i];
    uint32_t st = or_minstd_seed(or_hash((uint32_t)i));
    int any = 0;
    for (unsigned k = 0; k < 4; k++) {
      unsigned c = w + k;
      uint32_t val = (word >> (k * 8)) & 0xFFu;
      if (fabsf((float)val - bp[c]) > thresh) {
        any = 1;
        unsigned min_c = c > max_dist ? c - max_dist : 0;
        unsigned max_c = c < nchans - 1 - max_dist ? c + max_dist : nchans - 1;
        unsigned nc = or_uniform_uint(&st, min_c, max_c);
        int attempts = 0;
        uint32_t nv = (d[(size_t)t * stride + nc / 4] >> ((nc % 4) * 8)) & 0xFFu;
        while (fabsf((float)nv - bp[nc]) > thresh && ++attempts < 11) {
          nc = or_uniform_uint(&st, min_c, max_c);
          nv = (d[(size_t)t * stride + nc / 4] >> ((nc % 4) * 8)) & 0xFFu;
        }
        word &= ~(0xFFu << (k * 8));
        word |= nv << (k * 8);
      }
    }
    if (any) d[i] = word;
  }
}

/* The narrow-band branch (clean_filterbank_rfi.cu:303-351) on 8-bit data, in
 * place: per stretch of baseline_length / dt spectra, measure the bandpass
 * and zap with thresh = rfi_tol * rms and a draw radius of nchans / 60.
 * Returns -1 if the stretch is empty or nchans is not a multiple of 4 of at
 * least 20 (the reference's filters read outside the band then). */
int or_narrow_band(uint8_t* data, size_t nsamps, size_t nchans, float dt, float baseline_length,
                   float rfi_tol) {
  size_t nsmooth = (size_t)(baseline_length / (1 * dt));
  if (nsmooth == 0 || nchans % 4 != 0 || nchans < 20) return -1;
  unsigned stride = (unsigned)(nchans / 4);
  unsigned maxd = (unsigned)(nchans / 60);
  float* bp = (float*)malloc(nchans * sizeof(float));
  for (size_t g = 0; g < nsamps; g += nsmooth) {
    size_t ng = nsmooth < nsamps - g ? nsmooth : nsamps - g;
    float rms = 0.f;
    or_measure_bandpass(data + g * nchans, ng, nchans, bp, &rms);
    or_zap_narrow(data, g * stride, (g + ng) * stride, bp, rfi_tol * rms, stride,
                  (unsigned)nchans, maxd);
  }
  free(bp);
  return 0;
}

/* Test hook: when set, or_clean_filterbank_rfi runs the narrow-band branch
 * first and the broadband branch on its output (the reference with the
 * branch enabled: both read h_in_copy). */
static int g_narrow_band = 0;
void or_set_narrow_band(int enable) { g_narrow_band = enable; }

/* clean_filterbank_rfi (clean_filterbank_rfi.cu:256-528), broadband branch
 * only (the narrow-band branch is disabled at :303).  Returns 0, or -1 if the
 * resample radius is not below nsamps (the reference then reads outside the
 * filterbank). */
int or_clean_filterbank_rfi(const uint8_t* in, size_t nsamps, size_t nbits,
                            size_t nchans, float dt, float baseline_length,
                            float rfi_tol, size_t boxcar_max, size_t nbeams,
                            uint8_t* out, int* mask_out) {
  size_t beam_stride = nsamps / nbeams;
  size_t count = nsamps;          /* zero-DM plan: max delay 0 */
  size_t beam_nsamps = beam_stride;
  size_t nsamps_smooth = (size_t)(baseline_length / (2 * dt));
  if (nsamps_smooth / 4 >= nsamps) return -1;
  uint8_t* nb = NULL;
  if (g_narrow_band) {
    nb = (uint8_t*)malloc(nsamps * nchans + 16);
    memcpy(nb, in, nsamps * nchans);
    if (or_narrow_band(nb, nsamps, nchans, dt, baseline_length, rfi_tol) != 0) {
      free(nb);
      return -1;
    }
    in = nb;
  }
  float* s = (float*)calloc(count + 8, sizeof(float));
  for (size_t t = 0; t < count; t++) {
    int32_t acc = 0;
    for (size_t c = 0; c < nchans; c++) acc += in[t * nchans + c];
    s[t] = (float)acc;
  }
  or_remove_baseline(s, count, beam_stride, beam_nsamps, nsamps_smooth, nbeams);
  float* rms = (float*)calloc(nbeams, sizeof(float));
  or_rms_beams(s, rms, beam_stride, beam_nsamps, nbeams);
  or_normalise_beams(s, rms, beam_stride, count);
  int* mask = (int*)calloc(count + 8, sizeof(int));
  int* fm = (int*)calloc(count + 8, sizeof(int));
  int* sm = (int*)calloc(count + 8, sizeof(int));
  for (size_t t = 0; t < count; t++) mask[t] = fabsf(s[t]) > rfi_tol;
  float* S = (float*)calloc(count + 8, sizeof(float));
  or_exclusive_scan(s, count + 1, S);
  size_t nf = count + 1 - boxcar_max;
  float* F = (float*)calloc(nf + 8, sizeof(float));
  size_t off = boxcar_max / 2;
  for (size_t w = 1; w <= boxcar_max; w *= 2) {
    or_matched_filter(S, count + 1, boxcar_max, F, w, 1);
    float norm = (float)(1.0 / (double)sqrtf((float)w));
    for (size_t k = 0; k < nf; k++) F[k] = F[k] * norm;
    for (size_t k = 0; k < nf; k++) fm[off + k] = fabsf(F[k]) > rfi_tol;
    int sum = 0;
    for (size_t k = 0; k <= count; k++) { int tmp = fm[k]; sm[k] = sum; sum += tmp; }
    size_t ahead = (w - 1) / 2 + 1, behind = w / 2;
    for (size_t k = 0; k < nf; k++) fm[off + k] = sm[off + ahead + k] - sm[off - behind + k];
    for (size_t t = 0; t < count; t++) mask[t] = mask[t] || fm[t];
  }
  or_zap(mask, in, count, nbits, nchans, nsamps_smooth / 4, out);
  if (mask_out) memcpy(mask_out, mask, count * sizeof(int));
  free(s); free(rms); free(mask); free(fm); free(sm); free(S); free(F);
  free(nb);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Whole chain: Pipeline/pipeline.cu:233-887 (use_scrunching = 0)            */
/* ------------------------------------------------------------------------ */
static unsigned or_log2(size_t v) { unsigned r = 0; while ((v >> r) > 1) r++; return r; }

typedef struct {
  or_giants g[16];
  int       nw;
  int       stopped;  /* a break condition fired before this DM */
} or_dm_out;

/* Test hook: when set, or_hd_execute copies each DM trial's prefix sum
 * (nc + 1 values) to g_scan_capture + d * pitch. */
static float* g_scan_capture = NULL;
static size_t g_scan_capture_pitch = 0;
void or_set_scan_capture(float* buf, size_t pitch) {
  g_scan_capture = buf;
  g_scan_capture_pitch = pitch;
}

int or_hd_execute(const or_params* p, const uint8_t* fb, size_t nsamps, size_t nbits,
                  size_t first_idx, size_t nbeams, or_result* res) {
  (void)first_idx;
  memset(res, 0, sizeof(*res));
  if (nbits != 8 || nbeams == 0 || p->nchans % 4 != 0) { res->error = 8; return res->error; }
  if (p->min_tscrunch_width < 2) { res->error = 7; return res->error; }
  size_t C = p->nchans;
  int* km = (int*)malloc(C * sizeof(int));
  for (size_t c = 0; c < C; c++) km[c] = 1;
  const uint8_t* in = fb;
  uint8_t* clean = NULL;
  if (p->clean) {
    clean = (uint8_t*)malloc(nsamps * C + 16);
    if (or_clean_filterbank_rfi(fb, nsamps, nbits, C, p->dt, p->baseline_length,
                                p->rfi_tol, 64, nbeams, clean, NULL) != 0) {
      free(km); free(clean); res->error = 11; return res->error;
    }
    in = clean;
  }
  for (unsigned z = 0; z < p->num_channel_zaps; z++)
    for (size_t j = p->channel_zaps[2 * z]; j < p->channel_zaps[2 * z + 1]; j++)
      if (j < C) km[j] = 0;

  float dml[65536];
  size_t D = or_generate_dm_list(p->dm_min, p->dm_max, p->dt, p->dm_pulse_width, p->f0,
                                 p->df, C, p->dm_tol, dml, 65536);
  if (D > 65536) D = 65536;
  float* table = (float*)malloc(C * sizeof(float));
  or_delay_table(C, p->dt, p->f0, p->df, table);
  size_t max_delay = or_max_delay(dml, D, table, C);
  res->dm_count = D;
  res->max_delay = max_delay;
  if (nsamps <= max_delay) {
    free(km); free(clean); free(table); res->error = 11; return res->error;
  }
  size_t nc = nsamps - max_delay;
  res->nsamps_processed = nsamps - nbeams * (p->boxcar_max + max_delay);
  if (nsamps < nbeams * (p->boxcar_max + max_delay)) res->nsamps_processed = 0;

  size_t ostr = nc + 1;
  float* dd = (float*)malloc(D * ostr * sizeof(float));
  /* per-trial scrunch factors (pipeline.cu:187-196,344-345), all 1 without
   * adaptive dt */
  size_t* scr_list = (size_t*)malloc(D * sizeof(size_t));
  if (p->use_scrunching)
    or_scrunch_factors(dml, D, p->dt, p->dm_pulse_width, p->f0, p->df, C, p->scrunch_tol,
                       scr_list);
  else
    for (size_t d = 0; d < D; d++) scr_list[d] = 1;
  res->scrunch = scr_list;
  or_dedisperse_scrunched(in, nsamps, C, C, km, dml, D, table, scr_list, dd, ostr,
                          p->nthreads);

  size_t Bmax = p->boxcar_max;
  size_t nwidths = or_log2(Bmax) + 1;
  or_dm_out* per = (or_dm_out*)calloc(D, sizeof(or_dm_out));
  /* the DM loop's break conditions (pipeline.cu:497-502,632-637), per trial;
   * the first trial that trips one ends the search */
  for (size_t d = 0; d < D; d++) {
    size_t scr = scr_list[d];
    size_t cur_delay = max_delay / scr;
    size_t cur_bs = nsamps / nbeams / scr;
    per[d].stopped = (cur_delay >= cur_bs) || (cur_delay + Bmax / scr > cur_bs);
  }
  int stop_all = per[0].stopped;
  if (!stop_all) {
#ifdef _OPENMP
    int nt = p->nthreads > 0 ? p->nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
    for (long long dl = 0; dl < (long long)D; dl++) {
      size_t d = (size_t)dl;
      if (per[d].stopped) continue;
      size_t scr = scr_list[d], cur_nsamps = nc / scr;
      float cur_dt = p->dt * (float)scr;
      size_t cur_delay = max_delay / scr;
      size_t cur_bs = nsamps / nbeams / scr;
      size_t cur_bn = cur_bs - cur_delay;
      float* x = (float*)calloc(cur_nsamps + 8, sizeof(float));
      memcpy(x, dd + d * ostr, cur_nsamps * sizeof(float));
      size_t smooth = (size_t)(p->baseline_length / (2 * cur_dt));
      or_remove_baseline(x, cur_nsamps, cur_bs, cur_bn, smooth, nbeams);
      float rms[4096];
      or_rms_beams(x, rms, cur_bs, cur_bn, nbeams);
      or_normalise_beams(x, rms, cur_bs, cur_nsamps);
      size_t rel_bmax = Bmax / scr;
      size_t max_nf = cur_nsamps + 1 - rel_bmax;
      size_t cur_off = rel_bmax / 2;
      float* S = (float*)calloc(cur_nsamps + 8, sizeof(float));
      or_exclusive_scan(x, cur_nsamps + 1, S);
      if (g_scan_capture)
        memcpy(g_scan_capture + d * g_scan_capture_pitch, S, (cur_nsamps + 1) * sizeof(float));
      float* F = (float*)calloc(nc + 8, sizeof(float));
      int wi = 0;
      for (size_t fw = scr; fw <= Bmax; fw *= 2, wi++) {
        size_t rel_fw = fw / scr;
        size_t fidx = or_log2(fw);
        size_t rel_min_ts = p->min_tscrunch_width / scr; if (rel_min_ts < 1) rel_min_ts = 1;
        size_t ts = 2 * rel_fw / rel_min_ts; if (ts < 1) ts = 1;
        size_t rel_rel_fw = rel_fw / ts;
        or_matched_filter(S, cur_nsamps + 1, rel_bmax, F, rel_fw, ts);
        size_t nf = (max_nf - 1) / ts + 1;
        size_t cur_scr = scr * ts;
        size_t bn = cur_bs - (cur_delay + rel_bmax);
        float brms = or_rms_block(F, cur_bs, bn, nbeams);
        or_normalise_scalar(F, brms, nf);
        or_giants* G = &per[d].g[wi];
        or_giants_init(G);
        or_find_giants(F, nf, p->detect_thresh, p->cand_sep_time * rel_rel_fw, cur_bs, bn, G);
        size_t roff = cur_off / ts;
        for (size_t k = 0; k < G->count; k++) {
          G->inds[k] = (G->inds[k] + roff) * cur_scr;
          G->begins[k] = (G->begins[k] + roff) * cur_scr;
          G->ends[k] = (G->ends[k] + roff) * cur_scr;
          G->filter_inds[k] = fidx;
          G->dm_inds[k] = d;
          G->members[k] = 1;
        }
      }
      per[d].nw = wi;
      free(x); free(S); free(F);
    }
  }
  /* Append in (DM, width) order and apply the giant-rate bail-out
   * (pipeline.cu:779-787) in that same order. */
  or_giants* all = &res->giants;
  or_giants_init(all);
  int too_many = 0;
  float mins = (float)((double)((float)nsamps * p->dt) / 60.0);
  for (size_t d = 0; d < D && !stop_all && !too_many; d++) {
    if (per[d].stopped) break;
    for (int w = 0; w < per[d].nw && !too_many; w++) {
      or_giants* G = &per[d].g[w];
      or_giants_reserve(all, all->count + G->count + 1);
      for (size_t k = 0; k < G->count; k++) {
        size_t j = all->count++;
        all->peaks[j] = G->peaks[k]; all->inds[j] = G->inds[k];
        all->begins[j] = G->begins[k]; all->ends[j] = G->ends[k];
        all->filter_inds[j] = G->filter_inds[k]; all->dm_inds[j] = G->dm_inds[k];
        all->members[j] = 1;
      }
      if (p->max_giant_rate != 0.0f && ((float)all->count / mins > p->max_giant_rate))
        too_many = 1;
    }
  }
  for (size_t d = 0; d < D; d++)
    for (int w = 0; w < per[d].nw; w++) or_giants_free(&per[d].g[w]);
  free(per);
  (void)nwidths;
  if (!too_many) {
    size_t G = all->count;
    res->labels = (size_t*)malloc((G + 1) * sizeof(size_t));
    res->label_count = or_label_clusters(G, all, p->cand_sep_time, p->cand_sep_filter,
                                         p->cand_sep_dm, nsamps / nbeams, res->labels);
    or_giants_init(&res->groups);
    or_merge(G, res->labels, all, res->label_count, &res->groups);
    res->group_dms = (float*)malloc((res->groups.count + 1) * sizeof(float));
    for (size_t k = 0; k < res->groups.count; k++) res->group_dms[k] = dml[res->groups.dm_inds[k]];
    res->error = 0;
  } else {
    res->error = 12;
  }
  free(km); free(clean); free(table); free(dd);
  return res->error;
}

void or_result_free(or_result* res) {
  or_giants_free(&res->giants);
  or_giants_free(&res->groups);
  free(res->labels);
  free(res->group_dms);
  free(res->scrunch);
  memset(res, 0, sizeof(*res));
}
