/*
 * snr64.c -- the S/N part of or_hd_execute's chain held in double precision.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  The float chain (oracle.c, and the
 * product, which matches it bit for bit) computes each giant's S/N through
 * baseline removal, per-beam RMS, normalisation, a sequential prefix sum, the
 * boxcar difference of that sum and a block RMS of the boxcar series, all in
 * float (Pipeline/remove_baseline.cu:21-102, get_rms.cu:236-301,344-370,
 * matched_filter.cu:21-67).  These are the same steps with every value in
 * double: the same samples, the same medians (an exact selection picks the
 * same element in either precision), the same interpolation positions (their
 * index arithmetic stays as the reference writes it, in float); only the
 * rounding of the values differs.  or64_giant_snr evaluates that chain at
 * given giants, so a test can state the float chain's S/N error against it.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define D_CSWAP(x, y) do { if ((y) < (x)) { double t_ = (x); (x) = (y); (y) = t_; } } while (0)

static double d_median3(double a, double b, double c) {
  D_CSWAP(a, b);
  D_CSWAP(b, c);
  D_CSWAP(a, b);
  return b;
}

static double d_median4(double a, double b, double c, double d) {
  D_CSWAP(a, b);
  D_CSWAP(c, d);
  D_CSWAP(a, c);
  D_CSWAP(b, d);
  return 0.5 * (b + c);
}

static double d_median5(double a, double b, double c, double d, double e) {
  double v[5] = {a, b, c, d, e};
  for (int i = 1; i < 5; i++)
    for (int j = i; j > 0 && v[j] < v[j - 1]; j--) {
      double t = v[j]; v[j] = v[j - 1]; v[j - 1] = t;
    }
  return v[2];
}

static unsigned d_f2u(float x) { return (x != x) ? 0u : (unsigned)x; }

/* or_linear_stretch with double values (positions as the float chain's) */
static void d_linear_stretch(const double* in, size_t in_count, double* out, size_t out_count) {
  float step = (float)(in_count - 1) / (float)(out_count - 1);
  for (unsigned i = 0; i < (unsigned)out_count; i++) {
    float x = (float)i * step;
    unsigned j = d_f2u(x);
    float fr = x - (float)j;
    out[i] = in[j] + (((double)fr > 1e-5) ? (double)fr * (in[j + 1] - in[j]) : 0.0);
  }
}

static void d_linear_stretch_beam(const double* in, size_t in_count_beam, double* out,
                                  size_t out_count_beam, size_t nbeam) {
  float step = (float)(in_count_beam - 1) / (float)out_count_beam;
  size_t out_count = out_count_beam * nbeam;
  for (unsigned i = 0; i < (unsigned)out_count; i++) {
    size_t beam = i / out_count_beam;
    float x = (float)i * step;
    unsigned k = d_f2u(x + (float)beam);
    float o = (x - (float)k) + (float)beam;
    out[i] = in[k] + (((double)o > 1e-5) ? (double)o * (in[k + 1] - in[k]) : 0.0);
  }
}

static void d_median_scrunch5(const double* in, size_t count, double* out) {
  if (count == 1) out[0] = in[0];
  else if (count == 2) out[0] = 0.5 * (in[0] + in[1]);
  else if (count == 3) out[0] = d_median3(in[0], in[1], in[2]);
  else if (count == 4) out[0] = d_median4(in[0], in[1], in[2], in[3]);
  else {
    size_t oc = count / 5;
    for (size_t i = 0; i < oc; i++)
      out[i] = d_median5(in[5 * i], in[5 * i + 1], in[5 * i + 2], in[5 * i + 3], in[5 * i + 4]);
  }
}

static void d_median_scrunch5_beam(const double* in, size_t beam_stride, size_t nbeam,
                                   double* out) {
  if (beam_stride > 4) {
    size_t oc = beam_stride / 5, total = nbeam * oc;
    for (size_t o = 0; o < total; o++) {
      size_t beam = o / oc, i = (o % oc) * 5, off = beam * beam_stride + i;
      out[o] = d_median5(in[off], in[off + 1], in[off + 2], in[off + 3], in[off + 4]);
    }
  } else {
    for (size_t o = 0; o < nbeam; o++) {
      size_t off = o * beam_stride;
      if (beam_stride == 1) out[o] = in[off];
      else if (beam_stride == 2) out[o] = 0.5 * (in[off] + in[off + 1]);
      else if (beam_stride == 3) out[o] = d_median3(in[off], in[off + 1], in[off + 2]);
      else out[o] = d_median4(in[off], in[off + 1], in[off + 2], in[off + 3]);
    }
  }
}

/* or_remove_baseline in double; `data` holds one readable zero past its end */
static void d_remove_baseline(double* data, size_t beam_stride, size_t beam_count,
                              size_t smooth_radius, size_t nbeams) {
  size_t sample_count, nscr, count_round;
  or_baseline_plan(beam_stride, smooth_radius, &sample_count, &nscr, &count_round);
  if (sample_count == 0) return;
  size_t dm_delay = beam_stride - beam_count;
  size_t nbm = nbeams - 1;
  size_t nsamps = beam_stride * nbeams - dm_delay;
  double* buf1 = (double*)calloc(nbeams * count_round + 8, sizeof(double));
  double* buf2 = (double*)calloc(nbeams * (count_round / 5) + 8, sizeof(double));
  double* base = (double*)calloc(beam_stride * nbeams + 8, sizeof(double));
  d_linear_stretch_beam(data, beam_stride, buf1, count_round, nbm);
  d_linear_stretch(data + nbm * beam_stride, beam_count, buf1 + nbm * count_round, count_round);
  double* p1 = buf1;
  double* p2 = buf2;
  for (size_t size = count_round; size > sample_count; size /= 5) {
    d_median_scrunch5_beam(p1, size, nbeams, p2);
    double* t = p1; p1 = p2; p2 = t;
  }
  d_linear_stretch_beam(p1, sample_count, base, beam_stride, nbm);
  d_linear_stretch(p1 + nbm * sample_count, sample_count, base + nbm * beam_stride, beam_count);
  for (size_t i = 0; i < nsamps; i++) data[i] = data[i] - base[i];
  free(buf1); free(buf2); free(base);
}

static void d_reblock_abs_beam(const double* in, size_t in_stride, size_t in_length,
                               double* out, size_t nbeam) {
  size_t oc = in_length * nbeam;
  float delta = (float)(in_stride - in_length);
  for (unsigned o = 0; o < (unsigned)oc; o++) {
    size_t beam = o / in_length;
    size_t i = (size_t)((float)beam * delta + (float)o);
    out[o] = fabs(in[i]);
  }
}

static void d_rms_beams(const double* data, double* rms, size_t beam_stride, size_t beam_count,
                        size_t nbeams) {
  size_t count = nbeams * beam_count;
  double* b1 = (double*)calloc(count + 8, sizeof(double));
  double* b2 = (double*)calloc(count / 5 + 8, sizeof(double));
  d_reblock_abs_beam(data, beam_stride, beam_count, b1, nbeams);
  for (size_t size = beam_count; size > 1; size /= 5) {
    d_median_scrunch5_beam(b1, size, nbeams, b2);
    double* t = b1; b1 = b2; b2 = t;
  }
  for (size_t b = 0; b < nbeams; b++) rms[b] = b1[b] * 1.4862;
  free(b1); free(b2);
}

static double d_rms_block(const double* data, size_t beam_stride, size_t beam_count,
                          size_t nbeams) {
  size_t count = nbeams * beam_count;
  double* b1 = (double*)calloc(count + 8, sizeof(double));
  double* b2 = (double*)calloc(count / 5 + 8, sizeof(double));
  d_reblock_abs_beam(data, beam_stride, beam_count, b1, nbeams);
  for (size_t size = count; size > 1; size /= 5) {
    d_median_scrunch5(b1, size, b2);
    double* t = b1; b1 = b2; b2 = t;
  }
  double m = b1[0];
  free(b1); free(b2);
  return m * 1.4862;
}

static unsigned d_log2(size_t v) { unsigned r = 0; while ((v >> r) > 1) r++; return r; }

int or64_giant_snr(const or_params* p, const uint8_t* fb, size_t nsamps, size_t nbeams,
                   size_t n, const size_t* dm_inds, const size_t* filter_inds,
                   const size_t* inds, double* snr) {
  if (nbeams == 0 || p->nchans % 4 != 0 || p->min_tscrunch_width < 2) return 8;
  const size_t C = p->nchans;
  int* km = (int*)malloc(C * sizeof(int));
  for (size_t c = 0; c < C; c++) km[c] = 1;
  const uint8_t* in = fb;
  uint8_t* clean = NULL;
  if (p->clean) {
    /* the cleaned filterbank is bytes: the float chain's cleaning is the input */
    clean = (uint8_t*)malloc(nsamps * C + 16);
    if (or_clean_filterbank_rfi(fb, nsamps, 8, C, p->dt, p->baseline_length, p->rfi_tol, 64,
                                nbeams, clean, NULL) != 0) {
      free(km); free(clean); return 11;
    }
    in = clean;
  }
  for (unsigned z = 0; z < p->num_channel_zaps; z++)
    for (size_t j = p->channel_zaps[2 * z]; j < p->channel_zaps[2 * z + 1]; j++)
      if (j < C) km[j] = 0;
  float* dml = (float*)malloc(65536 * sizeof(float));
  size_t D = or_generate_dm_list(p->dm_min, p->dm_max, p->dt, p->dm_pulse_width, p->f0, p->df,
                                 C, p->dm_tol, dml, 65536);
  if (D > 65536) D = 65536;
  float* table = (float*)malloc(C * sizeof(float));
  or_delay_table(C, p->dt, p->f0, p->df, table);
  const size_t max_delay = or_max_delay(dml, D, table, C);
  if (nsamps <= max_delay) {
    free(km); free(clean); free(table); free(dml); return 11;
  }
  const size_t nc = nsamps - max_delay;
  const size_t Bmax = p->boxcar_max;
  const size_t cur_bs = nsamps / nbeams;
  const size_t cur_bn = cur_bs - max_delay;
  const size_t smooth = (size_t)(p->baseline_length / (2 * p->dt));
  const size_t rel_min_ts = p->min_tscrunch_width < 1 ? 1 : p->min_tscrunch_width;
  int err = 0;
  /* the DM trials that hold a giant, ascending */
  char* need = (char*)calloc(D, 1);
  for (size_t k = 0; k < n; k++) {
    if (dm_inds[k] >= D) err = 7;
    else need[dm_inds[k]] = 1;
  }
  size_t nu = 0;
  size_t* uq = (size_t*)malloc((D + 1) * sizeof(size_t));
  for (size_t d = 0; d < D; d++)
    if (need[d]) uq[nu++] = d;
  char* done = (char*)calloc(n + 1, 1);
  /* dedisperse the needed trials a chunk at a time (integer sums: exact in
   * either precision; a trial's first nc sums do not depend on which other
   * trials share the call), then run each trial's chain */
  enum { CHUNK = 128 };
  float* dsub = (float*)malloc(CHUNK * sizeof(float));
  float* rows = (float*)malloc((size_t)CHUNK * (nsamps + 8) * sizeof(float));
  for (size_t c0 = 0; c0 < nu && !err; c0 += CHUNK) {
    const size_t m = nu - c0 < (size_t)CHUNK ? nu - c0 : (size_t)CHUNK;
    for (size_t j = 0; j < m; j++) dsub[j] = dml[uq[c0 + j]];
    or_dedisperse(in, nsamps, C, C, km, dsub, m, table, rows, nsamps + 8, p->nthreads);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) reduction(max : err)
#endif
    for (long long jj = 0; jj < (long long)m; jj++) {
      const size_t d = uq[c0 + (size_t)jj];
      const float* row = rows + (size_t)jj * (nsamps + 8);
      double* x = (double*)calloc(nc + 8, sizeof(double));
      double* S = (double*)calloc(nc + 8, sizeof(double));
      double* F = (double*)calloc(nc + 8, sizeof(double));
      for (size_t t = 0; t < nc; t++) x[t] = (double)row[t];
      d_remove_baseline(x, cur_bs, cur_bn, smooth, nbeams);
      double rms[4096];
      d_rms_beams(x, rms, cur_bs, cur_bn, nbeams);
      for (unsigned i = 0; i < (unsigned)nc; i++) x[i] = x[i] / rms[i / cur_bs];
      double sum = 0.0;
      for (size_t k = 0; k < nc + 1; k++) { double t = x[k]; S[k] = sum; sum = sum + t; }
      const size_t max_nf = nc + 1 - Bmax;
      const size_t off = Bmax / 2;
      for (size_t fw = 1; fw <= Bmax; fw *= 2) {
        const size_t fidx = d_log2(fw);
        size_t ts = 2 * fw / rel_min_ts;
        if (ts < 1) ts = 1;
        const size_t ahead = (fw - 1) / 2 + 1, behind = fw / 2;
        const size_t nf = (max_nf - 1) / ts + 1;
        /* every width in turn, normalised in place as the float chain does:
         * a time-scrunched width's block RMS reads, past its own nf values,
         * the normalised values the previous widths left in F */
        for (size_t k = 0; k < nf; k++)
          F[k] = S[off + ahead + k * ts] - S[off - behind + k * ts];
        const size_t bn = cur_bs - (max_delay + Bmax);
        const double r = 1.0 / d_rms_block(F, cur_bs, bn, nbeams);
        for (size_t k = 0; k < nf; k++) F[k] = F[k] * r;
        const size_t roff = off / ts;
        for (size_t k = 0; k < n; k++) {
          if (dm_inds[k] != d || filter_inds[k] != fidx) continue;
          /* a giant's index is (filtered index + roff) * ts */
          const size_t q = inds[k] / ts;
          if (inds[k] % ts != 0 || q < roff || q - roff >= nf) { err = 9; continue; }
          snr[k] = F[q - roff];
          done[k] = 1;
        }
      }
      free(x); free(S); free(F);
    }
  }
  for (size_t k = 0; k < n && !err; k++)
    if (!done[k]) err = 10;  /* a filter index beyond boxcar_max */
  free(need); free(uq); free(dsub); free(rows);
  free(km); free(clean); free(table); free(dml);
  free(done);
  return err;
}
