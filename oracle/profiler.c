/*
 * profiler.c -- CPU restatement of the reference's candidate profiler
 * (Applications/candidate_profiler.C).  TEST INFRASTRUCTURE ONLY: the checker
 * of the GPU profiler (hd_profile_candidates).
 *
 *   or_profile_ft     gen_freq_time_plot (candidate_profiler.C:136-230)
 *   or_profile_dm     gen_dm_time_plot   (candidate_profiler.C:232-415)
 *   or_profile        main's plots and extractions (:443-640): the DM-time
 *                     plot, the DM-0 series, the freq-time plot, SNR vs DM
 *                     and SNR vs time
 *
 * The profiler reads a sigproc file; here the data are the file's spectra
 * (fb, nsamps x nchans bytes, 8-bit).  Where the reference reads outside the
 * file (a window that starts before the first spectrum or runs past the
 * last) it gets no data; here such samples read as 0.  Dedispersion uses the
 * dedisp restatement (oracle.c), with adaptive dt on the window's trials as
 * gen_dm_time_plot enables it (pulse width 40 us, tolerance 1.15).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

static uint8_t sample_at(const uint8_t* fb, size_t nsamps, size_t nchans, long long t, size_t c) {
  return (t >= 0 && t < (long long)nsamps) ? fb[(size_t)t * nchans + c] : 0;
}

static int cmp_f(const void* a, const void* b) {
  float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}

static float kth_of(const float* v, size_t n, size_t k, float* tmp) {
  memcpy(tmp, v, n * sizeof(float));
  qsort(tmp, n, sizeof(float), cmp_f);
  return tmp[k];
}

/* normalise_series_array (candidate_profiler.C:88-134) with its arithmetic
 * kept where a row has no deviation: the scale 1 / (mad * 1.4826) is then
 * infinite and the row becomes NaN (0 * inf) or +-inf, as in the reference. */
static void normalise_rows_ref(float* data, size_t n, size_t nrows) {
  float* tmp = (float*)malloc(n * sizeof(float));
  float* a = (float*)malloc(n * sizeof(float));
  for (size_t r = 0; r < nrows; r++) {
    float* x = data + r * n;
    float median1 = kth_of(x, n / 2, n / 4, tmp);
    float median2 = kth_of(x + n / 2, n - n / 2, n / 4, tmp);
    double gradient = (double)((median2 - median1) / (float)(n / 2));
    float median0 = (float)((double)median1 - gradient * (double)(n / 4));
    for (size_t j = 0; j < n; j++) {
      float baseline = (float)((double)median0 + (double)j * gradient);
      x[j] = x[j] - baseline;
      a[j] = fabsf(x[j]);
    }
    float mad = kth_of(a, n, n / 2, tmp);
    float stddev = (float)((double)mad * 1.4826);
    float val = (float)(1.0 / (double)stddev);
    for (size_t j = 0; j < n; j++) x[j] = x[j] * val;
  }
  free(tmp);
  free(a);
}

/* gen_freq_time_plot: the undispersed window around the candidate, scrunched
 * by tscrunch x fscrunch, each channel row normalised. */
int or_profile_ft(const uint8_t* fb, size_t nsamps, size_t nchans, float dt, float f0, float df,
                  size_t samp, size_t filter, float dm, size_t out_nsamps, size_t fscrunch,
                  float* out) {
  if (fscrunch == 0 || nchans % fscrunch != 0 || out_nsamps < 2) return -1;
  float* table = (float*)malloc(nchans * sizeof(float));
  or_delay_table(nchans, dt, f0, df, table);
  size_t max_delay = or_max_delay(&dm, 1, table, nchans);
  free(table);
  size_t delay = 2;
  size_t tscrunch = (size_t)1 << filter;
  size_t in_nsamps = out_nsamps * tscrunch;
  if (in_nsamps < max_delay) {
    while (delay < max_delay) delay *= 2;
    in_nsamps = delay;
    tscrunch = in_nsamps / out_nsamps;
  }
  long long first = (long long)(samp + max_delay / 2) - (long long)(in_nsamps / 2);
  const size_t out_nchans = nchans / fscrunch;
  for (size_t t = 0; t < in_nsamps; t += tscrunch) {
    if (t / tscrunch >= out_nsamps) break;
    for (size_t c = 0; c < nchans; c += fscrunch) {
      float sum = 0.f;
      for (size_t s = 0; s < tscrunch; ++s)
        for (size_t f = 0; f < fscrunch; ++f) {
          uint8_t x = sample_at(fb, nsamps, nchans, first + (long long)(t + s), c + f);
          sum += (float)x / 255.f * 255.f;
        }
      out[c / fscrunch * out_nsamps + t / tscrunch] = sum / (float)(tscrunch * fscrunch);
    }
  }
  normalise_rows_ref(out, out_nsamps, out_nchans);
  return 0;
}

/* gen_dm_time_plot: the window's trials [dm_begin, dm_end) around dm_idx,
 * re-dedispersed with adaptive dt, then either summed over the boxcar width
 * at the trial's resolution (do_filter 0) or unscrunched and boxcar-filtered
 * through an exclusive scan (do_filter 1); every row normalised.  Rows
 * [n_dm, out_dm_count) of `out` are left as they are.  Returns n_dm (0 on a
 * bad argument) and the first trial in *dm_begin_out. */
size_t or_profile_dm(const uint8_t* fb, size_t nsamps, size_t nchans, float dt, float f0,
                     float df, const float* dm_list, size_t dm_count, size_t samp, size_t filter,
                     size_t dm_idx, size_t out_nsamps, size_t out_dm_count, int do_filter,
                     float* out, size_t* dm_begin_out) {
  if (dm_idx >= dm_count || out_dm_count == 0 || out_nsamps < 2) return 0;
  size_t dm_begin = dm_idx >= out_dm_count / 2 ? dm_idx - out_dm_count / 2 : 0;
  size_t dm_end = dm_idx < dm_count - ((out_dm_count - 1) / 2 + 1)
                      ? dm_idx + (out_dm_count - 1) / 2 + 1
                      : dm_count;
  size_t n_dm = dm_end - dm_begin;
  const float* dms = dm_list + dm_begin;
  size_t* scr = (size_t*)malloc(n_dm * sizeof(size_t));
  or_scrunch_factors(dms, n_dm, dt, 40.0, f0, df, nchans, 1.15, scr);
  float* table = (float*)malloc(nchans * sizeof(float));
  or_delay_table(nchans, dt, f0, df, table);
  size_t max_delay = or_max_delay(dms, n_dm, table, nchans);
  size_t width = (size_t)1 << filter;
  size_t nd, in_nsamps, first;
  if (!do_filter) {
    nd = out_nsamps * width;
    first = samp >= out_nsamps / 2 * width ? samp - out_nsamps / 2 * width : 0;
  } else {
    nd = out_nsamps + width - 1;
    first = samp > out_nsamps / 2 + width / 2 ? samp - out_nsamps / 2 - width / 2 : 0;
  }
  in_nsamps = nd + max_delay;
  uint8_t* in = (uint8_t*)malloc(in_nsamps * nchans + 1);
  for (size_t t = 0; t < in_nsamps; t++)
    for (size_t c = 0; c < nchans; c++)
      in[t * nchans + c] = sample_at(fb, nsamps, nchans, (long long)(first + t), c);
  int* km = (int*)malloc(nchans * sizeof(int));
  for (size_t c = 0; c < nchans; c++) km[c] = 1;
  float* dd = (float*)calloc(nd * n_dm + 1, sizeof(float));
  or_dedisperse_scrunched(in, in_nsamps, nchans, nchans, km, dms, n_dm, table, scr, dd, nd, 1);
  if (!do_filter) {
    for (size_t d = 0; d < n_dm; ++d)
      for (size_t t = 0; t < out_nsamps; ++t) {
        float v = 0.f;
        size_t sc = scr[d];
        for (size_t j = 0; j < width / sc; ++j) v += dd[d * nd + t * (width / sc) + j];
        out[d * out_nsamps + t] = v;
      }
  } else {
    float* row = (float*)malloc((nd + 1) * sizeof(float));
    float* scanned = (float*)malloc((nd + 1) * sizeof(float));
    for (size_t d = 0; d < n_dm; ++d) {
      for (size_t t = 0; t < nd; ++t) row[t] = dd[d * nd + t / scr[d]];
      scanned[0] = 0.f;
      for (size_t i = 1; i < nd + 1; ++i) scanned[i] = scanned[i - 1] + row[i - 1];
      const size_t a = width / 2 + (width - 1) / 2 + 1;
      for (size_t t = 0; t < out_nsamps; ++t)
        out[d * out_nsamps + t] = scanned[a + t] - scanned[t];
    }
    free(row);
    free(scanned);
  }
  normalise_rows_ref(out, out_nsamps, n_dm);
  free(scr); free(table); free(in); free(km); free(dd);
  *dm_begin_out = dm_begin;
  return n_dm;
}

/* main (candidate_profiler.C:443-640): the DM-time plot (out_dm_count rows,
 * rows past the window's trials left 0), the DM-0 series, the freq-time plot
 * (filter - 2, at least 0), the first maximum of the DM-time plot, SNR vs DM
 * at that maximum's time (snr_dm[d] for trial dm_idx_start + d, d < the
 * window's trial count) and SNR vs time (per time bin: the maximum's row, the
 * rows above and below it (0 outside the plot), the DM-0 series, and the
 * bin's time in seconds, from the header's double tsamp).  Returns the
 * window's trial count, 0 on error. */
size_t or_profile(const uint8_t* fb, size_t nsamps, size_t nchans, double tsamp, double fch1,
                  double foff,
                  const float* dm_list, size_t dm_count, size_t samp, size_t filter,
                  size_t dm_idx, size_t out_nsamps, size_t out_dm_count, size_t fscrunch,
                  int do_filter, float* dm_time, float* dm0_time, float* freq_time,
                  size_t* max_idx_out, size_t* snr_dm_first, float* snr_dm, float* snr_time) {
  /* the dedisp plans take the header's values as float */
  const float dt = (float)tsamp, f0 = (float)fch1, df = (float)foff;
  memset(dm_time, 0, out_nsamps * out_dm_count * sizeof(float));
  memset(dm0_time, 0, out_nsamps * sizeof(float));
  size_t dm_begin = 0, dm0_begin = 0;
  size_t n_dm = or_profile_dm(fb, nsamps, nchans, dt, f0, df, dm_list, dm_count, samp, filter,
                              dm_idx, out_nsamps, out_dm_count, do_filter, dm_time, &dm_begin);
  if (!n_dm) return 0;
  if (!or_profile_dm(fb, nsamps, nchans, dt, f0, df, dm_list, dm_count, samp, filter, 0,
                     out_nsamps, 1, do_filter, dm0_time, &dm0_begin))
    return 0;
  size_t ft_filter = filter > 2 ? filter - 2 : 0;
  if (or_profile_ft(fb, nsamps, nchans, dt, f0, df, samp, ft_filter, dm_list[dm_idx], out_nsamps,
                    fscrunch, freq_time) != 0)
    return 0;
  size_t total = out_nsamps * out_dm_count, max_idx = 0;
  for (size_t i = 1; i < total; i++)
    if (dm_time[i] > dm_time[max_idx]) max_idx = i;
  *max_idx_out = max_idx;
  size_t dm_idx_start = dm_idx > out_dm_count / 2 ? dm_idx - out_dm_count / 2 : 0;
  *snr_dm_first = dm_idx_start;
  size_t t_max = max_idx % out_nsamps;
  for (size_t d = 0; d < out_dm_count; ++d)
    snr_dm[d] = d < n_dm ? dm_time[d * out_nsamps + t_max] : 0.f;
  size_t dmax = max_idx / out_nsamps;
  float width = (float)((size_t)1 << filter);
  for (size_t t = 0; t < out_nsamps; ++t) {
    float tt = (float)((double)((float)samp + ((float)t - (float)(out_nsamps / 2)) * width) *
                       tsamp);
    float* r = snr_time + t * 5;
    r[0] = tt;
    r[1] = dm_time[dmax * out_nsamps + t];
    r[2] = dmax > 0 ? dm_time[(dmax - 1) * out_nsamps + t] : 0.f;
    r[3] = dmax + 1 < out_dm_count ? dm_time[(dmax + 1) * out_nsamps + t] : 0.f;
    r[4] = dm0_time[t];
  }
  return n_dm;
}
