/*
 * oracle.h -- CPU restatement of Heimdall's per-gulp search chain.
 *
 * TEST INFRASTRUCTURE ONLY.  This code is the checker for the CUDA product in
 * heimdall_multibeam_b200/; it is never linked into, loaded by or called from
 * the product.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it.
 *
 * Every function restates one reference function with the same arithmetic
 * (same float/double types, same operation order, no FMA contraction) so the
 * product can be compared bit-for-bit.  Each definition cites the reference
 * file:line it follows.  Pinning: the DM-list generator reproduces
 * Share/dm2000.list; the stage functions are compared against the reference's
 * own stage code rebuilt on Thrust's OpenMP backend (oracle/Makefile, target
 * `ref`).  The dedispersion delay table follows the documented restatement in
 * include/dedisp.h (the real dedisp library is not in the reference tree).
 */
#ifndef HD_ORACLE_H
#define HD_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- selection networks (Pipeline/median_filter.cu:21-75) ---------------- */
float or_median3(float a, float b, float c);
float or_median4(float a, float b, float c, float d);
float or_median5(float a, float b, float c, float d, float e);

/* ---- dedisp restatement ------------------------------------------------- */
size_t or_generate_dm_list(float dm_start, float dm_end, double dt, double ti,
                           double f0, double df, size_t nchans, double tol,
                           float* out, size_t cap);
void   or_delay_table(size_t nchans, float dt, float f0, float df, float* table);
size_t or_delay(float dm, float table_c);
size_t or_max_delay(const float* dm_list, size_t dm_count, const float* table,
                    size_t nchans);
void   or_dedisperse(const uint8_t* in, size_t nsamps, size_t in_stride,
                     size_t nchans, const int* killmask, const float* dm_list,
                     size_t dm_count, const float* table, float* out,
                     size_t out_stride, int nthreads);
/* Per-trial scrunch factors of adaptive dt, and dedispersion with them
 * (oracle.c documents the restated rule and the scrunched input). */
void   or_scrunch_factors(const float* dm_list, size_t dm_count, double dt, double ti,
                          double f0, double df, size_t nchans, double tol, size_t* out);
void   or_dedisperse_scrunched(const uint8_t* in, size_t nsamps, size_t in_stride,
                               size_t nchans, const int* killmask, const float* dm_list,
                               size_t dm_count, const float* table, const size_t* scrunch,
                               float* out, size_t out_stride, int nthreads);

/* ---- stage restatements -------------------------------------------------- */
void  or_linear_stretch(const float* in, size_t in_count, float* out, size_t out_count);
void  or_linear_stretch_beam(const float* in, size_t in_count_beam, float* out,
                             size_t out_count_beam, size_t nbeam);
void  or_median_scrunch5(const float* in, size_t count, float* out);
void  or_median_scrunch5_beam(const float* in, size_t beam_stride, size_t nbeam,
                              float* out);
int   or_remove_baseline(float* data, size_t data_len, size_t beam_stride,
                         size_t beam_count, size_t smooth_radius, size_t nbeams);
void  or_baseline_plan(size_t beam_stride, size_t smooth_radius,
                       size_t* sample_count, size_t* nscrunches, size_t* count_round);
void  or_rms_beams(const float* data, float* rms, size_t beam_stride,
                   size_t beam_count, size_t nbeams);
float or_rms_block(const float* data, size_t beam_stride, size_t beam_count,
                   size_t nbeams);
void  or_normalise_beams(float* data, const float* rms, size_t beam_stride,
                         size_t count);
void  or_normalise_scalar(float* data, float rms, size_t count);
void  or_exclusive_scan(const float* in, size_t n_in, float* out);
void  or_matched_filter(const float* scanned, size_t scanned_size, size_t max_width,
                        float* out, size_t width, size_t tscrunch);

/* Giant list (Pipeline/find_giants.cu:101-316 + pipeline.cu:755-775). */
typedef struct {
  size_t  count, cap;
  float*  peaks;
  size_t* inds;
  size_t* begins;
  size_t* ends;
  size_t* filter_inds;
  size_t* dm_inds;
  size_t* members;
} or_giants;

void   or_giants_init(or_giants* g);
void   or_giants_free(or_giants* g);
size_t or_find_giants(const float* data, size_t count, float thresh, size_t merge_dist,
                      size_t beam_stride, size_t beam_count, or_giants* out);

size_t or_label_clusters(size_t count, const or_giants* g, size_t time_tol,
                         size_t filter_tol, size_t dm_tol, size_t nsamps_beam,
                         size_t* labels);
void   or_merge(size_t count, const size_t* labels, const or_giants* g,
                size_t label_count, or_giants* groups);

/* ---- RFI cleaning (Pipeline/clean_filterbank_rfi.cu) --------------------- */
uint32_t or_hash(uint32_t a);
uint32_t or_uniform_uint(uint32_t* state, uint32_t lo, uint32_t hi);
void     or_measure_bandpass(const uint8_t* fb, size_t nsamps, size_t nchans, float* bandpass,
                             float* rms);
int      or_narrow_band(uint8_t* data, size_t nsamps, size_t nchans, float dt,
                        float baseline_length, float rfi_tol);
void     or_set_narrow_band(int enable);
int      or_clean_filterbank_rfi(const uint8_t* in, size_t nsamps, size_t nbits,
                                 size_t nchans, float dt, float baseline_length,
                                 float rfi_tol, size_t boxcar_max, size_t nbeams,
                                 uint8_t* out, int* mask_out);

/* ---- whole chain (Pipeline/pipeline.cu:233-1087) ------------------------- */
typedef struct {
  size_t nchans;
  float  dt, f0, df;
  float  dm_min, dm_max, dm_tol, dm_pulse_width;
  float  baseline_length;
  float  rfi_tol;
  size_t boxcar_max;
  float  detect_thresh;
  size_t cand_sep_time, cand_sep_filter, cand_sep_dm;
  float  max_giant_rate;
  size_t min_tscrunch_width;
  int    clean;              /* run clean_filterbank_rfi (reference: -DCLEANING) */
  unsigned num_channel_zaps;
  const size_t* channel_zaps;  /* 2*num_channel_zaps: [start, end) pairs */
  int    nthreads;
  int    use_scrunching;     /* adaptive dt (pipeline.cu:187-196) */
  float  scrunch_tol;
} or_params;

typedef struct {
  int     error;               /* 0 ok, 12 too many events, 11 too few samples */
  size_t  nsamps_processed;
  size_t  dm_count;
  size_t  max_delay;
  or_giants giants;            /* every giant in append order */
  size_t* labels;              /* giants.count */
  size_t  label_count;
  or_giants groups;            /* merged candidates, label order */
  float*  group_dms;
  size_t* scrunch;             /* dm_count scrunch factors */
} or_result;

int  or_hd_execute(const or_params* p, const uint8_t* fb, size_t nsamps, size_t nbits,
                   size_t first_idx, size_t nbeams, or_result* res);
void or_result_free(or_result* res);
/* Test hook: keep every DM trial's prefix sum of the last or_hd_execute. */
void or_set_scan_capture(float* buf, size_t pitch);
/* The S/N of giants (DM trial, filter index, giant sample index as
 * or_hd_execute reports them) from the same chain with every value in
 * double (snr64.c).  Returns 0, or non-zero for a giant it cannot place. */
int  or64_giant_snr(const or_params* p, const uint8_t* fb, size_t nsamps, size_t nbeams,
                    size_t n, const size_t* dm_inds, const size_t* filter_inds,
                    const size_t* inds, double* snr);

/* ---- candidate profiler (Applications/candidate_profiler.C; profiler.c) ---- */
int    or_profile_ft(const uint8_t* fb, size_t nsamps, size_t nchans, float dt, float f0,
                     float df, size_t samp, size_t filter, float dm, size_t out_nsamps,
                     size_t fscrunch, float* out);
size_t or_profile_dm(const uint8_t* fb, size_t nsamps, size_t nchans, float dt, float f0,
                     float df, const float* dm_list, size_t dm_count, size_t samp,
                     size_t filter, size_t dm_idx, size_t out_nsamps, size_t out_dm_count,
                     int do_filter, float* out, size_t* dm_begin_out);
size_t or_profile(const uint8_t* fb, size_t nsamps, size_t nchans, double tsamp, double fch1,
                  double foff, const float* dm_list, size_t dm_count, size_t samp,
                  size_t filter, size_t dm_idx, size_t out_nsamps, size_t out_dm_count,
                  size_t fscrunch, int do_filter, float* dm_time, float* dm0_time,
                  float* freq_time, size_t* max_idx_out, size_t* snr_dm_first, float* snr_dm,
                  float* snr_time);

/* ---- classifier (Applications/candidate_profiler.C and the CNN) ---- */
void or_normalise_rows(float* data, size_t n, size_t nrows);
void or_patch_dm(const float* scans, size_t pitch, size_t len, size_t ndm, size_t dm,
                 size_t ind, size_t filter, float* out);
void or_patch_ft(const uint8_t* tf, size_t nsamps, size_t nchans, size_t max_delay,
                 size_t ind, size_t filter, float* out);
size_t or_cnn_param_count(void);
float or_bf16(float x);
void or_cnn_run(const float* params, const float* dm_time, const float* freq_time,
                const int* labels, size_t n, float* probs, float* grads, float* loss);

#ifdef __cplusplus
}
#endif
#endif
