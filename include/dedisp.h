/*
 * dedisp.h -- the dedispersion-plan C interface that Heimdall's pipeline calls.
 *
 * Heimdall links against an external "dedisp" library that is not part of the
 * reference tree and carries no pinned version (config/dedisp.m4:14-21).  This
 * header declares exactly the subset of that interface the reference calls,
 * with the argument meanings its call sites rely on:
 *
 *   Pipeline/pipeline.cu:171-196   create plan, generate DM list, adaptive dt
 *   Pipeline/pipeline.cu:335-365   getters, killmask, max delay
 *   Pipeline/pipeline.cu:453-462   dedisp_execute_adv over the whole gulp
 *   Pipeline/pipeline.cu:493       dedisp_get_dm_delay
 *   Pipeline/clean_filterbank_rfi.cu:361-397   zero-DM plan + dedisp_execute
 *   Pipeline/error.C:64-91         error enum members and error strings
 *   Applications/generate_dmlist.C:93-101      dedisp_generate_dm_list_guru
 *
 * Two implementations sit behind it:
 *   - libhdb200.so (heimdall_multibeam_b200/csrc): the product, sm_100a kernels;
 *   - oracle/dedisp_cpu.c: the CPU restatement used only as a test checker and
 *     to link the reference's own stage code for the CPU baseline.
 *
 * Semantics both implementations share (documented restatement; the real
 * dedisp is unpinned):
 *   delay_table[c] = K * ((f0 + c*df)^-2 - f0^-2) / dt      (float, K = 4148.808)
 *   delay(d, c)    = (dedisp_size)(dm_list[d] * delay_table[c] + 0.5f)
 *   out[d][t]      = (float) sum_c killmask[c] * in[t + delay(d,c)][c],
 *                    t in [0, nsamps - max_delay), summed exactly in int32.
 * With adaptive dt, trial d has a scrunch factor s_d (dedisp_get_dt_factors)
 * and is computed at sampling time s_d dt:
 *   in_s[c][u]     = (sum_{j<s} in[s u + j][c] + s/2) / s   (byte mean,
 *                    rounded half up), u < nsamps / s;
 *   out[d][u]      = (float) sum_c killmask[c] * in_s[c][u + delay(d,c) / s],
 *                    u in [0, (nsamps - max_delay) / s)   (integer divisions);
 * the rest of row d is left as it was.  Scrunch factors (the rule of
 * Barsdell et al. 2012, MNRAS 422, 379, restated; unpinned): the smearing of
 * trial DM at sampling time T is W(DM, T)^2 = T^2 + pulse_width^2 +
 * (a DM)^2 in microseconds, with the DM-list generator's a = 8.3 df / f^3
 * (df in MHz, f in GHz at the band centre); factors start at 1, never
 * decrease, and trial d doubles the previous factor s when
 * W(DM_d, 2 s dt) / W(DM_d, s dt) < tol.
 */
#ifndef HEIMDALL_B200_DEDISP_H
#define HEIMDALL_B200_DEDISP_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dedisp_plan_struct* dedisp_plan;
typedef size_t        dedisp_size;
typedef float         dedisp_float;
typedef unsigned char dedisp_byte;
typedef int           dedisp_bool;

typedef enum {
  DEDISP_NO_ERROR = 0,
  DEDISP_MEM_ALLOC_FAILED,
  DEDISP_MEM_COPY_FAILED,
  DEDISP_NCHANS_EXCEEDS_LIMIT,
  DEDISP_INVALID_PLAN,
  DEDISP_INVALID_POINTER,
  DEDISP_INVALID_STRIDE,
  DEDISP_NO_DM_LIST_SET,
  DEDISP_TOO_FEW_NSAMPS,
  DEDISP_INVALID_FLAG_COMBINATION,
  DEDISP_UNSUPPORTED_IN_NBITS,
  DEDISP_UNSUPPORTED_OUT_NBITS,
  DEDISP_INVALID_DEVICE_INDEX,
  DEDISP_DEVICE_ALREADY_SET,
  DEDISP_PRIOR_GPU_ERROR,
  DEDISP_INTERNAL_GPU_ERROR,
  DEDISP_UNKNOWN_ERROR
} dedisp_error;

/* Execution flags.  The reference passes only DEDISP_USE_DEFAULT (= host
 * pointers, synchronous).  DEDISP_DEVICE_POINTERS is an addition of this
 * library: `in` and `out` are device pointers on the current device. */
enum {
  DEDISP_USE_DEFAULT     = 0,
  DEDISP_HOST_POINTERS   = 1 << 1,
  DEDISP_DEVICE_POINTERS = 1 << 2
};

/* Plan: channel count, sampling time [s], frequency of channel 0 [MHz] and
 * channel width [MHz] (negative: channel 0 is the highest frequency).
 * pipeline.cu:171-173, clean_filterbank_rfi.cu:364 */
dedisp_error dedisp_create_plan(dedisp_plan* plan, dedisp_size nchans,
                                dedisp_float dt, dedisp_float f0, dedisp_float df);
void         dedisp_destroy_plan(dedisp_plan plan);

/* DM trials.  pipeline.cu:178-182, clean_filterbank_rfi.cu:373 */
dedisp_error dedisp_set_dm_list(dedisp_plan plan, const dedisp_float* dm_list,
                                dedisp_size count);
/* Trials spaced so the total smearing grows by at most `tol` per step, for an
 * intrinsic pulse width `ti` in microseconds.  pipeline.cu:178-182 */
dedisp_error dedisp_generate_dm_list(dedisp_plan plan, dedisp_float dm_start,
                                     dedisp_float dm_end, dedisp_float ti,
                                     dedisp_float tol);
/* Plan-free form; the returned list stays valid until the next call from the
 * same thread.  Applications/generate_dmlist.C:93-101 */
const dedisp_float* dedisp_generate_dm_list_guru(dedisp_float dm_start, dedisp_float dm_end,
                                                 double dt, double ti, double f0,
                                                 double df, dedisp_size nchans,
                                                 double tol, dedisp_size* dm_count);

/* Channel killmask: nchans ints, 0 = channel excluded.  pipeline.cu:363 */
dedisp_error dedisp_set_killmask(dedisp_plan plan, const dedisp_bool* killmask);

/* Adaptive time resolution (per-DM power-of-two scrunch, rule above);
 * tol must exceed 1.  The factors follow later changes of the DM list.
 * pipeline.cu:190, clean_filterbank_rfi.cu:369 */
dedisp_error dedisp_enable_adaptive_dt(dedisp_plan plan, dedisp_float pulse_width,
                                       dedisp_float tol);
dedisp_error dedisp_disable_adaptive_dt(dedisp_plan plan);

/* Getters.  pipeline.cu:335-345,365,493; clean_filterbank_rfi.cu:285,361-362 */
dedisp_size         dedisp_get_dm_count(const dedisp_plan plan);
const dedisp_float* dedisp_get_dm_list(const dedisp_plan plan);
const dedisp_size*  dedisp_get_dt_factors(const dedisp_plan plan);
dedisp_size         dedisp_get_max_delay(const dedisp_plan plan);
dedisp_size         dedisp_get_dm_delay(const dedisp_plan plan, int dm_trial);
dedisp_size         dedisp_get_channel_count(const dedisp_plan plan);
dedisp_float        dedisp_get_dt(const dedisp_plan plan);
dedisp_float        dedisp_get_f0(const dedisp_plan plan);
dedisp_float        dedisp_get_df(const dedisp_plan plan);

/* Brute-force dedispersion of nsamps spectra of `in` (in_stride = nchans *
 * in_nbits / 8 bytes apart, in_nbits = 1, 2, 4, 8 or 16 per channel, packed as
 * hd_execute documents) into dm_count series of nsamps - max_delay samples
 * (out_stride bytes apart, out_nbits per sample; 32 = float, the only output
 * width).  Sums are exact integers written as float (rounded once); 16-bit
 * samples are summed as low and high bytes, lo + 256 hi, and take no adaptive
 * dt (DEDISP_UNSUPPORTED_IN_NBITS).  Input in device memory
 * (DEDISP_DEVICE_POINTERS) must be 4-byte aligned (DEDISP_INVALID_POINTER).
 * pipeline.cu:459-462, clean_filterbank_rfi.cu:389-393 */
dedisp_error dedisp_execute_adv(const dedisp_plan plan, dedisp_size nsamps,
                                const dedisp_byte* in, dedisp_size in_nbits,
                                dedisp_size in_stride, dedisp_byte* out,
                                dedisp_size out_nbits, dedisp_size out_stride,
                                unsigned flags);
dedisp_error dedisp_execute(const dedisp_plan plan, dedisp_size nsamps,
                            const dedisp_byte* in, dedisp_size in_nbits,
                            dedisp_byte* out, dedisp_size out_nbits,
                            unsigned flags);

const char* dedisp_get_error_string(dedisp_error error);

#ifdef __cplusplus
}
#endif

#endif /* HEIMDALL_B200_DEDISP_H */
