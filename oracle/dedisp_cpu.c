/*
 * dedisp_cpu.c -- CPU implementation of include/dedisp.h on top of the
 * oracle's restatement.
 *
 * TEST INFRASTRUCTURE ONLY.  It exists so the reference's own stage code
 * (Pipeline/*.cu rebuilt on Thrust's OpenMP backend, oracle/Makefile target
 * `ref`) can link against a dedisp library: the reference tree does not ship
 * one (config/dedisp.m4).  The product implements the same interface in
 * heimdall_multibeam_b200/csrc with sm_100a kernels.
 */
#include <omp.h>
#include "dedisp.h"
#include "oracle.h"

#include <stdint.h>
#include <stdlib.h>
#include <string.h>

struct dedisp_plan_struct {
  dedisp_size  nchans;
  dedisp_float dt, f0, df;
  float*       table;
  float*       dm_list;
  dedisp_size  dm_count;
  int*         killmask;
  dedisp_size* dt_factors;
  int          adaptive;
  double       adaptive_width, adaptive_tol;
};

dedisp_error dedisp_create_plan(dedisp_plan* plan, dedisp_size nchans, dedisp_float dt,
                                dedisp_float f0, dedisp_float df) {
  if (!plan) return DEDISP_INVALID_POINTER;
  struct dedisp_plan_struct* p = (struct dedisp_plan_struct*)calloc(1, sizeof(*p));
  if (!p) return DEDISP_MEM_ALLOC_FAILED;
  p->nchans = nchans; p->dt = dt; p->f0 = f0; p->df = df;
  p->table = (float*)malloc(nchans * sizeof(float));
  p->killmask = (int*)malloc(nchans * sizeof(int));
  for (dedisp_size c = 0; c < nchans; c++) p->killmask[c] = 1;
  or_delay_table(nchans, dt, f0, df, p->table);
  *plan = p;
  return DEDISP_NO_ERROR;
}

void dedisp_destroy_plan(dedisp_plan p) {
  if (!p) return;
  free(p->table); free(p->dm_list); free(p->killmask); free(p->dt_factors); free(p);
}

static void set_list(dedisp_plan p, const float* l, dedisp_size n) {
  free(p->dm_list); free(p->dt_factors);
  p->dm_list = (float*)malloc((n + 1) * sizeof(float));
  memcpy(p->dm_list, l, n * sizeof(float));
  p->dm_count = n;
  p->dt_factors = (dedisp_size*)malloc((n + 1) * sizeof(dedisp_size));
  for (dedisp_size i = 0; i < n; i++) p->dt_factors[i] = 1;
  if (p->adaptive)
    or_scrunch_factors(p->dm_list, n, p->dt, p->adaptive_width, p->f0, p->df, p->nchans,
                       p->adaptive_tol, (size_t*)p->dt_factors);
}

dedisp_error dedisp_set_dm_list(dedisp_plan p, const dedisp_float* l, dedisp_size n) {
  if (!p || !l) return DEDISP_INVALID_POINTER;
  set_list(p, l, n);
  return DEDISP_NO_ERROR;
}

dedisp_error dedisp_generate_dm_list(dedisp_plan p, dedisp_float a, dedisp_float b,
                                     dedisp_float ti, dedisp_float tol) {
  if (!p) return DEDISP_INVALID_PLAN;
  size_t n = or_generate_dm_list(a, b, p->dt, ti, p->f0, p->df, p->nchans, tol, NULL, 0);
  float* l = (float*)malloc((n + 1) * sizeof(float));
  or_generate_dm_list(a, b, p->dt, ti, p->f0, p->df, p->nchans, tol, l, n);
  set_list(p, l, n);
  free(l);
  return DEDISP_NO_ERROR;
}

static __thread float* g_guru = NULL;
const dedisp_float* dedisp_generate_dm_list_guru(dedisp_float a, dedisp_float b, double dt,
                                                 double ti, double f0, double df,
                                                 dedisp_size nchans, double tol,
                                                 dedisp_size* count) {
  size_t n = or_generate_dm_list(a, b, dt, ti, f0, df, nchans, tol, NULL, 0);
  free(g_guru);
  g_guru = (float*)malloc((n + 1) * sizeof(float));
  or_generate_dm_list(a, b, dt, ti, f0, df, nchans, tol, g_guru, n);
  if (count) *count = n;
  return g_guru;
}

dedisp_error dedisp_set_killmask(dedisp_plan p, const dedisp_bool* km) {
  if (!p) return DEDISP_INVALID_PLAN;
  for (dedisp_size c = 0; c < p->nchans; c++) p->killmask[c] = km ? km[c] : 1;
  return DEDISP_NO_ERROR;
}

/* Adaptive dt: the per-trial scrunch factors of the oracle's restated rule
 * (or_scrunch_factors), recomputed whenever the DM list changes; execution
 * then dedisperses each trial at its factor (or_dedisperse_scrunched). */
dedisp_error dedisp_enable_adaptive_dt(dedisp_plan p, dedisp_float w, dedisp_float tol) {
  if (!p) return DEDISP_INVALID_PLAN;
  p->adaptive = 1;
  p->adaptive_width = w;
  p->adaptive_tol = tol;
  if (p->dm_count)
    or_scrunch_factors(p->dm_list, p->dm_count, p->dt, w, p->f0, p->df, p->nchans, tol,
                       (size_t*)p->dt_factors);
  return DEDISP_NO_ERROR;
}
dedisp_error dedisp_disable_adaptive_dt(dedisp_plan p) {
  if (!p) return DEDISP_INVALID_PLAN;
  p->adaptive = 0;
  for (dedisp_size i = 0; i < p->dm_count; i++) p->dt_factors[i] = 1;
  return DEDISP_NO_ERROR;
}

dedisp_size dedisp_get_dm_count(const dedisp_plan p) { return p->dm_count; }
const dedisp_float* dedisp_get_dm_list(const dedisp_plan p) { return p->dm_list; }
const dedisp_size* dedisp_get_dt_factors(const dedisp_plan p) { return p->dt_factors; }
dedisp_size dedisp_get_max_delay(const dedisp_plan p) {
  return or_max_delay(p->dm_list, p->dm_count, p->table, p->nchans);
}
dedisp_size dedisp_get_dm_delay(const dedisp_plan p, int d) {
  return or_max_delay(p->dm_list + d, 1, p->table, p->nchans);
}
dedisp_size dedisp_get_channel_count(const dedisp_plan p) { return p->nchans; }
dedisp_float dedisp_get_dt(const dedisp_plan p) { return p->dt; }
dedisp_float dedisp_get_f0(const dedisp_plan p) { return p->f0; }
dedisp_float dedisp_get_df(const dedisp_plan p) { return p->df; }

/* Threads of the brute-force dedisperser (0: every host core).  A caller that
 * runs several pipelines in parallel processes gives each its share. */
static int g_dedisp_threads = 0;
void dedisp_cpu_set_threads(int n) { g_dedisp_threads = n; }

dedisp_error dedisp_execute_adv(const dedisp_plan p, dedisp_size nsamps, const dedisp_byte* in,
                                dedisp_size in_nbits, dedisp_size in_stride, dedisp_byte* out,
                                dedisp_size out_nbits, dedisp_size out_stride, unsigned flags) {
  (void)flags;
  if (!p) return DEDISP_INVALID_PLAN;
  if (!in || !out) return DEDISP_INVALID_POINTER;
  if (!p->dm_count) return DEDISP_NO_DM_LIST_SET;
  if (in_nbits != 1 && in_nbits != 2 && in_nbits != 4 && in_nbits != 8 && in_nbits != 16)
    return DEDISP_UNSUPPORTED_IN_NBITS;
  if (in_nbits == 16 && p->adaptive) return DEDISP_UNSUPPORTED_IN_NBITS;
  if (out_nbits != 32) return DEDISP_UNSUPPORTED_OUT_NBITS;
  if (out_stride % 4) return DEDISP_INVALID_STRIDE;
  if ((p->nchans * in_nbits) % 32) return DEDISP_INVALID_STRIDE;
  size_t md = dedisp_get_max_delay(p);
  if (nsamps < md) return DEDISP_TOO_FEW_NSAMPS;
  /* every host core unless dedisp_cpu_set_threads() says otherwise, whatever
   * thread count the caller set for the stage code: the integer sums do not
   * depend on it */
  const int threads = g_dedisp_threads > 0 ? g_dedisp_threads : omp_get_num_procs();
  const size_t* factors = p->adaptive ? (const size_t*)p->dt_factors : NULL;
  if (in_nbits == 8) {
    or_dedisperse_scrunched(in, nsamps, in_stride, p->nchans, p->killmask, p->dm_list,
                            p->dm_count, p->table, factors, (float*)out, out_stride / 4, threads);
    return DEDISP_NO_ERROR;
  }
  /* packed samples: channel c of spectrum t is the in_nbits-bit field at bit
   * (c mod (32 / in_nbits)) * in_nbits of the little-endian 32-bit word
   * c / (32 / in_nbits) (the reference's writer, Formats/giant_maker.C:385-392).
   * Values below 256 are summed as bytes; 16-bit values as their low and high
   * bytes, sum = sum(lo) + 256 sum(hi), exact in integers. */
  const size_t C = p->nchans, cpw = 32 / in_nbits, mask = (in_nbits == 16) ? 0xFFFFu
                                                        : ((1u << in_nbits) - 1u);
  const int planes = in_nbits == 16 ? 2 : 1;
  unsigned char* u = (unsigned char*)malloc((size_t)planes * nsamps * C);
  if (!u) return DEDISP_MEM_ALLOC_FAILED;
  for (size_t t = 0; t < nsamps; t++) {
    const unsigned char* row = in + t * in_stride;
    for (size_t c = 0; c < C; c++) {
      const size_t w = c / cpw, k = c % cpw;
      const uint32_t word = (uint32_t)row[4 * w] | ((uint32_t)row[4 * w + 1] << 8) |
                            ((uint32_t)row[4 * w + 2] << 16) | ((uint32_t)row[4 * w + 3] << 24);
      const uint32_t v = (word >> (k * in_nbits)) & mask;
      u[t * C + c] = (unsigned char)(v & 0xFFu);
      if (planes == 2) u[nsamps * C + t * C + c] = (unsigned char)(v >> 8);
    }
  }
  float* o = (float*)out;
  const size_t opitch = out_stride / 4, nout = nsamps - md;
  or_dedisperse_scrunched(u, nsamps, C, C, p->killmask, p->dm_list, p->dm_count, p->table,
                          factors, o, opitch, threads);
  if (planes == 2) {
    float* hi = (float*)malloc(opitch * p->dm_count * sizeof(float));
    if (!hi) {
      free(u);
      return DEDISP_MEM_ALLOC_FAILED;
    }
    or_dedisperse_scrunched(u + nsamps * C, nsamps, C, C, p->killmask, p->dm_list,
                            p->dm_count, p->table, NULL, hi, opitch, threads);
    for (size_t d = 0; d < p->dm_count; d++)
      for (size_t t = 0; t < nout; t++) {
        const uint32_t v = (uint32_t)o[d * opitch + t] + 256u * (uint32_t)hi[d * opitch + t];
        o[d * opitch + t] = (float)v;
      }
    free(hi);
  }
  free(u);
  return DEDISP_NO_ERROR;
}

dedisp_error dedisp_execute(const dedisp_plan p, dedisp_size nsamps, const dedisp_byte* in,
                            dedisp_size in_nbits, dedisp_byte* out, dedisp_size out_nbits,
                            unsigned flags) {
  if (!p) return DEDISP_INVALID_PLAN;
  size_t md = dedisp_get_max_delay(p);
  if (nsamps < md) return DEDISP_TOO_FEW_NSAMPS;
  return dedisp_execute_adv(p, nsamps, in, in_nbits, p->nchans * in_nbits / 8, out, out_nbits,
                            (nsamps - md) * out_nbits / 8, flags);
}

const char* dedisp_get_error_string(dedisp_error e) {
  switch (e) {
    case DEDISP_NO_ERROR: return "No error";
    case DEDISP_MEM_ALLOC_FAILED: return "Memory allocation failed";
    case DEDISP_INVALID_PLAN: return "Invalid plan";
    case DEDISP_INVALID_POINTER: return "Invalid pointer";
    case DEDISP_INVALID_STRIDE: return "Invalid stride";
    case DEDISP_NO_DM_LIST_SET: return "No DM list has been set";
    case DEDISP_TOO_FEW_NSAMPS: return "No. samples < maximum delay";
    case DEDISP_INVALID_FLAG_COMBINATION: return "Invalid flag combination";
    case DEDISP_UNSUPPORTED_IN_NBITS: return "Unsupported in_nbits value";
    case DEDISP_UNSUPPORTED_OUT_NBITS: return "Unsupported out_nbits value";
    default: return "Unknown error";
  }
}
