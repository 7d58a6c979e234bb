/* ref_driver.cpp -- runs the reference's own hd_* pipeline (Pipeline/*.cu,
 * built on Thrust's OpenMP backend against oracle/dedisp_cpu.c) on one gulp
 * and writes its .cand file.  TEST INFRASTRUCTURE ONLY: the CPU reference arm
 * of bench.py and the parity tests call it through ctypes. */
#include <chrono>
#include <cstring>
#include <omp.h>

#include "hd/pipeline.h"
#include "hd/default_params.h"
#include "oracle.h"

static int run(const or_params* p, const unsigned char* fb, size_t nsamps, size_t nbits,
               size_t first_idx, size_t nbeams, const char* output_dir,
               size_t* nsamps_processed, double* seconds) {
  hd_params hp;
  hd_set_default_params(&hp);
  hp.verbosity = 0;
  hp.nchans = p->nchans;
  hp.dt = p->dt;
  hp.f0 = p->f0;
  hp.df = p->df;
  hp.dm_min = p->dm_min;
  hp.dm_max = p->dm_max;
  hp.dm_tol = p->dm_tol;
  hp.dm_pulse_width = p->dm_pulse_width;
  hp.baseline_length = p->baseline_length;
  hp.rfi_tol = p->rfi_tol;
  hp.boxcar_max = p->boxcar_max;
  hp.detect_thresh = p->detect_thresh;
  hp.cand_sep_time = p->cand_sep_time;
  hp.cand_sep_filter = p->cand_sep_filter;
  hp.cand_sep_dm = p->cand_sep_dm;
  hp.max_giant_rate = p->max_giant_rate;
  hp.min_tscrunch_width = p->min_tscrunch_width;
  hp.use_scrunching = p->use_scrunching != 0;
  hp.scrunch_tol = p->scrunch_tol;
  hp.output_dir = output_dir;
  hp.utc_start = 0;
  hp.spectra_per_second = (hd_size)(1.0 / p->dt + 0.5);
  hd_range_t zaps[64];
  hp.num_channel_zaps = p->num_channel_zaps < 64 ? p->num_channel_zaps : 64;
  for (unsigned z = 0; z < hp.num_channel_zaps; z++) {
    zaps[z].start = p->channel_zaps[2 * z];
    zaps[z].end = p->channel_zaps[2 * z + 1];
  }
  hp.channel_zaps = zaps;
  hd_pipeline pl;
  hd_error e = hd_create_pipeline(&pl, hp);
  if (e != HD_NO_ERROR) return e;
  hd_preallocate(pl, nsamps, nbeams);
  auto t0 = std::chrono::steady_clock::now();
  e = hd_execute(pl, fb, nsamps, nbits, first_idx, nbeams, nsamps_processed);
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  hd_destroy_pipeline(pl);
  return e;
}

/* The thread count applies to this call only: the process's OpenMP default
 * is put back, so later OpenMP work in the process keeps every thread. */
extern "C" int ref_execute(const or_params* p, const unsigned char* fb, size_t nsamps,
                           size_t nbits, size_t first_idx, size_t nbeams,
                           const char* output_dir, size_t* nsamps_processed,
                           double* seconds, int nthreads) {
  const int prev = omp_get_max_threads();
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const int e = run(p, fb, nsamps, nbits, first_idx, nbeams, output_dir, nsamps_processed,
                    seconds);
  omp_set_num_threads(prev);
  return e;
}
