// plan.h -- host-side dedispersion plan shared by the dedisp_* C interface and
// the hd_* pipeline.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "dedisp.h"

struct dedisp_plan_struct {
  dedisp_size nchans = 0;
  float dt = 0.f, f0 = 0.f, df = 0.f;
  std::vector<float> table;       // delay per unit DM per channel (samples)
  std::vector<float> dm_list;
  std::vector<int> killmask;
  std::vector<dedisp_size> dt_factors;
  bool adaptive = false;
  float adaptive_width = 0.f, adaptive_tol = 0.f;

  // derived / device state (rebuilt lazily when the list or killmask change)
  bool dirty = true;
  unsigned long long gen = 0;      // counts the rebuilds of the device tables
  std::vector<int> delays;         // [dm][chan]
  // per DM-block size (8, 16, 32 trials): [dm block][chan] minimum delay
  std::vector<int> blk_min[3];
  std::vector<int> active;         // channels with killmask != 0
  size_t max_delay = 0;
  size_t max_span[3] = {0, 0, 0};  // max over blocks/chans of (max - min) delay
  int* d_delays = nullptr;
  int* d_blk_min[3] = {nullptr, nullptr, nullptr};
  // dedispersion tile {dm_block, time_block, rows, source} per (nsamps,
  // units, scrunch group): the fastest of the candidates, timed on first use
  // (autotuner) or read from the persistent tile cache
  std::map<std::array<size_t, 3>, std::array<int, 4>> tiles;
  std::array<int, 3> last_tile = {16, 512, 8};
  // where last_tile came from (hd_get_dedisp_tile_source): 0 default,
  // 1 forced (HDB_DEDISP_TILE), 2 timed by the autotuner in this process,
  // 3 the persistent tile cache (HDB_TUNE_CACHE)
  int last_tile_source = 0;
  bool tune = true;
  int forced_dm_block = 0, forced_time_block = 0;  // HDB_DEDISP_TILE="DBxTB"
  int* d_active = nullptr;
  float* d_dm_list = nullptr;
  unsigned* d_err = nullptr;
  int device = -1;

  // adaptive dt: trials [d0, d1) share scrunch factor s and are dedispersed
  // at sampling time s dt from the scrunched input with delays delay / s
  // (one group of factor 1 over all trials when adaptive dt is off)
  struct Group {
    size_t d0 = 0, d1 = 0, s = 1;
    size_t max_delay = 0;            // largest scrunched delay of the group
    size_t max_span[3] = {0, 0, 0};  // per DM-block size
    std::vector<int> delays;         // [d1 - d0][chan]
    std::vector<int> blk_min[3];
    int* d_delays = nullptr;
    int* d_blk_min[3] = {nullptr, nullptr, nullptr};
  };
  std::vector<Group> groups;          // built only with adaptive dt
  uint8_t* d_scr = nullptr;           // scrunched channel-major input
  size_t d_scr_cap = 0;

  // scratch for dedisp_execute* with host pointers
  uint8_t* d_in_tf = nullptr;
  size_t d_in_tf_cap = 0;
  uint8_t* d_in_ft = nullptr;
  size_t d_in_ft_cap = 0;
  float* d_out = nullptr;
  size_t d_out_cap = 0;
  float* d_out_hi = nullptr;  // high-byte plane sums of 16-bit input
  size_t d_out_hi_cap = 0;
  cudaStream_t stream = nullptr;

  ~dedisp_plan_struct();
};

namespace hdb {

// include/dedisp.h restatement (float arithmetic as documented there).
void delay_table(size_t nchans, float dt, float f0, float df, float* table);
// Per-trial scrunch factors of adaptive dt (include/dedisp.h documents the
// rule).
std::vector<dedisp_size> scrunch_factors(const std::vector<float>& dm_list, double dt,
                                         double ti, double f0, double df, size_t nchans,
                                         double tol);
size_t delay_of(float dm, float table_c);
std::vector<float> generate_dm_list(float dm_start, float dm_end, double dt, double ti,
                                    double f0, double df, size_t nchans, double tol);

// Recomputes delays, block minima, active channels and uploads them.
dedisp_error plan_prepare(dedisp_plan p);

// Pitch (bytes) of the channel-major working copy for nsamps samples.
size_t ft_pitch(const dedisp_plan p, size_t nsamps);

// Dedisperses the FT copy already on the device into out (device floats).
// With units > 1, one launch dedisperses `units` filterbanks that lie
// in_unit bytes (inputs) and out_unit floats (outputs) apart.
dedisp_error plan_dedisperse_ft(dedisp_plan p, const uint8_t* d_ft, size_t pitch, size_t nsamps,
                                float* d_out, size_t out_pitch, cudaStream_t s, size_t units = 1,
                                size_t in_unit = 0, size_t out_unit = 0);

}  // namespace hdb
