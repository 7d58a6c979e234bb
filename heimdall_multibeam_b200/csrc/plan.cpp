// plan.cpp -- the dedisp_* C interface (include/dedisp.h) on sm_100a kernels.
//
// Plan semantics follow the reference's call sites (Pipeline/pipeline.cu:
// 171-196,335-365,453-462,493; clean_filterbank_rfi.cu:361-397) with the
// documented restatement of the external dedisp library: float delay table
// with K = 4148.808, delays rounded half up, exact integer channel sums
// written as float.
#include "plan.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>

#include <sys/stat.h>

#include "internal.h"

namespace hdb {

void delay_table(size_t nchans, float dt, float f0, float df, float* table) {
  const float K = 4148.808f;
  float b = 1.0f / f0;
  for (size_t c = 0; c < nchans; c++) {
    float fc = f0 + (float)c * df;
    float a = 1.0f / fc;
    table[c] = K * (a * a - b * b) / dt;
  }
}

size_t delay_of(float dm, float table_c) {
  float v = dm * table_c + 0.5f;
  if (!(v > 0.0f)) return 0;
  return (size_t)v;
}

// DM trial spacing for a smearing tolerance (dedisp's generator, golden
// vector Share/dm2000.list).  With times in microseconds, trial p has width
//   W(p)^2 = dt^2 + ti^2 + (a p)^2,  a = 8.3 df / f^3 (df MHz, f GHz, band
// centre); the next trial x satisfies
//   dt^2 + ti^2 + (a x)^2 + b^2 (x - p)^2 = tol^2 W(p)^2,  b = a nchans / 4,
// whose positive root is taken.  Trials are stored as float and the stored
// value seeds the next step; generation stops at the first trial >= dm_end.
std::vector<float> generate_dm_list(float dm_start, float dm_end, double dt, double ti,
                                    double f0, double df, size_t nchans, double tol) {
  double dt_us = dt * 1e6;
  double f = (f0 + ((double)(nchans / 2) - 0.5) * df) * 1e-3;
  double tol2 = tol * tol;
  double a = 8.3 * df / (f * f * f);
  double a2 = a * a;
  double b2 = a2 * ((double)(nchans * nchans) / 16.0);
  double c = (dt_us * dt_us + ti * ti) * (tol2 - 1.0);
  std::vector<float> out;
  out.push_back(dm_start);
  while (out.back() < dm_end && out.size() < (1u << 20)) {
    double p = (double)out.back();
    double k = c + tol2 * a2 * p * p;
    double x = (b2 * p + std::sqrt(-a2 * b2 * p * p + (a2 + b2) * k)) / (a2 + b2);
    out.push_back((float)x);
  }
  return out;
}

// Adaptive dt (dedisp_enable_adaptive_dt; the rule of Barsdell et al. 2012,
// MNRAS 422, 379, restated): the smearing of trial DM at sampling time T is
// the generator's model W(DM, T)^2 = T^2 + ti^2 + (a DM)^2 (microseconds,
// same a and band centre); factors start at 1, never decrease, and trial d
// takes twice the previous factor s when W(DM_d, 2 s dt) / W(DM_d, s dt) <
// tol.  Double precision throughout.
std::vector<dedisp_size> scrunch_factors(const std::vector<float>& dm_list, double dt,
                                         double ti, double f0, double df, size_t nchans,
                                         double tol) {
  const double dt_us = dt * 1e6;
  const double f = (f0 + ((double)(nchans / 2) - 0.5) * df) * 1e-3;
  const double a = 8.3 * df / (f * f * f);
  std::vector<dedisp_size> out(dm_list.size(), 1);
  dedisp_size s = 1;
  for (size_t d = 1; d < dm_list.size(); d++) {
    const double sm = a * (double)dm_list[d];
    const double t1 = (double)s * dt_us, t2 = 2.0 * (double)s * dt_us;
    const double w1 = std::sqrt(t1 * t1 + ti * ti + sm * sm);
    const double w2 = std::sqrt(t2 * t2 + ti * ti + sm * sm);
    if (w2 / w1 < tol) s *= 2;
    out[d] = s;
  }
  return out;
}

static void free_dev(void* p) {
  if (p) cudaFree(p);
}

static void free_groups(dedisp_plan p) {
  for (auto& g : p->groups) {
    free_dev(g.d_delays);
    for (int* b : g.d_blk_min) free_dev(b);
  }
  p->groups.clear();
}

// Trials of one scrunch factor: delays at that factor, per DM-block minima
// and spans, uploaded.
static dedisp_error build_groups(dedisp_plan p) {
  free_groups(p);
  if (!p->adaptive) return DEDISP_NO_ERROR;
  const size_t D = p->dm_list.size(), C = p->nchans;
  size_t d = 0;
  while (d < D) {
    dedisp_plan_struct::Group g;
    g.d0 = d;
    g.s = p->dt_factors[d];
    while (d < D && p->dt_factors[d] == g.s) d++;
    g.d1 = d;
    const size_t Dg = g.d1 - g.d0;
    g.delays.resize(Dg * C);
    for (size_t i = 0; i < Dg; i++)
      for (size_t c = 0; c < C; c++) {
        const int v = p->delays[(g.d0 + i) * C + c] / (int)g.s;
        g.delays[i * C + c] = v;
        g.max_delay = std::max(g.max_delay, (size_t)v);
      }
    for (int k = 0; k < 3; k++) {
      const size_t DB = (size_t)kDedispDmBlocks[k];
      const size_t nblk = (Dg + DB - 1) / DB;
      g.blk_min[k].assign(nblk * C, 0);
      for (size_t b = 0; b < nblk; b++)
        for (size_t c = 0; c < C; c++) {
          int lo = 0x7FFFFFFF, hi = 0;
          for (size_t i = b * DB; i < std::min(Dg, (b + 1) * DB); i++) {
            lo = std::min(lo, g.delays[i * C + c]);
            hi = std::max(hi, g.delays[i * C + c]);
          }
          g.blk_min[k][b * C + c] = lo;
          g.max_span[k] = std::max(g.max_span[k], (size_t)(hi - lo));
        }
    }
    p->groups.push_back(std::move(g));
    dedisp_plan_struct::Group& G = p->groups.back();
    if (dev_malloc(&G.d_delays, G.delays.size() * sizeof(int)) != cudaSuccess)
      return DEDISP_MEM_ALLOC_FAILED;
    if (cudaMemcpy(G.d_delays, G.delays.data(), G.delays.size() * sizeof(int),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return DEDISP_MEM_COPY_FAILED;
    for (int k = 0; k < 3; k++) {
      if (dev_malloc(&G.d_blk_min[k], G.blk_min[k].size() * sizeof(int)) != cudaSuccess)
        return DEDISP_MEM_ALLOC_FAILED;
      if (cudaMemcpy(G.d_blk_min[k], G.blk_min[k].data(), G.blk_min[k].size() * sizeof(int),
                     cudaMemcpyHostToDevice) != cudaSuccess)
        return DEDISP_MEM_COPY_FAILED;
    }
  }
  return DEDISP_NO_ERROR;
}

dedisp_error plan_prepare(dedisp_plan p) {
  if (!p->dirty) return DEDISP_NO_ERROR;
  if (p->dm_list.empty()) return DEDISP_NO_DM_LIST_SET;
  const size_t D = p->dm_list.size(), C = p->nchans;
  p->delays.assign(D * C, 0);
  p->max_delay = 0;
  for (size_t d = 0; d < D; d++)
    for (size_t c = 0; c < C; c++) {
      size_t v = delay_of(p->dm_list[d], p->table[c]);
      if (v > (size_t)0x3FFFFFFF) return DEDISP_TOO_FEW_NSAMPS;
      p->delays[d * C + c] = (int)v;
      p->max_delay = std::max(p->max_delay, v);
    }
  for (int k = 0; k < 3; k++) {
    const size_t DB = (size_t)kDedispDmBlocks[k];
    const size_t nblk = (D + DB - 1) / DB;
    p->blk_min[k].assign(nblk * C, 0);
    p->max_span[k] = 0;
    for (size_t b = 0; b < nblk; b++)
      for (size_t c = 0; c < C; c++) {
        int lo = 0x7FFFFFFF, hi = 0;
        for (size_t d = b * DB; d < std::min(D, (b + 1) * DB); d++) {
          lo = std::min(lo, p->delays[d * C + c]);
          hi = std::max(hi, p->delays[d * C + c]);
        }
        p->blk_min[k][b * C + c] = lo;
        p->max_span[k] = std::max(p->max_span[k], (size_t)(hi - lo));
      }
  }
  p->active.clear();
  for (size_t c = 0; c < C; c++)
    if (p->killmask[c]) p->active.push_back((int)c);
  p->tiles.clear();
  int dev = 0;
  cudaGetDevice(&dev);
  free_dev(p->d_delays); free_dev(p->d_active); free_dev(p->d_dm_list);
  p->d_delays = nullptr; p->d_active = nullptr; p->d_dm_list = nullptr;
  for (auto& b : p->d_blk_min) {
    free_dev(b);
    b = nullptr;
  }
  if (hdb::dev_malloc(&p->d_delays, p->delays.size() * sizeof(int)) != cudaSuccess ||
      hdb::dev_malloc(&p->d_active, (p->active.size() + 1) * sizeof(int)) != cudaSuccess ||
      hdb::dev_malloc(&p->d_dm_list, D * sizeof(float)) != cudaSuccess)
    return DEDISP_MEM_ALLOC_FAILED;
  for (int k = 0; k < 3; k++)
    if (hdb::dev_malloc(&p->d_blk_min[k], p->blk_min[k].size() * sizeof(int)) != cudaSuccess)
      return DEDISP_MEM_ALLOC_FAILED;
  if (!p->d_err && hdb::dev_malloc(&p->d_err, sizeof(unsigned)) != cudaSuccess)
    return DEDISP_MEM_ALLOC_FAILED;
  cudaMemset(p->d_err, 0, sizeof(unsigned));
  if (cudaMemcpy(p->d_delays, p->delays.data(), p->delays.size() * sizeof(int),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      (!p->active.empty() &&
       cudaMemcpy(p->d_active, p->active.data(), p->active.size() * sizeof(int),
                  cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemcpy(p->d_dm_list, p->dm_list.data(), D * sizeof(float), cudaMemcpyHostToDevice) !=
          cudaSuccess)
    return DEDISP_MEM_COPY_FAILED;
  for (int k = 0; k < 3; k++)
    if (cudaMemcpy(p->d_blk_min[k], p->blk_min[k].data(), p->blk_min[k].size() * sizeof(int),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return DEDISP_MEM_COPY_FAILED;
  dedisp_error ge = build_groups(p);
  if (ge != DEDISP_NO_ERROR) return ge;
  p->device = dev;
  p->dirty = false;
  p->gen++;
  return DEDISP_NO_ERROR;
}

static int dm_block_index(int dm_block) {
  for (int k = 0; k < 3; k++)
    if (kDedispDmBlocks[k] == dm_block) return k;
  return -1;
}

// Staged row bytes of a tile: the DM block's delay span for one channel, the
// time block, the 16-byte alignment of the copy and one word of look-ahead.
static int rowb_of(const size_t* max_span, int dm_block, int time_block) {
  size_t r = max_span[dm_block_index(dm_block)] + 16 + (size_t)time_block + 8;
  return (int)((r + 15) & ~(size_t)15);
}

// Row pitch of a channel-major input of nsamps samples whose trials reach
// max_delay and produce nout samples: room for the longest staged row of
// every candidate tile past the last time block.
static size_t ft_pitch_for(const size_t* max_span, size_t max_delay, size_t nsamps,
                           size_t nout) {
  size_t need = nsamps + 4;
  for (const auto& t : kDedispTiles) {
    const size_t tb = (size_t)t[1];
    const size_t ntb = (nout + tb - 1) / tb;
    need = std::max(need, ntb * tb + max_delay + (size_t)rowb_of(max_span, t[0], t[1]));
  }
  need += 64;
  return (need + 63) & ~(size_t)63;
}

size_t ft_pitch(const dedisp_plan p, size_t nsamps) {
  size_t nout = nsamps > p->max_delay ? nsamps - p->max_delay : 0;
  return ft_pitch_for(p->max_span, p->max_delay, nsamps, nout);
}

// ---------------------------------------------------------------------------
// Persistent tile cache.  The autotuner's choice is kept across processes in
// a text file, one line per tuned shape: "<key, 16 hex digits> <dm_block>
// <time_block> <rows>".  The key is a 64-bit FNV-1a hash of everything the
// kernel's speed depends on: the kernel generation, the device (name, SM
// count), the input and output lengths, the unit count and the trial-by-
// channel delay table of the launch (which fixes the DM list, the sampling
// time, the band and the active channels).  The file is HDB_TUNE_CACHE, else
// $XDG_CACHE_HOME/heimdall_b200/dedisp_tiles.txt, else
// $HOME/.cache/heimdall_b200/dedisp_tiles.txt; HDB_TUNE_CACHE=0 (or empty)
// turns the cache off.  Entries naming a tile that no longer fits are
// ignored and the shape is timed again.
// ---------------------------------------------------------------------------
namespace {
// bump when the dedispersion kernel changes, so stale choices are not reused
constexpr uint64_t kDedispKernelGeneration = 6;

struct TileCache {
  std::mutex mu;
  bool loaded = false;
  std::string path;
  std::map<uint64_t, std::array<int, 3>> entries;
};
TileCache& tile_cache() {
  static TileCache c;
  return c;
}

std::string tile_cache_path() {
  if (const char* e = std::getenv("HDB_TUNE_CACHE"))
    return (e[0] == 0 || std::strcmp(e, "0") == 0) ? std::string() : std::string(e);
  std::string base;
  if (const char* x = std::getenv("XDG_CACHE_HOME"); x && x[0]) base = x;
  else if (const char* h = std::getenv("HOME"); h && h[0]) base = std::string(h) + "/.cache";
  else return std::string();
  return base + "/heimdall_b200/dedisp_tiles.txt";
}

struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void bytes(const void* p, size_t n) {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    for (size_t i = 0; i < n; i++) h = (h ^ b[i]) * 1099511628211ull;
  }
  template <class T> void val(const T& v) { bytes(&v, sizeof v); }
};

uint64_t tile_key(const std::vector<int>& delays, const std::vector<int>& active, size_t nsamps,
                  size_t nout, size_t units) {
  Fnv f;
  f.val(kDedispKernelGeneration);
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) f.bytes(prop.name, std::strlen(prop.name));
  f.val(sms);
  f.val(nsamps);
  f.val(nout);
  f.val(units);
  const size_t n = delays.size();
  f.val(n);
  f.bytes(delays.data(), n * sizeof(int));
  const size_t na = active.size();
  f.val(na);
  f.bytes(active.data(), na * sizeof(int));
  return f.h;
}

// Looks the key up (loading the file on first use); false when absent or
// the cache is off.
bool tile_cache_get(uint64_t key, std::array<int, 3>* out) {
  TileCache& c = tile_cache();
  std::lock_guard<std::mutex> lock(c.mu);
  if (!c.loaded) {
    c.loaded = true;
    c.path = tile_cache_path();
    if (!c.path.empty())
      if (FILE* fp = std::fopen(c.path.c_str(), "r")) {
        unsigned long long k = 0;
        int a = 0, b = 0, r = 0;
        char line[128];
        while (std::fgets(line, sizeof line, fp))
          if (std::sscanf(line, "%llx %d %d %d", &k, &a, &b, &r) == 4) c.entries[k] = {a, b, r};
        std::fclose(fp);
      }
  }
  if (c.path.empty()) return false;
  auto it = c.entries.find(key);
  if (it == c.entries.end()) return false;
  *out = it->second;
  return true;
}

void tile_cache_put(uint64_t key, const std::array<int, 3>& t) {
  TileCache& c = tile_cache();
  std::lock_guard<std::mutex> lock(c.mu);
  if (c.path.empty()) return;
  c.entries[key] = t;
  // create the directory chain; a failure only means the choice is not kept
  for (size_t pos = c.path.find('/', 1); pos != std::string::npos; pos = c.path.find('/', pos + 1))
    mkdir(c.path.substr(0, pos).c_str(), 0755);
  if (FILE* fp = std::fopen(c.path.c_str(), "a")) {
    std::fprintf(fp, "%016llx %d %d %d\n", (unsigned long long)key, t[0], t[1], t[2]);
    std::fclose(fp);
  }
}
}  // namespace

// One launch set over trials whose delays are d_delays (dm_count rows; host
// copy h_delays) on a channel-major input of nsamps samples, nout output
// samples per trial; the tile is tuned per (nsamps, units, tune_key) and kept
// in the persistent tile cache.
static dedisp_error dedisperse_tables(dedisp_plan p, const std::vector<int>& h_delays,
                                      const int* d_delays, int* const* d_blk_min,
                                      const size_t* max_span, int dm_count, size_t nout,
                                      size_t tune_key, const uint8_t* d_ft, size_t pitch,
                                      size_t nsamps, float* d_out, size_t out_pitch,
                                      cudaStream_t s, size_t units, size_t in_unit,
                                      size_t out_unit) {
  if (nout == 0 || units == 0 || dm_count == 0) return DEDISP_NO_ERROR;
  if (p->active.empty()) {
    for (size_t u = 0; u < units; u++)
      if (cudaMemset2DAsync(d_out + u * out_unit, out_pitch * sizeof(float), 0,
                            nout * sizeof(float), (size_t)dm_count, s) != cudaSuccess)
        return DEDISP_INTERNAL_GPU_ERROR;
    return DEDISP_NO_ERROR;
  }
  DedispArgs a;
  a.in = d_ft;
  a.in_pitch = pitch;
  a.delays = d_delays;
  a.chans = p->d_active;
  a.nact = (int)p->active.size();
  a.nchans = (int)p->nchans;
  a.dm_count = dm_count;
  a.nout = nout;
  a.out = d_out;
  a.out_pitch = out_pitch;
  a.err = p->d_err;
  a.units = (int)units;
  a.in_unit = in_unit;
  a.out_unit = out_unit;
  a.wait_limit = kDedispWaitLimit;
  a.withhold_last = 0;
  a.one = 1;
  // error-path test (read per call so a test can clear it between gulps):
  // the last channel stage is withheld and the waits give up quickly
  if (const char* e = std::getenv("HDB_TEST_WITHHOLD_STAGE"))
    if (e[0] == '1') {
      a.withhold_last = 1;
      a.wait_limit = 1u << 12;
    }
  if (units > 65535) return DEDISP_INVALID_STRIDE;
  auto with_tile = [&](const std::array<int, 3>& t) {
    a.blk_min = d_blk_min[dm_block_index(t[0])];
    a.rowb = rowb_of(max_span, t[0], t[1]);
    return DedispTile{t[0], t[1], t[2]};
  };
  // candidate tiles whose staged rows fit shared memory
  std::vector<std::array<int, 3>> cand;
  for (const auto& t : kDedispTiles) {
    const int rows = dedisp_rows_per_stage(t[0], rowb_of(max_span, t[0], t[1]));
    if (rows) cand.push_back({t[0], t[1], rows});
  }
  // one channel row of the widest block's delay span must fit shared memory
  if (cand.empty()) return DEDISP_NCHANS_EXCEEDS_LIMIT;
  const std::array<size_t, 3> key = {nsamps, units, tune_key};
  auto it = p->tiles.find(key);
  if (it == p->tiles.end()) {
    // default: 16 DMs x 512 samples when it fits
    std::array<int, 3> best = cand[0];
    bool forced = false;
    int source = 0;
    for (const auto& t : cand)
      if (t[0] == 16 && t[1] == 512) best = t;
    for (const auto& t : cand)
      if (t[0] == p->forced_dm_block && t[1] == p->forced_time_block) {
        best = t;
        forced = true;
        source = 1;
      }
    uint64_t ckey = 0;
    bool cached = false;
    if (p->tune && !forced && cand.size() > 1) {
      ckey = tile_key(h_delays, p->active, nsamps, nout, units);
      std::array<int, 3> t;
      if (tile_cache_get(ckey, &t) && std::find(cand.begin(), cand.end(), t) != cand.end()) {
        best = t;
        cached = true;
        source = 3;
      }
    }
    if (p->tune && !forced && !cached && cand.size() > 1) {
      // autotuner: each candidate once to warm up and once timed; all give the
      // same sums, so the output of the last run stands
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      if (cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess) {
        float best_ms = 0.f;
        bool have = false;
        for (const auto& t : cand) {
          const DedispTile dt = with_tile(t);
          if (launch_dedisp(a, dt, s) != cudaSuccess) return DEDISP_INTERNAL_GPU_ERROR;
          cudaEventRecord(e0, s);
          if (launch_dedisp(a, dt, s) != cudaSuccess) return DEDISP_INTERNAL_GPU_ERROR;
          cudaEventRecord(e1, s);
          float ms = 0.f;
          if (cudaEventSynchronize(e1) != cudaSuccess ||
              cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
            return DEDISP_INTERNAL_GPU_ERROR;
          if (!have || ms < best_ms) {
            best_ms = ms;
            best = t;
            have = true;
          }
        }
      }
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
      source = 2;
      tile_cache_put(ckey, best);
    }
    it = p->tiles.emplace(key, std::array<int, 4>{best[0], best[1], best[2], source}).first;
  }
  p->last_tile = {it->second[0], it->second[1], it->second[2]};
  p->last_tile_source = it->second[3];
  if (launch_dedisp(a, with_tile(p->last_tile), s) != cudaSuccess) return DEDISP_INTERNAL_GPU_ERROR;
  return DEDISP_NO_ERROR;
}


dedisp_error plan_dedisperse_ft(dedisp_plan p, const uint8_t* d_ft, size_t pitch, size_t nsamps,
                                float* d_out, size_t out_pitch, cudaStream_t s, size_t units,
                                size_t in_unit, size_t out_unit) {
  dedisp_error de = plan_prepare(p);
  if (de != DEDISP_NO_ERROR) return de;
  if (nsamps < p->max_delay) return DEDISP_TOO_FEW_NSAMPS;
  const size_t nout = nsamps - p->max_delay;
  if (p->groups.empty())
    return dedisperse_tables(p, p->delays, p->d_delays, p->d_blk_min, p->max_span,
                             (int)p->dm_list.size(), nout, 0, d_ft, pitch, nsamps, d_out,
                             out_pitch, s, units, in_unit, out_unit);
  // adaptive dt: group g's trials [d0, d1) of every unit are rows
  // units * d0 + u * (d1 - d0) + i of the output (group-major)
  const size_t C = p->nchans;
  for (size_t gi = 0; gi < p->groups.size(); gi++) {
    const dedisp_plan_struct::Group& g = p->groups[gi];
    const size_t Dg = g.d1 - g.d0;
    const size_t nout_s = nout / g.s;
    float* out_g = d_out + units * g.d0 * out_pitch;
    if (g.s == 1) {
      de = dedisperse_tables(p, g.delays, g.d_delays, g.d_blk_min, g.max_span, (int)Dg, nout_s, gi + 1,
                             d_ft, pitch, nsamps, out_g, out_pitch, s, units, in_unit,
                             Dg * out_pitch);
    } else {
      const size_t ns = nsamps / g.s;
      const size_t pitch_s = ft_pitch_for(g.max_span, g.max_delay, ns, nout_s);
      const size_t need = units * pitch_s * C;
      if (p->d_scr_cap < need) {
        free_dev(p->d_scr);
        p->d_scr = nullptr;
        p->d_scr_cap = 0;
        if (dev_malloc(&p->d_scr, need) != cudaSuccess) return DEDISP_MEM_ALLOC_FAILED;
        p->d_scr_cap = need;
      }
      if (launch_scrunch_ft(d_ft, pitch, nsamps, (int)C, (int)g.s, p->d_scr, pitch_s, units,
                            in_unit, pitch_s * C, s) != cudaSuccess)
        return DEDISP_INTERNAL_GPU_ERROR;
      de = dedisperse_tables(p, g.delays, g.d_delays, g.d_blk_min, g.max_span, (int)Dg, nout_s, gi + 1,
                             p->d_scr, pitch_s, ns, out_g, out_pitch, s, units, pitch_s * C,
                             Dg * out_pitch);
    }
    if (de != DEDISP_NO_ERROR) return de;
  }
  return DEDISP_NO_ERROR;
}

}  // namespace hdb

dedisp_plan_struct::~dedisp_plan_struct() {
  hdb::free_dev(d_delays);
  for (int* b : d_blk_min) hdb::free_dev(b);
  hdb::free_dev(d_active);
  hdb::free_dev(d_dm_list);
  hdb::free_dev(d_err);
  hdb::free_dev(d_in_tf);
  hdb::free_dev(d_in_ft);
  hdb::free_dev(d_out);
  hdb::free_dev(d_out_hi);
  hdb::free_dev(d_scr);
  hdb::free_groups(this);
  if (stream) cudaStreamDestroy(stream);
}

// ===========================================================================
// C interface
// ===========================================================================
extern "C" {

dedisp_error dedisp_create_plan(dedisp_plan* plan, dedisp_size nchans, dedisp_float dt,
                                dedisp_float f0, dedisp_float df) {
  if (!plan) return DEDISP_INVALID_POINTER;
  *plan = nullptr;
  if (nchans == 0) return DEDISP_NCHANS_EXCEEDS_LIMIT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return DEDISP_PRIOR_GPU_ERROR;
  dedisp_plan p = new (std::nothrow) dedisp_plan_struct();
  if (!p) return DEDISP_MEM_ALLOC_FAILED;
  p->nchans = nchans;
  p->dt = dt;
  p->f0 = f0;
  p->df = df;
  p->table.resize(nchans);
  hdb::delay_table(nchans, dt, f0, df, p->table.data());
  p->killmask.assign(nchans, 1);
  // HDB_DEDISP_TUNE=0 keeps the default tile; HDB_DEDISP_TILE=DBxTB forces one
  if (const char* e = std::getenv("HDB_DEDISP_TUNE"))
    if (e[0] == '0') p->tune = false;
  if (const char* e = std::getenv("HDB_DEDISP_TILE")) {
    int db = 0, tb = 0;
    if (std::sscanf(e, "%dx%d", &db, &tb) == 2) {
      p->forced_dm_block = db;
      p->forced_time_block = tb;
    }
  }
  *plan = p;
  return DEDISP_NO_ERROR;
}

void dedisp_destroy_plan(dedisp_plan plan) { delete plan; }

// The per-trial scrunch factors follow the DM list (all 1 without adaptive dt).
static void set_factors(dedisp_plan p) {
  if (p->adaptive)
    p->dt_factors = hdb::scrunch_factors(p->dm_list, p->dt, p->adaptive_width, p->f0, p->df,
                                         p->nchans, p->adaptive_tol);
  else
    p->dt_factors.assign(p->dm_list.size(), 1);
  p->dirty = true;
}

dedisp_error dedisp_set_dm_list(dedisp_plan p, const dedisp_float* l, dedisp_size n) {
  if (!p) return DEDISP_INVALID_PLAN;
  if (!l) return DEDISP_INVALID_POINTER;
  p->dm_list.assign(l, l + n);
  set_factors(p);
  return DEDISP_NO_ERROR;
}

dedisp_error dedisp_generate_dm_list(dedisp_plan p, dedisp_float a, dedisp_float b,
                                     dedisp_float ti, dedisp_float tol) {
  if (!p) return DEDISP_INVALID_PLAN;
  p->dm_list = hdb::generate_dm_list(a, b, p->dt, ti, p->f0, p->df, p->nchans, tol);
  set_factors(p);
  return DEDISP_NO_ERROR;
}

static thread_local std::vector<float> g_guru;
const dedisp_float* dedisp_generate_dm_list_guru(dedisp_float a, dedisp_float b, double dt,
                                                 double ti, double f0, double df,
                                                 dedisp_size nchans, double tol,
                                                 dedisp_size* count) {
  g_guru = hdb::generate_dm_list(a, b, dt, ti, f0, df, nchans, tol);
  if (count) *count = g_guru.size();
  return g_guru.data();
}

dedisp_error dedisp_set_killmask(dedisp_plan p, const dedisp_bool* km) {
  if (!p) return DEDISP_INVALID_PLAN;
  // the device tables depend on the mask: rebuild them only when it changes
  bool changed = false;
  for (size_t c = 0; c < p->nchans; c++) {
    const int v = km ? (km[c] != 0) : 1;
    changed = changed || p->killmask[c] != v;
    p->killmask[c] = v;
  }
  if (changed) p->dirty = true;
  return DEDISP_NO_ERROR;
}

// Adaptive time resolution: per-trial scrunch factors (hdb::scrunch_factors),
// recomputed whenever the DM list changes.
dedisp_error dedisp_enable_adaptive_dt(dedisp_plan p, dedisp_float w, dedisp_float tol) {
  if (!p) return DEDISP_INVALID_PLAN;
  if (!(tol > 1.0f) || !(w >= 0.0f)) return DEDISP_INVALID_FLAG_COMBINATION;
  p->adaptive = true;
  p->adaptive_width = w;
  p->adaptive_tol = tol;
  set_factors(p);
  return DEDISP_NO_ERROR;
}

dedisp_error dedisp_disable_adaptive_dt(dedisp_plan p) {
  if (!p) return DEDISP_INVALID_PLAN;
  p->adaptive = false;
  set_factors(p);
  return DEDISP_NO_ERROR;
}

dedisp_size dedisp_get_dm_count(const dedisp_plan p) { return p ? p->dm_list.size() : 0; }
const dedisp_float* dedisp_get_dm_list(const dedisp_plan p) {
  return (p && !p->dm_list.empty()) ? p->dm_list.data() : nullptr;
}
const dedisp_size* dedisp_get_dt_factors(const dedisp_plan p) {
  return (p && !p->dt_factors.empty()) ? p->dt_factors.data() : nullptr;
}
dedisp_size dedisp_get_max_delay(const dedisp_plan p) {
  if (!p || p->dm_list.empty()) return 0;
  size_t m = 0;
  for (float dm : p->dm_list)
    for (size_t c = 0; c < p->nchans; c++) m = std::max(m, hdb::delay_of(dm, p->table[c]));
  return m;
}
dedisp_size dedisp_get_dm_delay(const dedisp_plan p, int d) {
  if (!p || d < 0 || (size_t)d >= p->dm_list.size()) return 0;
  size_t m = 0;
  for (size_t c = 0; c < p->nchans; c++) m = std::max(m, hdb::delay_of(p->dm_list[d], p->table[c]));
  return m;
}
dedisp_size dedisp_get_channel_count(const dedisp_plan p) { return p ? p->nchans : 0; }
dedisp_float dedisp_get_dt(const dedisp_plan p) { return p ? p->dt : 0.f; }
dedisp_float dedisp_get_f0(const dedisp_plan p) { return p ? p->f0 : 0.f; }
dedisp_float dedisp_get_df(const dedisp_plan p) { return p ? p->df : 0.f; }

dedisp_error dedisp_execute_adv(const dedisp_plan p, dedisp_size nsamps, const dedisp_byte* in,
                                dedisp_size in_nbits, dedisp_size in_stride, dedisp_byte* out,
                                dedisp_size out_nbits, dedisp_size out_stride, unsigned flags) {
  if (!p) return DEDISP_INVALID_PLAN;
  if (!in || !out) return DEDISP_INVALID_POINTER;
  if (p->dm_list.empty()) return DEDISP_NO_DM_LIST_SET;
  // 1, 2, 4, 8 or 16-bit samples (packed little-endian, channel-fastest);
  // adaptive dt averages byte values, so 16-bit input searches at native
  // resolution only
  if (!hdb::nbits_supported(in_nbits) || (in_nbits == 16 && p->adaptive))
    return DEDISP_UNSUPPORTED_IN_NBITS;
  if (out_nbits != 32) return DEDISP_UNSUPPORTED_OUT_NBITS;
  if ((p->nchans * in_nbits) % 32 != 0 || in_stride != p->nchans * in_nbits / 8 ||
      (p->nchans % 4) != 0)
    return DEDISP_INVALID_STRIDE;
  if (out_stride % 4) return DEDISP_INVALID_STRIDE;
  // spectra are read as 32-bit words: device input must be 4-byte aligned
  if ((flags & DEDISP_DEVICE_POINTERS) && (reinterpret_cast<uintptr_t>(in) & 3))
    return DEDISP_INVALID_POINTER;
  dedisp_error de = hdb::plan_prepare(p);
  if (de != DEDISP_NO_ERROR) return de;
  if (nsamps < p->max_delay) return DEDISP_TOO_FEW_NSAMPS;
  const size_t nout = nsamps - p->max_delay;
  const size_t D = p->dm_list.size();
  if (out_stride / 4 < nout) return DEDISP_INVALID_STRIDE;
  if (!p->stream && cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess)
    return DEDISP_PRIOR_GPU_ERROR;
  cudaStream_t s = p->stream;
  const size_t pitch = hdb::ft_pitch(p, nsamps);
  const bool dev_ptrs = (flags & DEDISP_DEVICE_POINTERS) != 0;
  const uint8_t* d_tf = in;
  if (!dev_ptrs) {
    size_t need = nsamps * in_stride;
    if (p->d_in_tf_cap < need) {
      hdb::free_dev(p->d_in_tf);
      p->d_in_tf = nullptr;
      if (hdb::dev_malloc(&p->d_in_tf, need) != cudaSuccess) return DEDISP_MEM_ALLOC_FAILED;
      p->d_in_tf_cap = need;
    }
    if (cudaMemcpyAsync(p->d_in_tf, in, need, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return DEDISP_MEM_COPY_FAILED;
    d_tf = p->d_in_tf;
  }
  const size_t plane = pitch * p->nchans;
  size_t need_ft = plane * (in_nbits == 16 ? 2 : 1);
  if (p->d_in_ft_cap < need_ft) {
    hdb::free_dev(p->d_in_ft);
    p->d_in_ft = nullptr;
    if (hdb::dev_malloc(&p->d_in_ft, need_ft) != cudaSuccess) return DEDISP_MEM_ALLOC_FAILED;
    cudaMemsetAsync(p->d_in_ft, 0, need_ft, s);
    p->d_in_ft_cap = need_ft;
  }
  if (cudaMemsetAsync(p->d_err, 0, sizeof(unsigned), s) != cudaSuccess ||
      hdb::input_to_ft(d_tf, nsamps, (int)p->nchans, (int)in_nbits, p->d_in_ft, pitch, s, 1,
                       plane) != cudaSuccess)
    return DEDISP_INTERNAL_GPU_ERROR;
  float* d_o = reinterpret_cast<float*>(out);
  size_t opitch = out_stride / 4;
  if (!dev_ptrs) {
    opitch = (nout + 3) & ~(size_t)3;
    size_t need = opitch * D;
    if (p->d_out_cap < need) {
      hdb::free_dev(p->d_out);
      p->d_out = nullptr;
      if (hdb::dev_malloc(&p->d_out, need * sizeof(float)) != cudaSuccess)
        return DEDISP_MEM_ALLOC_FAILED;
      p->d_out_cap = need;
    }
    d_o = p->d_out;
  } else if (opitch % 4) {
    return DEDISP_INVALID_STRIDE;
  }
  if (in_nbits == 16) {
    // high-byte plane, low-byte plane, then lo + 256 hi
    const size_t need = opitch * D;
    if (p->d_out_hi_cap < need) {
      hdb::free_dev(p->d_out_hi);
      p->d_out_hi = nullptr;
      if (hdb::dev_malloc(&p->d_out_hi, need * sizeof(float)) != cudaSuccess)
        return DEDISP_MEM_ALLOC_FAILED;
      p->d_out_hi_cap = need;
    }
    de = hdb::plan_dedisperse_ft(p, p->d_in_ft + plane, pitch, nsamps, p->d_out_hi, opitch, s);
    if (de != DEDISP_NO_ERROR) return de;
  }
  de = hdb::plan_dedisperse_ft(p, p->d_in_ft, pitch, nsamps, d_o, opitch, s);
  if (de != DEDISP_NO_ERROR) return de;
  if (in_nbits == 16 &&
      hdb::launch_combine_planes(d_o, p->d_out_hi, opitch, nout, D, s) != cudaSuccess)
    return DEDISP_INTERNAL_GPU_ERROR;
  if (!dev_ptrs) {
    if (cudaMemcpy2DAsync(out, out_stride, d_o, opitch * sizeof(float), nout * sizeof(float), D,
                          cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return DEDISP_MEM_COPY_FAILED;
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return DEDISP_INTERNAL_GPU_ERROR;
  unsigned err = 0;
  cudaMemcpy(&err, p->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost);
  if (err) return DEDISP_INTERNAL_GPU_ERROR;
  return DEDISP_NO_ERROR;
}

dedisp_error dedisp_execute(const dedisp_plan p, dedisp_size nsamps, const dedisp_byte* in,
                            dedisp_size in_nbits, dedisp_byte* out, dedisp_size out_nbits,
                            unsigned flags) {
  if (!p) return DEDISP_INVALID_PLAN;
  dedisp_size md = dedisp_get_max_delay(p);
  if (nsamps < md) return DEDISP_TOO_FEW_NSAMPS;
  return dedisp_execute_adv(p, nsamps, in, in_nbits, p->nchans * in_nbits / 8, out, out_nbits,
                            (nsamps - md) * out_nbits / 8, flags);
}

const char* dedisp_get_error_string(dedisp_error e) {
  switch (e) {
    case DEDISP_NO_ERROR: return "No error";
    case DEDISP_MEM_ALLOC_FAILED: return "Memory allocation failed";
    case DEDISP_MEM_COPY_FAILED: return "Memory copy failed";
    case DEDISP_NCHANS_EXCEEDS_LIMIT: return "No. channels exceeds internal limit";
    case DEDISP_INVALID_PLAN: return "Invalid plan";
    case DEDISP_INVALID_POINTER: return "Invalid pointer";
    case DEDISP_INVALID_STRIDE: return "Invalid stride";
    case DEDISP_NO_DM_LIST_SET: return "No DM list has been set";
    case DEDISP_TOO_FEW_NSAMPS: return "No. samples < maximum delay";
    case DEDISP_INVALID_FLAG_COMBINATION: return "Invalid flag combination";
    case DEDISP_UNSUPPORTED_IN_NBITS: return "Unsupported in_nbits value";
    case DEDISP_UNSUPPORTED_OUT_NBITS: return "Unsupported out_nbits value";
    case DEDISP_INVALID_DEVICE_INDEX: return "Invalid device index";
    case DEDISP_DEVICE_ALREADY_SET: return "Device is already set and cannot be changed";
    case DEDISP_PRIOR_GPU_ERROR: return "Prior GPU error.";
    case DEDISP_INTERNAL_GPU_ERROR: return "Internal GPU error.";
    default: return "Unknown error";
  }
}

}  // extern "C"
