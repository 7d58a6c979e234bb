// beamset.cpp -- beams of different shapes (channel count, gulp length,
// sampling time, band, DM range) searched in one call.
//
// Each beam keeps the reference's per-beam semantics: its candidates are
// those hd_execute gives for that beam with its own hd_params (one heimdall
// process per beam in the reference, Applications/heimdall.C).  The set runs
// them concurrently on one GPU:
//   * beams are grouped by configuration (every hd_params field but `beam`);
//     runs of beams with the same configuration and gulp length go through
//     one hd_execute_beams call (the batched kernels);
//   * the beams, ordered by configuration and then by decreasing length, are
//     split into nworkers contiguous chunks of about equal estimated work
//     (DM trials x samples x (channels + a per-sample search share)); one host
//     thread per chunk searches it with its own pipelines (one per
//     configuration in the chunk, each with its own non-blocking streams), so
//     the chunks overlap on the GPU: copies, small kernels and the host
//     synchronisations of one chunk (threshold and giant counts, clustering
//     rounds) hide behind the kernels of another;
//   * a worker keeps the pipelines of its chunk between calls (no device
//     allocation in steady state) and releases the others, so the device
//     memory stays near one pipeline per configuration.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "heimdall_b200.h"
#include "plan.h"

namespace {

constexpr size_t kMaxRun = 64;  // beams per hd_execute_beams call

// Configuration key: every field that changes the search or its output, with
// the pointed-to data of the pointer fields; `beam` is excluded.
std::string config_key(const hd_params& p) {
  std::string k;
  auto put = [&](const void* v, size_t n) { k.append(static_cast<const char*>(v), n); };
  hd_params q = p;
  q.beam = 0;
  q.sigproc_file = nullptr;
  q.coincidencer_host = nullptr;
  q.channel_zaps = nullptr;
  q.output_dir = nullptr;
  // field by field (no padding bytes in the key)
  put(&q.verbosity, sizeof q.verbosity);
  put(&q.nsamps_gulp, sizeof q.nsamps_gulp);
  put(&q.dm_gulp_size, sizeof q.dm_gulp_size);
  put(&q.baseline_length, sizeof q.baseline_length);
  put(&q.nbeams, sizeof q.nbeams);
  put(&q.nchans, sizeof q.nchans);
  put(&q.dt, sizeof q.dt);
  put(&q.f0, sizeof q.f0);
  put(&q.df, sizeof q.df);
  put(&q.dm_min, sizeof q.dm_min);
  put(&q.dm_max, sizeof q.dm_max);
  put(&q.dm_tol, sizeof q.dm_tol);
  put(&q.dm_pulse_width, sizeof q.dm_pulse_width);
  put(&q.dm_nbits, sizeof q.dm_nbits);
  const char flags[3] = {(char)q.use_scrunching, (char)q.override_beam, (char)q.yield_cpu};
  put(flags, 3);
  put(&q.scrunch_tol, sizeof q.scrunch_tol);
  put(&q.rfi_tol, sizeof q.rfi_tol);
  put(&q.rfi_min_beams, sizeof q.rfi_min_beams);
  put(&q.boxcar_max, sizeof q.boxcar_max);
  put(&q.detect_thresh, sizeof q.detect_thresh);
  put(&q.cand_sep_time, sizeof q.cand_sep_time);
  put(&q.cand_sep_filter, sizeof q.cand_sep_filter);
  put(&q.cand_sep_dm, sizeof q.cand_sep_dm);
  put(&q.cand_rfi_dm_cut, sizeof q.cand_rfi_dm_cut);
  put(&q.max_giant_rate, sizeof q.max_giant_rate);
  put(&q.min_tscrunch_width, sizeof q.min_tscrunch_width);
  put(&q.coincidencer_port, sizeof q.coincidencer_port);
  put(&q.beam_count, sizeof q.beam_count);
  put(&q.gpu_id, sizeof q.gpu_id);
  put(&q.utc_start, sizeof q.utc_start);
  put(&q.spectra_per_second, sizeof q.spectra_per_second);
  put(&p.num_channel_zaps, sizeof p.num_channel_zaps);
  if (p.channel_zaps && p.num_channel_zaps)
    put(p.channel_zaps, p.num_channel_zaps * sizeof(hd_range_t));
  const char* od = p.output_dir;
  k.push_back(od ? 1 : 0);
  if (od) k.append(od);
  k.push_back(0);
  return k;
}

}  // namespace

struct hd_beam_set_t {
  int device = 0;
  int nworkers = 1;
  bool cleaning = true;
  // distinct configurations with owned copies of their pointer fields
  struct Config {
    hd_params p;
    std::string output_dir;
    std::vector<hd_range_t> zaps;
  };
  std::vector<Config> configs;
  std::vector<double> cfg_trials;  // DM trials per configuration (work estimate)
  std::vector<int> cfg_of;       // beam -> configuration
  std::vector<hd_size> beam_no;  // beam -> hd_params.beam
  // pipelines kept between calls: pipes[worker][configuration]
  std::vector<std::map<int, hd_pipeline>> pipes;
  // results of the last call
  std::vector<std::vector<hd_candidate>> cands;

  ~hd_beam_set_t() {
    for (auto& m : pipes)
      for (auto& kv : m) hd_destroy_pipeline(kv.second);
  }
};

extern "C" {

hd_error hd_create_beam_set(hd_beam_set* set, const struct hd_params* params, hd_size nbeams,
                            int nworkers) {
  if (!set) return HD_INVALID_POINTER;
  *set = nullptr;
  if (!params || nbeams == 0) return HD_INVALID_POINTER;
  if (nworkers < 1 || nworkers > 64) return HD_INVALID_STRIDE;
  for (hd_size b = 1; b < nbeams; b++)
    if (params[b].gpu_id != params[0].gpu_id) return HD_INVALID_DEVICE_INDEX;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || params[0].gpu_id < 0 ||
      params[0].gpu_id >= ndev)
    return HD_INVALID_DEVICE_INDEX;
  hd_beam_set s = new (std::nothrow) hd_beam_set_t();
  if (!s) return HD_MEM_ALLOC_FAILED;
  s->device = params[0].gpu_id;
  s->nworkers = nworkers;
  std::map<std::string, int> index;
  s->cfg_of.resize(nbeams);
  s->beam_no.resize(nbeams);
  for (hd_size b = 0; b < nbeams; b++) {
    const std::string key = config_key(params[b]);
    auto it = index.find(key);
    int c;
    if (it == index.end()) {
      c = (int)s->configs.size();
      index.emplace(key, c);
      hd_beam_set_t::Config cf;
      cf.p = params[b];
      cf.p.beam = 0;
      if (params[b].output_dir) cf.output_dir = params[b].output_dir;
      if (params[b].channel_zaps && params[b].num_channel_zaps)
        cf.zaps.assign(params[b].channel_zaps,
                       params[b].channel_zaps + params[b].num_channel_zaps);
      s->configs.push_back(std::move(cf));
    } else {
      c = it->second;
    }
    s->cfg_of[b] = c;
    s->beam_no[b] = params[b].beam;
  }
  // the strings and zap tables now live in the set
  for (auto& cf : s->configs) {
    const std::vector<float> dms =
        hdb::generate_dm_list(cf.p.dm_min, cf.p.dm_max, cf.p.dt, cf.p.dm_pulse_width, cf.p.f0,
                              cf.p.df, cf.p.nchans, cf.p.dm_tol);
    s->cfg_trials.push_back((double)std::max<size_t>(dms.size(), 1));
    if (cf.p.output_dir) cf.p.output_dir = cf.output_dir.c_str();
    cf.p.channel_zaps = cf.zaps.empty() ? nullptr : cf.zaps.data();
    cf.p.num_channel_zaps = (unsigned)cf.zaps.size();
  }
  s->pipes.resize(nworkers);
  s->cands.resize(nbeams);
  *set = s;
  return HD_NO_ERROR;
}

hd_error hd_set_beam_set_cleaning(hd_beam_set s, int enable) {
  if (!s) return HD_INVALID_PIPELINE;
  s->cleaning = enable != 0;
  for (auto& m : s->pipes)
    for (auto& kv : m) hd_set_cleaning(kv.second, enable);
  return HD_NO_ERROR;
}

hd_size hd_get_beam_set_config_count(hd_beam_set s) { return s ? s->configs.size() : 0; }

hd_error hd_execute_beam_set(hd_beam_set s, const hd_byte* const* filterbanks,
                             const hd_size* nsamps, hd_size nbits, hd_size first_idx,
                             int on_device, hd_error* statuses, hd_size* nsamps_processed) {
  if (!s) return HD_INVALID_PIPELINE;
  const size_t n = s->cfg_of.size();
  if (!filterbanks || !nsamps) return HD_INVALID_POINTER;
  for (size_t b = 0; b < n; b++)
    if (!filterbanks[b]) return HD_INVALID_POINTER;
  if (nbits != 8) return HD_INVALID_NBITS;
  // order: by configuration, then by decreasing gulp length (runs of equal
  // length are batched), then by beam index
  std::vector<size_t> order(n);
  for (size_t b = 0; b < n; b++) order[b] = b;
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    if (s->cfg_of[a] != s->cfg_of[b]) return s->cfg_of[a] < s->cfg_of[b];
    if (nsamps[a] != nsamps[b]) return nsamps[a] > nsamps[b];
    return a < b;
  });
  std::vector<hd_error> st(n, HD_NO_ERROR);
  std::vector<hd_size> proc(n, 0);
  for (auto& v : s->cands) v.clear();
  // contiguous chunks of about equal estimated work, one per worker
  const int nw = (int)std::min<size_t>((size_t)s->nworkers, n);
  std::vector<double> cost(n);
  double total = 0.0;
  for (size_t i = 0; i < n; i++) {
    const size_t b = order[i];
    const hd_params& p = s->configs[s->cfg_of[b]].p;
    cost[i] = s->cfg_trials[s->cfg_of[b]] * (double)nsamps[b] * ((double)p.nchans + 256.0);
    total += cost[i];
  }
  std::vector<size_t> bound(nw + 1, n);
  bound[0] = 0;
  {
    double acc = 0.0;
    int w = 1;
    for (size_t i = 0; i < n && w < nw; i++) {
      acc += cost[i];
      // close chunk w - 1 after beam i once it holds its share, leaving at
      // least one beam for each later chunk
      if (acc >= total * w / nw && n - (i + 1) >= (size_t)(nw - w)) bound[w++] = i + 1;
    }
    for (; w < nw; w++) bound[w] = std::max(bound[w - 1], n - (size_t)(nw - w));
  }
  std::atomic<int> setup_error{HD_NO_ERROR};

  auto work = [&](int w) {
    if (cudaSetDevice(s->device) != cudaSuccess) {
      setup_error.store(HD_INVALID_DEVICE_INDEX);
      return;
    }
    std::map<int, hd_pipeline>& mine = s->pipes[w];
    const size_t c0 = bound[w], c1 = bound[w + 1];
    // release pipelines of configurations outside this chunk
    for (auto it = mine.begin(); it != mine.end();) {
      bool used = false;
      for (size_t i = c0; i < c1 && !used; i++) used = s->cfg_of[order[i]] == it->first;
      if (used) {
        ++it;
      } else {
        hd_destroy_pipeline(it->second);
        it = mine.erase(it);
      }
    }
    std::vector<const hd_byte*> fbs;
    std::vector<hd_size> bn;
    std::vector<hd_error> ust;
    std::vector<hd_candidate> buf;
    for (size_t i0 = c0; i0 < c1;) {
      const size_t b0 = order[i0];
      size_t i1 = i0 + 1;
      while (i1 < c1 && i1 - i0 < kMaxRun && s->cfg_of[order[i1]] == s->cfg_of[b0] &&
             nsamps[order[i1]] == nsamps[b0])
        i1++;
      const int cfg = s->cfg_of[b0];
      hd_pipeline pl = nullptr;
      auto it = mine.find(cfg);
      if (it != mine.end()) {
        pl = it->second;
      } else {
        hd_error e = hd_create_pipeline(&pl, s->configs[cfg].p);
        if (e != HD_NO_ERROR) {
          for (size_t i = i0; i < i1; i++) st[order[i]] = e;
          i0 = i1;
          continue;
        }
        hd_set_cleaning(pl, s->cleaning);
        // one pipeline serves beams of many gulp lengths: each length is a
        // shape of its own whose graph would be captured, and its buffers
        // regrown, for every new length, so the set stays on the
        // host-sized path
        hd_set_graphs(pl, 0);
        mine.emplace(cfg, pl);
      }
      const size_t U = i1 - i0;
      fbs.resize(U);
      bn.resize(U);
      ust.assign(U, HD_NO_ERROR);
      for (size_t u = 0; u < U; u++) {
        fbs[u] = filterbanks[order[i0 + u]];
        bn[u] = s->beam_no[order[i0 + u]];
      }
      hd_size processed = 0;
      const hd_error e = hd_execute_beams(pl, fbs.data(), U, nsamps[b0], nbits, first_idx, 1,
                                          bn.data(), on_device, ust.data(), &processed);
      for (size_t u = 0; u < U; u++) {
        const size_t b = order[i0 + u];
        st[b] = (e == HD_NO_ERROR || e == HD_TOO_MANY_EVENTS) ? ust[u] : e;
        proc[b] = processed;
        hd_size cnt = 0;
        hd_get_beam_candidates(pl, u, nullptr, &cnt);
        buf.resize(cnt);
        if (cnt) hd_get_beam_candidates(pl, u, buf.data(), &cnt);
        s->cands[b].assign(buf.begin(), buf.begin() + cnt);
      }
      i0 = i1;
    }
  };

  std::vector<std::thread> th;
  for (int w = 1; w < nw; w++) th.emplace_back(work, w);
  work(0);
  for (auto& t : th) t.join();
  if (setup_error.load() != HD_NO_ERROR) return setup_error.load();

  hd_error first = HD_NO_ERROR;
  for (size_t b = 0; b < n; b++) {
    if (statuses) statuses[b] = st[b];
    if (nsamps_processed) nsamps_processed[b] = proc[b];
    if (first == HD_NO_ERROR && st[b] != HD_NO_ERROR) first = st[b];
  }
  return first;
}

hd_error hd_get_beam_set_candidates(hd_beam_set s, hd_size beam, hd_candidate* out,
                                    hd_size* count) {
  if (!s) return HD_INVALID_PIPELINE;
  if (!count) return HD_INVALID_POINTER;
  if (beam >= s->cands.size()) return HD_INVALID_STRIDE;
  const std::vector<hd_candidate>& v = s->cands[beam];
  const size_t k = std::min(*count, (hd_size)v.size());
  if (out && k) std::memcpy(out, v.data(), k * sizeof(hd_candidate));
  *count = v.size();
  return HD_NO_ERROR;
}

void hd_destroy_beam_set(hd_beam_set s) {
  if (!s) return;
  cudaSetDevice(s->device);
  delete s;
}

}  // extern "C"
