// pipeline.cpp -- the hd_* pipeline (Pipeline/pipeline.cu:138-1100) on the
// sm_100a kernels.
//
// One gulp runs as a fixed sequence of kernels on the pipeline's own stream:
//   H2D (TF filterbank)
//   clean_filterbank_rfi: zero-DM sums -> baseline -> RMS -> normalise+scan ->
//       RFI mask -> zap (writes the channel-major working copy)   [optional]
//   dedispersion of all DM trials (TMA-staged, exact int32 sums)
//   per-DM baseline, robust RMS, normalise + prefix sum        (all DMs at once)
//   per-width block RMS, threshold + ordered hit compaction    (all DMs x widths)
//   giant segmentation, clustering, merge, DM gather
//   D2H of the merged candidate rows; .cand file on the host.
// Host synchronisations: the hit and giant totals (to size buffers), the
// clustering convergence flag and the final candidate rows.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <new>
#include <string>
#include <vector>

#include <cuda.h>

#include "heimdall_b200.h"
#include "internal.h"
#include "plan.h"

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  ~DevBuf() { if (p) cudaFree(p); }
  template <class T>
  T* as() { return reinterpret_cast<T*>(p); }
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t b = std::max<size_t>(bytes, 256);
    cudaError_t e = hdb::dev_malloc(&p, b);
    if (e == cudaSuccess) cap = b;
    return e;
  }
};

}  // namespace

// Merged candidate rows read back with the group count, before it is known
// (the rest follow in a second copy when there are more).
constexpr size_t kSpecRows = 2048;

// Host filterbanks of a batched gulp are copied in up to kMaxChunks pieces so
// that the transpose and dedispersion of one piece overlap the next copy.
constexpr int kMaxChunks = 8;

struct hd_pipeline_t {
  hd_params params;
  std::string output_dir;
  bool has_output_dir = true;
  std::vector<hd_range_t> zaps;
  dedisp_plan plan = nullptr;
  // clean_filterbank_rfi: off as in the reference's shipped build (it is
  // compiled in only under -DCLEANING); hd_set_cleaning turns it on
  bool cleaning = false;
  bool narrow_band = false;  // the reference's disabled narrow-band branch
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // host->device copies overlapped with compute
  cudaEvent_t ev[10] = {};
  cudaEvent_t chunk_ev[kMaxChunks] = {};
  // double-buffered ingest (hd_prefetch_beams / hd_execute_prefetched): two
  // slots of filterbanks copied on copy_stream ahead of their search
  struct Prefetch {
    DevBuf buf;
    cudaEvent_t done = nullptr;
    bool pending = false;
    unsigned long long tag = 0;
    size_t units = 0, nsamps = 0;
  } pf[2];
  unsigned long long pf_seq = 0;
  // set by hd_execute_prefetched: the gulp already sits in fb_tf (the slot's
  // buffer was swapped in), so execute_units copies nothing
  bool fb_resident = false;
  float timing[8] = {};

  DevBuf fb_tf, fb_ft, fb_tf_clean;
  DevBuf dm0, dm0_scan, base, rms, mask, fmask, rms0, nb_scratch;
  DevBuf dd, dd_hi, scan;
  DevBuf ws_a, ws_b;
  DevBuf winfo, norm, gmax, tile_list;
  DevBuf tile_cnt, tile_off, sw_cnt, sw_off, hit_ind, hit_val, hit_sw;
  DevBuf head, gid;
  // a giant list's arrays
  struct GiantSet {
    DevBuf key, peak, ind, begin, end, filter, dm, label;
    void view(hdb::GiantBuffers& g) {
      g.key = key.as<unsigned long long>();
      g.peak = peak.as<float>();
      g.ind = ind.as<unsigned long long>();
      g.begin = begin.as<unsigned long long>();
      g.end = end.as<unsigned long long>();
      g.filter = filter.as<int>();
      g.dm = dm.as<int>();
      g.label = label.as<int>();
    }
  };
  GiantSet main_giants;           // the gulp's giant list
  std::vector<GiantSet> gsets;    // per scrunch group (adaptive dt)
  DevBuf place_base;
  DevBuf scan_tmp, small;  // small: totals / flags
  DevBuf root_flag, root_off, mkey, rows, unit_off;
  DevBuf h_small_dev;

  // Gulps captured as CUDA graphs (hd_execute_beams with device input and
  // hd_execute_prefetched).  The first gulp of a shape runs on the
  // host-sized path and fixes the shape's hit and giant capacities and its
  // number of clustering sweep pairs; later gulps of the shape replay one
  // graph per set of device buffers.
  struct GraphShape {
    std::vector<size_t> key;
    unsigned hcap = 0, gcap = 0, pairs = 0;
    bool broken = false;  // capture failed: this shape stays on the host-sized path
  };
  struct GraphGulp {
    std::vector<size_t> key;   // shape key followed by the buffers' addresses and sizes
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;    // kernel nodes per replay
    bool events = false;       // the stage events are graph nodes
    unsigned long long used = 0;
  };
  std::vector<GraphShape> graph_shapes;
  std::vector<GraphGulp> graphs;
  unsigned long long graph_clock = 0;
  bool use_graphs = true;
  bool last_graph = false;     // the last gulp ran as a graph replay
  unsigned long long graph_replays = 0;
  std::vector<size_t> pending_shape;  // registered once its host-sized gulp succeeds
  DevBuf geo, gflags;
  // what the last host-sized gulp saw (sizes a new shape's capacities)
  unsigned obs_hits = 0, obs_giants = 0, obs_pairs = 0;
  void drop_graphs(const std::vector<size_t>& shape) {
    for (size_t i = 0; i < graphs.size();) {
      const auto& k = graphs[i].key;
      if (k.size() >= shape.size() && std::equal(shape.begin(), shape.end(), k.begin())) {
        if (graphs[i].exec) cudaGraphExecDestroy(graphs[i].exec);
        graphs.erase(graphs.begin() + i);
      } else {
        i++;
      }
    }
  }

  unsigned* h_small = nullptr;  // pinned host words

  std::vector<hd_candidate> cands;                     // all units, unit by unit
  std::vector<std::vector<hd_candidate>> unit_cands;   // per unit
  // per candidate (parallel to cands): filterbank, series index, DM trial,
  // width index -- what the patch extraction needs
  struct CandMeta { unsigned unit, ind; int dm, filter; };
  std::vector<std::vector<CandMeta>> unit_meta;
  std::vector<CandMeta> meta;
  // the last gulp's search geometry (valid when searched)
  bool searched = false;
  size_t last_nsamps = 0, last_len = 0, last_scan_pitch = 0, last_units = 0;
  DevBuf patch_jobs, patch_dm, patch_ft;
  std::vector<unsigned> unit_first;                    // first giant of each unit
  // the last gulp's giant list stays on the device (main_giants); it is
  // copied only when hd_get_giants asks for it
  size_t last_giants = 0, last_gap = 1;
  // merged candidate rows read back (pinned)
  hdb::GroupRow* h_rows = nullptr;
  size_t h_rows_cap = 0;
  cudaError_t ensure_rows_host(size_t n) {
    if (n <= h_rows_cap) return cudaSuccess;
    if (h_rows) cudaFreeHost(h_rows);
    h_rows = nullptr;
    h_rows_cap = 0;
    cudaError_t e = cudaMallocHost(&h_rows, n * sizeof(hdb::GroupRow));
    if (e == cudaSuccess) h_rows_cap = n;
    else cudaGetLastError();
    return e;
  }

  ~hd_pipeline_t() {
    for (auto& g : graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    if (plan) dedisp_destroy_plan(plan);
    for (auto& e : ev) if (e) cudaEventDestroy(e);
    for (auto& e : chunk_ev) if (e) cudaEventDestroy(e);
    for (auto& q : pf) if (q.done) cudaEventDestroy(q.done);
    if (stream) cudaStreamDestroy(stream);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (h_small) cudaFreeHost(h_small);
    if (h_rows) cudaFreeHost(h_rows);
  }
};

namespace {

hd_error cuda_err(cudaError_t e) {
  if (e == cudaSuccess) return HD_NO_ERROR;
  if (e == cudaErrorMemoryAllocation) return HD_MEM_ALLOC_FAILED;
  if (e == cudaErrorInvalidDevice) return HD_INVALID_DEVICE_INDEX;
  return HD_INTERNAL_GPU_ERROR;
}

hd_error dedisp_err(dedisp_error e) {
  switch (e) {
    case DEDISP_NO_ERROR: return HD_NO_ERROR;
    case DEDISP_MEM_ALLOC_FAILED: return HD_MEM_ALLOC_FAILED;
    case DEDISP_MEM_COPY_FAILED: return HD_MEM_COPY_FAILED;
    case DEDISP_INVALID_DEVICE_INDEX: return HD_INVALID_DEVICE_INDEX;
    case DEDISP_DEVICE_ALREADY_SET: return HD_DEVICE_ALREADY_SET;
    case DEDISP_INVALID_POINTER: return HD_INVALID_POINTER;
    case DEDISP_INVALID_STRIDE: return HD_INVALID_STRIDE;
    case DEDISP_TOO_FEW_NSAMPS: return HD_TOO_FEW_NSAMPS;
    case DEDISP_PRIOR_GPU_ERROR: return HD_PRIOR_GPU_ERROR;
    case DEDISP_INTERNAL_GPU_ERROR: return HD_INTERNAL_GPU_ERROR;
    // a block's delay span too long for one staged row (dedispersion limit)
    case DEDISP_NCHANS_EXCEEDS_LIMIT: return HD_INVALID_STRIDE;
    default: return HD_UNKNOWN_ERROR;
  }
}

#define HD_TRY(x)                                   \
  do {                                              \
    cudaError_t e_ = (x);                           \
    if (e_ != cudaSuccess) return cuda_err(e_);     \
  } while (0)

unsigned log2u(size_t v) {
  unsigned r = 0;
  while ((v >> r) > 1) r++;
  return r;
}

size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// The allocation that contains p (CUDA device or page-locked host memory):
// false for memory CUDA does not know (pageable host memory), or when the
// driver's pointer-range query is unavailable.
bool allocation_range(const void* p, uintptr_t* base, size_t* size) {
  using Fn = CUresult (*)(void*, CUpointer_attribute, CUdeviceptr);
  static Fn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &f, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    cudaGetLastError();
    return reinterpret_cast<Fn>(f);
  }();
  if (!fn) return false;
  CUdeviceptr b = 0;
  size_t n = 0;
  const CUdeviceptr d = (CUdeviceptr) reinterpret_cast<uintptr_t>(p);
  if (fn(&b, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, d) != CUDA_SUCCESS ||
      fn(&n, CU_POINTER_ATTRIBUTE_RANGE_SIZE, d) != CUDA_SUCCESS)
    return false;
  *base = (uintptr_t)b;
  *size = n;
  return true;
}

// Copies filterbanks u0 .. u1-1 of `bytes` each, from srcs[u] to dst + u *
// bytes, with one cudaMemcpyAsync per run of sources that lie back to back
// inside one allocation (one call for a caller's contiguous block of
// filterbanks).  Page-locked or device buffers that merely sit next to each
// other are separate allocations, which one copy may not span; pageable host
// buffers that do are read as plain host memory.
cudaError_t copy_units(uint8_t* dst, const hd_byte* const* srcs, size_t u0, size_t u1,
                       size_t bytes, cudaMemcpyKind kind, cudaStream_t s) {
  size_t u = u0;
  while (u < u1) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(srcs[u]);
    uintptr_t rb = 0;
    size_t rn = 0;
    const bool known = u + 1 < u1 && allocation_range(srcs[u], &rb, &rn);
    size_t v = u + 1;
    while (v < u1 && reinterpret_cast<uintptr_t>(srcs[v]) == a + (v - u) * bytes &&
           (!known || a + (v - u + 1) * bytes <= rb + rn))
      v++;
    const cudaError_t e = cudaMemcpyAsync(dst + u * bytes, srcs[u], (v - u) * bytes, kind, s);
    if (e != cudaSuccess) return e;
    u = v;
  }
  return cudaSuccess;
}

// Scratch needed by the median trees of `nseg` segments of `count` values.
size_t tree_cap(size_t nseg, size_t count) { return nseg * (count / 3125 + 8) + 64; }

// Device clean_filterbank_rfi (Pipeline/clean_filterbank_rfi.cu:256-528) of
// `units` independent filterbanks (TF, nsamps x nchans bytes each, one after
// the other at tf).  Writes each zapped filterbank channel-major into
// fb_ft + u * nchans * pitch and, if out_tf, also time-major.  The zero-DM
// series of all units are baselined, normalised and summed as one batch.
hd_error clean_units(hd_pipeline pl, size_t units, const uint8_t* tf, size_t nsamps,
                     size_t nchans, float dt, float baseline_length, float rfi_tol,
                     size_t boxcar_max, size_t nbeams, uint8_t* fb_ft, size_t pitch,
                     uint8_t* out_tf) {
  cudaStream_t s = pl->stream;
  const size_t nsmooth = (size_t)(baseline_length / (2 * dt));
  if (nsamps < boxcar_max + 1 || nsmooth / 4 >= nsamps) return HD_TOO_FEW_NSAMPS;
  const size_t spitch = round_up(nsamps + 8, 64);
  const size_t U = units;
  HD_TRY(pl->dm0.ensure(U * spitch * sizeof(float)));
  HD_TRY(pl->dm0_scan.ensure(U * spitch * sizeof(float)));
  HD_TRY(pl->mask.ensure((U * nsamps + 64) * sizeof(int)));
  HD_TRY(pl->fmask.ensure((nsamps + 256) * sizeof(int)));
  HD_TRY(pl->rms0.ensure(U * nbeams * sizeof(float) + 64));
  HD_TRY(pl->base.ensure((U * nbeams * hdb::baseline_samples(nsamps / nbeams, nsmooth) + 64) *
                         sizeof(float)));
  size_t cap = std::max(tree_cap(U * nbeams, nsamps),
                        hdb::baseline_scratch(nsamps / nbeams, nsmooth, U * nbeams));
  HD_TRY(pl->ws_a.ensure(cap * sizeof(float)));
  HD_TRY(pl->ws_b.ensure(cap * sizeof(float)));
  if (pl->narrow_band) {
    // clean_filterbank_rfi.cu:303-351 with its `&& false` removed: zap
    // narrow-band RFI first; the broadband branch then reads the result.
    // tf is the pipeline's own device copy of the input.
    if (nchans < 20 || (size_t)(baseline_length / (1 * dt)) == 0) return HD_INVALID_STRIDE;
    HD_TRY(pl->nb_scratch.ensure(
        hdb::narrow_band_scratch_bytes(U, nsamps, (int)nchans, dt, baseline_length)));
    HD_TRY(hdb::narrow_band(const_cast<uint8_t*>(tf), U, nsamps, (int)nchans, dt,
                            baseline_length, rfi_tol, pl->nb_scratch.p, s));
  }
  float* x = pl->dm0.as<float>();
  HD_TRY(cudaMemsetAsync(x, 0, U * spitch * sizeof(float), s));
  for (size_t u = 0; u < U; u++)
    HD_TRY(hdb::launch_dm0_sum(tf + u * nsamps * nchans, nsamps, (int)nchans, x + u * spitch, s));
  hdb::SeriesBatch sb{x, spitch, (int)U, nsamps, nsamps / nbeams, nsamps / nbeams, (int)nbeams};
  hdb::TreeScratch ws{pl->ws_a.as<float>(), pl->ws_b.as<float>(), pl->ws_a.cap / sizeof(float)};
  HD_TRY(hdb::remove_baseline(sb, nsmooth, pl->base.as<float>(), ws, s));
  HD_TRY(hdb::rms_beams(sb, pl->rms0.as<float>(), ws, s));
  HD_TRY(hdb::normalise_scan(sb, pl->rms0.as<float>(), pl->dm0_scan.as<float>(), spitch, x, s,
                             pl->plan->d_err));
  for (size_t u = 0; u < U; u++) {
    int* mask = pl->mask.as<int>() + u * nsamps;
    HD_TRY(hdb::rfi_mask(x + u * spitch, pl->dm0_scan.as<float>() + u * spitch, nsamps,
                         boxcar_max, rfi_tol, mask, pl->fmask.as<int>(), s));
    HD_TRY(hdb::launch_zap(tf + u * nsamps * nchans, nsamps, (int)nchans, mask,
                           (unsigned)(nsmooth / 4), fb_ft ? fb_ft + u * nchans * pitch : nullptr,
                           pitch, out_tf ? out_tf + u * nsamps * nchans : nullptr, s));
  }
  return HD_NO_ERROR;
}

void write_cand_file(hd_pipeline pl, const std::vector<hd_candidate>& cands, size_t beam,
                     size_t first_idx) {
  if (!pl->has_output_dir) return;
  char buffer[64];
  time_t off = pl->params.spectra_per_second
                   ? (time_t)(first_idx / pl->params.spectra_per_second)
                   : (time_t)0;
  time_t now = pl->params.utc_start + off;
  struct tm tmv;
  gmtime_r(&now, &tmv);
  strftime(buffer, sizeof(buffer), "%Y-%m-%d-%H:%M:%S", &tmv);
  char bname[32];
  snprintf(bname, sizeof(bname), "%02zu", beam + 1);
  std::string fn = pl->output_dir + "/" + buffer + "_" + bname + ".cand";
  FILE* f = fopen(fn.c_str(), "w");
  if (!f) {
    fprintf(stdout, "Skipping dump due to bad file open on %s\n", fn.c_str());
    return;
  }
  for (const hd_candidate& c : cands)
    fprintf(f, "%g\t%zu\t%g\t%zu\t%zu\t%g\t%zu\t%zu\t%zu\t%zu\t\n", (double)c.snr, c.samp_idx,
            (double)c.time, c.filter, c.dm_trial, (double)c.dm, c.members, c.begin, c.end,
            c.beam);
  fclose(f);
}

}  // namespace

extern "C" {

hd_error hd_create_pipeline(hd_pipeline* pipeline_, hd_params params) {
  if (!pipeline_) return HD_INVALID_POINTER;
  *pipeline_ = nullptr;
  hd_pipeline pl = new (std::nothrow) hd_pipeline_t();
  if (!pl) return HD_MEM_ALLOC_FAILED;
  pl->params = params;
  if (params.output_dir) pl->output_dir = params.output_dir;
  else pl->has_output_dir = false;
  pl->params.output_dir = pl->has_output_dir ? pl->output_dir.c_str() : nullptr;
  for (unsigned z = 0; z < params.num_channel_zaps && params.channel_zaps; z++)
    pl->zaps.push_back(params.channel_zaps[z]);
  pl->params.channel_zaps = pl->zaps.empty() ? nullptr : pl->zaps.data();
  pl->params.coincidencer_host = nullptr;
  pl->params.sigproc_file = nullptr;
  // allocate_gpu (pipeline.cu:80-124)
  cudaError_t ce = cudaSetDevice(params.gpu_id);
  if (ce != cudaSuccess) { delete pl; return cuda_err(ce); }
  pl->device = params.gpu_id;
  if (const char* g = std::getenv("HDB_NO_GRAPH"))
    if (g[0] == '1') pl->use_graphs = false;
  if (cudaStreamCreateWithFlags(&pl->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&pl->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete pl;
    return HD_PRIOR_GPU_ERROR;
  }
  for (auto& e : pl->ev) cudaEventCreate(&e);
  for (auto& e : pl->chunk_ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  for (auto& q : pl->pf) cudaEventCreateWithFlags(&q.done, cudaEventDisableTiming);
  if (cudaMallocHost(&pl->h_small, 64 * sizeof(unsigned)) != cudaSuccess) {
    delete pl;
    return HD_MEM_ALLOC_FAILED;
  }
  dedisp_error de = dedisp_create_plan(&pl->plan, params.nchans, params.dt, params.f0, params.df);
  if (de == DEDISP_NO_ERROR)
    de = dedisp_generate_dm_list(pl->plan, params.dm_min, params.dm_max, params.dm_pulse_width,
                                 params.dm_tol);
  // adaptive dt (pipeline.cu:187-196)
  if (de == DEDISP_NO_ERROR && params.use_scrunching)
    de = dedisp_enable_adaptive_dt(pl->plan, params.dm_pulse_width, params.scrunch_tol);
  if (de != DEDISP_NO_ERROR) {
    delete pl;
    return dedisp_err(de);
  }
  *pipeline_ = pl;
  return HD_NO_ERROR;
}

hd_size hd_get_max_overlap(hd_pipeline pl, hd_size nbeams) {
  if (!pl) return 0;
  return (pl->params.boxcar_max + dedisp_get_max_delay(pl->plan)) * nbeams;
}

hd_error hd_preallocate(hd_pipeline pl, hd_size nsamps, hd_size nbeams) {
  if (!pl) return HD_INVALID_PIPELINE;
  (void)nsamps;
  (void)nbeams;
  return HD_NO_ERROR;
}

hd_error hd_set_narrow_band(hd_pipeline pl, int enable) {
  if (!pl) return HD_INVALID_PIPELINE;
  pl->narrow_band = enable != 0;
  return HD_NO_ERROR;
}

hd_error hd_set_cleaning(hd_pipeline pl, int enable) {
  if (!pl) return HD_INVALID_PIPELINE;
  pl->cleaning = enable != 0;
  return HD_NO_ERROR;
}

// One gulp of `U` units (independent filterbanks of nsamps x nchans bytes,
// each holding nbeams time-concatenated beams) through one batched pass:
// every stage runs over all units' DM series at once; giants carry a DM key
// that keeps units more than dm_tol apart, so clustering never links units
// and each unit's result equals a separate hd_execute of it.
// Per-width constants of the boxcar loop (pipeline.cu:657-776) for trials
// searched at scrunch factor scr: nc_s filtered-input samples, stride_s
// samples per beam, cur_delay the scrunched largest delay.
static std::vector<hdb::WidthInfo> widths_for(const hd_params& P, size_t scr, size_t nc_s,
                                              size_t stride_s, size_t cur_delay) {
  std::vector<hdb::WidthInfo> wi;
  const size_t Bmax = P.boxcar_max;
  const size_t rel_bmax = Bmax / scr;
  const size_t max_nf = nc_s + 1 - rel_bmax;
  const size_t cur_off = rel_bmax / 2;
  for (size_t fw = scr; fw <= Bmax; fw *= 2) {
    hdb::WidthInfo w{};
    const size_t rel_fw = fw / scr;
    size_t rel_min_ts = std::max<size_t>(P.min_tscrunch_width / scr, 1);
    size_t ts = std::max<size_t>(2 * rel_fw / rel_min_ts, 1);
    w.width = (int)rel_fw;
    w.ts = (int)ts;
    w.ahead = (int)((rel_fw - 1) / 2 + 1);
    w.behind = (int)(rel_fw / 2);
    w.filter_idx = (int)log2u(fw);
    w.n = (unsigned)((max_nf - 1) / ts + 1);
    w.bn = (unsigned)(stride_s - (cur_delay + rel_bmax));
    w.merge_dist = (unsigned)(P.cand_sep_time * (rel_fw / ts));
    w.rel_off = (unsigned)(cur_off / ts);
    w.prev_cover = (int)wi.size() - 1;
    w.scr = (int)(scr * ts);
    wi.push_back(w);
  }
  return wi;
}

// Giant-rate bail-out per unit (pipeline.cu:779-787) from each unit's first
// giant (first[u] .. first[u + 1]): the running count only grows, so it
// trips exactly when the final count does.
static void giant_rate_bail_out(hd_pipeline pl, size_t U, size_t nsamps,
                                const std::vector<unsigned>& first, hd_error* statuses,
                                std::vector<char>& too_many, bool& any_ok, bool& any_too_many) {
  const hd_params& P = pl->params;
  too_many.assign(U, 0);
  any_ok = any_too_many = false;
  float mins = (float)((double)((float)nsamps * P.dt) / 60.0);
  for (size_t u = 0; u < U; u++) {
    unsigned gu = first[u + 1] - first[u];
    if (P.max_giant_rate != 0.0f && ((float)gu / mins > P.max_giant_rate)) too_many[u] = 1;
    if (too_many[u]) any_too_many = true;
    else any_ok = true;
    if (statuses && too_many[u]) statuses[u] = HD_TOO_MANY_EVENTS;
  }
}

// Merged candidate rows -> each unit's candidates and .cand file
// (pipeline.cu:1012-1039).
static void emit_candidates(hd_pipeline pl, size_t U, const hdb::GroupRow* rows,
                            unsigned ngroups, const std::vector<char>& too_many, size_t nsamps,
                            size_t nbeams, size_t first_idx, const hd_size* beams,
                            size_t nsamps_processed) {
  const hd_params& P = pl->params;
  const unsigned nsamps_beam = (unsigned)(nsamps / nbeams);
  const unsigned nsamps_valid = (unsigned)(nsamps_processed / nbeams);
  for (unsigned i = 0; i < ngroups; i++) {
    const hdb::GroupRow& r = rows[i];
    const size_t u = (size_t)r.unit;
    if (u >= U || too_many[u]) continue;
    const size_t beam_base = beams ? (size_t)beams[u] : (size_t)P.beam + u * nbeams;
    size_t ind = (size_t)r.ind;
    size_t beam_idx = (size_t)std::floor((float)ind / (float)nsamps_beam);
    size_t beam_start = beam_idx * nsamps_beam + (P.boxcar_max / 2);
    size_t beam_end = beam_start + nsamps_valid;
    if (!(beam_start <= ind && ind < beam_end)) continue;
    hd_candidate c;
    size_t samp_off = ind - (size_t)nsamps_beam * beam_idx;
    c.samp_idx = first_idx + samp_off;
    c.snr = std::isinf(r.peak) ? 0.0f : r.peak;
    c.time = P.dt * (float)c.samp_idx;
    c.filter = (hd_size)r.filter;
    c.dm_trial = (hd_size)r.dm_ind;
    c.dm = r.dm;
    c.members = (hd_size)r.members;
    c.begin = first_idx + ((size_t)r.begin % nsamps_beam);
    c.end = first_idx + ((size_t)r.end % nsamps_beam);
    c.beam = beam_base + beam_idx + 1;
    pl->unit_cands[u].push_back(c);
    pl->unit_meta[u].push_back({(unsigned)u, (unsigned)ind, (int)r.dm_ind, (int)r.filter});
  }
  for (size_t u = 0; u < U; u++) {
    const size_t beam_base = beams ? (size_t)beams[u] : (size_t)P.beam + u * nbeams;
    write_cand_file(pl, pl->unit_cands[u], beam_base, first_idx);
    pl->cands.insert(pl->cands.end(), pl->unit_cands[u].begin(), pl->unit_cands[u].end());
    pl->meta.insert(pl->meta.end(), pl->unit_meta[u].begin(), pl->unit_meta[u].end());
  }
}

// ---- the gulp as a CUDA graph -------------------------------------------------
// Capture-safe enqueue of one gulp of U device-resident 8-bit filterbanks at
// native resolution: no host synchronisation, no allocation (every buffer was
// sized by graph_gulp), hits and giants at the shape's capacities, clustering
// as `pairs` sweep pairs that stop themselves at the fixed point.
struct GulpGeom {
  size_t U, nsamps, nbeams, C, D, max_delay, dm_tol, gap, nc, fb_bytes, pitch, ft_unit,
      dd_pitch, NS, stride, bcount, scan_pitch, nsmooth, nsw, gcap_groups;
  unsigned ntiles;
};

// With `events`, the stage boundaries of hd_get_timing are recorded by event
// nodes of the graph (the events of the host-sized path, at the same points).
static hd_error enqueue_gulp(hd_pipeline pl, const hd_byte* const* fbs, bool resident,
                             const GulpGeom& g, const std::vector<hdb::WidthInfo>& wi,
                             unsigned hcap, unsigned gcap, unsigned pairs, bool events) {
  const hd_params& P = pl->params;
  dedisp_plan plan = pl->plan;
  cudaStream_t s = pl->stream;
  auto mark = [&](int k) {
    return events ? cudaEventRecordWithFlags(pl->ev[k], s, cudaEventRecordExternal)
                  : cudaSuccess;
  };
  HD_TRY(cudaMemsetAsync(plan->d_err, 0, sizeof(unsigned), s));
  if (!resident)
    HD_TRY(copy_units(pl->fb_tf.as<uint8_t>(), fbs, 0, g.U, g.fb_bytes, cudaMemcpyDeviceToDevice,
                      s));
  HD_TRY(mark(1));
  if (pl->cleaning) {
    hd_error he = clean_units(pl, g.U, pl->fb_tf.as<uint8_t>(), g.nsamps, g.C, P.dt,
                              P.baseline_length, P.rfi_tol, 64, g.nbeams,
                              pl->fb_ft.as<uint8_t>(), g.pitch, nullptr);
    if (he != HD_NO_ERROR) return he;
  } else {
    HD_TRY(hdb::input_to_ft(pl->fb_tf.as<uint8_t>(), g.nsamps, (int)g.C, 8,
                            pl->fb_ft.as<uint8_t>(), g.pitch, s, g.U, g.ft_unit));
  }
  HD_TRY(mark(2));
  float* dd = pl->dd.as<float>();
  dedisp_error de = hdb::plan_dedisperse_ft(plan, pl->fb_ft.as<uint8_t>(), g.pitch, g.nsamps, dd,
                                            g.dd_pitch, s, g.U, g.ft_unit, g.D * g.dd_pitch);
  if (de != DEDISP_NO_ERROR) return dedisp_err(de);
  HD_TRY(cudaMemset2DAsync(dd + g.nc, g.dd_pitch * sizeof(float), 0, sizeof(float), g.NS, s));
  HD_TRY(mark(3));

  hdb::SeriesBatch sb{dd, g.dd_pitch, (int)g.NS, g.nc, g.stride, g.bcount, (int)g.nbeams};
  hdb::TreeScratch ws{pl->ws_a.as<float>(), pl->ws_b.as<float>(), pl->ws_a.cap / sizeof(float)};
  float* scan = pl->scan.as<float>();
  HD_TRY(hdb::remove_baseline(sb, g.nsmooth, pl->base.as<float>(), ws, s));
  HD_TRY(hdb::rms_beams(sb, pl->rms.as<float>(), ws, s));
  HD_TRY(hdb::normalise_scan(sb, pl->rms.as<float>(), scan, g.scan_pitch, nullptr, s, plan->d_err));
  HD_TRY(mark(4));

  const int nw = (int)wi.size();
  hdb::WidthCtx wctx{};
  wctx.scan = scan;
  wctx.scan_pitch = g.scan_pitch;
  wctx.nser = (int)g.NS;
  wctx.stride = g.stride;
  wctx.nbeams = (int)g.nbeams;
  wctx.offset = (int)(P.boxcar_max / 2);
  wctx.nw = nw;
  wctx.winfo = pl->winfo.as<hdb::WidthInfo>();
  wctx.host_winfo = wi.data();
  wctx.scan_len = g.nc + 1;
  wctx.dms_per_unit = (int)g.D;
  wctx.dm_key_gap = (int)g.gap;
  wctx.dm_offset = 0;
  wctx.norm = pl->norm.as<float>();
  wctx.thresh = P.detect_thresh;
  wctx.gmax = pl->gmax.as<float>();
  wctx.gmax_cap = g.gcap_groups;
  int n_ts1 = 0;
  while (n_ts1 < nw && wi[n_ts1].ts == 1) n_ts1++;
  if (n_ts1 > 0) HD_TRY(hdb::block_rms(wctx, wi.data(), 0, n_ts1, ws, s));
  for (int w = n_ts1; w < nw; w++) HD_TRY(hdb::block_rms(wctx, wi.data(), w, w + 1, ws, s));

  hdb::HitBuffers hb{};
  hb.tile_list = pl->tile_list.as<unsigned>();
  hb.tile_list_n = hb.tile_list + g.NS * g.ntiles;
  hb.tile_cnt = pl->tile_cnt.as<unsigned>();
  hb.tile_off = pl->tile_off.as<unsigned>();
  hb.sw_cnt = pl->sw_cnt.as<unsigned>();
  hb.sw_off = pl->sw_off.as<unsigned>();
  HD_TRY(hdb::count_hits(wctx, hb, g.ntiles, s));
  HD_TRY(hdb::scan_hit_counts(wctx, hb, s));
  unsigned* small = pl->small.as<unsigned>();
  unsigned* scan_tmp = pl->scan_tmp.as<unsigned>();
  HD_TRY(hdb::scan_u32(hb.sw_cnt, hb.sw_off, g.nsw, small, scan_tmp, s));
  hb.ind = pl->hit_ind.as<unsigned>();
  hb.val = pl->hit_val.as<float>();
  hb.sw = pl->hit_sw.as<unsigned>();
  hb.cap = hcap;
  HD_TRY(hdb::write_hits(wctx, hb, s));
  HD_TRY(mark(5));

  hdb::GiantBuffers gb{};
  pl->main_giants.view(gb);
  gb.head = pl->head.as<unsigned>();
  gb.gid = pl->gid.as<unsigned>();
  gb.cap = gcap;
  HD_TRY(hdb::giants_dev(wctx, hb, small, hcap, gb, gcap, small + 1, scan_tmp, s));
  HD_TRY(mark(6));
  hdb::ClusterArgs ca{0, P.cand_sep_time, P.cand_sep_filter, g.dm_tol,
                      (unsigned long long)(g.nsamps / g.nbeams), 0};
  HD_TRY(hdb::cluster_merge_dev(ca, gb, gcap, small + 1, (int)g.U, (int)g.gap,
                                pl->unit_off.as<unsigned>(), pl->geo.as<int>(), small + 32,
                                (int)pairs, plan->d_dm_list, pl->root_flag.as<unsigned>(),
                                pl->root_off.as<unsigned>(), small + 16, scan_tmp,
                                pl->mkey.as<unsigned long long>(), pl->rows.as<hdb::GroupRow>(),
                                s));
  return HD_NO_ERROR;
}

// Capacity for a total first seen as n: room for 4x as many, at least `floor`.
static unsigned graph_capacity(unsigned n, unsigned floor) {
  const unsigned long long c = std::max<unsigned long long>(4ull * n + 1024, floor);
  return (unsigned)std::min<unsigned long long>((c + 1023) / 1024 * 1024, 0x7FFFF000ull);
}

// One gulp as a CUDA graph replay.  Returns false when the host-sized path is
// to search this gulp instead: a shape seen for the first time (that search
// sizes the shape's capacities), a gulp with nothing to search, a failed
// capture, or a replay whose totals overflowed the capacities or whose
// clustering needed more sweeps than were captured (the capacities grow for
// the next gulp of the shape, and no clamped result is reported).  Returns
// true with *result set when the graph's results stand or a CUDA call failed.
static bool graph_gulp(hd_pipeline pl, const hd_byte* const* fbs, size_t U, bool resident,
                       size_t nsamps, size_t nbeams, size_t first_idx, const hd_size* beams,
                       hd_error* statuses, size_t nsamps_processed, hd_error* result) {
  const hd_params& P = pl->params;
  dedisp_plan plan = pl->plan;
  GulpGeom g{};
  g.U = U;
  g.nsamps = nsamps;
  g.nbeams = nbeams;
  g.C = P.nchans;
  g.D = plan->dm_list.size();
  g.max_delay = plan->max_delay;
  g.stride = nsamps / nbeams;
  const size_t Bmax = P.boxcar_max;
  if (g.max_delay >= g.stride || g.max_delay + Bmax > g.stride) return false;
  bool withhold = false;
  if (const char* e = std::getenv("HDB_TEST_WITHHOLD_STAGE")) withhold = e[0] == '1';
  const std::vector<size_t> shape = {U, nsamps, nbeams, g.C, g.D, g.max_delay,
                                     (size_t)pl->cleaning, (size_t)resident,
                                     (size_t)plan->forced_dm_block,
                                     (size_t)plan->forced_time_block, (size_t)plan->tune,
                                     (size_t)withhold, (size_t)plan->gen};
  hd_pipeline_t::GraphShape* gs = nullptr;
  for (auto& x : pl->graph_shapes)
    if (x.key == shape) gs = &x;
  if (!gs) {
    pl->pending_shape = shape;
    return false;
  }
  if (gs->broken) return false;
  const unsigned hcap = gs->hcap, gcap = gs->gcap, pairs = gs->pairs;

  g.dm_tol = std::min<size_t>(P.cand_sep_dm, g.D);
  g.gap = g.D + g.dm_tol + 2;
  g.nc = nsamps - g.max_delay;
  g.fb_bytes = nsamps * g.C;
  g.pitch = hdb::ft_pitch(plan, nsamps);
  g.ft_unit = g.pitch * g.C;
  g.dd_pitch = round_up(g.nc + 1, 4);
  g.NS = U * g.D;
  g.bcount = g.stride - g.max_delay;
  g.scan_pitch = round_up(g.nc + 1, 4);
  g.nsmooth = (size_t)(P.baseline_length / (2 * P.dt));
  const std::vector<hdb::WidthInfo> wi = widths_for(P, 1, g.nc, g.stride, g.max_delay);
  if (wi.empty()) return false;
  const size_t nw = wi.size();
  g.ntiles = (unsigned)((wi[0].n + 2047) / 2048);
  g.nsw = g.NS * nw;
  g.gcap_groups = g.NS * nw * (nbeams * g.stride / 3125 + 5);

  // every buffer at the size the host-sized path gives this shape, with the
  // hit and giant lists at the capacities
  cudaError_t ae = cudaSuccess;
  auto need = [&](DevBuf& b, size_t bytes) {
    if (ae == cudaSuccess) ae = b.ensure(bytes);
  };
  if (!resident) need(pl->fb_tf, U * g.fb_bytes);
  need(pl->fb_ft, U * g.ft_unit);
  need(pl->dd, g.NS * g.dd_pitch * sizeof(float));
  const size_t tcap = std::max({tree_cap(g.NS * nbeams, g.stride),
                                tree_cap(g.NS * (log2u(Bmax) + 1), nbeams * g.stride),
                                hdb::baseline_scratch(g.stride, g.nsmooth, g.NS * nbeams)});
  need(pl->ws_a, tcap * sizeof(float));
  need(pl->ws_b, tcap * sizeof(float));
  need(pl->base, (g.NS * nbeams * hdb::baseline_samples(g.stride, g.nsmooth) + 64) *
                     sizeof(float));
  need(pl->rms, g.NS * nbeams * sizeof(float) + 64);
  need(pl->scan, g.NS * g.scan_pitch * sizeof(float));
  need(pl->small, 64 * sizeof(unsigned));
  need(pl->winfo, nw * sizeof(hdb::WidthInfo));
  need(pl->norm, g.NS * nw * sizeof(float));
  need(pl->gmax, g.gcap_groups * sizeof(float));
  need(pl->tile_cnt, g.nsw * g.ntiles * sizeof(unsigned));
  need(pl->tile_off, g.nsw * g.ntiles * sizeof(unsigned));
  need(pl->sw_cnt, (g.nsw + 1) * sizeof(unsigned));
  need(pl->sw_off, (g.nsw + 1) * sizeof(unsigned));
  need(pl->tile_list, (g.NS * g.ntiles + 1) * sizeof(unsigned));
  const size_t H = (size_t)hcap + 1, G = (size_t)gcap + 1;
  need(pl->hit_ind, H * sizeof(unsigned));
  need(pl->hit_val, H * sizeof(float));
  need(pl->hit_sw, H * sizeof(unsigned));
  need(pl->head, H * sizeof(unsigned));
  need(pl->gid, H * sizeof(unsigned));
  hd_pipeline_t::GiantSet& m = pl->main_giants;
  need(m.key, G * sizeof(unsigned long long));
  need(m.peak, G * sizeof(float));
  need(m.ind, G * sizeof(unsigned long long));
  need(m.begin, G * sizeof(unsigned long long));
  need(m.end, G * sizeof(unsigned long long));
  need(m.filter, G * sizeof(int));
  need(m.dm, G * sizeof(int));
  need(m.label, G * sizeof(int));
  need(pl->scan_tmp,
       hdb::scan_tmp_words(std::max({g.nsw, (size_t)hcap, (size_t)gcap})) * sizeof(unsigned));
  need(pl->root_flag, G * sizeof(unsigned));
  need(pl->root_off, G * sizeof(unsigned));
  need(pl->mkey, 2 * G * sizeof(unsigned long long));
  need(pl->rows, G * sizeof(hdb::GroupRow));
  need(pl->unit_off, (U + 1) * sizeof(unsigned));
  need(pl->geo, 4 * sizeof(int));
  if (ae != cudaSuccess) return false;  // the host-sized path reports it
  const size_t spec = std::min<size_t>(gcap, kSpecRows);
  if (pl->ensure_rows_host(std::max<size_t>(spec, 1)) != cudaSuccess) return false;

  // the graph's key: the shape, then every device address it uses
  std::vector<size_t> key = shape;
  key.push_back(hcap);
  key.push_back(gcap);
  key.push_back(pairs);
  for (size_t u = 0; u < U; u++) key.push_back(resident ? 0 : (size_t)fbs[u]);
  for (const DevBuf* b : {&pl->fb_tf, &pl->fb_ft, &pl->dm0, &pl->dm0_scan, &pl->base, &pl->rms,
                          &pl->mask, &pl->fmask, &pl->rms0, &pl->dd, &pl->scan, &pl->ws_a,
                          &pl->ws_b, &pl->winfo, &pl->norm, &pl->gmax, &pl->tile_list,
                          &pl->tile_cnt, &pl->tile_off, &pl->sw_cnt, &pl->sw_off, &pl->hit_ind,
                          &pl->hit_val, &pl->hit_sw, &pl->head, &pl->gid, &m.key, &m.peak,
                          &m.ind, &m.begin, &m.end, &m.filter, &m.dm, &m.label, &pl->scan_tmp,
                          &pl->small, &pl->root_flag, &pl->root_off, &pl->mkey, &pl->rows,
                          &pl->unit_off, &pl->geo}) {
    key.push_back((size_t)b->p);
    key.push_back(b->cap);
  }
  for (const void* q : {(const void*)plan->d_delays, (const void*)plan->d_blk_min[0],
                        (const void*)plan->d_blk_min[1], (const void*)plan->d_blk_min[2],
                        (const void*)plan->d_active, (const void*)plan->d_dm_list,
                        (const void*)plan->d_err})
    key.push_back((size_t)q);

  cudaStream_t s = pl->stream;
  hd_pipeline_t::GraphGulp* gg = nullptr;
  for (auto& x : pl->graphs)
    if (x.key == key) gg = &x;
  if (!gg) {
    hd_pipeline_t::GraphGulp ng;
    ng.key = key;
    cudaError_t ce = cudaErrorUnknown;
    hd_error he = HD_NO_ERROR;
    // with the stage events first; without them if that capture fails
    for (int events = 1; events >= 0 && !ng.exec; events--) {
      const unsigned long long l0 = hdb::launch_count();
      ce = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
      if (ce == cudaSuccess) {
        he = enqueue_gulp(pl, fbs, resident, g, wi, hcap, gcap, pairs, events != 0);
        cudaGraph_t graph = nullptr;
        ce = cudaStreamEndCapture(s, &graph);
        if (he == HD_NO_ERROR && ce == cudaSuccess && graph)
          ce = cudaGraphInstantiate(&ng.exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
      }
      ng.launches = (long long)(hdb::launch_count() - l0);
      hdb::add_launches(-ng.launches);
      if (!ng.exec) cudaGetLastError();
      ng.events = events != 0;
    }
    if (ce != cudaSuccess || he != HD_NO_ERROR || !ng.exec) {
      // not capturable here: this shape stays on the host-sized path
      if (ng.exec) cudaGraphExecDestroy(ng.exec);
      cudaGetLastError();
      gs->broken = true;
      return false;
    }
    // a few graphs per pipeline (the prefetched form rotates three input
    // buffers); the least recently used goes
    if (pl->graphs.size() >= 6) {
      size_t old = 0;
      for (size_t i = 1; i < pl->graphs.size(); i++)
        if (pl->graphs[i].used < pl->graphs[old].used) old = i;
      cudaGraphExecDestroy(pl->graphs[old].exec);
      pl->graphs.erase(pl->graphs.begin() + old);
    }
    pl->graphs.push_back(ng);
    gg = &pl->graphs.back();
  }
  gg->used = ++pl->graph_clock;

#define GG_TRY(x)                         \
  do {                                    \
    cudaError_t e_ = (x);                 \
    if (e_ != cudaSuccess) {              \
      *result = cuda_err(e_);             \
      return true;                        \
    }                                     \
  } while (0)
  // the width table is the pipeline's (another shape's gulp may have
  // replaced it since the capture)
  GG_TRY(cudaMemcpyAsync(pl->winfo.p, wi.data(), nw * sizeof(hdb::WidthInfo),
                         cudaMemcpyHostToDevice, s));
  cudaEventRecord(pl->ev[0], s);
  GG_TRY(cudaGraphLaunch(gg->exec, s));
  hdb::add_launches(gg->launches);
  std::vector<unsigned>& first = pl->unit_first;
  first.assign(U + 1, 0);
  GG_TRY(cudaMemcpyAsync(pl->h_small, pl->small.p, 64 * sizeof(unsigned), cudaMemcpyDeviceToHost,
                         s));
  GG_TRY(cudaMemcpyAsync(pl->h_small + 20, plan->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                         s));
  GG_TRY(cudaMemcpyAsync(first.data(), pl->unit_off.p, (U + 1) * sizeof(unsigned),
                         cudaMemcpyDeviceToHost, s));
  GG_TRY(cudaMemcpyAsync(pl->h_rows, pl->rows.p, spec * sizeof(hdb::GroupRow),
                         cudaMemcpyDeviceToHost, s));
  cudaEventRecord(pl->ev[7], s);
  GG_TRY(cudaStreamSynchronize(s));
  const unsigned nh = pl->h_small[0], ngi = pl->h_small[1];
  if (nh > hcap || ngi > gcap) {
    gs->hcap = std::max(hcap, graph_capacity(nh, hcap));
    gs->gcap = std::max(gcap, graph_capacity(ngi, gcap));
    pl->drop_graphs(shape);
    return false;
  }
  int conv = -1;
  for (unsigned p = 0; p < pairs && conv < 0; p++)
    if (pl->h_small[32 + 2 * p + 1] == 0) conv = (int)p;
  if (conv < 0) {
    gs->pairs = std::min(pairs + 2, 16u);
    if (gs->pairs == pairs) gs->broken = true;
    pl->drop_graphs(shape);
    return false;
  }
  if (pl->h_small[20]) {
    *result = HD_INTERNAL_GPU_ERROR;
    return true;
  }
  unsigned ngroups = pl->h_small[16];
  if (ngroups > spec) {
    std::vector<hdb::GroupRow> head(pl->h_rows, pl->h_rows + spec);
    GG_TRY(pl->ensure_rows_host(ngroups));
    std::copy(head.begin(), head.end(), pl->h_rows);
    GG_TRY(cudaMemcpyAsync(pl->h_rows + spec, pl->rows.as<hdb::GroupRow>() + spec,
                           (ngroups - spec) * sizeof(hdb::GroupRow), cudaMemcpyDeviceToHost, s));
    GG_TRY(cudaStreamSynchronize(s));
  }
#undef GG_TRY
  std::vector<char> too_many;
  bool any_ok = false, any_too_many = false;
  giant_rate_bail_out(pl, U, nsamps, first, statuses, too_many, any_ok, any_too_many);
  if (!any_ok) ngroups = 0;
  pl->searched = true;
  pl->last_nsamps = nsamps;
  pl->last_len = g.nc;
  pl->last_scan_pitch = g.scan_pitch;
  pl->last_units = U;
  pl->last_giants = (any_ok && ngi > 0) ? ngi : 0;
  pl->last_gap = g.gap;
  pl->obs_hits = nh;
  pl->obs_giants = ngi;
  pl->obs_pairs = (unsigned)conv + 1;
  emit_candidates(pl, U, pl->h_rows, ngroups, too_many, nsamps, nbeams, first_idx, beams,
                  nsamps_processed);
  auto el = [&](int a, int b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pl->ev[a], pl->ev[b]) != cudaSuccess) ms = 0.f;
    return ms;
  };
  pl->timing[0] = el(0, 7);
  if (gg->events) {
    pl->timing[7] = el(0, 1);
    pl->timing[1] = el(1, 2);
    pl->timing[2] = el(2, 3);
    pl->timing[3] = el(3, 4);
    pl->timing[4] = el(4, 5);
    pl->timing[5] = el(5, 6);
    pl->timing[6] = el(6, 7);
  }
  cudaGetLastError();
  pl->last_graph = true;
  pl->graph_replays++;
  *result = any_too_many ? HD_TOO_MANY_EVENTS : HD_NO_ERROR;
  return true;
}

static hd_error execute_units(hd_pipeline pl, const hd_byte* const* fbs, size_t U, bool on_device,
                              hd_size nsamps, hd_size nbits, hd_size first_idx, hd_size nbeams,
                              const hd_size* beams, hd_error* statuses,
                              hd_size* nsamps_processed, bool graph = false) {
  if (!pl) return HD_INVALID_PIPELINE;
  const bool resident = pl->fb_resident;
  pl->fb_resident = false;
  if (!fbs || !nsamps_processed || U == 0) return HD_INVALID_POINTER;
  for (size_t u = 0; u < U; u++)
    if (!fbs[u]) return HD_INVALID_POINTER;
  // 1, 2, 4, 8 or 16-bit samples (dedisp's widths; packed little-endian,
  // channel-fastest).  Cleaning and the resident prefetched gulp work on
  // bytes; adaptive dt averages byte values, so 16-bit input searches at
  // native resolution.
  if (!hdb::nbits_supported(nbits)) return HD_INVALID_NBITS;
  if (nbits != 8 && (pl->cleaning || resident)) return HD_INVALID_NBITS;
  if (nbits == 16 && pl->plan->adaptive) return HD_INVALID_NBITS;
  const hd_params& P = pl->params;
  const size_t C = P.nchans;
  if (C % 4 != 0 || nbeams == 0 || (C * nbits) % 32 != 0) return HD_INVALID_STRIDE;
  if (nbits != 8)
    for (size_t u = 0; u < U; u++)
      if (on_device && (reinterpret_cast<uintptr_t>(fbs[u]) & 3)) return HD_INVALID_POINTER;
  if (P.min_tscrunch_width < 2) return HD_INVALID_STRIDE;
  // sample, hit and giant indices are kept in 31/32 bits on the device
  if (nsamps >= 0x7FFFFFFFull) return HD_INVALID_STRIDE;
  if (cudaSetDevice(pl->device) != cudaSuccess) return HD_INVALID_DEVICE_INDEX;
  cudaStream_t s = pl->stream;
  pl->cands.clear();
  pl->unit_cands.assign(U, {});
  pl->meta.clear();
  pl->unit_meta.assign(U, {});
  pl->searched = false;
  pl->unit_first.assign(U + 1, 0);
  pl->last_giants = 0;
  std::memset(pl->timing, 0, sizeof(pl->timing));
  if (statuses)
    for (size_t u = 0; u < U; u++) statuses[u] = HD_NO_ERROR;

  // killmask: manual channel zaps (clean_filterbank_rfi.cu:530-545)
  std::vector<int> km(C, 1);
  for (const hd_range_t& z : pl->zaps)
    for (size_t j = z.start; j < z.end; j++)
      if (j < C) km[j] = 0;
  dedisp_set_killmask(pl->plan, km.data());
  dedisp_error de = hdb::plan_prepare(pl->plan);
  if (de != DEDISP_NO_ERROR) return dedisp_err(de);
  const size_t max_delay = pl->plan->max_delay;
  const size_t D = pl->plan->dm_list.size();
  // series of all units share the kernels' y/z grid dimensions
  if (U * D > 65535) return HD_INVALID_STRIDE;
  // DM keys: unit u's trial d is u * gap + d with gap - (D - 1) > dm_tol
  const size_t dm_tol = std::min<size_t>(P.cand_sep_dm, D);
  const size_t gap = D + dm_tol + 2;
  if ((U + 1) * gap > 0x7FFFFFFFull) return HD_INVALID_STRIDE;
  if (nsamps <= max_delay) {
    *nsamps_processed = 0;
    return HD_TOO_FEW_NSAMPS;
  }
  const size_t nc = nsamps - max_delay;  // nsamps_computed
  *nsamps_processed = nsamps - nbeams * (P.boxcar_max + max_delay);
  if (nsamps < nbeams * (P.boxcar_max + max_delay)) *nsamps_processed = 0;

  // the batched forms with device-resident input: a shape seen before runs as
  // one CUDA graph replay
  pl->last_graph = false;
  pl->pending_shape.clear();
  if (graph && on_device && nbits == 8 && pl->use_graphs && pl->plan->groups.empty() &&
      !pl->narrow_band) {
    hd_error ge = HD_NO_ERROR;
    if (graph_gulp(pl, fbs, U, resident, nsamps, nbeams, first_idx, beams, statuses,
                   *nsamps_processed, &ge))
      return ge;
  }

  cudaEventRecord(pl->ev[0], s);
  HD_TRY(cudaMemsetAsync(pl->plan->d_err, 0, sizeof(unsigned), s));
  // ---- H2D, clean or channel-major copy, dedispersion ------------------------
  const size_t fb_bytes = nsamps * C * nbits / 8;
  const size_t pitch = hdb::ft_pitch(pl->plan, nsamps);
  const size_t ft_unit = pitch * C;
  const size_t dd_pitch = round_up(nc + 1, 4);
  const size_t NS = U * D;  // series of the batch, unit-major
  HD_TRY(pl->fb_tf.ensure(U * fb_bytes));
  // 16-bit input: the low-byte planes, then the high-byte planes
  HD_TRY(pl->fb_ft.ensure(U * ft_unit * (nbits == 16 ? 2 : 1)));
  HD_TRY(pl->dd.ensure(NS * dd_pitch * sizeof(float)));
  float* dd = pl->dd.as<float>();
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (!on_device && !pl->cleaning && U > 1 && pl->plan->groups.empty() && nbits == 8) {
    // pipelined: copy chunk k on the copy stream while chunk k - 1 is
    // transposed and dedispersed on the compute stream (the unit-major series
    // layout; adaptive dt lays series out by scrunch factor and dedisperses
    // all units at once)
    const size_t nch = std::min<size_t>(U, kMaxChunks);
    HD_TRY(cudaEventRecord(pl->ev[9], s));
    HD_TRY(cudaStreamWaitEvent(pl->copy_stream, pl->ev[9], 0));
    for (size_t k = 0; k < nch; k++) {
      const size_t u0 = U * k / nch, u1 = U * (k + 1) / nch;
      HD_TRY(copy_units(pl->fb_tf.as<uint8_t>(), fbs, u0, u1, fb_bytes, kind,
                        pl->copy_stream));
      HD_TRY(cudaEventRecord(pl->chunk_ev[k], pl->copy_stream));
    }
    HD_TRY(cudaEventRecord(pl->ev[1], pl->copy_stream));
    for (size_t k = 0; k < nch; k++) {
      const size_t u0 = U * k / nch, u1 = U * (k + 1) / nch;
      HD_TRY(cudaStreamWaitEvent(s, pl->chunk_ev[k], 0));
      HD_TRY(hdb::launch_transpose_tf_ft(pl->fb_tf.as<uint8_t>() + u0 * fb_bytes, nsamps,
                                         (int)C, pl->fb_ft.as<uint8_t>() + u0 * ft_unit, pitch,
                                         s, u1 - u0, ft_unit));
      if (k + 1 == nch) cudaEventRecord(pl->ev[2], s);
      de = hdb::plan_dedisperse_ft(pl->plan, pl->fb_ft.as<uint8_t>() + u0 * ft_unit, pitch,
                                   nsamps, dd + u0 * D * dd_pitch, dd_pitch, s, u1 - u0, ft_unit,
                                   D * dd_pitch);
      if (de != DEDISP_NO_ERROR) return dedisp_err(de);
    }
  } else {
    if (!resident) HD_TRY(copy_units(pl->fb_tf.as<uint8_t>(), fbs, 0, U, fb_bytes, kind, s));
    cudaEventRecord(pl->ev[1], s);
    if (pl->cleaning) {
      hd_error he = clean_units(pl, U, pl->fb_tf.as<uint8_t>(), nsamps, C, P.dt,
                                P.baseline_length, P.rfi_tol, 64, nbeams,
                                pl->fb_ft.as<uint8_t>(), pitch, nullptr);
      if (he != HD_NO_ERROR) return he;
    } else {
      HD_TRY(hdb::input_to_ft(pl->fb_tf.as<uint8_t>(), nsamps, (int)C, (int)nbits,
                              pl->fb_ft.as<uint8_t>(), pitch, s, U, ft_unit));
    }
    cudaEventRecord(pl->ev[2], s);
    if (nbits == 16) {
      // the high-byte plane's sums, then the low plane's, then lo + 256 hi
      HD_TRY(pl->dd_hi.ensure(NS * dd_pitch * sizeof(float)));
      de = hdb::plan_dedisperse_ft(pl->plan, pl->fb_ft.as<uint8_t>() + U * ft_unit, pitch,
                                   nsamps, pl->dd_hi.as<float>(), dd_pitch, s, U, ft_unit,
                                   D * dd_pitch);
      if (de != DEDISP_NO_ERROR) return dedisp_err(de);
    }
    de = hdb::plan_dedisperse_ft(pl->plan, pl->fb_ft.as<uint8_t>(), pitch, nsamps, dd, dd_pitch,
                                 s, U, ft_unit, D * dd_pitch);
    if (de != DEDISP_NO_ERROR) return dedisp_err(de);
    if (nbits == 16)
      HD_TRY(hdb::launch_combine_planes(dd, pl->dd_hi.as<float>(), dd_pitch, nc, NS, s));
  }
  // the element after each series is read (never used) by the baseline stretch
  if (pl->plan->groups.empty()) {
    HD_TRY(cudaMemset2DAsync(dd + nc, dd_pitch * sizeof(float), 0, sizeof(float), NS, s));
  } else {
    for (const auto& g : pl->plan->groups)
      HD_TRY(cudaMemset2DAsync(dd + U * g.d0 * dd_pitch + nc / g.s, dd_pitch * sizeof(float), 0,
                               sizeof(float), U * (g.d1 - g.d0), s));
  }
  cudaEventRecord(pl->ev[3], s);

  const size_t stride = nsamps / nbeams;
  const size_t Bmax = P.boxcar_max;
  // scrunch groups: trials [d0, d1) searched at factor s (one group of factor
  // 1 without adaptive dt); the series rows are group-major, group g's U * (d1
  // - d0) rows (unit-major inside) starting at row U * d0
  struct GroupSpec { size_t d0, d1, s; };
  std::vector<GroupSpec> groups;
  if (pl->plan->groups.empty()) {
    groups.push_back({0, D, 1});
  } else {
    for (const auto& g : pl->plan->groups) groups.push_back({g.d0, g.d1, g.s});
  }
  // the DM loop's break conditions (pipeline.cu:497-502,632-637): the first
  // trial that trips one ends the search, so only the groups before it run
  size_t ngs = 0;
  while (ngs < groups.size()) {
    const size_t scr = groups[ngs].s;
    const size_t cur_delay = max_delay / scr, stride_s = nsamps / nbeams / scr;
    if (cur_delay >= stride_s || cur_delay + Bmax / scr > stride_s) break;
    ngs++;
  }
  // the first (unscrunched) width of a trial must not be time-scrunched: its
  // block-RMS window would read the previous trial's filtered output
  for (size_t gi = 0; gi < ngs; gi++)
    if (std::max<size_t>(P.min_tscrunch_width / groups[gi].s, 1) < 2) return HD_INVALID_STRIDE;
  const bool search = ngs > 0;
  const bool multi = groups.size() > 1;
  unsigned nhits = 0, ngiants = 0;
  std::vector<hdb::WidthInfo> wi;
  hdb::WidthCtx wctx{};
  hdb::HitBuffers hb{};
  hdb::GiantBuffers gb{};
  std::vector<unsigned> group_giants(ngs, 0);
  const size_t scan_pitch = round_up(nc + 1, 4);
  if (search) {
    const size_t cap = std::max({tree_cap(NS * nbeams, stride),
                                 tree_cap(NS * (log2u(Bmax) + 1), nbeams * stride),
                                 hdb::baseline_scratch(stride, (size_t)(P.baseline_length /
                                                                        (2 * P.dt)),
                                                       NS * nbeams)});
    HD_TRY(pl->ws_a.ensure(cap * sizeof(float)));
    HD_TRY(pl->ws_b.ensure(cap * sizeof(float)));
    HD_TRY(pl->base.ensure((NS * nbeams *
                                hdb::baseline_samples(stride, (size_t)(P.baseline_length /
                                                                       (2 * P.dt))) +
                            64) * sizeof(float)));
    HD_TRY(pl->rms.ensure(NS * nbeams * sizeof(float) + 64));
    HD_TRY(pl->scan.ensure(NS * scan_pitch * sizeof(float)));
    HD_TRY(pl->small.ensure(64 * sizeof(unsigned)));
    pl->searched = !multi;  // patches read unscrunched series only
    pl->last_nsamps = nsamps;
    pl->last_len = nc;
    pl->last_scan_pitch = scan_pitch;
    pl->last_units = U;
    if (multi && pl->gsets.size() < ngs) pl->gsets.resize(ngs);
  }
  for (size_t gi = 0; gi < ngs; gi++) {
    const GroupSpec& G = groups[gi];
    const size_t scr = G.s, Dg = G.d1 - G.d0, NSg = U * Dg, row0 = U * G.d0;
    const size_t nc_s = nc / scr;
    const size_t cur_delay = max_delay / scr;
    const size_t stride_s = nsamps / nbeams / scr;
    const size_t rel_bmax = Bmax / scr;
    // ---- per-DM baseline, RMS, normalise + scan ------------------------------
    const size_t bcount = stride_s - cur_delay;
    float* ddg = dd + row0 * dd_pitch;
    float* scan_g = pl->scan.as<float>() + row0 * scan_pitch;
    hdb::SeriesBatch sb{ddg, dd_pitch, (int)NSg, nc_s, stride_s, bcount, (int)nbeams};
    const float cur_dt = P.dt * (float)scr;
    const size_t nsmooth = (size_t)(P.baseline_length / (2 * cur_dt));
    hdb::TreeScratch ws{pl->ws_a.as<float>(), pl->ws_b.as<float>(), pl->ws_a.cap / sizeof(float)};
    HD_TRY(hdb::remove_baseline(sb, nsmooth, pl->base.as<float>(), ws, s));
    HD_TRY(hdb::rms_beams(sb, pl->rms.as<float>(), ws, s));
    HD_TRY(hdb::normalise_scan(sb, pl->rms.as<float>(), scan_g, scan_pitch, nullptr, s,
                               pl->plan->d_err));
    if (gi == 0) cudaEventRecord(pl->ev[4], s);

    // ---- widths (pipeline.cu:657-776 at this group's factor) ------------------
    wi = widths_for(P, scr, nc_s, stride_s, cur_delay);
    const size_t cur_off = rel_bmax / 2;
    const int nw = (int)wi.size();
    if (nw == 0) continue;  // the trials' factor exceeds the widest boxcar
    HD_TRY(pl->winfo.ensure(nw * sizeof(hdb::WidthInfo)));
    HD_TRY(cudaMemcpyAsync(pl->winfo.p, wi.data(), nw * sizeof(hdb::WidthInfo),
                           cudaMemcpyHostToDevice, s));
    HD_TRY(pl->norm.ensure(NSg * nw * sizeof(float)));
    wctx.scan = scan_g;
    wctx.scan_pitch = scan_pitch;
    wctx.nser = (int)NSg;
    wctx.stride = stride_s;
    wctx.nbeams = (int)nbeams;
    wctx.offset = (int)cur_off;
    wctx.nw = nw;
    wctx.winfo = pl->winfo.as<hdb::WidthInfo>();
    wctx.host_winfo = wi.data();
    wctx.scan_len = nc_s + 1;
    wctx.dms_per_unit = (int)Dg;
    wctx.dm_key_gap = (int)gap;
    wctx.dm_offset = (int)G.d0;
    wctx.norm = pl->norm.as<float>();
    wctx.thresh = P.detect_thresh;
    // largest |boxcar| per block-RMS group (at most nbeams * stride / 5^5 + 4
    // groups per series), read by the count pass to skip quiet tiles
    const size_t gcap = NSg * (size_t)nw * (nbeams * stride_s / 3125 + 5);
    HD_TRY(pl->gmax.ensure(gcap * sizeof(float)));
    wctx.gmax = pl->gmax.as<float>();
    wctx.gmax_cap = gcap;
    int n_ts1 = 0;
    while (n_ts1 < nw && wi[n_ts1].ts == 1) n_ts1++;
    if (n_ts1 > 0) HD_TRY(hdb::block_rms(wctx, wi.data(), 0, n_ts1, ws, s));
    for (int w = n_ts1; w < nw; w++) HD_TRY(hdb::block_rms(wctx, wi.data(), w, w + 1, ws, s));

    // ---- threshold + ordered compaction -------------------------------------
    const unsigned ntiles = (unsigned)((wi[0].n + 2047) / 2048);
    const size_t nsw = NSg * nw;
    HD_TRY(pl->tile_cnt.ensure(nsw * ntiles * sizeof(unsigned)));
    HD_TRY(pl->tile_off.ensure(nsw * ntiles * sizeof(unsigned)));
    HD_TRY(pl->sw_cnt.ensure((nsw + 1) * sizeof(unsigned)));
    HD_TRY(pl->sw_off.ensure((nsw + 1) * sizeof(unsigned)));
    HD_TRY(pl->tile_list.ensure((NSg * ntiles + 1) * sizeof(unsigned)));
    hb.tile_list = pl->tile_list.as<unsigned>();
    hb.tile_list_n = hb.tile_list + NSg * ntiles;
    hb.tile_cnt = pl->tile_cnt.as<unsigned>();
    hb.tile_off = pl->tile_off.as<unsigned>();
    hb.sw_cnt = pl->sw_cnt.as<unsigned>();
    hb.sw_off = pl->sw_off.as<unsigned>();
    HD_TRY(hdb::count_hits(wctx, hb, ntiles, s));
    HD_TRY(hdb::scan_hit_counts(wctx, hb, s));
    HD_TRY(pl->scan_tmp.ensure(hdb::scan_tmp_words(nsw) * sizeof(unsigned)));
    unsigned* totals = pl->small.as<unsigned>();
    HD_TRY(hdb::scan_u32(hb.sw_cnt, hb.sw_off, nsw, totals, pl->scan_tmp.as<unsigned>(), s));
    HD_TRY(cudaMemcpyAsync(pl->h_small, totals, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    HD_TRY(cudaStreamSynchronize(s));
    const unsigned gh = pl->h_small[0];
    nhits += gh;
    HD_TRY(pl->hit_ind.ensure((size_t)(gh + 1) * sizeof(unsigned)));
    HD_TRY(pl->hit_val.ensure((size_t)(gh + 1) * sizeof(float)));
    HD_TRY(pl->hit_sw.ensure((size_t)(gh + 1) * sizeof(unsigned)));
    hb.ind = pl->hit_ind.as<unsigned>();
    hb.val = pl->hit_val.as<float>();
    hb.sw = pl->hit_sw.as<unsigned>();
    hb.cap = gh;
    if (gh) HD_TRY(hdb::write_hits(wctx, hb, s));
    if (gi == 0) cudaEventRecord(pl->ev[5], s);

    // ---- giants ------------------------------------------------------------
    if (!gh) continue;
    HD_TRY(pl->head.ensure((size_t)(gh + 1) * sizeof(unsigned)));
    HD_TRY(pl->gid.ensure((size_t)(gh + 1) * sizeof(unsigned)));
    hdb::GiantBuffers gg{};
    gg.head = pl->head.as<unsigned>();
    gg.gid = pl->gid.as<unsigned>();
    HD_TRY(hdb::giant_heads(wctx, hb, gh, gg, s));
    HD_TRY(pl->scan_tmp.ensure(hdb::scan_tmp_words(gh) * sizeof(unsigned)));
    HD_TRY(hdb::scan_u32(gg.head, gg.gid, gh, totals + 1, pl->scan_tmp.as<unsigned>(), s));
    HD_TRY(cudaMemcpyAsync(pl->h_small + 1, totals + 1, sizeof(unsigned),
                           cudaMemcpyDeviceToHost, s));
    HD_TRY(cudaStreamSynchronize(s));
    const unsigned gn = pl->h_small[1];
    group_giants[gi] = gn;
    ngiants += gn;
    // one group: straight into the giant list; several: into the group's
    // own buffers, placed unit-major once every group is done
    hd_pipeline_t::GiantSet& gs = multi ? pl->gsets[gi] : pl->main_giants;
    const size_t Gc = (size_t)gn + 1;
    HD_TRY(gs.key.ensure(Gc * sizeof(unsigned long long)));
    HD_TRY(gs.peak.ensure(Gc * sizeof(float)));
    HD_TRY(gs.ind.ensure(Gc * sizeof(unsigned long long)));
    HD_TRY(gs.begin.ensure(Gc * sizeof(unsigned long long)));
    HD_TRY(gs.end.ensure(Gc * sizeof(unsigned long long)));
    HD_TRY(gs.filter.ensure(Gc * sizeof(int)));
    HD_TRY(gs.dm.ensure(Gc * sizeof(int)));
    HD_TRY(gs.label.ensure(Gc * sizeof(int)));
    gs.view(gg);
    gg.cap = gn;
    HD_TRY(hdb::giant_fill(wctx, hb, gh, gn, gg, s));
  }
  if (search && ngiants) {
    hd_pipeline_t::GiantSet& m = pl->main_giants;
    if (multi) {
      // giants unit-major across groups: unit u's giants of group 0, then of
      // group 1, ... (the order the reference's DM loop appends them in)
      const size_t Gc = (size_t)ngiants + 1;
      HD_TRY(m.key.ensure(Gc * sizeof(unsigned long long)));
      HD_TRY(m.peak.ensure(Gc * sizeof(float)));
      HD_TRY(m.ind.ensure(Gc * sizeof(unsigned long long)));
      HD_TRY(m.begin.ensure(Gc * sizeof(unsigned long long)));
      HD_TRY(m.end.ensure(Gc * sizeof(unsigned long long)));
      HD_TRY(m.filter.ensure(Gc * sizeof(int)));
      HD_TRY(m.dm.ensure(Gc * sizeof(int)));
      HD_TRY(m.label.ensure(Gc * sizeof(int)));
      hdb::GiantBuffers dst{};
      m.view(dst);
      // per-group unit offsets, then each group's destination per unit
      std::vector<unsigned> firsts(ngs * (U + 1), 0);
      HD_TRY(pl->unit_off.ensure(ngs * (U + 1) * sizeof(unsigned)));
      HD_TRY(pl->place_base.ensure(ngs * (U + 1) * sizeof(unsigned)));
      for (size_t gi = 0; gi < ngs; gi++) {
        if (!group_giants[gi]) continue;
        hdb::GiantBuffers src{};
        pl->gsets[gi].view(src);
        HD_TRY(hdb::unit_giant_offsets(src, (int)group_giants[gi], (int)gap, (int)U,
                                       pl->unit_off.as<unsigned>() + gi * (U + 1), s));
      }
      HD_TRY(cudaMemcpyAsync(firsts.data(), pl->unit_off.p, ngs * (U + 1) * sizeof(unsigned),
                             cudaMemcpyDeviceToHost, s));
      HD_TRY(cudaStreamSynchronize(s));
      std::vector<unsigned> base(ngs * (U + 1), 0);
      unsigned at = 0;
      for (size_t u = 0; u < U; u++)
        for (size_t gi = 0; gi < ngs; gi++) {
          base[gi * (U + 1) + u] = at;
          if (group_giants[gi])
            at += firsts[gi * (U + 1) + u + 1] - firsts[gi * (U + 1) + u];
        }
      HD_TRY(cudaMemcpyAsync(pl->place_base.p, base.data(), base.size() * sizeof(unsigned),
                             cudaMemcpyHostToDevice, s));
      for (size_t gi = 0; gi < ngs; gi++) {
        if (!group_giants[gi]) continue;
        hdb::GiantBuffers src{};
        pl->gsets[gi].view(src);
        HD_TRY(hdb::giant_place(src, group_giants[gi], (int)gap,
                                pl->unit_off.as<unsigned>() + gi * (U + 1),
                                pl->place_base.as<unsigned>() + gi * (U + 1), dst, s));
      }
      // the host base table must outlive the copy
      HD_TRY(cudaStreamSynchronize(s));
    }
    m.view(gb);
    gb.head = pl->head.as<unsigned>();
    gb.gid = pl->gid.as<unsigned>();
    gb.cap = ngiants;
  }
  cudaEventRecord(pl->ev[6], s);

  // giants of each unit: they are unit-major, so unit u holds [first[u], first[u+1])
  std::vector<unsigned>& first = pl->unit_first;
  if (U == 1 || ngiants == 0) {
    for (size_t u = 1; u <= U; u++) first[u] = ngiants;
  } else {
    HD_TRY(pl->unit_off.ensure((U + 1) * sizeof(unsigned)));
    HD_TRY(hdb::unit_giant_offsets(gb, (int)ngiants, (int)gap, (int)U,
                                   pl->unit_off.as<unsigned>(), s));
    HD_TRY(cudaMemcpyAsync(first.data(), pl->unit_off.p, (U + 1) * sizeof(unsigned),
                           cudaMemcpyDeviceToHost, s));
    HD_TRY(cudaStreamSynchronize(s));
  }

  std::vector<char> too_many;
  bool any_ok = false, any_too_many = false;
  giant_rate_bail_out(pl, U, nsamps, first, statuses, too_many, any_ok, any_too_many);

  unsigned ngroups = 0;
  std::vector<hdb::GroupRow> rows;
  pl->obs_hits = nhits;
  pl->obs_giants = ngiants;
  pl->obs_pairs = 0;
  if (any_ok && ngiants > 0) {
    // ---- clustering ----------------------------------------------------------
    HD_TRY(hdb::cluster_init(gb, (int)ngiants, s));
    unsigned max_unit = 0;
    for (size_t u = 0; u < U; u++) max_unit = std::max(max_unit, first[u + 1] - first[u]);
    hdb::ClusterArgs ca{(int)ngiants, P.cand_sep_time, P.cand_sep_filter, dm_tol,
                        (unsigned long long)(nsamps / nbeams), (int)max_unit};
    // sweeps until one changes nothing; the fixed point is idempotent, so
    // the sweeps run in pairs, each with its own flag, and the host reads
    // both flags once per pair: the loop ends when the pair's second sweep
    // changed nothing (half the host round trips, no sweep beyond the one
    // that confirms the fixed point)
    unsigned* changed = pl->small.as<unsigned>() + 8;
    for (unsigned it = 0; it <= ngiants; it += 2) {
      pl->obs_pairs++;
      HD_TRY(cudaMemsetAsync(changed, 0, 2 * sizeof(unsigned), s));
      HD_TRY(hdb::cluster_sweep(ca, gb, changed, s));
      HD_TRY(hdb::cluster_sweep(ca, gb, changed + 1, s));
      HD_TRY(cudaMemcpyAsync(pl->h_small + 8, changed, 2 * sizeof(unsigned),
                             cudaMemcpyDeviceToHost, s));
      HD_TRY(cudaStreamSynchronize(s));
      if (pl->h_small[9] == 0) break;
    }
    // ---- merge -----------------------------------------------------------------
    size_t G = ngiants;
    HD_TRY(pl->root_flag.ensure((G + 1) * sizeof(unsigned)));
    HD_TRY(pl->root_off.ensure((G + 1) * sizeof(unsigned)));
    HD_TRY(pl->mkey.ensure(2 * (G + 1) * sizeof(unsigned long long)));
    HD_TRY(pl->rows.ensure((G + 1) * sizeof(hdb::GroupRow)));
    HD_TRY(pl->scan_tmp.ensure(hdb::scan_tmp_words(G) * sizeof(unsigned)));
    unsigned* nroots = pl->small.as<unsigned>() + 16;
    HD_TRY(hdb::merge_groups(gb, (int)G, (int)gap, pl->plan->d_dm_list,
                             pl->root_flag.as<unsigned>(), pl->root_off.as<unsigned>(), nroots,
                             pl->scan_tmp.as<unsigned>(), pl->mkey.as<unsigned long long>(),
                             pl->rows.as<hdb::GroupRow>(), s));
    // the group count, the error word and the first rows in one round trip
    // (the giants stay on the device until hd_get_giants asks for them)
    const size_t spec = std::min<size_t>(G, kSpecRows);
    HD_TRY(pl->ensure_rows_host(std::max<size_t>(spec, 1)));
    HD_TRY(cudaMemcpyAsync(pl->h_small + 16, nroots, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    HD_TRY(cudaMemcpyAsync(pl->h_small + 17, pl->plan->d_err, sizeof(unsigned),
                           cudaMemcpyDeviceToHost, s));
    HD_TRY(cudaMemcpyAsync(pl->h_rows, pl->rows.p, spec * sizeof(hdb::GroupRow),
                           cudaMemcpyDeviceToHost, s));
    cudaEventRecord(pl->ev[7], s);
    HD_TRY(cudaStreamSynchronize(s));
    ngroups = pl->h_small[16];
    if (ngroups > spec) {
      std::vector<hdb::GroupRow> head(pl->h_rows, pl->h_rows + spec);
      HD_TRY(pl->ensure_rows_host(ngroups));
      std::copy(head.begin(), head.end(), pl->h_rows);
      HD_TRY(cudaMemcpyAsync(pl->h_rows + spec, pl->rows.as<hdb::GroupRow>() + spec,
                             (ngroups - spec) * sizeof(hdb::GroupRow), cudaMemcpyDeviceToHost, s));
      HD_TRY(cudaStreamSynchronize(s));
    }
    rows.assign(pl->h_rows, pl->h_rows + ngroups);
    pl->last_giants = G;
  } else {
    HD_TRY(cudaMemcpyAsync(pl->h_small + 17, pl->plan->d_err, sizeof(unsigned),
                           cudaMemcpyDeviceToHost, s));
    cudaEventRecord(pl->ev[7], s);
    HD_TRY(cudaStreamSynchronize(s));
  }
  pl->last_gap = gap;
  if (pl->h_small[17]) return HD_INTERNAL_GPU_ERROR;

  emit_candidates(pl, U, rows.data(), ngroups, too_many, nsamps, nbeams, first_idx, beams,
                  *nsamps_processed);

  // stage timings
  auto el = [&](int a, int b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pl->ev[a], pl->ev[b]) != cudaSuccess) ms = 0.f;
    return ms;
  };
  pl->timing[0] = el(0, 7);
  pl->timing[7] = el(0, 1);
  pl->timing[1] = el(1, 2);
  pl->timing[2] = el(2, 3);
  if (search) {
    pl->timing[3] = el(3, 4);
    pl->timing[4] = el(4, 5);
    pl->timing[5] = el(5, 6);
  }
  pl->timing[6] = el(6, 7);
  if (!pl->pending_shape.empty()) {
    // a new shape for the graph form: capacities from what this gulp saw
    if (pl->graph_shapes.size() >= 64) pl->graph_shapes.erase(pl->graph_shapes.begin());
    hd_pipeline_t::GraphShape gsh;
    gsh.key = pl->pending_shape;
    gsh.hcap = graph_capacity(pl->obs_hits, 1u << 16);
    gsh.gcap = graph_capacity(pl->obs_giants, 1u << 14);
    gsh.pairs = std::min(std::max(pl->obs_pairs + 1, 2u), 16u);
    // HDB_GRAPH_CAPS="hits,giants,pairs" sets a new shape's starting
    // capacities instead (tests of the overflow and extra-sweep paths)
    if (const char* c = std::getenv("HDB_GRAPH_CAPS")) {
      unsigned h = 0, g = 0, q = 0;
      if (std::sscanf(c, "%u,%u,%u", &h, &g, &q) == 3 && h && g && q && q <= 16) {
        gsh.hcap = h;
        gsh.gcap = g;
        gsh.pairs = q;
      }
    }
    pl->graph_shapes.push_back(gsh);
    pl->pending_shape.clear();
  }
  return any_too_many ? HD_TOO_MANY_EVENTS : HD_NO_ERROR;
}

hd_error hd_execute(hd_pipeline pl, const hd_byte* h_filterbank, hd_size nsamps, hd_size nbits,
                    hd_size first_idx, hd_size nbeams, hd_size* nsamps_processed) {
  if (!h_filterbank) return pl ? HD_INVALID_POINTER : HD_INVALID_PIPELINE;
  return execute_units(pl, &h_filterbank, 1, false, nsamps, nbits, first_idx, nbeams, nullptr,
                       nullptr, nsamps_processed);
}

hd_error hd_execute_device(hd_pipeline pl, const hd_byte* d_filterbank, hd_size nsamps,
                           hd_size nbits, hd_size first_idx, hd_size nbeams,
                           hd_size* nsamps_processed) {
  if (!d_filterbank) return pl ? HD_INVALID_POINTER : HD_INVALID_PIPELINE;
  return execute_units(pl, &d_filterbank, 1, true, nsamps, nbits, first_idx, nbeams, nullptr,
                       nullptr, nsamps_processed);
}

hd_error hd_execute_beams(hd_pipeline pl, const hd_byte* const* filterbanks,
                          hd_size nfilterbanks, hd_size nsamps, hd_size nbits,
                          hd_size first_idx, hd_size nbeams, const hd_size* beams,
                          int on_device, hd_error* statuses, hd_size* nsamps_processed) {
  return execute_units(pl, filterbanks, nfilterbanks, on_device != 0, nsamps, nbits, first_idx,
                       nbeams, beams, statuses, nsamps_processed, true);
}

hd_error hd_prefetch_beams(hd_pipeline pl, const hd_byte* const* filterbanks,
                           hd_size nfilterbanks, hd_size nsamps, hd_size nbits) {
  if (!pl) return HD_INVALID_PIPELINE;
  if (!filterbanks || nfilterbanks == 0) return HD_INVALID_POINTER;
  for (size_t u = 0; u < nfilterbanks; u++)
    if (!filterbanks[u]) return HD_INVALID_POINTER;
  if (nbits != 8) return HD_INVALID_NBITS;
  int slot = -1;
  for (int i = 0; i < 2; i++)
    if (!pl->pf[i].pending) {
      slot = i;
      break;
    }
  if (slot < 0) return HD_INVALID_STRIDE;  // two gulps already queued
  if (cudaSetDevice(pl->device) != cudaSuccess) return HD_INVALID_DEVICE_INDEX;
  hd_pipeline_t::Prefetch& q = pl->pf[slot];
  const size_t fb_bytes = nsamps * pl->params.nchans;
  HD_TRY(q.buf.ensure(nfilterbanks * fb_bytes + 64));
  // the slot may still be read by a search queued earlier on the compute stream
  HD_TRY(cudaEventRecord(q.done, pl->stream));
  HD_TRY(cudaStreamWaitEvent(pl->copy_stream, q.done, 0));
  HD_TRY(copy_units(q.buf.as<uint8_t>(), filterbanks, 0, nfilterbanks, fb_bytes,
                    cudaMemcpyHostToDevice, pl->copy_stream));
  HD_TRY(cudaEventRecord(q.done, pl->copy_stream));
  q.pending = true;
  q.tag = ++pl->pf_seq;
  q.units = nfilterbanks;
  q.nsamps = nsamps;
  return HD_NO_ERROR;
}

hd_error hd_execute_prefetched(hd_pipeline pl, hd_size first_idx, hd_size nbeams,
                               const hd_size* beams, hd_error* statuses,
                               hd_size* nsamps_processed) {
  if (!pl) return HD_INVALID_PIPELINE;
  int slot = -1;
  for (int i = 0; i < 2; i++)
    if (pl->pf[i].pending && (slot < 0 || pl->pf[i].tag < pl->pf[slot].tag)) slot = i;
  if (slot < 0) return HD_INVALID_POINTER;  // nothing queued
  if (cudaSetDevice(pl->device) != cudaSuccess) return HD_INVALID_DEVICE_INDEX;
  hd_pipeline_t::Prefetch& q = pl->pf[slot];
  HD_TRY(cudaStreamWaitEvent(pl->stream, q.done, 0));
  // the slot's buffer becomes the pipeline's time-major input (no copy); the
  // previous input buffer becomes the slot's, to be filled by a later
  // hd_prefetch_beams once the work queued on the compute stream is done
  std::swap(pl->fb_tf.p, q.buf.p);
  std::swap(pl->fb_tf.cap, q.buf.cap);
  const size_t fb_bytes = q.nsamps * pl->params.nchans;
  std::vector<const hd_byte*> fbs(q.units);
  for (size_t u = 0; u < q.units; u++) fbs[u] = pl->fb_tf.as<uint8_t>() + u * fb_bytes;
  pl->fb_resident = true;
  const hd_error e = execute_units(pl, fbs.data(), q.units, true, q.nsamps, 8, first_idx,
                                   nbeams, beams, statuses, nsamps_processed, true);
  q.pending = false;
  return e;
}

unsigned long long hd_get_launch_count(void) { return hdb::launch_count(); }

hd_error hd_set_graphs(hd_pipeline pl, int enable) {
  if (!pl) return HD_INVALID_PIPELINE;
  pl->use_graphs = enable != 0;
  if (!pl->use_graphs) {
    cudaSetDevice(pl->device);
    for (auto& g : pl->graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    pl->graphs.clear();
  }
  return HD_NO_ERROR;
}

unsigned long long hd_get_graph_replays(hd_pipeline pl) { return pl ? pl->graph_replays : 0; }

void hd_destroy_pipeline(hd_pipeline pl) {
  if (!pl) return;
  cudaSetDevice(pl->device);
  delete pl;
}

hd_error hd_clean_filterbank_rfi(hd_pipeline pl, const hd_byte* h_in, hd_size nsamps,
                                 hd_size nbits, hd_byte* h_out, int* h_mask, hd_float dt,
                                 hd_float baseline_length, hd_float rfi_tol, hd_size boxcar_max,
                                 hd_size nbeams) {
  if (!pl) return HD_INVALID_PIPELINE;
  if (!h_in || !h_out) return HD_INVALID_POINTER;
  if (nbits != 8) return HD_INVALID_NBITS;
  const size_t C = pl->params.nchans;
  if (C % 4 != 0 || nbeams == 0) return HD_INVALID_STRIDE;
  // one flag bit per boxcar width in a byte: widths 1..128
  if (boxcar_max > 128) return HD_INVALID_STRIDE;
  cudaSetDevice(pl->device);
  cudaStream_t s = pl->stream;
  // the plan's device error word records a bounded wait that gave up
  dedisp_error de = hdb::plan_prepare(pl->plan);
  if (de != DEDISP_NO_ERROR) return dedisp_err(de);
  HD_TRY(cudaMemsetAsync(pl->plan->d_err, 0, sizeof(unsigned), s));
  HD_TRY(pl->fb_tf.ensure(nsamps * C));
  HD_TRY(pl->fb_tf_clean.ensure(nsamps * C));
  HD_TRY(cudaMemcpyAsync(pl->fb_tf.p, h_in, nsamps * C, cudaMemcpyHostToDevice, s));
  hd_error he = clean_units(pl, 1, pl->fb_tf.as<uint8_t>(), nsamps, C, dt, baseline_length,
                            rfi_tol, boxcar_max, nbeams, nullptr, 0,
                            pl->fb_tf_clean.as<uint8_t>());
  if (he != HD_NO_ERROR) return he;
  HD_TRY(cudaMemcpyAsync(h_out, pl->fb_tf_clean.p, nsamps * C, cudaMemcpyDeviceToHost, s));
  if (h_mask)
    HD_TRY(cudaMemcpyAsync(h_mask, pl->mask.p, nsamps * sizeof(int), cudaMemcpyDeviceToHost, s));
  HD_TRY(cudaMemcpyAsync(pl->h_small + 24, pl->plan->d_err, sizeof(unsigned),
                         cudaMemcpyDeviceToHost, s));
  HD_TRY(cudaStreamSynchronize(s));
  if (pl->h_small[24]) return HD_INTERNAL_GPU_ERROR;
  return HD_NO_ERROR;
}

hd_error hd_get_candidates(hd_pipeline pl, hd_candidate* out, hd_size* count) {
  if (!pl) return HD_INVALID_PIPELINE;
  if (!count) return HD_INVALID_POINTER;
  size_t n = std::min(*count, pl->cands.size());
  if (out && n) std::memcpy(out, pl->cands.data(), n * sizeof(hd_candidate));
  *count = pl->cands.size();
  return HD_NO_ERROR;
}

hd_error hd_get_beam_candidates(hd_pipeline pl, hd_size index, hd_candidate* out,
                                hd_size* count) {
  if (!pl) return HD_INVALID_PIPELINE;
  if (!count) return HD_INVALID_POINTER;
  if (index >= pl->unit_cands.size()) return HD_INVALID_STRIDE;
  const std::vector<hd_candidate>& v = pl->unit_cands[index];
  size_t n = std::min(*count, v.size());
  if (out && n) std::memcpy(out, v.data(), n * sizeof(hd_candidate));
  *count = v.size();
  return HD_NO_ERROR;
}

hd_error hd_get_raw_candidates(hd_pipeline pl, struct RawCandidates* out, hd_size* count) {
  if (!pl) return HD_INVALID_PIPELINE;
  if (!out || !count) return HD_INVALID_POINTER;
  const std::vector<hd_candidate>& v = pl->cands;
  const size_t n = std::min(*count, v.size());
  for (size_t i = 0; i < n; i++) {
    const hd_candidate& c = v[i];
    if (out->peaks) out->peaks[i] = c.snr;
    if (out->inds) out->inds[i] = c.samp_idx;
    if (out->begins) out->begins[i] = c.begin;
    if (out->ends) out->ends[i] = c.end;
    if (out->filter_inds) out->filter_inds[i] = c.filter;
    if (out->dm_inds) out->dm_inds[i] = c.dm_trial;
    if (out->members) out->members[i] = c.members;
  }
  *count = v.size();
  return HD_NO_ERROR;
}

namespace {
// Patches of the first k candidates of the last gulp into pl->patch_dm /
// pl->patch_ft (device), on the pipeline's stream.
hd_error patches_on_device(hd_pipeline pl, size_t k) {
  const size_t C = pl->params.nchans;
  if (!pl->searched || C % 64 != 0) return HD_INVALID_STRIDE;
  if (cudaSetDevice(pl->device) != cudaSuccess) return HD_INVALID_DEVICE_INDEX;
  cudaStream_t s = pl->stream;
  const size_t D = pl->plan->dm_list.size();
  std::vector<hdb::PatchJob> jobs(k);
  for (size_t i = 0; i < k; i++) {
    const hd_pipeline_t::CandMeta& m = pl->meta[i];
    hdb::PatchJob& j = jobs[i];
    j.series0 = (unsigned)(m.unit * D);
    j.dm = m.dm;
    j.ndm = (int)D;
    j.ind = m.ind;
    j.filter = m.filter;
    j.unit = m.unit;
    // gen_freq_time_plot: window of 256 bins of 2^filter samples, widened to
    // the next power of two >= the DM's largest delay, centred half a sweep
    // after the candidate
    size_t md = 0;
    for (size_t c = 0; c < C; c++) md = std::max(md, (size_t)pl->plan->delays[(size_t)m.dm * C + c]);
    size_t ts = (size_t)1 << m.filter;
    size_t in_n = 256 * ts;
    if (in_n < md) {
      size_t delay = 2;
      while (delay < md) delay *= 2;
      in_n = delay;
      ts = in_n / 256;
    }
    j.ft_ts = (unsigned)ts;
    j.ft_first = (long long)(m.ind + md / 2) - (long long)(in_n / 2);
  }
  HD_TRY(pl->patch_jobs.ensure(k * sizeof(hdb::PatchJob)));
  HD_TRY(pl->patch_dm.ensure(k * HD_PATCH_DM_TIME * sizeof(float)));
  HD_TRY(pl->patch_ft.ensure(k * HD_PATCH_FREQ_TIME * sizeof(float)));
  HD_TRY(cudaMemcpyAsync(pl->patch_jobs.p, jobs.data(), k * sizeof(hdb::PatchJob),
                         cudaMemcpyHostToDevice, s));
  HD_TRY(hdb::extract_patches(pl->scan.as<float>(), pl->last_scan_pitch, pl->last_len,
                              pl->fb_tf.as<uint8_t>(), pl->last_nsamps, (int)C,
                              pl->patch_jobs.as<hdb::PatchJob>(), (int)k,
                              pl->patch_dm.as<float>(), pl->patch_ft.as<float>(), s));
  return HD_NO_ERROR;
}
}  // namespace

hd_error hd_extract_patches(hd_pipeline pl, hd_float* dm_time, hd_float* freq_time,
                            hd_size* count) {
  if (!pl) return HD_INVALID_PIPELINE;
  if (!count) return HD_INVALID_POINTER;
  const size_t n = pl->cands.size();
  const size_t k = std::min(*count, n);
  *count = n;
  if (k == 0 || (!dm_time && !freq_time)) return HD_NO_ERROR;
  hd_error he = patches_on_device(pl, k);
  if (he != HD_NO_ERROR) return he;
  cudaStream_t s = pl->stream;
  if (dm_time)
    HD_TRY(cudaMemcpyAsync(dm_time, pl->patch_dm.p, k * HD_PATCH_DM_TIME * sizeof(float),
                           cudaMemcpyDeviceToHost, s));
  if (freq_time)
    HD_TRY(cudaMemcpyAsync(freq_time, pl->patch_ft.p, k * HD_PATCH_FREQ_TIME * sizeof(float),
                           cudaMemcpyDeviceToHost, s));
  HD_TRY(cudaStreamSynchronize(s));
  return HD_NO_ERROR;
}

hd_error hd_score_candidates(hd_pipeline pl, hd_classifier clf, hd_float* scores,
                             hd_size* count) {
  if (!pl) return HD_INVALID_PIPELINE;
  if (!clf) return HD_INVALID_PIPELINE;
  if (!count) return HD_INVALID_POINTER;
  const size_t n = pl->cands.size();
  const size_t k = std::min(*count, n);
  *count = n;
  if (k == 0) return HD_NO_ERROR;
  if (!scores) return HD_INVALID_POINTER;
  if (hdb::classifier_device(clf) != pl->device) return HD_INVALID_DEVICE_INDEX;
  hd_error he = patches_on_device(pl, k);
  if (he != HD_NO_ERROR) return he;
  // the classifier's stream waits for the patches; nothing leaves the device
  // but the scores
  HD_TRY(cudaEventRecord(pl->ev[8], pl->stream));
  HD_TRY(hdb::classifier_score_device(clf, pl->patch_dm.as<float>(), pl->patch_ft.as<float>(),
                                      k, pl->ev[8], scores));
  return HD_NO_ERROR;
}

hd_error hd_get_giants(hd_pipeline pl, hd_float* peaks, hd_size* inds, hd_size* begins,
                       hd_size* ends, hd_size* filter_inds, hd_size* dm_inds, hd_size* labels,
                       hd_size* count) {
  if (!pl) return HD_INVALID_PIPELINE;
  if (!count) return HD_INVALID_POINTER;
  const size_t G = pl->last_giants;
  const size_t n = std::min(*count, G);
  *count = G;
  if (n == 0) return HD_NO_ERROR;
  if (cudaSetDevice(pl->device) != cudaSuccess) return HD_INVALID_DEVICE_INDEX;
  // the last gulp's giants, from the device
  hdb::GiantBuffers gb{};
  pl->main_giants.view(gb);
  cudaStream_t s = pl->stream;
  std::vector<unsigned long long> u64(n);
  std::vector<int> i32(n);
  auto widen64 = [&](const unsigned long long* src, hd_size* dst) -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(u64.data(), src, n * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    for (size_t g = 0; e == cudaSuccess && g < n; g++) dst[g] = (hd_size)u64[g];
    return e;
  };
  auto widen32 = [&](const int* src, hd_size* dst, size_t mod) -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(i32.data(), src, n * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    for (size_t g = 0; e == cudaSuccess && g < n; g++)
      dst[g] = mod ? (hd_size)((unsigned)i32[g] % mod) : (hd_size)i32[g];
    return e;
  };
  if (peaks) {
    HD_TRY(cudaMemcpyAsync(peaks, gb.peak, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    HD_TRY(cudaStreamSynchronize(s));
  }
  if (inds) HD_TRY(widen64(gb.ind, inds));
  if (begins) HD_TRY(widen64(gb.begin, begins));
  if (ends) HD_TRY(widen64(gb.end, ends));
  if (filter_inds) HD_TRY(widen32(gb.filter, filter_inds, 0));
  // DM trial of the key unit * gap + trial
  if (dm_inds) HD_TRY(widen32(gb.dm, dm_inds, pl->last_gap));
  if (labels) HD_TRY(widen32(gb.label, labels, 0));
  return HD_NO_ERROR;
}

}  // extern "C"

namespace hdb {
int pipeline_device(hd_pipeline pl) { return pl ? pl->device : 0; }
}  // namespace hdb

extern "C" {

hd_error hd_get_dedisp_tile(hd_pipeline pl, int* dm_block, int* time_block, int* rows) {
  if (!pl) return HD_INVALID_PIPELINE;
  const std::array<int, 3>& t = pl->plan->last_tile;
  if (dm_block) *dm_block = t[0];
  if (time_block) *time_block = t[1];
  if (rows) *rows = t[2];
  return HD_NO_ERROR;
}

int hd_get_dedisp_tile_source(hd_pipeline pl) {
  if (!pl) return -1;
  return pl->plan->last_tile_source;
}

hd_error hd_get_timing(hd_pipeline pl, float* ms, int n) {
  if (!pl) return HD_INVALID_PIPELINE;
  if (!ms) return HD_INVALID_POINTER;
  for (int i = 0; i < n && i < 8; i++) ms[i] = pl->timing[i];
  return HD_NO_ERROR;
}

}  // extern "C"
