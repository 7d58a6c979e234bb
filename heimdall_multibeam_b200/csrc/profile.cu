// profile.cu -- the candidate profiler (Applications/candidate_profiler.C) on
// the GPU for a batch of candidates of one filterbank.
//
// Per candidate, as the reference's application computes them:
//   * the DM-time plot (gen_dm_time_plot, candidate_profiler.C:232-415): the
//     trials [dm_begin, dm_end) around the candidate's trial re-dedispersed
//     over a window of the filterbank with adaptive dt on those trials (pulse
//     width 40 us, tolerance 1.15), then either summed over the boxcar at each
//     trial's resolution or (do_filter) unscrunched and boxcar-filtered
//     through a float prefix sum; each row normalised
//     (normalise_series_array, :88-134, with its division by zero kept);
//   * the DM-0 series: the same with the list's first trial alone;
//   * the freq-time plot (gen_freq_time_plot, :136-230) at filter - 2;
//   * from these, on the host: the plot's first maximum, SNR vs DM at its time
//     and SNR vs time along its row (:560-640).
// Windows are read from the filterbank as the application reads its file:
// samples past the end read as 0; a freq-time window that would start before
// the first sample reads 0 there.
//
// Kernels: k_prof_dedisp computes each window trial's dedispersed samples
// (exact integer sums over channels of the byte-mean scrunched input, as
// include/dedisp.h defines them) into a scratch row; k_prof_boxcar and
// k_prof_filter form the plot rows in the reference's float order;
// k_prof_ft sums the freq-time pixels; normalise_rows normalises every row.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "heimdall_b200.h"
#include "internal.h"
#include "plan.h"

namespace hdb {
namespace {

// One dedispersed row of a candidate's window (a trial of its DM-time plot
// or its DM-0 series).
struct ProfRow {
  float dm;            // trial DM
  int s;               // scrunch factor
  unsigned nd;         // samples of the row before scrunching (valid: nd / s)
  long long first;     // first filterbank sample of the window
  size_t off;          // float offset of the row in the scratch (nd + 1 floats)
  size_t out;          // float offset of the plot row in the output
  int width;           // boxcar width of the plot (1 << filter)
};

// dedispersed[u] = sum_c in_s[c][u + delay(dm, c) / s] for u < nd / s, with
// in_s the byte mean of s samples (rounded half up) from the window start
__global__ void k_prof_dedisp(const uint8_t* __restrict__ tf, size_t nsamps, int nchans,
                              const float* __restrict__ table, const ProfRow* __restrict__ rows,
                              float* __restrict__ scratch) {
  const ProfRow r = rows[blockIdx.y];
  const unsigned u = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned n = r.nd / (unsigned)r.s;
  if (u >= n) return;
  int acc = 0;
  for (int c = 0; c < nchans; c++) {
    const float v = __fadd_rn(__fmul_rn(r.dm, table[c]), 0.5f);
    const unsigned dl = v > 0.f ? (unsigned)v : 0u;
    const long long t0 = r.first + (long long)r.s * (long long)(u + dl / (unsigned)r.s);
    unsigned sum = 0;
    for (int k = 0; k < r.s; k++) {
      const long long t = t0 + k;
      sum += (t < (long long)nsamps) ? tf[(size_t)t * nchans + c] : 0u;
    }
    acc += (int)((sum + (unsigned)(r.s / 2)) / (unsigned)r.s);
  }
  scratch[r.off + u] = (float)acc;
}

// do_filter = 0: out[t] = sum over the boxcar at the trial's resolution,
// sum_{j < width / s} d[t * (width / s) + j] in float, left to right
__global__ void k_prof_boxcar(const ProfRow* __restrict__ rows, const float* __restrict__ scratch,
                              int out_nsamps, float* __restrict__ out) {
  const ProfRow r = rows[blockIdx.y];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= out_nsamps) return;
  const unsigned k = (unsigned)r.width / (unsigned)r.s;
  const float* d = scratch + r.off + (size_t)t * k;
  float v = 0.f;
  for (unsigned j = 0; j < k; j++) v = __fadd_rn(v, d[j]);
  out[r.out + t] = v;
}

// do_filter = 1: the row unscrunched (sample t takes d[t / s]), its exclusive
// float prefix sum, and out[t] = S[t + width/2 + (width-1)/2 + 1] - S[t]; one
// thread per row walks the sum in order
__global__ void k_prof_filter(const ProfRow* __restrict__ rows, int nrows,
                              float* __restrict__ scratch, float* __restrict__ prefix,
                              int out_nsamps, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrows) return;
  const ProfRow r = rows[i];
  const float* d = scratch + r.off;
  float* S = prefix + r.off;
  float acc = 0.f;
  S[0] = 0.f;
  for (unsigned t = 0; t < r.nd; t++) {
    acc = __fadd_rn(acc, d[t / (unsigned)r.s]);
    S[t + 1] = acc;
  }
  const unsigned a = (unsigned)(r.width / 2 + (r.width - 1) / 2 + 1);
  for (int t = 0; t < out_nsamps; t++) out[r.out + t] = __fsub_rn(S[a + t], S[t]);
}

struct FtJob {
  long long first;   // first sample of the window (may be < 0)
  unsigned ts;       // samples per bin
  size_t out;        // float offset of the candidate's plot
};

// pixel (channel group cs, bin ti): the float sum, time outer and channel
// inner, of x / 255 * 255 over ts samples x fs channels, divided by ts * fs
__global__ void k_prof_ft(const uint8_t* __restrict__ tf, size_t nsamps, int nchans, int fs,
                          int out_nsamps, const FtJob* __restrict__ jobs,
                          float* __restrict__ out) {
  __shared__ float lut[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = prof_scale((unsigned)i);
  __syncthreads();
  const FtJob jb = jobs[blockIdx.z];
  const int cs = blockIdx.y;
  const int ti = blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= out_nsamps) return;
  const long long t0 = jb.first + (long long)ti * jb.ts;
  float sum = 0.f;
  for (unsigned s = 0; s < jb.ts; s++) {
    const long long t = t0 + s;
    // outside the filterbank every sample is 0 and adds +0 (a no-op on a
    // sum >= +0)
    if (t < 0 || t >= (long long)nsamps) continue;
    const uint8_t* row = tf + (size_t)t * nchans + (size_t)cs * fs;
    for (int f = 0; f < fs; f++) sum = __fadd_rn(sum, lut[row[f]]);
  }
  out[jb.out + (size_t)cs * out_nsamps + ti] =
      __fdiv_rn(sum, (float)((size_t)jb.ts * (size_t)fs));
}

struct DevMem {
  void* p = nullptr;
  ~DevMem() { if (p) cudaFree(p); }
  template <class T> T* as() { return reinterpret_cast<T*>(p); }
};

}  // namespace
}  // namespace hdb

extern "C" hd_error hd_profile_candidates(
    const hd_byte* filterbank, hd_size nsamps, hd_size nchans, int on_device, double tsamp,
    double fch1, double foff, const hd_float* dm_list, hd_size dm_count,
    const hd_profile_request* cands, hd_size ncands, hd_size out_nsamps, hd_size out_dm_count,
    hd_size fscrunch, int do_filter, hd_profile* out) {
  using namespace hdb;
  if (!filterbank || !dm_list || !cands || !out) return HD_INVALID_POINTER;
  if (ncands == 0) return HD_NO_ERROR;
  if (nchans == 0 || fscrunch == 0 || nchans % fscrunch != 0 || out_nsamps < 2 ||
      out_nsamps > 4096 || out_dm_count == 0 || dm_count == 0 || nsamps == 0)
    return HD_INVALID_STRIDE;
  for (size_t i = 0; i < ncands; i++)
    if (cands[i].dm_idx >= dm_count || cands[i].filter > 24) return HD_INVALID_STRIDE;
  const size_t C = nchans, out_nchans = nchans / fscrunch;
  // the dedisp plans take the header's values as float
  const float dt = (float)tsamp, f0 = (float)fch1, df = (float)foff;
  std::vector<float> table(C);
  delay_table(C, dt, f0, df, table.data());
  auto max_delay_of = [&](const float* dms, size_t n) {
    size_t m = 0;
    for (size_t d = 0; d < n; d++)
      for (size_t c = 0; c < C; c++) m = std::max(m, delay_of(dms[d], table[c]));
    return m;
  };
  const std::vector<float> dml(dm_list, dm_list + dm_count);

  // ---- host plan of every window ------------------------------------------
  std::vector<ProfRow> rows;
  std::vector<FtJob> ftj(ncands);
  std::vector<size_t> n_dm(ncands), dm_begin(ncands);
  const size_t plot = out_dm_count * out_nsamps;  // floats of one DM-time plot
  size_t scratch = 0;
  for (size_t i = 0; i < ncands; i++) {
    const size_t samp = cands[i].samp, filter = cands[i].filter, dm_idx = cands[i].dm_idx;
    const size_t width = (size_t)1 << filter;
    // DM-time plot (candidate_profiler.C:265-344) and the DM-0 series
    for (int pass = 0; pass < 2; pass++) {
      const size_t di = pass == 0 ? dm_idx : 0;
      const size_t odc = pass == 0 ? out_dm_count : 1;
      const size_t b = di >= odc / 2 ? di - odc / 2 : 0;
      const size_t e = di < dm_count - ((odc - 1) / 2 + 1) ? di + (odc - 1) / 2 + 1 : dm_count;
      const size_t nd_trials = e - b;
      const std::vector<float> sub(dml.begin() + b, dml.begin() + e);
      const std::vector<dedisp_size> scr = scrunch_factors(sub, dt, 40.0, f0, df, C, 1.15);
      const size_t md = max_delay_of(sub.data(), sub.size());
      size_t nd, first;
      if (!do_filter) {
        nd = out_nsamps * width;
        first = samp >= out_nsamps / 2 * width ? samp - out_nsamps / 2 * width : 0;
      } else {
        nd = out_nsamps + width - 1;
        first = samp > out_nsamps / 2 + width / 2 ? samp - out_nsamps / 2 - width / 2 : 0;
      }
      (void)md;
      if (nd >= 0x7FFFFFFFu) return HD_INVALID_STRIDE;
      for (size_t d = 0; d < nd_trials; d++) {
        ProfRow r{};
        r.dm = sub[d];
        r.s = (int)scr[d];
        r.nd = (unsigned)nd;
        r.first = (long long)first;
        r.off = scratch;
        scratch += nd + 1;
        r.out = pass == 0 ? i * plot + d * out_nsamps : i * out_nsamps;
        r.width = (int)width;
        rows.push_back(r);
      }
      if (pass == 0) {
        n_dm[i] = nd_trials;
        dm_begin[i] = b;
      }
    }
    // freq-time plot (candidate_profiler.C:136-184) at filter - 2
    const size_t ftf = filter > 2 ? filter - 2 : 0;
    const float dmv = dml[dm_idx];
    const size_t md = max_delay_of(&dmv, 1);
    size_t delay = 2, ts = (size_t)1 << ftf, in_n = out_nsamps * ts;
    if (in_n < md) {
      while (delay < md) delay *= 2;
      in_n = delay;
      ts = in_n / out_nsamps;
    }
    if (ts >= 0x7FFFFFFFu) return HD_INVALID_STRIDE;
    ftj[i].first = (long long)(samp + md / 2) - (long long)(in_n / 2);
    ftj[i].ts = (unsigned)ts;
    ftj[i].out = i * out_nchans * out_nsamps;
  }
  if (rows.size() > 65535) return HD_INVALID_STRIDE;  // grid y

  // ---- device work ------------------------------------------------------------
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
    return HD_PRIOR_GPU_ERROR;
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{s};
  DevMem d_fb, d_table, d_rows, d_ftj, d_scr, d_pre, d_dm, d_dm0, d_ft;
  const uint8_t* tf = filterbank;
  auto alloc = [&](DevMem& m, size_t bytes) { return dev_malloc(&m.p, std::max<size_t>(bytes, 16)); };
  if (!on_device) {
    if (alloc(d_fb, nsamps * C) != cudaSuccess) return HD_MEM_ALLOC_FAILED;
    if (cudaMemcpyAsync(d_fb.p, filterbank, nsamps * C, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return HD_MEM_COPY_FAILED;
    tf = d_fb.as<uint8_t>();
  }
  const size_t ft_floats = ncands * out_nchans * out_nsamps;
  if (alloc(d_table, C * sizeof(float)) != cudaSuccess ||
      alloc(d_rows, rows.size() * sizeof(ProfRow)) != cudaSuccess ||
      alloc(d_ftj, ncands * sizeof(FtJob)) != cudaSuccess ||
      alloc(d_scr, scratch * sizeof(float)) != cudaSuccess ||
      (do_filter && alloc(d_pre, scratch * sizeof(float)) != cudaSuccess) ||
      alloc(d_dm, ncands * plot * sizeof(float)) != cudaSuccess ||
      alloc(d_dm0, ncands * out_nsamps * sizeof(float)) != cudaSuccess ||
      alloc(d_ft, ft_floats * sizeof(float)) != cudaSuccess)
    return HD_MEM_ALLOC_FAILED;
  if (cudaMemcpyAsync(d_table.p, table.data(), C * sizeof(float), cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(d_rows.p, rows.data(), rows.size() * sizeof(ProfRow),
                      cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(d_ftj.p, ftj.data(), ncands * sizeof(FtJob), cudaMemcpyHostToDevice, s) ||
      cudaMemsetAsync(d_dm.p, 0, ncands * plot * sizeof(float), s))
    return HD_MEM_COPY_FAILED;
  unsigned max_n = 0;
  for (const ProfRow& r : rows) max_n = std::max(max_n, r.nd / (unsigned)r.s);
  const unsigned nrows = (unsigned)rows.size();
  k_prof_dedisp<<<dim3((max_n + 127) / 128, nrows), 128, 0, s>>>(
      tf, nsamps, (int)C, d_table.as<float>(), d_rows.as<ProfRow>(), d_scr.as<float>());
  note_launch();
  // plot rows: the DM-time rows and the DM-0 rows share the row list; the
  // output offset of a DM-0 row indexes the DM-0 buffer
  std::vector<ProfRow> dm_rows, dm0_rows;
  for (size_t i = 0, k = 0; i < ncands; i++) {
    for (size_t d = 0; d < n_dm[i]; d++) dm_rows.push_back(rows[k++]);
    dm0_rows.push_back(rows[k++]);
  }
  DevMem d_rows_dm, d_rows_dm0;
  if (alloc(d_rows_dm, dm_rows.size() * sizeof(ProfRow)) != cudaSuccess ||
      alloc(d_rows_dm0, dm0_rows.size() * sizeof(ProfRow)) != cudaSuccess)
    return HD_MEM_ALLOC_FAILED;
  if (cudaMemcpyAsync(d_rows_dm.p, dm_rows.data(), dm_rows.size() * sizeof(ProfRow),
                      cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(d_rows_dm0.p, dm0_rows.data(), dm0_rows.size() * sizeof(ProfRow),
                      cudaMemcpyHostToDevice, s))
    return HD_MEM_COPY_FAILED;
  const int on = (int)out_nsamps;
  if (!do_filter) {
    k_prof_boxcar<<<dim3((on + 127) / 128, (unsigned)dm_rows.size()), 128, 0, s>>>(
        d_rows_dm.as<ProfRow>(), d_scr.as<float>(), on, d_dm.as<float>());
    note_launch();
    k_prof_boxcar<<<dim3((on + 127) / 128, (unsigned)dm0_rows.size()), 128, 0, s>>>(
        d_rows_dm0.as<ProfRow>(), d_scr.as<float>(), on, d_dm0.as<float>());
    note_launch();
  } else {
    k_prof_filter<<<((unsigned)dm_rows.size() + 63) / 64, 64, 0, s>>>(
        d_rows_dm.as<ProfRow>(), (int)dm_rows.size(), d_scr.as<float>(), d_pre.as<float>(), on,
        d_dm.as<float>());
    note_launch();
    k_prof_filter<<<((unsigned)dm0_rows.size() + 63) / 64, 64, 0, s>>>(
        d_rows_dm0.as<ProfRow>(), (int)dm0_rows.size(), d_scr.as<float>(), d_pre.as<float>(),
        on, d_dm0.as<float>());
    note_launch();
  }
  k_prof_ft<<<dim3((on + 127) / 128, (unsigned)out_nchans, (unsigned)ncands), 128, 0, s>>>(
      tf, nsamps, (int)C, (int)fscrunch, on, d_ftj.as<FtJob>(), d_ft.as<float>());
  note_launch();
  if (cudaGetLastError() != cudaSuccess) return HD_INTERNAL_GPU_ERROR;
  // normalise: each candidate's n_dm plot rows (a run of rows per candidate
  // when every window has the same trial count; else candidate by candidate)
  bool uniform = true;
  for (size_t i = 1; i < ncands; i++) uniform = uniform && n_dm[i] == n_dm[0];
  cudaError_t e = cudaSuccess;
  if (uniform) {
    e = normalise_rows(d_dm.as<float>(), on, ncands * n_dm[0], out_nsamps, (int)n_dm[0], plot,
                       false, s);
  } else {
    for (size_t i = 0; i < ncands && e == cudaSuccess; i++)
      e = normalise_rows(d_dm.as<float>() + i * plot, on, n_dm[i], out_nsamps, (int)n_dm[i],
                         plot, false, s);
  }
  if (e == cudaSuccess)
    e = normalise_rows(d_dm0.as<float>(), on, ncands, out_nsamps, 1, out_nsamps, false, s);
  if (e == cudaSuccess)
    e = normalise_rows(d_ft.as<float>(), on, ncands * out_nchans, out_nsamps, 1, out_nsamps,
                       false, s);
  if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? HD_MEM_ALLOC_FAILED
                                                              : HD_INTERNAL_GPU_ERROR;

  // ---- results to the host and the extractions (candidate_profiler.C:560-640)
  std::vector<float> h_dm(ncands * plot), h_dm0(ncands * out_nsamps);
  if (cudaMemcpyAsync(h_dm.data(), d_dm.p, h_dm.size() * sizeof(float), cudaMemcpyDeviceToHost,
                      s) ||
      cudaMemcpyAsync(h_dm0.data(), d_dm0.p, h_dm0.size() * sizeof(float),
                      cudaMemcpyDeviceToHost, s))
    return HD_MEM_COPY_FAILED;
  for (size_t i = 0; i < ncands; i++)
    if (out[i].freq_time &&
        cudaMemcpyAsync(out[i].freq_time, d_ft.as<float>() + i * out_nchans * out_nsamps,
                        out_nchans * out_nsamps * sizeof(float), cudaMemcpyDeviceToHost, s))
      return HD_MEM_COPY_FAILED;
  if (cudaStreamSynchronize(s) != cudaSuccess) return HD_INTERNAL_GPU_ERROR;
  for (size_t i = 0; i < ncands; i++) {
    hd_profile& o = out[i];
    const float* dmt = h_dm.data() + i * plot;
    const float* dm0 = h_dm0.data() + i * out_nsamps;
    if (o.dm_time) std::memcpy(o.dm_time, dmt, plot * sizeof(float));
    if (o.dm0_time) std::memcpy(o.dm0_time, dm0, out_nsamps * sizeof(float));
    // first maximum (std::max_element: a NaN never replaces a number)
    size_t mx = 0;
    for (size_t k = 1; k < plot; k++)
      if (dmt[mx] < dmt[k]) mx = k;
    o.max_idx = mx;
    o.n_dm = n_dm[i];
    o.dm_begin = dm_begin[i];
    const size_t dm_idx = cands[i].dm_idx;
    o.snr_dm_first = dm_idx > out_dm_count / 2 ? dm_idx - out_dm_count / 2 : 0;
    const size_t tmax = mx % out_nsamps, dmax = mx / out_nsamps;
    if (o.snr_dm)
      for (size_t d = 0; d < out_dm_count; d++)
        o.snr_dm[d] = d < n_dm[i] ? dmt[d * out_nsamps + tmax] : 0.f;
    if (o.snr_time) {
      const float width = (float)((size_t)1 << cands[i].filter);
      for (size_t t = 0; t < out_nsamps; t++) {
        float* r = o.snr_time + t * 5;
        r[0] = (float)((double)((float)cands[i].samp +
                                ((float)t - (float)(out_nsamps / 2)) * width) *
                       tsamp);
        r[1] = dmt[dmax * out_nsamps + t];
        r[2] = dmax > 0 ? dmt[(dmax - 1) * out_nsamps + t] : 0.f;
        r[3] = dmax + 1 < out_dm_count ? dmt[(dmax + 1) * out_nsamps + t] : 0.f;
        r[4] = dm0[t];
      }
    }
  }
  return HD_NO_ERROR;
}
