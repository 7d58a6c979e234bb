// internal.h -- declarations shared by the host pipeline and the kernels.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

struct hd_classifier_t;
struct hd_pipeline_t;

namespace hdb {

// cudaMalloc that, when it fails, also clears the failure from the runtime's
// last-error state (an allocation failure is not sticky; left there, it would
// be reported by the next launch check of an unrelated call).
template <class T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
  }
  return e;
}

// Kernel launches made by this library in this process (additive counter,
// read through hd_get_launch_count).
void note_launch();
unsigned long long launch_count();
// Adds n (may be negative) to the counter: a CUDA graph's kernel nodes are
// counted when the graph is launched, not when they are captured.
void add_launches(long long n);

// Raises the dynamic shared-memory limit of kernel `func` on the current
// device to at least `bytes`.  The limit is a process-wide attribute of the
// function and is never lowered here: host threads that launch the same
// kernel with different shared-memory sizes (the workers of a beam set) can
// then not pull it below what another thread's launch needs.
cudaError_t raise_smem_limit(const void* func, size_t bytes);
template <class F>
cudaError_t raise_smem_limit(F* func, size_t bytes) {
  return raise_smem_limit(reinterpret_cast<const void*>(func), bytes);
}

// ---- filterbank kernels (kernels_fb.cu) ------------------------------------
struct DedispArgs {
  const uint8_t* in;      // FT rows, channel c at in + c*in_pitch
  size_t in_pitch;
  const int* delays;      // [dm_count][nchans] delay in samples
  const int* blk_min;     // [n_dm_blocks][nchans] min delay over the block's DMs
  const int* chans;       // active (not killed) channel indices
  int nact;
  int nchans;
  int dm_count;
  size_t nout;            // output samples per DM
  float* out;
  size_t out_pitch;       // floats between DM rows (multiple of 4)
  int rowb;               // shared-memory row bytes (multiple of 16)
  unsigned* err;          // device error word (bit 0: staging wait timed out)
  int units;              // independent filterbanks dedispersed by one launch
  size_t in_unit;         // bytes between units' FT inputs
  size_t out_unit;        // floats between units' outputs
  unsigned wait_limit;    // polls of each bounded mbarrier wait
  // test of the error path: the producer issues no copy for the last stage,
  // so the consumers' wait on it runs out (HDB_TEST_WITHHOLD_STAGE=1)
  int withhold_last;
  // always 1: the multiplier of the kernel's multiply-add accumulations.  A
  // runtime value keeps them multiply-adds, which issue to the FMA pipe and
  // leave the ALU pipe (shifts, byte permutes, adds) to the rest of the work
  unsigned one;
};

// Dedispersion tile: DMs and output samples per CTA, channel rows staged per
// pipeline stage.  Every tile gives the same (exact integer) sums.
struct DedispTile {
  int dm_block, time_block, rows;
};
constexpr int kDedispDmBlocks[3] = {8, 16, 32};
// polls of a dedispersion mbarrier wait before it gives up and reports
constexpr unsigned kDedispWaitLimit = 1u << 22;
// candidate {dm_block, time_block} pairs: time_block = 128 K G with K output
// words per lane (1, 3 or 5) in G groups; the launcher maps each pair to its
// kernel instance
constexpr int kDedispTiles[11][2] = {{8, 1024}, {8, 640},  {8, 768},  {8, 1152},
                                     {8, 1280}, {16, 512}, {16, 384}, {16, 640},
                                     {16, 768}, {32, 256}, {32, 384}};
// rows per stage that fit shared memory for staged rows of rowb bytes (0: none)
int dedisp_rows_per_stage(int dm_block, int rowb);
size_t dedisp_smem_bytes(int dm_block, int rows, int rowb);
cudaError_t launch_dedisp(const DedispArgs& a, const DedispTile& t, cudaStream_t s);
// TF -> channel-major copy of `units` filterbanks (nsamps x nchans bytes each,
// consecutive in `in`); unit u's copy starts at out + u * out_unit.
cudaError_t launch_transpose_tf_ft(const uint8_t* in, size_t nsamps, int nchans, uint8_t* out,
                                   size_t pitch, cudaStream_t s, size_t units = 1,
                                   size_t out_unit = 0);
// The same from packed samples of nbits = 1, 2, 4 or 16 bits (nchans * nbits a
// multiple of 32; `in` 4-byte aligned): byte rows of the sample values, or for
// 16 bits the low bytes at `out` and the high bytes at `out + hi_off`.
cudaError_t launch_unpack_tf_ft(const uint8_t* in, size_t nsamps, int nchans, int nbits,
                                uint8_t* out, size_t pitch, cudaStream_t s, size_t units,
                                size_t out_unit, size_t hi_off);
// lo[r * pitch + k] = RN(lo + 256 hi) for k < n, r < rows (the two byte planes'
// exact integer sums of 16-bit input).
cudaError_t launch_combine_planes(float* lo, const float* hi, size_t pitch, size_t n, size_t rows,
                                  cudaStream_t s);
// Channel-major byte rows of `units` filterbanks of nbits-bit samples (8: a
// transpose; 1, 2, 4: unpacked; 16: low and high byte planes, the high plane
// `units * out_unit` bytes after the low one).
inline cudaError_t input_to_ft(const uint8_t* in, size_t nsamps, int nchans, int nbits,
                               uint8_t* out, size_t pitch, cudaStream_t s, size_t units,
                               size_t out_unit) {
  if (nbits == 8) return launch_transpose_tf_ft(in, nsamps, nchans, out, pitch, s, units, out_unit);
  return launch_unpack_tf_ft(in, nsamps, nchans, nbits, out, pitch, s, units, out_unit,
                             units * out_unit);
}
// Input sample widths the search and the dedisp_* calls accept.
inline bool nbits_supported(size_t nbits) {
  return nbits == 1 || nbits == 2 || nbits == 4 || nbits == 8 || nbits == 16;
}
// Scrunched channel-major copy of `units` inputs: out[c][u] = the mean of
// in[c][s u .. s u + s), rounded half up, for u < nsamps / s, and 0 from
// there to out_pitch.
cudaError_t launch_scrunch_ft(const uint8_t* in, size_t in_pitch, size_t nsamps, int nchans,
                              int s, uint8_t* out, size_t out_pitch, size_t units,
                              size_t in_unit, size_t out_unit, cudaStream_t st);
// Narrow-band RFI zapping of `units` TF filterbanks of nsamps spectra in
// place (the branch Pipeline/clean_filterbank_rfi.cu:303-351 disables);
// scratch of narrow_band_scratch_bytes().
size_t narrow_band_scratch_bytes(size_t units, size_t nsamps, int nchans, float dt,
                                 float baseline_length);
cudaError_t narrow_band(uint8_t* tf, size_t units, size_t nsamps, int nchans, float dt,
                        float baseline_length, float rfi_tol, void* scratch, cudaStream_t s);
cudaError_t launch_dm0_sum(const uint8_t* in, size_t nsamps, int nchans, float* out,
                           cudaStream_t s);
cudaError_t launch_zap(const uint8_t* in, size_t nsamps, int nchans, const int* mask,
                       unsigned max_resample_dist, uint8_t* out_ft, size_t pitch,
                       uint8_t* out_tf, cudaStream_t s);

// ---- series kernels (kernels_search.cu) ------------------------------------
// A batch of `nser` time series of `len` valid floats each, `pitch` floats
// apart, every series holding `nbeams` beams of `stride` samples (the last
// beam truncated by the dispersion delay: beam_count valid samples).
struct SeriesBatch {
  float* data;
  size_t pitch;
  int nser;
  size_t len;
  size_t stride;      // beam stride
  size_t beam_count;  // valid samples per beam
  int nbeams;
};

// Workspace for the median-of-5 trees (two ping-pong arrays).
struct TreeScratch {
  float* a;
  float* b;
  size_t cap;  // floats in each
};

// The baseline subtraction of remove_baseline (remove_baseline.cu:90-102):
// sample i < nsub of series ser becomes x - (stretched baseline at i).
struct BaselineSub {
  const float* base = nullptr;  // [ser][nbeams][sc] scrunched baseline samples
  unsigned sc = 0, stride = 0, last_start = 0, nsub = 0;
  int nbeams = 1;
  float step2 = 0.f, step3 = 0.f;  // stretch steps: beams 0..n-2, last beam
};

// Samples per beam of the scrunched baseline (remove_baseline.cu:38) and the
// tree scratch (floats per buffer) remove_baseline needs for nseg beams.
size_t baseline_samples(size_t stride, size_t smooth_radius);
size_t baseline_scratch(size_t stride, size_t smooth_radius, size_t nseg);
// RemoveBaselinePlan::exec for every series (Pipeline/remove_baseline.cu:21-160):
// the baseline is subtracted from the series in place.
cudaError_t remove_baseline(const SeriesBatch& sb, size_t smooth_radius, float* base_out,
                            TreeScratch& ws, cudaStream_t s);
// GetRMSPlanMB::exec_multibeam, vector form (Pipeline/get_rms.cu:236-270):
// rms[ser*nbeams + b].
cudaError_t rms_beams(const SeriesBatch& sb, float* rms, TreeScratch& ws, cudaStream_t s);
// normalise_multibeam (get_rms.cu:372-382) fused with the exclusive prefix sum
// of MatchedFilterPlan::prep (matched_filter.cu:21-32), sequential association:
// scan[ser][0..len] (len + 1 values, pitch scan_pitch).  norm_out (nullable,
// same layout as the batch) receives the normalised series.
// err (nullable): bit 1 is set if a staging wait timed out.
cudaError_t normalise_scan(const SeriesBatch& sb, const float* rms, float* scan,
                           size_t scan_pitch, float* norm_out, cudaStream_t s,
                           unsigned* err = nullptr);

// Per-width constants of the boxcar loop (Pipeline/pipeline.cu:657-776).
struct WidthInfo {
  int width;          // rel_filter_width
  int ts;             // rel_tscrunch_width
  int ahead, behind;  // matched_filter.cu:44-45
  int filter_idx;
  unsigned n;         // cur_nsamps_filtered
  unsigned bn;        // cur_beam_nsamps for the block RMS / giant window
  unsigned merge_dist;
  unsigned rel_off;   // rel_cur_filtered_offset
  int prev_cover;     // index of the latest earlier width whose n covers more
  int scr;            // cur_scrunch: trial scrunch x ts (index rescale)
};

struct WidthCtx {
  const float* scan;
  size_t scan_pitch;
  int nser;
  size_t stride;
  int nbeams;
  int offset;         // rel_boxcar_max / 2
  int nw;             // widths per series
  const WidthInfo* winfo;       // device copy
  const WidthInfo* host_winfo;  // host copy (launch decisions)
  size_t scan_len;              // valid prefix-sum entries per series (len + 1)
  int dms_per_unit;             // series per independent unit (beam searched alone)
  int dm_key_gap;               // giant DM key = unit * dm_key_gap + DM index
  int dm_offset;                // DM index of each unit's first series
  float* norm;        // [nser][nw]  1 / block_rms
  float thresh;
  // Largest |boxcar value| of each block-RMS group (gsize consecutive
  // filtered samples, ngroups complete groups per series) for the
  // unscrunched widths [0, gmax_nw): [nser][gmax_nw][ngroups].  block_rms
  // records it when gmax is set and the group geometry fits gmax_cap floats
  // (else ngroups = 0); count_hits skips the tiles whose covering groups
  // stay below every width's threshold.
  float* gmax;
  size_t gmax_cap;
  unsigned gsize, ngroups;
  int gmax_nw;
};

// Block RMS of width wi for every series (get_rms.cu:274-301 on the filtered
// series) -> ctx.norm[ser][wi].  Widths in [w_begin, w_end) are handled
// together; widths with ts > 1 must be passed one at a time after all earlier
// widths (their RMS window reads the earlier widths' normalised output).
cudaError_t block_rms(WidthCtx& ctx, const WidthInfo* host_winfo, int w_begin, int w_end,
                      TreeScratch& ws, cudaStream_t s);

// Threshold + ordered compaction of every (series, width) into hit lists.
struct HitBuffers {
  // tiles (ser * ntiles + tile) with at least one hit of an unscrunched width,
  // listed by count_hits for write_hits (list_valid when the list is complete)
  unsigned* tile_list;  // capacity nser * ntiles
  unsigned* tile_list_n;
  bool list_valid;
  unsigned* tile_cnt;   // [nser][nw][ntiles]
  unsigned* sw_cnt;     // [nser*nw + 1]
  unsigned* sw_off;     // [nser*nw + 1]
  unsigned* tile_off;   // [nser][nw][ntiles]
  unsigned* ind;        // hits
  float* val;
  unsigned* sw;
  size_t cap;
  unsigned ntiles;
};
cudaError_t count_hits(const WidthCtx& ctx, HitBuffers& hb, unsigned ntiles, cudaStream_t s);
cudaError_t scan_hit_counts(const WidthCtx& ctx, HitBuffers& hb, cudaStream_t s);
cudaError_t write_hits(const WidthCtx& ctx, HitBuffers& hb, cudaStream_t s);

// Device-wide exclusive scan of n unsigned values (out may alias in); the
// total is written to *total.  tmp needs scan_tmp_words(n) words.
size_t scan_tmp_words(size_t n);
cudaError_t scan_u32(const unsigned* in, unsigned* out, size_t n, unsigned* total, unsigned* tmp,
                     cudaStream_t s);

// Giant list (find_giants.cu + pipeline.cu:755-775).
struct GiantBuffers {
  unsigned* head;       // [hits]
  unsigned* gid;        // [hits]
  unsigned long long* key;  // [giants]
  float* peak;
  unsigned long long* ind;
  unsigned long long* begin;
  unsigned long long* end;
  int* filter;
  int* dm;
  int* label;
  size_t cap;
};
cudaError_t giant_heads(const WidthCtx& ctx, const HitBuffers& hb, unsigned nhits,
                        GiantBuffers& gb, cudaStream_t s);
cudaError_t giant_fill(const WidthCtx& ctx, const HitBuffers& hb, unsigned nhits,
                       unsigned ngiants, GiantBuffers& gb, cudaStream_t s);

// Places the n giants of one scrunch group (unit-major within the group) at
// dst_base[u] + (i - first[u]) of the combined list (unit u from the DM key);
// labels and keys are not copied.
cudaError_t giant_place(const GiantBuffers& src, unsigned n, int dm_key_gap,
                        const unsigned* first, const unsigned* dst_base, GiantBuffers& dst,
                        cudaStream_t s);

// label_candidate_clusters (Pipeline/label_candidate_clusters.cu:203-394),
// sequential-sweep semantics; iterates until stable.
struct ClusterArgs {
  int ngiants;
  unsigned long long time_tol, filter_tol, dm_tol, nsamps_beam;
  // giants per unit at most (a giant's DM window never leaves its unit):
  // sizes the sweep grid's chunks of earlier giants (0: ngiants)
  int max_unit_giants;
};
cudaError_t cluster_init(GiantBuffers& gb, int ngiants, cudaStream_t s);
cudaError_t cluster_sweep(const ClusterArgs& a, GiantBuffers& gb, unsigned* changed,
                          cudaStream_t s);

// merge_candidates (Pipeline/merge_candidates.cu:74-134) + DM gather.
struct GroupRow {
  float peak;
  float dm;
  unsigned long long ind, begin, end, filter, dm_ind, members, unit;
};
// offs[u] = first giant of unit u (u = 0..units; offs[units] = n).
cudaError_t unit_giant_offsets(const GiantBuffers& gb, int n, int dm_key_gap, int units,
                               unsigned* offs, cudaStream_t s);
cudaError_t merge_groups(const GiantBuffers& gb, int ngiants, int dm_key_gap, const float* dm_list,
                         unsigned* root_flag, unsigned* root_off, unsigned* nroots,
                         unsigned* scan_tmp, unsigned long long* gkey, GroupRow* rows,
                         cudaStream_t s);

// Device-count forms of the stages after thresholding, for a gulp captured as
// a CUDA graph: the totals are device words (*nhits from the hit scan,
// *ngiants written here), the grids are sized by the capacities hcap and
// gcap, and every kernel clamps to them.
// giants_dev: heads over hcap hit slots, their scan (-> *ngiants), giant
// maxima, begin/end, filter, DM key, peak and index.  scan_tmp needs
// scan_tmp_words(max(hcap, gcap)) words.
cudaError_t giants_dev(const WidthCtx& ctx, const HitBuffers& hb, const unsigned* nhits,
                       unsigned hcap, GiantBuffers& gb, unsigned gcap, unsigned* ngiants,
                       unsigned* scan_tmp, cudaStream_t s);
// cluster_merge_dev: unit offsets (unit_off[0..units]), `pairs` pairs of
// clustering sweeps (flags[2 pairs]: flag 2p + 1 stays 0 when pair p reached
// the fixed point; later pairs do nothing), then the merge into rows with the
// group count in *nroots.  geo: 2 device ints.  gkey: 2 gcap words.
cudaError_t cluster_merge_dev(const ClusterArgs& a, GiantBuffers& gb, unsigned gcap,
                              const unsigned* ngiants, int units, int dm_key_gap,
                              unsigned* unit_off, int* geo, unsigned* flags, int pairs,
                              const float* dm_list, unsigned* root_flag, unsigned* root_off,
                              unsigned* nroots, unsigned* scan_tmp, unsigned long long* gkey,
                              GroupRow* rows, cudaStream_t s);

// RFI mask of clean_filterbank_rfi (clean_filterbank_rfi.cu:447-506) from the
// normalised zero-DM series and its prefix sum.
cudaError_t rfi_mask(const float* x, const float* scan, size_t count, size_t boxcar_max,
                     float rfi_tol, int* mask, int* fmask, cudaStream_t s);

// One candidate's patch extraction (Applications/candidate_profiler.C).
struct PatchJob {
  unsigned series0;    // first series of the candidate's filterbank (unit x D)
  int dm, ndm;         // DM trial, trials per filterbank
  unsigned ind;        // sample index in the dedispersed series
  int filter;          // boxcar width index (width 2^filter)
  unsigned unit;       // filterbank of the batch
  long long ft_first;  // first input sample of the freq-time window (may be < 0)
  unsigned ft_ts;      // samples per freq-time bin
};
// DM-time (64 x 64) and freq-time (64 x 256) patches of njobs candidates
// (device job list), normalised per row; outputs njobs x 4096 / 16384 floats.
cudaError_t extract_patches(const float* scan, size_t scan_pitch, size_t len, const uint8_t* tf,
                            size_t nsamps, int nchans, const PatchJob* jobs, int njobs,
                            float* dm_out, float* ft_out, cudaStream_t s);

// BF16 GEMM on tcgen05 (umma.cu): C(m, n) (+)= sum_k A[m*lda + k] B[n*ldb + k]
// with C(m, n) at C[m*scm + n*scn]; N <= 128, K, lda, ldb multiples of 8,
// A and B 16-byte aligned (else cudaErrorNotSupported).  splits > 1 splits K
// and needs a workspace of umma_workspace_floats() floats; the splits are
// added in order.  *err records a bounded wait that gave up.
size_t umma_workspace_floats(int M, int N, int K, int splits);
cudaError_t umma_gemm(int M, int N, int K, const void* A, long long lda, const void* B,
                      long long ldb, float* C, long long scm, long long scn, int accumulate,
                      int splits, float* ws, unsigned* err, cudaStream_t s);

// normalise_series_array (candidate_profiler.C:88-134) on nrows rows of n
// floats: row r at data + (r / rows_per_group) * group_pitch + (r %
// rows_per_group) * pitch.  zero_flat: a row with zero deviation becomes 0
// (else the reference's division by zero is kept).
cudaError_t normalise_rows(float* data, int n, size_t nrows, size_t pitch, int rows_per_group,
                           size_t group_pitch, bool zero_flat, cudaStream_t s);
// 256 entries of x / 255 * 255 in float (the profiler's sample scaling)
__device__ __forceinline__ float prof_scale(unsigned x) {
  return __fmul_rn(__fdiv_rn((float)x, 255.f), 255.f);
}

// Scores of n device-resident patch pairs with the classifier, after `after`
// (an event recorded where the patches were written); scores to host memory.
cudaError_t classifier_score_device(struct ::hd_classifier_t* c, const float* d_dm,
                                    const float* d_ft, size_t n, cudaEvent_t after,
                                    float* scores);
int classifier_device(struct ::hd_classifier_t* c);
int pipeline_device(struct ::hd_pipeline_t* p);

}  // namespace hdb
