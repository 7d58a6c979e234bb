/*
 * heimdall_b200.h -- C interface of the B200 single-pulse search library
 * (libhdb200.so).
 *
 * Drop-in for Heimdall's pipeline API.  Each declaration below replaces the
 * reference interface cited beside it with the same name, argument meaning,
 * error codes and ownership rules:
 *
 *   Pipeline/hd/types.h:12-48           hd_byte/hd_size/hd_float, hd_pipeline,
 *                                       RawCandidates, ConstRawCandidates,
 *                                       Candidates (C++), hd_range_t
 *   Pipeline/hd/params.h:19-78          struct hd_params (same fields, order)
 *   Pipeline/hd/error.h:19-41           hd_error codes, hd_get_error_string
 *   Pipeline/hd/pipeline.h:10-28        hd_create_pipeline, hd_preallocate,
 *                                       hd_get_max_overlap, hd_execute,
 *                                       hd_destroy_pipeline
 *   Pipeline/hd/default_params.h:16     hd_set_default_params
 *   Pipeline/hd/parse_command_line.h:16-17  hd_parse_command_line, hd_print_usage
 *   Pipeline/hd/clean_filterbank_rfi.h  hd_clean_filterbank_rfi
 *
 * Additions (no reference counterpart; the reference only writes candidates to
 * a .cand file or a socket): hd_set_cleaning, hd_set_narrow_band,
 * hd_execute_device, hd_execute_beams, hd_get_candidates,
 * hd_get_beam_candidates, hd_get_raw_candidates, hd_get_giants, hd_get_timing,
 * hd_get_dedisp_tile, hd_get_dedisp_tile_source, hd_get_launch_count, hd_measure_int_add_rate,
 * hd_clean_filterbank_rfi_noalloc, hd_set_graphs, hd_get_graph_replays;
 * beam sets (hd_*_beam_set*); sigproc input and the gulp loop
 * (hd_read_sigproc_header, hd_mjd_to_utc, hd_params_from_sigproc,
 * hd_search_sigproc_file, hd_search_sigproc_files); the coincidencer (hd_coincide,
 * hd_write_coincident_candidates); the candidate classifier
 * (hd_extract_patches, hd_score_candidates, hd_classifier_*); the candidate
 * profiler (hd_profile_candidates, Applications/candidate_profiler.C).
 *
 * Ownership and threading: the caller owns every host buffer it passes; the
 * pipeline owns all device memory, its CUDA stream and events.  A pipeline
 * object is used by one thread at a time; separate pipelines are independent
 * (no global state), so one pipeline per thread or per GPU is safe.
 *
 * The struct layout of hd_params depends on HAVE_PSRDADA exactly as in the
 * reference: build the library and the caller with the same setting.
 */
#ifndef HEIMDALL_B200_H
#define HEIMDALL_B200_H

#include <stdbool.h>
#include <stddef.h>
#include <time.h>
#ifdef HAVE_PSRDADA
#include <sys/types.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned char          hd_byte;
typedef size_t                 hd_size;
typedef float                  hd_float;
typedef struct hd_pipeline_t*  hd_pipeline;

/* Candidate arrays (Pipeline/hd/types.h:18-42): one entry per candidate in
 * each array. */
struct RawCandidates {
  hd_float* peaks;
  hd_size*  inds;
  hd_size*  begins;
  hd_size*  ends;
  hd_size*  filter_inds;
  hd_size*  dm_inds;
  hd_size*  members;
};
struct ConstRawCandidates {
  const hd_float* peaks;
  const hd_size*  inds;
  const hd_size*  begins;
  const hd_size*  ends;
  const hd_size*  filter_inds;
  const hd_size*  dm_inds;
  const hd_size*  members;
};

typedef struct hd_range {
  hd_size start;
  hd_size end;
} hd_range_t;

struct hd_params {
  int          verbosity;
#ifdef HAVE_PSRDADA
  key_t        dada_id;
#endif
  const char*  sigproc_file;
  bool         yield_cpu;
  hd_size      nsamps_gulp;
  hd_size      dm_gulp_size;
  hd_float     baseline_length;     /* seconds */
  hd_size      beam;                /* 0-based index of the first beam */
  hd_size      nbeams;
  bool         override_beam;
  hd_size      nchans;
  hd_float     dt;                  /* seconds */
  hd_float     f0;                  /* MHz, channel 0 */
  hd_float     df;                  /* MHz per channel */
  hd_float     dm_min;
  hd_float     dm_max;
  hd_float     dm_tol;
  hd_float     dm_pulse_width;      /* microseconds */
  hd_size      dm_nbits;
  bool         use_scrunching;
  hd_float     scrunch_tol;
  hd_float     rfi_tol;
  hd_size      rfi_min_beams;
  hd_size      boxcar_max;
  hd_float     detect_thresh;
  hd_size      cand_sep_time;
  hd_size      cand_sep_filter;
  hd_size      cand_sep_dm;
  hd_size      cand_rfi_dm_cut;
  hd_float     max_giant_rate;
  hd_size      min_tscrunch_width;
  const char*  coincidencer_host;
  int          coincidencer_port;
  unsigned int num_channel_zaps;
  hd_range_t*  channel_zaps;
  hd_size      beam_count;
  int          gpu_id;
  time_t       utc_start;
  hd_size      spectra_per_second;
  const char*  output_dir;
};

typedef int hd_error;
enum {
  HD_NO_ERROR = 0,
  HD_MEM_ALLOC_FAILED,
  HD_MEM_COPY_FAILED,
  HD_INVALID_DEVICE_INDEX,
  HD_DEVICE_ALREADY_SET,
  HD_INVALID_PIPELINE,
  HD_INVALID_POINTER,
  HD_INVALID_STRIDE,
  HD_INVALID_NBITS,
  HD_PRIOR_GPU_ERROR,
  HD_INTERNAL_GPU_ERROR,
  HD_TOO_FEW_NSAMPS,
  HD_TOO_MANY_EVENTS,
  HD_UNKNOWN_ERROR
};

const char* hd_get_error_string(hd_error error);

void hd_set_default_params(struct hd_params* params);
int  hd_parse_command_line(int argc, char* argv[], struct hd_params* params);
void hd_print_usage(void);

hd_error hd_create_pipeline(hd_pipeline* pipeline, struct hd_params params);
hd_error hd_preallocate(hd_pipeline pipeline, hd_size nsamps, hd_size nbeams);
hd_size  hd_get_max_overlap(hd_pipeline pipeline, hd_size nbeams);
/* One gulp: nsamps spectra (nbeams beams of nsamps/nbeams spectra each, time
 * concatenated) of nchans*nbits/8 bytes.  nbits is 1, 2, 4, 8 or 16 (the
 * widths dedisp reads; samples packed little-endian, channel c the nbits-bit
 * field at bit (c mod (32/nbits))*nbits of 32-bit word c/(32/nbits), as the
 * reference's writer packs them, Formats/giant_maker.C:385-392); nchans a
 * multiple of 4 and nchans*nbits a multiple of 32 (whole 32-bit words per
 * spectrum, as Pipeline/clean_filterbank_rfi.cu:202-212 assumes), else
 * HD_INVALID_NBITS / HD_INVALID_STRIDE.  Widths other than 8 are refused
 * (HD_INVALID_NBITS) with cleaning on (hd_set_cleaning), with a prefetched
 * gulp, and, for 16 bits, with adaptive dt; every width is searched through
 * the same integer sums, so a gulp of values below 256 gives the same
 * candidates at any width.  Candidates go to
 * <output_dir>/<UTC>_<beam+1>.cand as in Pipeline/pipeline.cu:1001-1044
 * (output_dir == NULL: no file).  Returns HD_TOO_MANY_EVENTS (soft) when the
 * giant rate exceeds max_giant_rate. */
hd_error hd_execute(hd_pipeline pipeline, const hd_byte* h_filterbank, hd_size nsamps,
                    hd_size nbits, hd_size first_idx, hd_size nbeams,
                    hd_size* nsamps_processed);
void     hd_destroy_pipeline(hd_pipeline pipeline);

/* Zero-DM RFI excision of Pipeline/clean_filterbank_rfi.cu:256-528 on host
 * buffers (8-bit data): h_out receives the cleaned filterbank, h_mask (may be
 * NULL) the per-spectrum RFI mask. */
hd_error hd_clean_filterbank_rfi(hd_pipeline pipeline, const hd_byte* h_in, hd_size nsamps,
                                 hd_size nbits, hd_byte* h_out, int* h_mask,
                                 hd_float dt, hd_float baseline_length, hd_float rfi_tol,
                                 hd_size boxcar_max, hd_size nbeams);

/* ---- additions ---------------------------------------------------------- */

/* Switches the zero-DM RFI cleaning stage on or off (default: off).  The
 * reference selects it at compile time (Pipeline/pipeline.cu:72-74,255-299,
 * #ifdef CLEANING) and its shipped build leaves it off; enabling it here is
 * the reference built with -DCLEANING. */
hd_error hd_set_cleaning(hd_pipeline pipeline, int enable);
/* Narrow-band RFI zapping before the broadband stage when cleaning is on: the
 * branch of Pipeline/clean_filterbank_rfi.cu:303-351 that the reference
 * disables (`nbits > 4 && false`), with measure_bandpass.cu:45-275.  Off by
 * default, as in the reference.  Per stretch of baseline_length / dt spectra
 * the bandpass and its deviation are measured from 3125 drawn spectra and
 * bytes further than rfi_tol deviations from the bandpass are replaced by
 * nearby channels; the reference's functor reads the bytes it is rewriting,
 * and the result here is the one it gives in index order.  Needs nchans >= 20. */
hd_error hd_set_narrow_band(hd_pipeline pipeline, int enable);

/* hd_execute on a filterbank already in device memory (same layout; a
 * device-to-device copy replaces the host-to-device one). */
hd_error hd_execute_device(hd_pipeline pipeline, const hd_byte* d_filterbank, hd_size nsamps,
                           hd_size nbits, hd_size first_idx, hd_size nbeams,
                           hd_size* nsamps_processed);

/* Batched search of independent filterbanks.  No counterpart in the
 * reference, which runs one heimdall process per beam of a multibeam receiver
 * (each calling hd_execute on its own stream of data).
 *
 * Searches nfilterbanks filterbanks of the same shape (nsamps x nchans bytes
 * each, every one holding nbeams time-concatenated beams as in hd_execute)
 * with this pipeline's configuration in one pass: each stage runs over the
 * DM trials of all of them at once, and giants are never clustered across
 * filterbanks.  The result for filterbank u -- its candidates, its .cand file
 * and its status -- is identical to hd_execute(filterbanks[u], nsamps, nbits,
 * first_idx, nbeams, ...) on a pipeline whose params.beam is beams[u]
 * (beams may be NULL: params.beam + u * nbeams).
 *
 * filterbanks: host pointers, or device pointers when on_device != 0.
 * statuses (may be NULL): per filterbank HD_NO_ERROR or HD_TOO_MANY_EVENTS
 * (giant-rate bail-out, whose candidates are dropped).  The call returns
 * HD_TOO_MANY_EVENTS if any filterbank bailed out, else the first error.
 * Limit: nfilterbanks x (number of DM trials) <= 65535 (HD_INVALID_STRIDE
 * otherwise).  Candidates: hd_get_candidates (all, filterbank by filterbank)
 * or hd_get_beam_candidates (one filterbank). */
hd_error hd_execute_beams(hd_pipeline pipeline, const hd_byte* const* filterbanks,
                          hd_size nfilterbanks, hd_size nsamps, hd_size nbits,
                          hd_size first_idx, hd_size nbeams, const hd_size* beams,
                          int on_device, hd_error* statuses, hd_size* nsamps_processed);

/* Allocation-free zero-DM RFI cleaning.  No counterpart in the reference.
 *
 * For callers that must not allocate device memory while they run -- a
 * real-time ingest loop where a cudaMalloc/cudaFree would synchronise the
 * device and stall other streams, or a process whose device memory is
 * committed up front.  Same computation as hd_clean_filterbank_rfi, but on
 * caller-owned device buffers (d_in: nsamps x nchans bytes, d_out: same size,
 * d_mask: nsamps ints), queued on `stream` (a cudaStream_t, NULL = default
 * stream) without waiting for it, and with every scratch buffer taken from one
 * fixed array of HD_NOALLOC_SCRATCH_BYTES that this library reserves on each
 * GPU where its device code is loaded, until the process exits.  It performs
 * no cudaMalloc, cudaFree or other allocating call.
 *
 * Limits: nsamps <= HD_NOALLOC_MAX_NSAMPS, nbeams <= HD_NOALLOC_MAX_BEAMS,
 * boxcar_max <= 128, and beams long enough for the baseline's median trees to
 * fit the array; other requests return HD_INVALID_STRIDE (with a message on
 * stderr).  The first call on each device looks up the scratch array's device
 * address (cudaGetSymbolAddress), so make that first call before any stream
 * capture; the address is kept for the life of the process, so the call is not
 * for use after cudaDeviceReset.  All calls share the one array: calls whose
 * work overlaps on the GPU (e.g. on two streams at once) race and must be
 * serialised by the caller.
 *
 * d_status (a caller-owned device word, may be NULL) receives 0, or a nonzero
 * value if a bounded wait inside the cleaning kernels gave up (the mask and
 * the cleaned bytes are then not valid); it is written on `stream`, so read
 * it after the stream has finished the call's work. */
#define HD_NOALLOC_MAX_NSAMPS    524288u
#define HD_NOALLOC_MAX_BEAMS     64u
#define HD_NOALLOC_SCRATCH_BYTES 11534336u
hd_error hd_clean_filterbank_rfi_noalloc(const hd_byte* d_in, hd_size nsamps, hd_size nchans,
                                         hd_size nbits, hd_byte* d_out, int* d_mask,
                                         hd_float dt, hd_float baseline_length,
                                         hd_float rfi_tol, hd_size boxcar_max, hd_size nbeams,
                                         void* stream, unsigned* d_status);

/* ---- Candidate profiler (Applications/candidate_profiler.C) on the GPU ----
 *
 * The reference's candidate_profiler application makes, for one candidate of
 * a sigproc file, a DM-time plot (candidate_profiler.C:232-415, the trials
 * around the candidate re-dedispersed over a window of the file with adaptive
 * dt), a DM-0 series, a freq-time plot (:136-230), SNR vs DM and SNR vs time
 * (:560-640), and writes them to freq_time.dat, snr_dm.dat, snr_time.dat and
 * dm_time.pgm.  hd_profile_candidates computes the same arrays on the GPU for
 * a batch of candidates of one filterbank (nsamps x nchans bytes, 8-bit,
 * time-major; host memory, or device memory with on_device) whose header
 * values are tsamp, fch1 and foff, with the DM list dm_list.  Samples past the
 * end of the filterbank read as 0, as past the end of the file; a freq-time
 * window that would start before the first sample reads 0 there.  Rows with
 * no deviation come out NaN or +-inf (the reference's division by zero).
 * Per candidate (out[i]; any array may be NULL):
 *   dm_time   out_dm_count x out_nsamps: rows [0, n_dm) are trials
 *             dm_begin ... of the window, later rows 0;
 *   dm0_time  out_nsamps;
 *   freq_time (nchans / fscrunch) x out_nsamps;
 *   max_idx   index of the first maximum of dm_time;
 *   snr_dm    out_dm_count: dm_time at max_idx's time for trial
 *             snr_dm_first + d (0 for d >= n_dm);
 *   snr_time  out_nsamps x 5: time (s), dm_time on max_idx's row, on the rows
 *             above and below it (0 outside the plot), and dm0_time.
 * Limits: out_nsamps in [2, 4096], nchans a multiple of fscrunch, at most
 * 65535 dedispersed rows (candidates x (window trials + 1)) per call.  The
 * call allocates its device memory and returns when the results are on the
 * host. */
typedef struct hd_profile_request {
  hd_size samp;     /* sample index of the candidate in the filterbank */
  hd_size filter;   /* boxcar width index (width 2^filter) */
  hd_size dm_idx;   /* trial of dm_list */
} hd_profile_request;
typedef struct hd_profile {
  hd_float* dm_time;
  hd_float* dm0_time;
  hd_float* freq_time;
  hd_float* snr_dm;
  hd_float* snr_time;
  hd_size   max_idx, n_dm, dm_begin, snr_dm_first;
} hd_profile;
hd_error hd_profile_candidates(const hd_byte* filterbank, hd_size nsamps, hd_size nchans,
                               int on_device, double tsamp, double fch1, double foff,
                               const hd_float* dm_list, hd_size dm_count,
                               const hd_profile_request* cands, hd_size ncands,
                               hd_size out_nsamps, hd_size out_dm_count, hd_size fscrunch,
                               int do_filter, hd_profile* out);

/* ---- Learned candidate classifier (no counterpart in the reference) ----
 *
 * Patches per candidate (float, row-major): a DM-time patch of 64 DM trials
 * (the candidate's trial at row 32) x 64 boxcar-filtered samples, and a
 * frequency-time patch of 64 sub-bands x 256 time bins of the undispersed
 * filterbank around the candidate, each row detrended and scaled as the
 * reference's candidate profiler does (Applications/candidate_profiler.C:
 * 88-134 normalise_series_array, 136-230 gen_freq_time_plot, 232-415
 * gen_dm_time_plot).  The classifier is a two-branch CNN (3 conv layers per
 * branch, 2 fully connected layers, 175666 parameters) trained and evaluated
 * on the GPU with BF16 tensor-core GEMMs accumulating in FP32; patch values
 * enter the network limited to +-16.  Its score
 * (probability of a dispersed pulse) only ranks or flags candidates; the
 * candidate list itself is unchanged. */
#define HD_PATCH_DM_TIME   4096   /* 64 x 64 floats per candidate */
#define HD_PATCH_FREQ_TIME 16384  /* 64 x 256 floats per candidate */
typedef struct hd_classifier_t* hd_classifier;

/* Patches of every candidate of the last hd_execute / hd_execute_beams, in
 * hd_get_candidates order.  Copies min(*count, available) patches (either
 * output may be NULL) and sets *count to the number available.  Needs
 * nchans a multiple of 64 and a gulp searched at the native resolution
 * (HD_INVALID_STRIDE after a gulp with adaptive dt, whose trials have
 * different lengths).  Call before the next execute (it reads that gulp's
 * device buffers). */
hd_error hd_extract_patches(hd_pipeline pipeline, hd_float* dm_time, hd_float* freq_time,
                            hd_size* count);

hd_size  hd_classifier_param_count(void);
hd_error hd_classifier_create(hd_classifier* classifier, int gpu_id, unsigned long long seed);
void     hd_classifier_destroy(hd_classifier classifier);
/* FP32 parameters, layout: per conv layer (branch A layers 1-3, then branch
 * B) W [co][ci*9] then b [co]; W1 [16][10240], b1 [16], W2 [2][16], b2 [2]. */
hd_error hd_classifier_get_params(hd_classifier classifier, hd_float* params, hd_size count);
hd_error hd_classifier_set_params(hd_classifier classifier, const hd_float* params,
                                  hd_size count);
/* Gradient of the mean cross-entropy over n labelled patches (one batch,
 * n <= 4096), without updating the parameters. */
hd_error hd_classifier_gradients(hd_classifier classifier, const hd_float* dm_time,
                                 const hd_float* freq_time, const int* labels, hd_size n,
                                 hd_float* grads, hd_float* loss);
/* Adam training on n labelled patches (label 1 = dispersed pulse); the mean
 * loss of each epoch goes to epoch_loss[epoch] (may be NULL). */
hd_error hd_classifier_train(hd_classifier classifier, const hd_float* dm_time,
                             const hd_float* freq_time, const int* labels, hd_size n,
                             int epochs, int batch, hd_float lr, unsigned long long seed,
                             hd_float* epoch_loss);
/* Probability of a dispersed pulse for each of n patches. */
hd_error hd_classifier_score(hd_classifier classifier, const hd_float* dm_time,
                             const hd_float* freq_time, hd_size n, hd_float* scores);
/* The same with the patches in device memory of the classifier's GPU
 * (n x HD_PATCH_DM_TIME and n x HD_PATCH_FREQ_TIME floats); scores to host. */
hd_error hd_classifier_score_device(hd_classifier classifier, const hd_float* d_dm_time,
                                    const hd_float* d_freq_time, hd_size n, hd_float* scores);
/* Scores of the candidates of the last hd_execute / hd_execute_beams, in
 * hd_get_candidates order: patches are extracted and scored on the GPU (the
 * pipeline and the classifier must share it) and only the scores are copied
 * back.  Writes min(*count, available) scores and sets *count to the number
 * available.  The candidate list is not changed. */
hd_error hd_score_candidates(hd_pipeline pipeline, hd_classifier classifier, hd_float* scores,
                             hd_size* count);
/* Device time (ms, CUDA events on the classifier's stream) of the last
 * scoring call, from its first upload or conversion to its last score copy. */
hd_error hd_classifier_get_timing(hd_classifier classifier, hd_float* ms);
/* The classifier's GEMM on device operands, for testing: C (m x n, FP32) =
 * A (m x k, BF16) x B (k x n, BF16) with element strides A(i, l) =
 * A[i*sam + l*sak], B(l, j) = B[l*sbk + j*sbn], C(i, j) = C[i*scm + j*scn];
 * accumulate adds to C; splits > 1 sums K in parts atomically into C. */
hd_error hd_bf16_gemm(int m, int n, int k, const void* d_a, long long sam, long long sak,
                      const void* d_b, long long sbk, long long sbn, float* d_c,
                      long long scm, long long scn, int accumulate, int splits);
/* The same product on the fifth-generation tensor cores, as the classifier's
 * training runs its convolutions and fully connected layer (tcgen05.mma with
 * FP32 accumulators in tensor memory, operands staged by TMA), for testing:
 * A and B K-major (sak == 1, sbk == 1), n <= 128, k, sam and sbn multiples of
 * 8 and 16-byte aligned operands (else HD_INVALID_STRIDE); splits > 1 sums K
 * in parts through a workspace, added in order (deterministic). */
hd_error hd_bf16_gemm_tc(int m, int n, int k, const void* d_a, long long sam, long long sak,
                         const void* d_b, long long sbk, long long sbn, float* d_c,
                         long long scm, long long scn, int accumulate, int splits);

/* Dedispersion tile of the last gulp: DM trials and output samples per CTA
 * and channel rows staged per pipeline stage.  The first gulp of each shape
 * times every tile that fits shared memory and keeps the fastest (environment:
 * HDB_DEDISP_TUNE=0 keeps 16 x 512, HDB_DEDISP_TILE=DBxTB forces one); all
 * tiles give the same sums.  The choice is kept across processes in a tile
 * cache file, keyed by the device, the gulp shape and the delay table:
 * HDB_TUNE_CACHE=path, else $XDG_CACHE_HOME/heimdall_b200/dedisp_tiles.txt,
 * else $HOME/.cache/heimdall_b200/dedisp_tiles.txt; HDB_TUNE_CACHE=0 turns it
 * off. */
hd_error hd_get_dedisp_tile(hd_pipeline pipeline, int* dm_block, int* time_block, int* rows);

/* Where the last gulp's dedispersion tile came from: 0 the default tile,
 * 1 forced by HDB_DEDISP_TILE, 2 timed by the autotuner in this process,
 * 3 read from the tile cache; -1 for a null pipeline. */
int hd_get_dedisp_tile_source(hd_pipeline pipeline);

/* Number of kernels this library has launched in this process (a CUDA
 * graph's kernels counted at each replay). */
unsigned long long hd_get_launch_count(void);

/* The batched calls with device-resident input (hd_execute_beams with
 * on_device != 0, hd_execute_prefetched) run each gulp as one CUDA graph
 * replay once its shape (filterbank count, spectra, beams, cleaning, DM
 * trials) has been searched once: the first gulp of a shape runs on the
 * host-sized path and fixes the shape's hit and giant capacities and its
 * number of clustering sweeps; later gulps of the shape launch one captured
 * graph (one per set of input buffers) with every total kept on the device,
 * and the host reads the results once.  A gulp whose totals exceed the
 * capacities, or whose clustering needs more sweeps, is searched again on
 * the host-sized path and the shape's capacities grow: results never depend
 * on the form.  Adaptive dt, narrow-band zapping and input other than 8-bit
 * stay on the host-sized path.  hd_set_graphs(p, 0) turns the graph form off
 * (the environment variable HDB_NO_GRAPH=1 does so for new pipelines);
 * hd_get_graph_replays counts the gulps it served.  No reference
 * counterpart (the reference synchronises after every stage). */
hd_error hd_set_graphs(hd_pipeline pipeline, int enable);
unsigned long long hd_get_graph_replays(hd_pipeline pipeline);

/* Measured throughput of 32-bit integer adds on `device` (adds per second):
 * independent add chains on every SM, timed with CUDA events (best of three
 * launches after one warm-up).  The denominator of the integer-add roofline
 * of the dedispersion kernel.  No reference counterpart. */
hd_error hd_measure_int_add_rate(int device, double* adds_per_second);

/* One row of the .cand file (Pipeline/pipeline.cu:1028-1038). */
typedef struct hd_candidate {
  hd_float snr;
  hd_size  samp_idx;
  hd_float time;
  hd_size  filter;
  hd_size  dm_trial;
  hd_float dm;
  hd_size  members;
  hd_size  begin;
  hd_size  end;
  hd_size  beam;
} hd_candidate;

/* Cross-beam coincidence of candidate lists on the GPU (no C counterpart:
 * the reference's coincidencer does it in C++, Applications/Candidates.C
 * compute_coincidence 236-291 with Candidate::is_coincident 64-77).
 * cands[i].beam (1..nbeams) selects each candidate's beam list; within a
 * beam, the input order is the list order.  For every candidate, out[i]
 * holds the number of beams with a coincident candidate (itself included),
 * the beam and S/N of the brightest first-coincident one (itself when none
 * is brighter). */
typedef struct {
  unsigned int nbeams;
  unsigned int primary_beam;
  hd_float     max_snr;
} hd_coincidence;
hd_error hd_coincide(const hd_candidate* candidates, hd_size count, hd_size nbeams,
                     unsigned int sep_time, unsigned int sep_filter, int gpu_id,
                     hd_coincidence* out);
/* The reference's _all.cand lines (Candidates.C:85-93, 293-326): beam by
 * beam, each with the coincidence columns. */
hd_error hd_write_coincident_candidates(const char* path, const hd_candidate* candidates,
                                        const hd_coincidence* coincidence, hd_size count);

/* Sigproc filterbank input and the gulp loop (no C counterpart in the
 * reference: Formats/hd/header.h and SigprocFile.C read the file in C++,
 * Applications/heimdall.C:153-292 runs the loop).
 *
 * The header fields the reference reads (Formats/hd/header.h:26-56);
 * strings are NUL-terminated, size is the header's length in bytes, and a
 * missing nsamples is the whole file's size over one spectrum's bytes
 * (header.h:190-193, header included). */
typedef struct {
  char   source_name[80];
  char   rawdatafile[80];
  double az_start, za_start, src_raj, src_dej, tstart, tsamp, period, fch1, foff, refdm;
  int    nchans, telescope_id, machine_id, data_type, ibeam, nbeams, nbits, barycentric,
         pulsarcentric, nbins, nsamples, nifs, npuls;
  unsigned char signed_data;
  int    size;
  int    unknown_keys;   /* keywords the reader does not know (the reference warns) */
} hd_sigproc_header;

hd_error hd_read_sigproc_header(const char* path, hd_sigproc_header* header);
/* MJD -> Unix time as the reference's data sources convert tstart
 * (Formats/hd/DataSource.h:49-82, local time zone through mktime). */
long long hd_mjd_to_utc(double mjd);
/* The hd_params fields heimdall.C takes from its data source: nchans, dt,
 * f0, df, nbeams, beam (ibeam - 1 unless override_beam), utc_start and
 * spectra_per_second. */
hd_error hd_params_from_sigproc(const hd_sigproc_header* header, struct hd_params* params);
/* Called after every gulp with that gulp's candidates (as hd_get_candidates)
 * and the first sample index of the gulp. */
typedef void (*hd_gulp_callback)(void* user, const hd_candidate* candidates, hd_size count,
                                 hd_size first_idx);
/* Searches a sigproc file of 1, 2, 4, 8 or 16-bit samples (packed as
 * hd_execute documents; the same width limits) gulp by gulp as heimdall.C's
 * loop does: the
 * first gulp is nsamps_gulp spectra, each later one the previous gulp's
 * unprocessed overlap (boxcar_max + max_delay per beam) followed by
 * nsamps_gulp new spectra; a block shorter than nsamps_gulp ends the search
 * and is not searched.  With nbeams > 1 in the header each block holds the
 * beams in sequence.  The overlap stays on the device; the next block is
 * read from the file and copied to the device while the GPU searches.
 * Candidates go to the pipeline's .cand files and to on_gulp (may be NULL). */
hd_error hd_search_sigproc_file(hd_pipeline pipeline, const char* path, hd_size nsamps_gulp,
                                hd_gulp_callback on_gulp, void* user, hd_size* total_nsamps,
                                hd_size* ngulps);
/* The same loop over nfiles files read in lockstep, e.g. one file per beam
 * of a multibeam receiver (no reference counterpart: heimdall.C runs one
 * process per file).  Every file needs the same channels, bits, sampling
 * time, band and beams per file (else HD_INVALID_STRIDE).  Each gulp is one
 * hd_execute_beams call over the files' gulps, with file u as unit u (beam
 * numbers params.beam + u * nbeams); the first short block of any file ends
 * the search.  on_gulp receives all files' candidates, unit by unit. */
hd_error hd_search_sigproc_files(hd_pipeline pipeline, const char* const* paths, hd_size nfiles,
                                 hd_size nsamps_gulp, hd_gulp_callback on_gulp, void* user,
                                 hd_size* total_nsamps, hd_size* ngulps);

/* Candidates of the last hd_execute, in .cand order.  Copies
 * min(*count, available) rows into out (out may be NULL to query) and sets
 * *count to the number available. */
hd_error hd_get_candidates(hd_pipeline pipeline, hd_candidate* out, hd_size* count);

/* Double-buffered ingest for streaming callers (no reference counterpart:
 * heimdall.C copies and searches each gulp in turn).  hd_prefetch_beams
 * queues the copy of the next gulp's filterbanks (host memory, pinned for the
 * copy to overlap) on the pipeline's copy stream and returns at once; up to
 * two gulps may be queued.  hd_execute_prefetched searches the oldest queued
 * gulp exactly as hd_execute_beams would (same arguments after the data).
 * Calling hd_prefetch_beams for gulp k+1 before hd_execute_prefetched for
 * gulp k overlaps the copy of one gulp with the search of the other.  The
 * host buffers must stay unchanged until the gulp's search returns.  A third
 * hd_prefetch_beams while two gulps are queued returns HD_INVALID_STRIDE;
 * hd_execute_prefetched with nothing queued returns HD_INVALID_POINTER. */
hd_error hd_prefetch_beams(hd_pipeline pipeline, const hd_byte* const* filterbanks,
                           hd_size nfilterbanks, hd_size nsamps, hd_size nbits);
hd_error hd_execute_prefetched(hd_pipeline pipeline, hd_size first_idx, hd_size nbeams,
                               const hd_size* beams, hd_error* statuses,
                               hd_size* nsamps_processed);

/* Candidates of filterbank `index` of the last hd_execute_beams (index 0 after
 * hd_execute), same copy rules as hd_get_candidates. */
hd_error hd_get_beam_candidates(hd_pipeline pipeline, hd_size index, hd_candidate* out,
                                hd_size* count);
/* The candidates of the last gulp (hd_get_candidates order) as RawCandidates
 * arrays the caller provides, each of *count entries: peaks = S/N, inds =
 * sample index, begins/ends, filter_inds, dm_inds = DM trial, members.  Any
 * array pointer may be NULL; copies min(*count, available) and sets *count
 * to the number available. */
hd_error hd_get_raw_candidates(hd_pipeline pipeline, struct RawCandidates* out, hd_size* count);

/* Beams of different shapes in one call.  No counterpart in the reference,
 * which runs one heimdall process (one pipeline) per beam
 * (Applications/heimdall.C).  params[b] describes beam b (channel count,
 * sampling time, band, DM range, boxcar_max ...; all on one gpu_id); beam b's
 * candidates, .cand file and status are those hd_execute gives for
 * filterbanks[b] (nsamps[b] spectra of one beam, 8-bit) with a pipeline made
 * from params[b].  Beams are grouped by configuration (every field but
 * `beam`); runs of equal configuration and gulp length are searched by one
 * hd_execute_beams, and nworkers host threads, each with its own pipelines
 * and streams, search runs concurrently on the GPU.  hd_execute_beam_set
 * returns HD_NO_ERROR, or the status of the lowest-numbered beam that did
 * not succeed; statuses[b] and nsamps_processed[b] (both may be NULL) give
 * every beam's.  Filterbanks are host pointers, or device pointers with
 * on_device != 0. */
typedef struct hd_beam_set_t* hd_beam_set;
hd_error hd_create_beam_set(hd_beam_set* set, const struct hd_params* params, hd_size nbeams,
                            int nworkers);
hd_error hd_set_beam_set_cleaning(hd_beam_set set, int enable);
hd_size  hd_get_beam_set_config_count(hd_beam_set set);
hd_error hd_execute_beam_set(hd_beam_set set, const hd_byte* const* filterbanks,
                             const hd_size* nsamps, hd_size nbits, hd_size first_idx,
                             int on_device, hd_error* statuses, hd_size* nsamps_processed);
/* Candidates of beam `beam` of the last hd_execute_beam_set (copy rules of
 * hd_get_candidates). */
hd_error hd_get_beam_set_candidates(hd_beam_set set, hd_size beam, hd_candidate* out,
                                    hd_size* count);
void     hd_destroy_beam_set(hd_beam_set set);

/* Every giant of the last hd_execute in detection order (DM, width, time),
 * before clustering, with its cluster label (the index of the cluster's first
 * giant).  After hd_execute_beams: filterbank by filterbank, dm_inds local to
 * each filterbank, labels indexing the whole list.  Giants are reported only
 * when some filterbank did not bail out.  Any pointer may be NULL.  The giants
 * stay in device memory after the gulp and are copied by this call, so call
 * it before the next execute on the pipeline. */
hd_error hd_get_giants(hd_pipeline pipeline, hd_float* peaks, hd_size* inds, hd_size* begins,
                       hd_size* ends, hd_size* filter_inds, hd_size* dm_inds,
                       hd_size* labels, hd_size* count);

/* Device time of the last hd_execute per stage, milliseconds (CUDA events):
 * [0] total, [1] clean, [2] dedisperse, [3] baseline+normalise+scan,
 * [4] boxcar+threshold, [5] giants, [6] cluster+merge, [7] host->device copy.
 * When hd_execute_beams copies host filterbanks in pieces overlapped with
 * their transpose and dedispersion (cleaning off), [7] ends when the last
 * piece has landed, [1] then covers the last piece's transpose and [2] its
 * dedispersion. */
hd_error hd_get_timing(hd_pipeline pipeline, float* ms, int n);

#ifdef __cplusplus
}  /* extern "C" */

/* Full candidate info including derived quantities (Pipeline/hd/types.h:38-43). */
struct Candidates : public RawCandidates {
  hd_float* dms;
  hd_size*  flags;
  hd_size*  beam_counts;
  hd_size*  beam_masks;
};
#endif

#endif /* HEIMDALL_B200_H */
