// kernels_search.cu -- per-DM-series kernels of the single-pulse search:
// baseline removal, robust RMS, normalisation + prefix sum, boxcar block RMS,
// thresholding, giant segmentation, clustering and merging.
//
// Every float operation mirrors the cited reference expression (same types,
// same order; the file is compiled with -fmad=false), so outputs are
// bit-identical to the reference's stage code.  Where the reference iterates
// a median-of-5 scrunch level by level through global memory
// (Pipeline/median_filter.cu:288-395), these kernels evaluate several levels
// per block in shared memory: level-k value j of a tree depends only on the
// aligned input block [j*5^k, (j+1)*5^k), and the reference's per-level
// truncation (size/5) keeps exactly the complete blocks.
#include <algorithm>

#include "common.cuh"
#include "internal.h"

namespace hdb {

namespace {

constexpr int TREE_THREADS = 128;

__host__ __device__ inline size_t pow5(int m) {
  size_t r = 1;
  for (int i = 0; i < m; i++) r *= 5;
  return r;
}

// Level-m median of the 5^m source values src(0 .. 5^m-1) (m >= 1).  Result
// valid in every thread after the call.  sm needs 5^(m-1) + 5^(m-2) floats.
template <class F>
__device__ float block_tree(F src, int m, float* sm) {
  const int tid = threadIdx.x;
  int n = (int)pow5(m - 1);
  float* cur = sm;
  float* nxt = sm + n;
  for (int k = tid; k < n; k += blockDim.x)
    cur[k] = med5(src(5 * k), src(5 * k + 1), src(5 * k + 2), src(5 * k + 3), src(5 * k + 4));
  __syncthreads();
  for (int lev = 2; lev <= m; lev++) {
    n /= 5;
    for (int k = tid; k < n; k += blockDim.x)
      nxt[k] = med5(cur[5 * k], cur[5 * k + 1], cur[5 * k + 2], cur[5 * k + 3], cur[5 * k + 4]);
    __syncthreads();
    float* t = cur; cur = nxt; nxt = t;
  }
  float r = cur[0];
  __syncthreads();
  return r;
}

// Number of median-of-5 levels the reference performs on `count` values
// before the remainder is <= 4, and that remainder.
inline void tree_levels(size_t count, int* levels, size_t* rem) {
  int l = 0;
  size_t s = count;
  while (s > 4) { s /= 5; l++; }
  *levels = l;
  *rem = s;
}

// Final step of a tree: count (1..4) values -> one value, the reference's
// special cases (median_filter.cu:217-235 and 295-311).
__device__ __forceinline__ float tree_tail(const float* v, size_t count) {
  if (count <= 1) return v[0];
  if (count == 2) return __fmul_rn(0.5f, __fadd_rn(v[0], v[1]));
  if (count == 3) return med3(v[0], v[1], v[2]);
  return med4(v[0], v[1], v[2], v[3]);
}

// ---- generic level pass over an array: in[seg][n_in] -> out[seg][n_in/5^m]
__global__ void k_tree_array(const float* __restrict__ in, size_t in_pitch, int m,
                             float* __restrict__ out, size_t out_pitch) {
  __shared__ float sm[625 + 125];
  const size_t seg = blockIdx.y + (size_t)blockIdx.z * gridDim.y;
  const size_t g = blockIdx.x;
  const float* p = in + seg * in_pitch + g * pow5(m);
  float r = block_tree([&](int i) { return p[i]; }, m, sm);
  if (threadIdx.x == 0) out[seg * out_pitch + g] = r;
}

// Runs the remaining tree levels of `nseg` segments held in `cur` (pitch
// cur_pitch, `count` values each) down to <= 4 values per segment, using the
// scratch ping-pong buffers.  Returns the array holding the last level.
cudaError_t tree_reduce_array(float* cur, size_t cur_pitch, size_t count, size_t nseg,
                              TreeScratch& ws, cudaStream_t s, float** out, size_t* out_pitch,
                              size_t* out_count) {
  int levels;
  size_t rem;
  tree_levels(count, &levels, &rem);
  float* bufs[2] = {ws.a, ws.b};
  int which = (cur == ws.a) ? 1 : 0;
  while (levels > 0) {
    int m = levels < 5 ? levels : 5;
    size_t ng = count / pow5(m);
    float* dst = bufs[which];
    if (ng * nseg > ws.cap) return cudaErrorMemoryAllocation;
    dim3 grid((unsigned)ng, (unsigned)(nseg > 65535 ? 65535 : nseg),
              (unsigned)((nseg + 65534) / 65535));
    if (nseg > 65535) {
      // segments are laid out contiguously: fold into y*z with exact division
      size_t y = 1;
      for (size_t c = 65535; c >= 1; c--) if (nseg % c == 0) { y = c; break; }
      grid.y = (unsigned)y;
      grid.z = (unsigned)(nseg / y);
    }
    k_tree_array<<<grid, TREE_THREADS, 0, s>>>(cur, cur_pitch, m, dst, ng); note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cur = dst;
    cur_pitch = ng;
    count = ng;
    levels -= m;
    which ^= 1;
  }
  *out = cur;
  *out_pitch = cur_pitch;
  *out_count = count;
  return cudaSuccess;
}

inline dim3 seg_grid(size_t ng, size_t nseg_y, size_t nseg_z) {
  return dim3((unsigned)ng, (unsigned)nseg_y, (unsigned)nseg_z);
}

}  // namespace

// ===========================================================================
// Baseline removal (Pipeline/remove_baseline.cu:21-102)
// ===========================================================================
struct BaselinePlan {
  size_t sample_count, nscrunches, count_round;
};

static BaselinePlan baseline_plan(size_t beam_stride, size_t smooth_radius) {
  // remove_baseline.cu:36-46, same float/double arithmetic
  BaselinePlan p{0, 0, 0};
  if (smooth_radius == 0) return p;
  float oversample = 2;
  float q = oversample * (float)beam_stride / (float)(2 * smooth_radius);
  size_t sc = (size_t)((double)q + 0.5);
  p.sample_count = sc;
  if (sc == 0) return p;
  p.nscrunches = (size_t)(log((double)(beam_stride / sc)) / log(5.));
  p.count_round = (size_t)(pow(5., (double)p.nscrunches) * (double)sc);
  return p;
}

// Stretch of every beam to count_round samples followed by m median levels.
__global__ void k_baseline_down(const float* __restrict__ data, size_t pitch, int nbeams,
                                size_t stride, size_t beam_count, size_t cr, int m,
                                float step_b, float step_last, float* __restrict__ out,
                                size_t out_pitch_beam) {
  __shared__ float sm[625 + 125];
  const int b = blockIdx.y;
  const size_t ser = blockIdx.z;
  const size_t g = blockIdx.x;
  const float* d = data + ser * pitch;
  const size_t base_i = g * pow5(m);
  float r;
  if (b < nbeams - 1) {
    const unsigned gi0 = (unsigned)((size_t)b * cr + base_i);
    r = block_tree([&](int i) { return stretch_beam_at(d, gi0 + (unsigned)i, step_b,
                                                       (unsigned long long)b); }, m, sm);
  } else {
    const float* dl = d + (size_t)(nbeams - 1) * stride;
    r = block_tree([&](int i) { return stretch_at(dl, (unsigned)(base_i + i), step_last); },
                   m, sm);
  }
  if (threadIdx.x == 0) out[(ser * nbeams + b) * out_pitch_beam + g] = r;
}

__global__ void k_baseline_stretch0(const float* __restrict__ data, size_t pitch, int nbeams,
                                    size_t stride, size_t cr, float step_b, float step_last,
                                    float* __restrict__ out) {
  const int b = blockIdx.y;
  const size_t ser = blockIdx.z;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cr) return;
  const float* d = data + ser * pitch;
  float v = (b < nbeams - 1)
                ? stretch_beam_at(d, (unsigned)((size_t)b * cr + i), step_b, (unsigned long long)b)
                : stretch_at(d + (size_t)(nbeams - 1) * stride, (unsigned)i, step_last);
  out[(ser * nbeams + b) * cr + i] = v;
}

// Exact int <-> float conversions on the FMA pipe (the conversion unit runs
// at a fraction of its rate), valid for 0 <= v < 2^23: 2^23 + u is the float
// with exponent 23 and mantissa u, and adding 2^23 to x with rounding toward
// zero leaves floor(x) in the mantissa (the binade [2^23, 2^24) has ulp 1).
__device__ __forceinline__ float u2f_small(unsigned u) {
  return __fsub_rn(__uint_as_float(0x4B000000u | u), 8388608.f);
}
__device__ __forceinline__ unsigned trunc_small(float x) {
  return __float_as_uint(__fadd_rz(x, 8388608.f)) & 0x7FFFFFu;
}

// stretch_at / stretch_beam_at with those conversions (same float results;
// arguments outside their range take the general functions)
__device__ __forceinline__ float stretch_at_nc(const float* in, unsigned i, float step) {
  if (i >= (1u << 23)) return stretch_at(in, i, step);
  const float x = __fmul_rn(u2f_small(i), step);
  if (!(x >= 0.f && x < 8388608.f)) return stretch_at(in, i, step);
  const unsigned j = trunc_small(x);
  const float fr = __fsub_rn(x, u2f_small(j));
  const float add = (fr > kStretchEps) ? __fmul_rn(fr, __fsub_rn(in[j + 1], in[j])) : 0.f;
  return __fadd_rn(in[j], add);
}
__device__ __forceinline__ float stretch_beam_at_nc(const float* in, unsigned i, float step,
                                                    unsigned beam) {
  if (i >= (1u << 23) || beam >= (1u << 23))
    return stretch_beam_at(in, i, step, (unsigned long long)beam);
  const float x = __fmul_rn(u2f_small(i), step);
  const float fb = u2f_small(beam);
  const float xs = __fadd_rn(x, fb);
  if (!(x >= 0.f && xs < 8388608.f)) return stretch_beam_at(in, i, step, (unsigned long long)beam);
  const unsigned k = trunc_small(xs);
  const float o = __fadd_rn(__fsub_rn(x, u2f_small(k)), fb);
  const float add = (o > kStretchEps) ? __fmul_rn(o, __fsub_rn(in[k + 1], in[k])) : 0.f;
  return __fadd_rn(in[k], add);
}

// x - stretched baseline at sample i of series ser (i < nsub), else x
__device__ __forceinline__ float sub_baseline(const BaselineSub& b, size_t ser, unsigned i,
                                              float x) {
  if (i >= b.nsub) return x;
  const float* bs = b.base + ser * (size_t)b.nbeams * b.sc;
  const float v = (i < b.last_start)
                      ? stretch_beam_at_nc(bs, i, b.step2, i / b.stride)
                      : stretch_at_nc(bs + (size_t)(b.nbeams - 1) * b.sc, i - b.last_start,
                                      b.step3);
  return __fsub_rn(x, v);
}

// data[i] -= stretched baseline, lo <= i < nbeams*stride - dm_delay
__global__ void k_baseline_sub(float* __restrict__ data, size_t pitch, BaselineSub b,
                               unsigned lo) {
  const size_t ser = blockIdx.y;
  float* d = data + ser * pitch;
  const unsigned nsub = b.nsub;
  // four consecutive samples per thread (rows are 16-byte aligned)
  for (unsigned i = (lo & ~3u) + 4u * (blockIdx.x * blockDim.x + threadIdx.x); i < nsub;
       i += 4u * gridDim.x * blockDim.x) {
    float4 x;
    const bool full = i >= lo && i + 3 < nsub;
    if (full) x = *reinterpret_cast<const float4*>(d + i);
    float* xs = reinterpret_cast<float*>(&x);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const unsigned ij = i + j;
      if (!full) xs[j] = (ij >= lo && ij < nsub) ? d[ij] : 0.f;
      xs[j] = sub_baseline(b, ser, ij, xs[j]);
    }
    if (full) {
      *reinterpret_cast<float4*>(d + i) = x;
    } else {
      for (int j = 0; j < 4; j++)
        if (i + j >= lo && i + j < nsub) d[i + j] = xs[j];
    }
  }
}

static cudaError_t launch_baseline_sub(const SeriesBatch& sb, const BaselineSub& b, unsigned lo,
                                       cudaStream_t s) {
  if (lo >= b.nsub) return cudaSuccess;
  const size_t nq = (b.nsub - (lo & ~3u) + 3) / 4;
  dim3 grid((unsigned)((nq + 255) / 256 < 4096 ? (nq + 255) / 256 : 4096), sb.nser);
  k_baseline_sub<<<grid, 256, 0, s>>>(sb.data, sb.pitch, b, lo); note_launch();
  return cudaGetLastError();
}

size_t baseline_samples(size_t stride, size_t smooth_radius) {
  return baseline_plan(stride, smooth_radius).sample_count;
}

size_t baseline_scratch(size_t stride, size_t smooth_radius, size_t nseg) {
  BaselinePlan p = baseline_plan(stride, smooth_radius);
  size_t m1 = p.nscrunches < 5 ? p.nscrunches : 5;
  size_t ng1 = p.count_round / pow5((int)m1);
  return nseg * (ng1 + 8) + 64;
}

// The scrunched baseline of every series into base_out and the description
// of its subtraction (b->base stays null when there is no baseline).
static cudaError_t baseline_prepare(const SeriesBatch& sb, size_t smooth_radius,
                                    float* base_out, TreeScratch& ws, cudaStream_t s,
                                    BaselineSub* bp) {
  *bp = BaselineSub();
  BaselinePlan p = baseline_plan(sb.stride, smooth_radius);
  if (p.sample_count == 0) return cudaSuccess;
  const size_t sc = p.sample_count, cr = p.count_round;
  const int k = (int)p.nscrunches;
  const float step_b = (float)(sb.stride - 1) / (float)cr;            // median_filter.cu:490
  const float step_last = (float)(sb.beam_count - 1) / (float)(cr - 1);  // median_filter.cu:457
  const size_t nseg = (size_t)sb.nser * sb.nbeams;
  float* lev_out;
  int m1 = k < 5 ? k : 5;
  size_t ng1 = cr / pow5(m1);
  if (nseg * ng1 > ws.cap) return cudaErrorMemoryAllocation;
  if (k == 0) {
    // no scrunch levels: the baseline samples are the stretched values
    k_baseline_stretch0<<<dim3((unsigned)((cr + 127) / 128), sb.nbeams, sb.nser), 128, 0, s>>>(
        sb.data, sb.pitch, sb.nbeams, sb.stride, cr, step_b, step_last, ws.a); note_launch();
  } else {
    k_baseline_down<<<seg_grid(ng1, sb.nbeams, sb.nser), TREE_THREADS, 0, s>>>(
        sb.data, sb.pitch, sb.nbeams, sb.stride, sb.beam_count, cr, m1, step_b, step_last, ws.a,
        ng1); note_launch();
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  float* cur = ws.a;
  size_t cur_pitch = ng1, count = ng1;
  int left = k - m1;
  float* bufs[2] = {ws.b, ws.a};
  int w = 0;
  while (left > 0) {
    int m = left < 5 ? left : 5;
    size_t ng = count / pow5(m);
    float* dst = bufs[w];
    k_tree_array<<<seg_grid(ng, sb.nbeams, sb.nser), TREE_THREADS, 0, s>>>(cur, cur_pitch, m,
                                                                           dst, ng); note_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cur = dst; cur_pitch = ng; count = ng; left -= m; w ^= 1;
  }
  // cur[seg][sc] holds the scrunched baseline samples
  lev_out = cur;
  if (cur_pitch != sc) return cudaErrorInvalidValue;
  e = cudaMemcpyAsync(base_out, lev_out, nseg * sc * sizeof(float), cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return e;
  const float step2 = (float)(sc - 1) / (float)sb.stride;              // stretch back, beams 0..n-2
  const float step3 = (float)(sc - 1) / (float)(sb.beam_count - 1);    // last beam
  const size_t dm_delay = sb.stride - sb.beam_count;
  const size_t nsub = sb.stride * sb.nbeams - dm_delay;
  if (nsub >= 0xFFFFFF00u || sb.pitch % 4 || (reinterpret_cast<uintptr_t>(sb.data) & 15))
    return cudaErrorInvalidValue;
  BaselineSub b;
  b.base = base_out;
  b.sc = (unsigned)sc;
  b.stride = (unsigned)sb.stride;
  b.last_start = (unsigned)((size_t)(sb.nbeams - 1) * sb.stride);
  b.nsub = (unsigned)nsub;
  b.nbeams = sb.nbeams;
  b.step2 = step2;
  b.step3 = step3;
  *bp = b;
  return cudaSuccess;
}

cudaError_t remove_baseline(const SeriesBatch& sb, size_t smooth_radius, float* base_out,
                            TreeScratch& ws, cudaStream_t s) {
  BaselineSub b;
  cudaError_t e = baseline_prepare(sb, smooth_radius, base_out, ws, s, &b);
  if (e != cudaSuccess || !b.base) return e;
  return launch_baseline_sub(sb, b, 0, s);
}

// ===========================================================================
// Robust RMS per beam (Pipeline/get_rms.cu:236-270, reblock_abs_beam 384-418)
// ===========================================================================
__device__ __forceinline__ size_t reblock_index(size_t beam, float delta, unsigned o) {
  return (size_t)__fadd_rn(__fmul_rn(__ull2float_rn(beam), delta), __uint2float_rn(o));
}

__global__ void k_rms_beams_pass1(const float* __restrict__ data, size_t pitch, int nbeams,
                                  size_t beam_count, float delta, int m,
                                  float* __restrict__ out, size_t out_pitch_beam) {
  __shared__ float sm[625 + 125];
  const int b = blockIdx.y;
  const size_t ser = blockIdx.z;
  const size_t g = blockIdx.x;
  const float* d = data + ser * pitch;
  const size_t o0 = (size_t)b * beam_count + g * pow5(m);
  float r = block_tree([&](int i) {
    unsigned o = (unsigned)(o0 + i);
    return fabsf(d[reblock_index((size_t)b, delta, o)]);
  }, m, sm);
  if (threadIdx.x == 0) out[(ser * nbeams + b) * out_pitch_beam + g] = r;
}

__global__ void k_rms_beams_final(const float* __restrict__ lev, size_t lev_pitch, size_t count,
                                  int nseg, const float* __restrict__ data, size_t pitch,
                                  int nbeams, size_t beam_count, float delta, int from_data,
                                  float* __restrict__ rms) {
  int seg = blockIdx.x * blockDim.x + threadIdx.x;
  if (seg >= nseg) return;
  float v[4];
  if (from_data) {
    int ser = seg / nbeams, b = seg % nbeams;
    const float* d = data + (size_t)ser * pitch;
    for (size_t i = 0; i < count && i < 4; i++)
      v[i] = fabsf(d[reblock_index((size_t)b, delta, (unsigned)((size_t)b * beam_count + i))]);
  } else {
    for (size_t i = 0; i < count && i < 4; i++) v[i] = lev[(size_t)seg * lev_pitch + i];
  }
  float m = tree_tail(v, count);
  rms[seg] = __fmul_rn(m, (float)1.4862);  // multiplies<hd_float>(x, 1.4862)
}

cudaError_t rms_beams(const SeriesBatch& sb, float* rms, TreeScratch& ws, cudaStream_t s) {
  int levels;
  size_t rem;
  tree_levels(sb.beam_count, &levels, &rem);
  const float delta = (float)(sb.stride - sb.beam_count);
  const size_t nseg = (size_t)sb.nser * sb.nbeams;
  cudaError_t e;
  if (levels == 0) {
    k_rms_beams_final<<<(unsigned)((nseg + 127) / 128), 128, 0, s>>>(
        nullptr, 0, rem, (int)nseg, sb.data, sb.pitch, sb.nbeams, sb.beam_count, delta, 1, rms); note_launch();
    return cudaGetLastError();
  }
  int m1 = levels < 5 ? levels : 5;
  size_t ng1 = sb.beam_count / pow5(m1);
  if (nseg * ng1 > ws.cap) return cudaErrorMemoryAllocation;
  k_rms_beams_pass1<<<seg_grid(ng1, sb.nbeams, sb.nser), TREE_THREADS, 0, s>>>(
      sb.data, sb.pitch, sb.nbeams, sb.beam_count, delta, m1, ws.a, ng1); note_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  float* fin;
  size_t fin_pitch, fin_count;
  e = tree_reduce_array(ws.a, ng1, ng1, nseg, ws, s, &fin, &fin_pitch, &fin_count);
  if (e != cudaSuccess) return e;
  k_rms_beams_final<<<(unsigned)((nseg + 127) / 128), 128, 0, s>>>(
      fin, fin_pitch, fin_count, (int)nseg, nullptr, 0, sb.nbeams, sb.beam_count, delta, 0, rms); note_launch();
  return cudaGetLastError();
}

// ===========================================================================
// Normalise + exclusive prefix sum with the sequential association of the
// reference's scan (Thrust's sequential exclusive_scan: out[0] = 0,
// out[k+1] = out[k] + in[k]), for up to 8 series per block.
//
// The left-to-right float sum of a series is one dependent chain (~4 cycles
// per sample), so the block is split by role:
//   warp 0       the chains: lane l owns series l of the block and runs its
//                chain over one stage of its row in shared memory;
//   warps 1..np  a stage's rows arrive by TMA bulk copies requested SC_DEPTH
//                stages ahead; these warps divide them in place by their
//                beam's RMS, and write them out once the chain warp has
//                replaced them with their prefix sums.
// Stage k lives in buffer k % SC_NB.  At step k the producers normalise stage
// k and store stage k - 2 while the chain warp scans stage k - 1, and stage
// k + SC_DEPTH is requested into the buffer that held stage k - 3 (stored at
// step k - 1).  One block barrier ends each step.
// ===========================================================================
// Stages in flight ahead of the one being normalised, and the ring of stage
// buffers (depth + 3).  Stages of 256 samples: depth 3 (a ring of 6, 50 KB for
// 8 series) keeps four blocks on an SM, with each copy still requested about
// 5 us before it is read; stages of 512 samples (blocks of few series): 5.
__host__ __device__ constexpr int sc_depth(int ch) { return ch >= 512 ? 5 : 3; }
__host__ __device__ constexpr int sc_nb(int ch) { return sc_depth(ch) + 3; }
constexpr int SC_MAXRMS = 2048;      // series x beams whose RMS stays in shared memory
constexpr uint32_t SC_WAIT_LIMIT = 1u << 22;

// a / b correctly rounded, given y = RN(1/b) (__frcp_rn): q0 = RN(a*y), the
// residual a - b*q0 (exact by FMA), and one correction q0 + r*y (Markstein's
// theorem: P. W. Markstein, IBM J. Res. Dev. 34(1):111-119, 1990; Muller et
// al., Handbook of Floating-Point Arithmetic, 2nd ed., 2018, ch. 4).  The
// theorem needs the quotient and residual clear of underflow and overflow,
// which |a|, |b| in [2^-40, 2^40] guarantees; other operands (zeros, tiny,
// huge and non-finite values) take __fdiv_rn.
__device__ __forceinline__ float div_rn_by(float a, float b, float y) {
  const float aa = fabsf(a), ab = fabsf(b);
  if (aa >= 0x1p-40f && aa <= 0x1p40f && ab >= 0x1p-40f && ab <= 0x1p40f) {
    const float q0 = __fmul_rn(a, y);
    const float r = __fmaf_rn(-b, q0, a);
    return __fmaf_rn(r, y, q0);
  }
  return __fdiv_rn(a, b);
}

size_t scan_smem_bytes(int ser, int nbeams, int ch) {
  size_t b = 128 + (size_t)sc_nb(ch) * ser * (ch + 4) * sizeof(float);
  if ((size_t)ser * nbeams <= SC_MAXRMS) b += 2 * (size_t)ser * nbeams * sizeof(float);
  return b;
}

// CH samples per series per stage (128, 256 or 512): blocks of few series use
// long stages, so the per-stage fixed cost (barrier, copy issue, waits) is
// spread over more samples and each producer lane has CH / 128 independent
// float4 values in flight.
template <int CH>
__global__ void __launch_bounds__(256, CH >= 512 ? 3 : 4) k_normalise_scan(
    const float* __restrict__ data, size_t pitch, int nser, unsigned len, unsigned stride,
    int nbeams, const float* __restrict__ rms, float* __restrict__ scan, size_t scan_pitch,
    float* norm_out, int ser_per_block, unsigned* err) {
  constexpr int SC_DEPTH = sc_depth(CH);
  constexpr int SC_NB = sc_nb(CH);
  constexpr int ROW = CH + 4;  // row pitch in floats: lane l's 16 bytes hit banks 4l..4l+3
  constexpr int QN = CH / 128; // float4 per lane per row
  extern __shared__ __align__(128) float sc_smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(sc_smem);  // [SC_NB], first 128 bytes
  const int S = ser_per_block;
  float* rows = sc_smem + 32;                             // [SC_NB][S][ROW]
  float* srms = rows + (size_t)SC_NB * S * ROW;           // [S][nbeams]
  float* sy = srms + S * nbeams;                          // reciprocals
  const int s0 = blockIdx.x * S;
  const int nb = min(S, nser - s0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int np = (int)(blockDim.x >> 5) - 1;
  const bool rms_smem = nb * nbeams <= SC_MAXRMS;
  const unsigned nstage = len / CH + 1;     // outputs 0..len
  const unsigned len4 = (len + 3u) & ~3u;   // copies round up to 16 bytes (inside the row pitch)

  if (threadIdx.x == 0) {
    for (int b = 0; b < SC_NB; b++) mbar_init(&full[b], 1);
    fence_mbar_init();
  }
  if (rms_smem)
    for (int k = threadIdx.x; k < nb * nbeams; k += blockDim.x) {
      const float r = rms[(size_t)s0 * nbeams + k];
      srms[k] = r;
      sy[k] = __frcp_rn(r);
    }
  __syncthreads();

  // stage st -> its buffer; warp 1, one row per lane; a stage past the data
  // completes its barrier phase with a plain arrival
  auto request = [&](unsigned st) {
    uint64_t* bar = &full[st % SC_NB];
    const unsigned base = st * CH;
    const unsigned end = min(base + (unsigned)CH, len4);
    const unsigned bytes = end > base ? (end - base) * 4u : 0u;
    if (bytes == 0) {
      if (lane == 0) mbar_arrive(bar);
      return;
    }
    if (lane == 0) mbar_expect_tx(bar, bytes * (unsigned)nb);
    __syncwarp();
    // the buffer was last written by this block's threads (generic proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (lane < nb)
      bulk_g2s(rows + ((size_t)(st % SC_NB) * S + lane) * ROW,
               data + (size_t)(s0 + lane) * pitch + base, bytes, bar);
  };
  if (warp == 1)
    for (unsigned st = 0; st < (unsigned)SC_DEPTH && st < nstage; st++) request(st);

  float sum = 0.f;     // chain of series s0 + lane (warp 0)
  bool failed = false;
  for (unsigned k = 0; k < nstage + 2; k++) {
    if (warp == 0) {
      // ---- the chains: stage k - 1 ----
      if (k >= 1 && k - 1 < nstage && lane < nb) {
        float* row = rows + ((size_t)((k - 1) % SC_NB) * S + lane) * ROW;
#pragma unroll 8
        for (int e = 0; e < CH; e += 4) {
          const float4 v = *reinterpret_cast<const float4*>(row + e);
          float4 o;
          o.x = sum; sum = __fadd_rn(sum, v.x);
          o.y = sum; sum = __fadd_rn(sum, v.y);
          o.z = sum; sum = __fadd_rn(sum, v.z);
          o.w = sum; sum = __fadd_rn(sum, v.w);
          *reinterpret_cast<float4*>(row + e) = o;
        }
      }
    } else {
      const int p = warp - 1;
      if (warp == 1 && k + SC_DEPTH < nstage) request(k + SC_DEPTH);
      // ---- store stage k - 2 ----
      if (k >= 2 && k - 2 < nstage) {
        const unsigned st = k - 2;
        for (int sl = p; sl < nb; sl += np) {
          const float* rrow = rows + ((size_t)(st % SC_NB) * S + sl) * ROW;
          float* orow = scan + (size_t)(s0 + sl) * scan_pitch;
#pragma unroll
          for (int q = 0; q < QN; q++) {
            const unsigned e = 4u * lane + 128u * q;
            const unsigned i = st * CH + e;
            const float4 v = *reinterpret_cast<const float4*>(rrow + e);
            float* o = orow + i;
            if (i + 3 <= len) {
              *reinterpret_cast<float4*>(o) = v;
            } else {
              if (i <= len) o[0] = v.x;
              if (i + 1 <= len) o[1] = v.y;
              if (i + 2 <= len) o[2] = v.z;
            }
          }
        }
      }
      // ---- normalise stage k (get_rms.cu:344-356): x / rms[beam of sample] ----
      if (k < nstage) {
        if (!mbar_wait(&full[k % SC_NB], (k / SC_NB) & 1u, SC_WAIT_LIMIT)) {
          if (!failed && err && lane == 0) atomicOr(err, 2u);
          failed = true;
        }
        const unsigned base = k * CH;
        unsigned b0 = base / stride;
        if (b0 > (unsigned)nbeams - 1) b0 = (unsigned)nbeams - 1;
        const unsigned bend = (b0 + 1) * stride;
        // common case: the stage lies inside the data and inside one beam, so
        // one divisor (and its reciprocal) serves the whole row
        const bool uniform = rms_smem && base + CH <= len && stride >= (unsigned)CH &&
                             (b0 + 1 >= (unsigned)nbeams || bend >= base + CH);
        if (uniform) {
          for (int sl = p; sl < nb; sl += np) {
            float* crow = rows + ((size_t)(k % SC_NB) * S + sl) * ROW;
            const int q0 = sl * nbeams + (int)b0;
            const float rb = srms[q0], y = sy[q0];
            float4 x[QN];
#pragma unroll
            for (int q = 0; q < QN; q++) x[q] = *reinterpret_cast<const float4*>(crow + 4 * lane + 128 * q);
#pragma unroll
            for (int q = 0; q < QN; q++) {
              x[q].x = div_rn_by(x[q].x, rb, y);
              x[q].y = div_rn_by(x[q].y, rb, y);
              x[q].z = div_rn_by(x[q].z, rb, y);
              x[q].w = div_rn_by(x[q].w, rb, y);
              *reinterpret_cast<float4*>(crow + 4 * lane + 128 * q) = x[q];
              if (norm_out)
                *reinterpret_cast<float4*>(norm_out + (size_t)(s0 + sl) * pitch + base + 4 * lane +
                                           128 * q) = x[q];
            }
          }
        } else {
          for (int sl = p; sl < nb; sl += np) {
#pragma unroll
            for (int q = 0; q < QN; q++) {
              const unsigned i = base + 4u * lane + 128u * q;
              float4* cell = reinterpret_cast<float4*>(rows + ((size_t)(k % SC_NB) * S + sl) * ROW +
                                                       4 * lane + 128 * q);
              float x[4];
              *reinterpret_cast<float4*>(x) = *cell;
#pragma unroll
              for (int j = 0; j < 4; j++) {
                const unsigned ij = i + j;
                if (ij >= len) { x[j] = 0.f; continue; }
                unsigned b;
                if (stride >= (unsigned)CH) b = (ij >= bend && b0 + 1 < (unsigned)nbeams) ? b0 + 1 : b0;
                else b = min(ij / stride, (unsigned)nbeams - 1);
                if (rms_smem) {
                  const int qq = sl * nbeams + (int)b;
                  x[j] = div_rn_by(x[j], srms[qq], sy[qq]);
                } else {
                  x[j] = __fdiv_rn(x[j], rms[(size_t)(s0 + sl) * nbeams + b]);
                }
              }
              *cell = *reinterpret_cast<float4*>(x);
              if (norm_out) {
                float* o = norm_out + (size_t)(s0 + sl) * pitch + i;
                if (i + 3 < len) {
                  *reinterpret_cast<float4*>(o) = *reinterpret_cast<float4*>(x);
                } else {
                  for (int j = 0; j < 4; j++)
                    if (i + j < len) o[j] = x[j];
                }
              }
            }
          }
        }
      }
    }
    __syncthreads();
  }
  // every copy has been waited for at its normalise step; after a timed-out
  // wait, let the buffers' last copies land before the block exits
  if (failed && warp == 1)
    for (unsigned st = (nstage > SC_NB ? nstage - SC_NB : 0); st < nstage; st++)
      mbar_wait(&full[st % SC_NB], (st / SC_NB) & 1u, SC_WAIT_LIMIT);
}

template <int CH>
static cudaError_t launch_scan(const SeriesBatch& sb, const float* rms, float* scan,
                               size_t scan_pitch, float* norm_out, cudaStream_t s, unsigned* err,
                               int ser) {
  const int np = ser < 7 ? ser : 7;
  const size_t smem = scan_smem_bytes(ser, sb.nbeams, CH);
  cudaError_t e = raise_smem_limit(k_normalise_scan<CH>, smem);
  if (e != cudaSuccess) return e;
  k_normalise_scan<CH><<<(unsigned)((sb.nser + ser - 1) / ser), 32 * (np + 1), smem, s>>>(
      sb.data, sb.pitch, sb.nser, (unsigned)sb.len, (unsigned)sb.stride, sb.nbeams, rms, scan,
      scan_pitch, norm_out, ser, err); note_launch();
  return cudaGetLastError();
}

cudaError_t normalise_scan(const SeriesBatch& sb, const float* rms, float* scan,
                           size_t scan_pitch, float* norm_out, cudaStream_t s, unsigned* err) {
  if (sb.len >= 0xFFFFFF00u || sb.pitch % 4 || scan_pitch % 4 || sb.stride == 0 ||
      sb.pitch < ((sb.len + 3) & ~(size_t)3) || scan_pitch < sb.len + 1 ||
      (reinterpret_cast<uintptr_t>(sb.data) & 15) || (reinterpret_cast<uintptr_t>(scan) & 15) ||
      (norm_out && (reinterpret_cast<uintptr_t>(norm_out) & 15)))
    return cudaErrorInvalidValue;
  if (sb.nser <= 0) return cudaSuccess;
  // series per block: enough blocks to cover the SMs twice where possible, at
  // most 8 (measured: 8 series with 256-sample stages beat 16 with 128 on the
  // multibeam gulp, and 4 with 512 beat 2 with 512 on the survey gulp)
  int ser = 8;
  while (ser > 1 && (sb.nser + ser - 1) / ser < 296) ser /= 2;
  if (ser <= 4) return launch_scan<512>(sb, rms, scan, scan_pitch, norm_out, s, err, ser);
  return launch_scan<256>(sb, rms, scan, scan_pitch, norm_out, s, err, ser);
}

// ===========================================================================
// Boxcar filter helpers (Pipeline/matched_filter.cu:37-67)
// ===========================================================================
__device__ __forceinline__ float boxcar(const float* sc, int offset, const WidthInfo& w,
                                        size_t i) {
  size_t p = (size_t)i * (size_t)w.ts;
  return __fsub_rn(sc[offset + w.ahead + p], sc[offset - w.behind + p]);
}

// Value the reference's block-RMS window reads at filtered index i for width
// wi: fresh (unnormalised) output of wi if i < n, otherwise the normalised
// output of the latest earlier width that wrote index i.
__device__ __forceinline__ float rms_window_value(const float* sc, int offset,
                                                  const WidthInfo* winfo, const float* norm,
                                                  int wi, size_t i) {
  const WidthInfo& w = winfo[wi];
  if (i < w.n) return boxcar(sc, offset, w, i);
  int pw = w.prev_cover;
  while (pw >= 0 && i >= winfo[pw].n) pw = winfo[pw].prev_cover;
  if (pw < 0) return 0.f;
  return __fmul_rn(boxcar(sc, offset, winfo[pw], i), norm[pw]);
}

// Pass 1 of the block RMS: level-m medians of |window| over aligned groups of
// the reblocked index q (get_rms.cu:274-301; reblock_abs_beam with a float
// delta).  Widths [w0, w0 + gridDim.y) of every series.
__global__ void k_block_rms_pass1(WidthCtx ctx, int w0, int m, float* __restrict__ out,
                                  size_t out_pitch) {
  __shared__ float sm[625 + 125];
  const int wi = w0 + blockIdx.y;
  const size_t ser = blockIdx.z;
  const size_t g = blockIdx.x;
  const WidthInfo& w = ctx.winfo[wi];
  const float* sc = ctx.scan + ser * ctx.scan_pitch;
  const float* norm = ctx.norm + ser * ctx.nw;
  const float delta = (float)(ctx.stride - w.bn);
  const size_t q0 = g * pow5(m);
  float r = block_tree([&](int k) {
    unsigned q = (unsigned)(q0 + k);
    size_t beam = q / w.bn;
    size_t i = reblock_index(beam, delta, q);
    return fabsf(rms_window_value(sc, ctx.offset, ctx.winfo, norm, wi, i));
  }, m, sm);
  if (threadIdx.x == 0) out[(ser * gridDim.y + blockIdx.y) * out_pitch + g] = r;
}

// Pass 1 for several unscrunched widths at once: the group's prefix-sum window
// is staged in shared memory once and every width's boxcar is read from it.
// Falls back to global loads when the group's samples are not contiguous
// (a multibeam group straddling a beam gap) or the window does not fit.
constexpr int MULTI_SMEM_FLOATS = 12288;

__global__ void k_block_rms_pass1_multi(WidthCtx ctx, int w0, int nwb, int m, int win,
                                        float* __restrict__ out, size_t out_pitch) {
  extern __shared__ float dyn[];
  float* tile = dyn;                         // win floats
  float* sm = dyn + win;                     // tree buffers
  const size_t ser = blockIdx.y;
  const size_t g = blockIdx.x;
  const WidthInfo& w_first = ctx.winfo[w0];
  const float* sc = ctx.scan + ser * ctx.scan_pitch;
  const float delta = (float)(ctx.stride - w_first.bn);
  const size_t gsz = pow5(m);
  const size_t q0 = g * gsz;
  const size_t i_first = reblock_index((unsigned)q0 / w_first.bn, delta, (unsigned)q0);
  const size_t q1 = q0 + gsz - 1;
  const size_t i_last = reblock_index((unsigned)q1 / w_first.bn, delta, (unsigned)q1);
  const int offset = ctx.offset;
  const bool contig = (i_last - i_first == gsz - 1);
  const size_t span = (i_last - i_first) + 2 * (size_t)offset + 2;
  const bool staged = contig && span <= (size_t)win;
  if (staged) {
    for (size_t k = threadIdx.x; k < span; k += blockDim.x) tile[k] = sc[i_first + k];
    __syncthreads();
  }
  for (int wl = 0; wl < nwb; wl++) {
    const WidthInfo& w = ctx.winfo[w0 + wl];
    const int a = offset + w.ahead, b = offset - w.behind;
    float r;
    if (staged) {
      r = block_tree([&](int k) { return fabsf(__fsub_rn(tile[k + a], tile[k + b])); }, m, sm);
    } else {
      r = block_tree([&](int k) {
        unsigned q = (unsigned)(q0 + k);
        size_t i = reblock_index(q / w.bn, delta, q);
        return fabsf(__fsub_rn(sc[i + a], sc[i + b]));
      }, m, sm);
    }
    if (threadIdx.x == 0) out[(ser * nwb + wl) * out_pitch + g] = r;
  }
}

// Pass 1 for several unscrunched widths, one median level of every width per
// block barrier.  Level 1 works on runs of 4 consecutive medians (20
// consecutive samples): with the boxcar offset a multiple of 4, both ends of a
// width >= 8 boxcar are 16-byte aligned in the staged window and load as
// float4 (a thread stride of 80 bytes keeps the 8 lanes of each access phase
// on distinct banks); widths 1, 2 and 4 read one 28-value window.
constexpr int BRV_THREADS = 512;  // at most 16 warps: one per boxcar width
constexpr int VH_MAXW = 16;  // unscrunched widths the vector kernels handle at once

template <int AH, int BH>
__device__ __forceinline__ void brv_small(const float* win, float* v) {
#pragma unroll
  for (int r = 0; r < 20; r++) v[r] = fabsf(__fsub_rn(win[4 + r + AH], win[4 + r - BH]));
}

template <bool MM>
__device__ __forceinline__ float brv_med5(float a, float b, float c, float d, float e) {
  return MM ? med5_mm(a, b, c, d, e) : med5(a, b, c, d, e);
}

__device__ __forceinline__ float max5(float a, float b, float c, float d, float e) {
  return fmaxf(fmaxf(fmaxf(a, b), fmaxf(c, d)), e);
}

__host__ __device__ constexpr int pow5c(int k) { return k <= 0 ? 1 : 5 * pow5c(k - 1); }

// The median levels of one group for every width slot, M levels in the block
// (compile-time).  Warp w takes width slots w, w + nwarps, ... (the launcher
// gives a block one warp per slot, up to 16), and each slot's work -- level
// 1 over the staged window, levels 2..M in the slot's own rows of la and lb,
// and the group maximum -- stays inside its warp: branches are uniform, and
// no block barrier is needed until the next group's window.
template <bool MM, int M>
__device__ void brv_levels(const WidthCtx& ctx, const float* tile, int offset, int w0, int nwb,
                           float* la, float* lb, float* __restrict__ out, size_t out_pitch,
                           size_t ser, size_t g, float* srun, bool rec) {
  constexpr int n1 = pow5c(M - 1);
  constexpr int n1p = (n1 + 3) & ~3;
  constexpr int lbp = n1 / 5 + 1;
  // srun[wl][q]: largest |boxcar| of level-1 item q of width slot wl (runs of
  // 20 samples, then the < 4 remaining single medians)
  constexpr int nq = n1 / 4, rem = n1 - 4 * nq;
  constexpr int rp = nq + 4;
  const int lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  for (int wl = threadIdx.x >> 5; wl < nwb; wl += nwarps) {
    const int wi = w0 + wl;
    float* la_w = la + wl * n1p;
    float* srun_w = srun + wl * rp;

    // ---- level 1: runs of 4 medians (20 consecutive samples) per lane ----
    if (wi < 3) {
      for (int q = lane; q < nq; q += 32) {
        const int k0 = 4 * q;
        float v[20], wv[28];
        const float4* p = reinterpret_cast<const float4*>(tile + 5 * k0 + offset - 4);
#pragma unroll
        for (int r = 0; r < 7; r++) {
          const float4 x = p[r];
          wv[4 * r] = x.x; wv[4 * r + 1] = x.y; wv[4 * r + 2] = x.z; wv[4 * r + 3] = x.w;
        }
        if (wi == 0) brv_small<1, 0>(wv, v);
        else if (wi == 1) brv_small<1, 1>(wv, v);
        else brv_small<2, 2>(wv, v);
        float4 o;
        o.x = brv_med5<MM>(v[0], v[1], v[2], v[3], v[4]);
        o.y = brv_med5<MM>(v[5], v[6], v[7], v[8], v[9]);
        o.z = brv_med5<MM>(v[10], v[11], v[12], v[13], v[14]);
        o.w = brv_med5<MM>(v[15], v[16], v[17], v[18], v[19]);
        *reinterpret_cast<float4*>(la_w + k0) = o;
        if (rec)
          srun_w[q] = fmaxf(fmaxf(max5(v[0], v[1], v[2], v[3], v[4]), max5(v[5], v[6], v[7], v[8], v[9])),
                            fmaxf(max5(v[10], v[11], v[12], v[13], v[14]),
                                  max5(v[15], v[16], v[17], v[18], v[19])));
      }
    } else {
      const int h = 1 << (wi - 1);  // ahead = behind = width / 2 (the launcher checks)
      const float* ta = tile + offset + h;
      const float* tb = tile + offset - h;
      for (int q = lane; q < nq; q += 32) {
        const float4* pa = reinterpret_cast<const float4*>(ta + 20 * q);
        const float4* pb = reinterpret_cast<const float4*>(tb + 20 * q);
        float v[20];
#pragma unroll
        for (int r = 0; r < 5; r++) {
          const float4 a = pa[r], b = pb[r];
          v[4 * r] = fabsf(__fsub_rn(a.x, b.x));
          v[4 * r + 1] = fabsf(__fsub_rn(a.y, b.y));
          v[4 * r + 2] = fabsf(__fsub_rn(a.z, b.z));
          v[4 * r + 3] = fabsf(__fsub_rn(a.w, b.w));
        }
        float4 o;
        o.x = brv_med5<MM>(v[0], v[1], v[2], v[3], v[4]);
        o.y = brv_med5<MM>(v[5], v[6], v[7], v[8], v[9]);
        o.z = brv_med5<MM>(v[10], v[11], v[12], v[13], v[14]);
        o.w = brv_med5<MM>(v[15], v[16], v[17], v[18], v[19]);
        *reinterpret_cast<float4*>(la_w + 4 * q) = o;
        if (rec)
          srun_w[q] = fmaxf(fmaxf(max5(v[0], v[1], v[2], v[3], v[4]), max5(v[5], v[6], v[7], v[8], v[9])),
                            fmaxf(max5(v[10], v[11], v[12], v[13], v[14]),
                                  max5(v[15], v[16], v[17], v[18], v[19])));
      }
    }
    if constexpr (rem > 0)
      if (lane < rem) {
        const int k = 4 * nq + lane;
        const WidthInfo& w = ctx.winfo[wi];
        const int a = offset + w.ahead, b = offset - w.behind;
        float v[5];
#pragma unroll
        for (int r = 0; r < 5; r++) v[r] = fabsf(__fsub_rn(tile[5 * k + r + a], tile[5 * k + r + b]));
        la_w[k] = brv_med5<MM>(v[0], v[1], v[2], v[3], v[4]);
        if (rec) srun_w[nq + lane] = max5(v[0], v[1], v[2], v[3], v[4]);
      }
    __syncwarp();  // the slot's level-1 row and run maxima are complete

    if (rec) {
      // values are non-negative or NaN, so their bit patterns order as
      // unsigned (a NaN maximum only ever keeps a tile from being skipped);
      // fmaxf above drops a NaN unless all its operands are NaN, and no sample
      // is then left out of a maximum that decides a skip: a NaN boxcar never
      // passes the test
      unsigned mk = 0;
      for (int q = lane; q < nq + rem; q += 32) mk = max(mk, __float_as_uint(srun_w[q]));
      mk = __reduce_max_sync(0xffffffffu, mk);
      if (lane == 0) ctx.gmax[(ser * nwb + wl) * ctx.ngroups + g] = __uint_as_float(mk);
    }

    // ---- levels 2..M: rows alternate between the slot's lb and la rows ----
    float* rows[2] = {lb + wl * lbp, la_w};
    const float* cur = la_w;
    int n = n1;
#pragma unroll
    for (int lev = 2; lev <= M; lev++) {
      float* nxt = rows[lev & 1 ? 1 : 0];
      const int nn = n / 5;
      for (int k = lane; k < nn; k += 32) {
        const float* c = cur + 5 * k;
        nxt[k] = brv_med5<MM>(c[0], c[1], c[2], c[3], c[4]);
      }
      __syncwarp();  // every lane reaches it: the level is complete
      cur = nxt;
      n = nn;
    }
    // n == 1: one value per width
    if (lane == 0) out[(ser * nwb + wl) * out_pitch + g] = cur[0];
    __syncwarp();  // the rows are free for the slot's next use
  }
}

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" :: "r"(smem_addr(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(smem_addr(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory");
}

// Block (x, y): groups [x * gpb, (x + 1) * gpb) of series y.  The next
// group's window is copied into the other half of a double buffer (cp.async)
// while the current group's medians are computed.
template <int M>
__global__ void __launch_bounds__(BRV_THREADS) k_block_rms_pass1_vec(WidthCtx ctx, int w0,
                                                                     int nwb, int win,
                                                                     float* __restrict__ out,
                                                                     size_t out_pitch,
                                                                     int ngroups, int gpb) {
  extern __shared__ __align__(16) float dyn[];
  const int win4 = (win + 3) & ~3;
  float* tiles = dyn;                    // [2][win4]
  constexpr int n1 = pow5c(M - 1);       // level-1 medians per width
  const int n1p = (n1 + 3) & ~3;         // row pitch: 16-byte aligned rows
  float* la = dyn + 2 * win4;            // [nwb][n1p]
  float* lb = la + nwb * n1p;            // [nwb][n1 / 5 + 1]
  float* srun = lb + nwb * (n1 / 5 + 1); // [nwb][n1 / 4 + 4] (group maxima)
  const size_t ser = blockIdx.y;
  const int g_begin = blockIdx.x * gpb;
  const int g_end = min(g_begin + gpb, ngroups);
  const WidthInfo& w_first = ctx.winfo[w0];
  const float* sc = ctx.scan + ser * ctx.scan_pitch;
  const float delta = (float)(ctx.stride - w_first.bn);
  constexpr size_t gsz = pow5c(M);
  const int offset = ctx.offset;
  // the launcher guarantees contiguous groups (one beam) whose window fits
  auto first_of = [&](int g) {
    const size_t q0 = (size_t)g * gsz;
    return reblock_index((unsigned)q0 / w_first.bn, delta, (unsigned)q0);
  };
  const size_t span = gsz - 1 + 2 * (size_t)offset + 2;
  auto prefetch = [&](int g, float* tile) {
    const float* src = sc + first_of(g);
    for (size_t k = threadIdx.x; k < span; k += blockDim.x) cp_async4(tile + k, src + k);
    cp_async_commit();
  };
  // A prefix sum that is finite at its end is finite everywhere (a non-finite
  // term would stay non-finite), so every boxcar value is NaN-free and the
  // min/max median network selects the same values as the reference's.
  const float last = sc[ctx.scan_len - 1];
  const bool finite = fabsf(last) <= 3.402823466e38f;
  if (g_begin >= g_end || span > (size_t)win) return;
  const bool rec = ctx.gmax != nullptr && ctx.ngroups > 0;
  prefetch(g_begin, tiles);
  for (int g = g_begin; g < g_end; g++) {
    float* tile = tiles + (size_t)((g - g_begin) & 1) * win4;
    // the previous group's levels (and final reads of la/lb) are finished
    __syncthreads();
    if (g + 1 < g_end) {
      prefetch(g + 1, tiles + (size_t)((g + 1 - g_begin) & 1) * win4);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if (finite)
      brv_levels<true, M>(ctx, tile, offset, w0, nwb, la, lb, out, out_pitch, ser, g, srun, rec);
    else
      brv_levels<false, M>(ctx, tile, offset, w0, nwb, la, lb, out, out_pitch, ser, g, srun, rec);
  }
}

__global__ void k_block_rms_final(WidthCtx ctx, int w0, int nwb, const float* __restrict__ lev,
                                  size_t lev_pitch, size_t count, int from_window) {
  int seg = blockIdx.x * blockDim.x + threadIdx.x;
  if (seg >= ctx.nser * nwb) return;
  int ser = seg / nwb, wl = seg % nwb, wi = w0 + wl;
  float v[4];
  if (from_window) {
    const WidthInfo& w = ctx.winfo[wi];
    const float* sc = ctx.scan + (size_t)ser * ctx.scan_pitch;
    const float* norm = ctx.norm + (size_t)ser * ctx.nw;
    const float delta = (float)(ctx.stride - w.bn);
    for (size_t k = 0; k < count && k < 4; k++) {
      size_t beam = (unsigned)k / w.bn;
      v[k] = fabsf(rms_window_value(sc, ctx.offset, ctx.winfo, norm, wi,
                                    reblock_index(beam, delta, (unsigned)k)));
    }
  } else {
    for (size_t k = 0; k < count && k < 4; k++) v[k] = lev[(size_t)seg * lev_pitch + k];
  }
  float m = tree_tail(v, count);
  float rms = (float)((double)m * 1.4862);          // get_rms.cu:298
  ctx.norm[(size_t)ser * ctx.nw + wi] = __fdiv_rn(1.0f, rms);  // get_rms.cu:365
}

cudaError_t block_rms(WidthCtx& ctx, const WidthInfo* hw, int w_begin, int w_end,
                      TreeScratch& ws, cudaStream_t s) {
  if (w_begin == 0) ctx.ngroups = 0;  // no group maxima unless recorded below
  const int nwb = w_end - w_begin;
  const size_t cnt = (size_t)ctx.nbeams * hw[w_begin].bn;
  for (int wi = w_begin; wi < w_end; wi++)
    if ((size_t)ctx.nbeams * hw[wi].bn != cnt) return cudaErrorInvalidValue;
  int levels;
  size_t rem;
  tree_levels(cnt, &levels, &rem);
  const size_t nseg = (size_t)ctx.nser * nwb;
  cudaError_t e;
  if (levels == 0) {
    k_block_rms_final<<<(unsigned)((nseg + 127) / 128), 128, 0, s>>>(ctx, w_begin, nwb, nullptr,
                                                                     0, rem, 1); note_launch();
    return cudaGetLastError();
  }
  int m1 = levels < 5 ? levels : 5;
  size_t ng1 = cnt / pow5(m1);
  if (nseg * ng1 > ws.cap) return cudaErrorMemoryAllocation;
  bool unscrunched = true;
  for (int wi = w_begin; wi < w_end; wi++) unscrunched = unscrunched && hw[wi].ts == 1;
  bool vec = unscrunched && ctx.offset >= 4 && (ctx.offset & 3) == 0;
  for (int wi = w_begin; vec && wi < w_end; wi++) {
    const WidthInfo& w = hw[wi];
    vec = w.width == (1 << wi) && w.ahead == (w.width - 1) / 2 + 1 && w.behind == w.width / 2;
  }
  // a group of samples is contiguous unless it straddles a beam gap
  // (nbeams > 1); single-beam series always take the vector kernel
  if (vec && ctx.nbeams == 1) {
    const size_t win = pow5(m1) + 2 * (size_t)ctx.offset + 2;
    const size_t n1 = pow5(m1 - 1);
    const size_t smem = (2 * ((win + 3) & ~(size_t)3) + nwb * ((n1 + 3) & ~(size_t)3) +
                         nwb * (n1 / 5 + 1) + nwb * (n1 / 4 + 4)) *
                        sizeof(float);
    if (smem <= 200 * 1024) {
      auto kern = m1 == 5 ? k_block_rms_pass1_vec<5>
                  : m1 == 4 ? k_block_rms_pass1_vec<4>
                  : m1 == 3 ? k_block_rms_pass1_vec<3>
                  : m1 == 2 ? k_block_rms_pass1_vec<2>
                            : k_block_rms_pass1_vec<1>;
      if ((e = raise_smem_limit(kern, smem)) != cudaSuccess) return e;
      // the group maxima of the widths [0, nwb) for count_hits
      if (ctx.gmax && w_begin == 0 && nwb <= VH_MAXW && nseg * ng1 <= ctx.gmax_cap) {
        ctx.gsize = (unsigned)pow5(m1);
        ctx.ngroups = (unsigned)ng1;
        ctx.gmax_nw = nwb;
      }
      // about 8 consecutive groups per block, spread evenly
      const size_t nblk_x = (ng1 + 7) / 8;
      const size_t gpb = (ng1 + nblk_x - 1) / nblk_x;
      const unsigned nthreads = 32u * (unsigned)std::min(nwb, BRV_THREADS / 32);
      kern<<<dim3((unsigned)((ng1 + gpb - 1) / gpb), ctx.nser), nthreads, smem, s>>>(
          ctx, w_begin, nwb, (int)win, ws.a, ng1, (int)ng1, (int)gpb); note_launch();
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      float* fin;
      size_t fin_pitch, fin_count;
      e = tree_reduce_array(ws.a, ng1, ng1, nseg, ws, s, &fin, &fin_pitch, &fin_count);
      if (e != cudaSuccess) return e;
      k_block_rms_final<<<(unsigned)((nseg + 127) / 128), 128, 0, s>>>(ctx, w_begin, nwb, fin,
                                                                       fin_pitch, fin_count, 0); note_launch();
      return cudaGetLastError();
    }
  }
  if (unscrunched) {
    // window: one group of samples plus the widest boxcar on either side
    const size_t win = std::min<size_t>(pow5(m1) + 2 * (size_t)ctx.offset + 2, MULTI_SMEM_FLOATS);
    const size_t smem = (win + 625 + 125) * sizeof(float);
    if ((e = raise_smem_limit(k_block_rms_pass1_multi, smem)) != cudaSuccess) return e;
    k_block_rms_pass1_multi<<<dim3((unsigned)ng1, ctx.nser), TREE_THREADS, smem, s>>>(
        ctx, w_begin, nwb, m1, (int)win, ws.a, ng1); note_launch();
  } else {
    k_block_rms_pass1<<<seg_grid(ng1, nwb, ctx.nser), TREE_THREADS, 0, s>>>(ctx, w_begin, m1,
                                                                           ws.a, ng1); note_launch();
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  float* fin;
  size_t fin_pitch, fin_count;
  e = tree_reduce_array(ws.a, ng1, ng1, nseg, ws, s, &fin, &fin_pitch, &fin_count);
  if (e != cudaSuccess) return e;
  k_block_rms_final<<<(unsigned)((nseg + 127) / 128), 128, 0, s>>>(ctx, w_begin, nwb, fin,
                                                                   fin_pitch, fin_count, 0); note_launch();
  return cudaGetLastError();
}

// ===========================================================================
// Thresholding (find_giants.cu:47-60,137-183): hits are filtered indices i
// with (i % beam_stride) < bn and normalised value > thresh.
// ===========================================================================
constexpr int HIT_TILE = 2048;
constexpr int HIT_THREADS = 256;
constexpr int HIT_PER_THREAD = HIT_TILE / HIT_THREADS;

__device__ __forceinline__ bool hit_at(const WidthCtx& ctx, const float* sc, float norm,
                                       const WidthInfo& w, size_t i, float* val) {
  if (i >= w.n) return false;
  if ((i % ctx.stride) >= w.bn) return false;
  float v = __fmul_rn(boxcar(sc, ctx.offset, w, i), norm);
  *val = v;
  return v > ctx.thresh;
}

__global__ void __launch_bounds__(HIT_THREADS) k_count_hits(WidthCtx ctx, HitBuffers hb,
                                                            int w_base) {
  const int wi = w_base + blockIdx.y;
  const size_t ser = blockIdx.z;
  const unsigned tile = blockIdx.x;
  const WidthInfo& w = ctx.winfo[wi];
  const float* sc = ctx.scan + ser * ctx.scan_pitch;
  const float norm = ctx.norm[ser * ctx.nw + wi];
  const size_t i0 = (size_t)tile * HIT_TILE + (size_t)threadIdx.x * HIT_PER_THREAD;
  unsigned c = 0;
  float v;
  if (i0 < w.n) {
#pragma unroll
    for (int k = 0; k < HIT_PER_THREAD; k++) c += hit_at(ctx, sc, norm, w, i0 + k, &v);
  }
  __shared__ unsigned red[HIT_THREADS / 32];
#pragma unroll
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned t = 0;
    for (int k = 0; k < HIT_THREADS / 32; k++) t += red[k];
    size_t sw = ser * ctx.nw + wi;
    hb.tile_cnt[sw * hb.ntiles + tile] = t;
    if (t) atomicAdd(&hb.sw_cnt[sw], t);
  }
}

// exclusive scan of each (series, width)'s tile counts, one warp per row
__global__ void k_scan_tiles(const unsigned* __restrict__ cnt, unsigned* __restrict__ off,
                             unsigned ntiles, size_t nrows) {
  size_t row = (size_t)blockIdx.x * 4 + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (row >= nrows) return;
  const unsigned* c = cnt + row * ntiles;
  unsigned* o = off + row * ntiles;
  unsigned carry = 0;
  for (unsigned b = 0; b < ntiles; b += 32) {
    unsigned v = (b + lane < ntiles) ? c[b + lane] : 0u;
    unsigned x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      unsigned y = __shfl_up_sync(0xffffffffu, x, d);
      if (lane >= d) x += y;
    }
    if (b + lane < ntiles) o[b + lane] = carry + x - v;
    carry += __shfl_sync(0xffffffffu, x, 31);
  }
}

__global__ void __launch_bounds__(HIT_THREADS) k_write_hits(WidthCtx ctx, HitBuffers hb,
                                                            int w_base) {
  const int wi = w_base + blockIdx.y;
  const size_t ser = blockIdx.z;
  const unsigned tile = blockIdx.x;
  const size_t sw = ser * ctx.nw + wi;
  if (hb.tile_cnt[sw * hb.ntiles + tile] == 0) return;
  const WidthInfo& w = ctx.winfo[wi];
  const float* sc = ctx.scan + ser * ctx.scan_pitch;
  const float norm = ctx.norm[sw];
  const size_t i0 = (size_t)tile * HIT_TILE + (size_t)threadIdx.x * HIT_PER_THREAD;
  unsigned flags = 0;
  float vals[HIT_PER_THREAD];
#pragma unroll
  for (int k = 0; k < HIT_PER_THREAD; k++) {
    vals[k] = 0.f;
    if (hit_at(ctx, sc, norm, w, i0 + k, &vals[k])) flags |= 1u << k;
  }
  unsigned c = __popc(flags);
  // block exclusive scan of c
  __shared__ unsigned wsum[HIT_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned x = c;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    unsigned y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  unsigned wpre = 0;
  for (int k = 0; k < warp; k++) wpre += wsum[k];
  unsigned pos = hb.sw_off[sw] + hb.tile_off[sw * hb.ntiles + tile] + wpre + x - c;
#pragma unroll
  for (int k = 0; k < HIT_PER_THREAD; k++) {
    if (flags & (1u << k)) {
      if (pos < hb.cap) {
        hb.ind[pos] = (unsigned)(i0 + k);
        hb.val[pos] = vals[k];
        hb.sw[pos] = (unsigned)sw;
      }
      pos++;
    }
  }
}

// All unscrunched widths [0, nw1) of one tile, from one shared-memory window of
// the prefix sum (tile + boxcar_max + 1 values).
__device__ __forceinline__ void load_hit_tile(const float* sc, size_t i0, float* tile,
                                              size_t span, size_t slen) {
  for (size_t k = threadIdx.x; k < span; k += blockDim.x)
    tile[k] = (i0 + k < slen) ? sc[i0 + k] : 0.f;
  __syncthreads();
}

// Sample j of a tile (j = k * HIT_THREADS + thread) so consecutive lanes read
// consecutive words of the staged window (no bank conflicts).  The in-window
// test (n, beam-local bn) is the same for every unscrunched width, so it is
// evaluated once per sample.
__device__ __forceinline__ unsigned hit_window_mask(const WidthCtx& ctx, const WidthInfo& w,
                                                    size_t i0) {
  unsigned m = 0;
  const unsigned ustride = (unsigned)ctx.stride;
#pragma unroll
  for (int k = 0; k < HIT_PER_THREAD; k++) {
    const unsigned i = (unsigned)(i0 + (size_t)k * HIT_THREADS + threadIdx.x);
    if (i < w.n && (i % ustride) < w.bn) m |= 1u << k;
  }
  return m;
}

__global__ void __launch_bounds__(HIT_THREADS) k_count_hits_multi(WidthCtx ctx, HitBuffers hb,
                                                                  int nw1, size_t slen) {
  extern __shared__ float tile[];
  const size_t ser = blockIdx.y;
  const unsigned t = blockIdx.x;
  const float* sc = ctx.scan + ser * ctx.scan_pitch;
  const size_t i0 = (size_t)t * HIT_TILE;
  const size_t span = HIT_TILE + 2 * (size_t)ctx.offset + 2;
  load_hit_tile(sc, i0, tile, span, slen);
  __shared__ unsigned red[HIT_THREADS / 32];
  const unsigned inwin = hit_window_mask(ctx, ctx.winfo[0], i0);
  for (int wi = 0; wi < nw1; wi++) {
    const WidthInfo& w = ctx.winfo[wi];
    const float norm = ctx.norm[ser * ctx.nw + wi];
    const int a = ctx.offset + w.ahead, b = ctx.offset - w.behind;
    unsigned c = 0;
#pragma unroll
    for (int k = 0; k < HIT_PER_THREAD; k++) {
      const unsigned kl = k * HIT_THREADS + threadIdx.x;
      const float v = __fmul_rn(__fsub_rn(tile[kl + a], tile[kl + b]), norm);
      c += ((inwin >> k) & 1u) && (v > ctx.thresh);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned tot = 0;
      for (int k = 0; k < HIT_THREADS / 32; k++) tot += red[k];
      const size_t sw = ser * ctx.nw + wi;
      hb.tile_cnt[sw * hb.ntiles + t] = tot;
      if (tot) atomicAdd(&hb.sw_cnt[sw], tot);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(HIT_THREADS) k_write_hits_multi(WidthCtx ctx, HitBuffers hb,
                                                                  int nw1, size_t slen) {
  extern __shared__ float tile[];
  const size_t ser = blockIdx.y;
  const unsigned t = blockIdx.x;
  unsigned any = 0;
  for (int wi = 0; wi < nw1; wi++) any |= hb.tile_cnt[(ser * ctx.nw + wi) * hb.ntiles + t];
  if (!any) return;
  const float* sc = ctx.scan + ser * ctx.scan_pitch;
  const size_t i0 = (size_t)t * HIT_TILE;
  const size_t span = HIT_TILE + 2 * (size_t)ctx.offset + 2;
  load_hit_tile(sc, i0, tile, span, slen);
  constexpr int NWARP = HIT_THREADS / 32;
  __shared__ unsigned wcnt[HIT_PER_THREAD][NWARP];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const unsigned inwin = hit_window_mask(ctx, ctx.winfo[0], i0);
  for (int wi = 0; wi < nw1; wi++) {
    const size_t sw = ser * ctx.nw + wi;
    if (hb.tile_cnt[sw * hb.ntiles + t] == 0) continue;  // uniform across the block
    const WidthInfo& w = ctx.winfo[wi];
    const float norm = ctx.norm[sw];
    const int a = ctx.offset + w.ahead, b = ctx.offset - w.behind;
    float vals[HIT_PER_THREAD];
    unsigned bal[HIT_PER_THREAD];
#pragma unroll
    for (int k = 0; k < HIT_PER_THREAD; k++) {
      const unsigned kl = k * HIT_THREADS + threadIdx.x;
      vals[k] = __fmul_rn(__fsub_rn(tile[kl + a], tile[kl + b]), norm);
      const bool f = ((inwin >> k) & 1u) && (vals[k] > ctx.thresh);
      bal[k] = __ballot_sync(0xffffffffu, f);
      if (lane == 0) wcnt[k][warp] = __popc(bal[k]);
    }
    __syncthreads();
    // hits before this thread's sample k in index order: all samples of
    // rounds < k, then lower warps and lower lanes of round k
    unsigned base = hb.sw_off[sw] + hb.tile_off[sw * hb.ntiles + t];
#pragma unroll
    for (int k = 0; k < HIT_PER_THREAD; k++) {
      unsigned before = 0, round = 0;
#pragma unroll
      for (int ww = 0; ww < NWARP; ww++) {
        const unsigned cw = wcnt[k][ww];
        round += cw;
        before += (ww < warp) ? cw : 0u;
      }
      if ((bal[k] >> lane) & 1u) {
        const unsigned pos = base + before + __popc(bal[k] & lt);
        if (pos < hb.cap) {
          hb.ind[pos] = (unsigned)(i0 + (size_t)k * HIT_THREADS + threadIdx.x);
          hb.val[pos] = vals[k];
          hb.sw[pos] = (unsigned)sw;
        }
      }
      base += round;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Vector form of the unscrunched-width kernels, used when the boxcar offset is
// a multiple of 4 (boxcar_max >= 8): every thread owns runs of 4 consecutive
// samples (j = 4t + q and 1024 + 4t + q), so both ends of a boxcar of width
// >= 8 are 16-byte aligned in the staged window and load as float4; widths
// 1, 2 and 4 read one 12-value window around the run.  Consecutive lanes read
// consecutive 16-byte words (no bank conflicts).  Per-width counts are kept
// in 16-bit halves of registers and reduced once per tile.
// ---------------------------------------------------------------------------

struct VecTile {
  float* tile;
  unsigned valid;  // bit g*4+q: sample (g, q) of this thread is in a searched window
};

// In-window bits of this thread's 8 samples of the tile at i0
// (find_giants.cu:47-60): i < n and (i mod beam stride) < bn, the same for
// every unscrunched width.  *all is set when the whole tile is inside one
// beam's searched window (uniform across the block).
__device__ __forceinline__ unsigned vec_valid(const WidthCtx& ctx, size_t i0, bool* all) {
  const WidthInfo& w = ctx.winfo[0];
  const unsigned stride = (unsigned)ctx.stride;
  const unsigned ui0 = (unsigned)i0;
  if (ui0 + HIT_TILE <= w.n && (ui0 % stride) + HIT_TILE <= w.bn) {
    *all = true;
    return 0xFFu;
  }
  *all = false;
  unsigned valid = 0;
#pragma unroll
  for (int g = 0; g < 2; g++)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const unsigned i = ui0 + 1024u * g + 4u * threadIdx.x + q;
      if (i < w.n && (i % stride) < w.bn) valid |= 1u << (g * 4 + q);
    }
  return valid;
}

// Asynchronous copy of the window of the tile at i0 (span4 floats, zero past
// slen) into shared memory; completes with cp_async_wait + a barrier.
__device__ __forceinline__ void vec_prefetch(const float* sc, size_t i0, float* tile,
                                             size_t span4, size_t slen) {
  for (size_t k = 4 * threadIdx.x; k < span4; k += 4 * blockDim.x) {
    if (i0 + k + 3 < slen) {
      cp_async16(tile + k, sc + i0 + k);
    } else {
      tile[k] = (i0 + k < slen) ? sc[i0 + k] : 0.f;
      tile[k + 1] = (i0 + k + 1 < slen) ? sc[i0 + k + 1] : 0.f;
      tile[k + 2] = (i0 + k + 2 < slen) ? sc[i0 + k + 2] : 0.f;
      tile[k + 3] = 0.f;
    }
  }
  cp_async_commit();
}

__device__ __forceinline__ VecTile vec_stage(const WidthCtx& ctx, const float* sc, size_t i0,
                                             float* tile, size_t span4, size_t slen) {
  for (size_t k = 4 * threadIdx.x; k < span4; k += 4 * blockDim.x) {
    float4 v;
    if (i0 + k + 3 < slen) {
      v = *reinterpret_cast<const float4*>(sc + i0 + k);
    } else {
      v.x = (i0 + k < slen) ? sc[i0 + k] : 0.f;
      v.y = (i0 + k + 1 < slen) ? sc[i0 + k + 1] : 0.f;
      v.z = (i0 + k + 2 < slen) ? sc[i0 + k + 2] : 0.f;
      v.w = 0.f;
    }
    *reinterpret_cast<float4*>(tile + k) = v;
  }
  // in-window test (find_giants.cu:47-60): i < n and (i mod beam stride) < bn,
  // the same for every unscrunched width
  const WidthInfo& w = ctx.winfo[0];
  const unsigned stride = (unsigned)ctx.stride;
  const unsigned ui0 = (unsigned)i0;
  unsigned valid;
  const unsigned r0 = ui0 % stride;
  if (ui0 + HIT_TILE <= w.n && r0 + HIT_TILE <= w.bn) {
    valid = 0xFFu;  // the whole tile lies inside one beam's searched window
  } else {
    valid = 0;
#pragma unroll
    for (int g = 0; g < 2; g++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const unsigned i = ui0 + 1024u * g + 4u * threadIdx.x + q;
        if (i < w.n && (i % stride) < w.bn) valid |= 1u << (g * 4 + q);
      }
  }
  __syncthreads();
  return VecTile{tile, valid};
}

// Boxcar values of width wi for the 4 samples of run j0 (window: the 12 staged
// values from j0 + offset - 4).
template <int AH, int BH>
__device__ __forceinline__ void win_boxcar(const float* win, float* d) {
#pragma unroll
  for (int q = 0; q < 4; q++) d[q] = __fsub_rn(win[4 + q + AH], win[4 + q - BH]);
}

// widths 1, 2, 4: ahead = (w - 1) / 2 + 1, behind = w / 2 (matched_filter.cu:37-67)
__device__ __forceinline__ void vec_boxcar(const float* tile, int j0, int offset, int wi,
                                           int ahead, int behind, const float* win,
                                           float* d) {
  if (wi == 0) {
    win_boxcar<1, 0>(win, d);
  } else if (wi == 1) {
    win_boxcar<1, 1>(win, d);
  } else if (wi == 2) {
    win_boxcar<2, 2>(win, d);
  } else {
    const float4 va = *reinterpret_cast<const float4*>(tile + j0 + offset + ahead);
    const float4 vb = *reinterpret_cast<const float4*>(tile + j0 + offset - behind);
    d[0] = __fsub_rn(va.x, vb.x);
    d[1] = __fsub_rn(va.y, vb.y);
    d[2] = __fsub_rn(va.z, vb.z);
    d[3] = __fsub_rn(va.w, vb.w);
  }
}

__device__ __forceinline__ void vec_window(const float* tile, int j0, int offset, float* win) {
  const float4* p = reinterpret_cast<const float4*>(tile + j0 + offset - 4);
  const float4 x0 = p[0], x1 = p[1], x2 = p[2];
  win[0] = x0.x; win[1] = x0.y; win[2] = x0.z; win[3] = x0.w;
  win[4] = x1.x; win[5] = x1.y; win[6] = x1.z; win[7] = x1.w;
  win[8] = x2.x; win[9] = x2.y; win[10] = x2.z; win[11] = x2.w;
}

// For a positive finite norm, RN(d * norm) is non-decreasing in d, so the
// threshold test RN(d * norm) > thresh holds exactly for d >= dmin, the
// smallest float that passes it.  dmin starts from RN(thresh / norm) and is
// moved by single ulps until it passes and its predecessor does not.
// Returns false (use the product) when no such bound is found.
__device__ bool hit_bound(float nrm, float thresh, float* dmin) {
  if (!(nrm > 0.f) || !(nrm <= 3.402823466e38f)) return false;
  float d = __fdiv_rn(thresh, nrm);
  if (!(fabsf(d) <= 3.402823466e38f)) return false;
  for (int it = 0; it < 16 && !(__fmul_rn(d, nrm) > thresh); it++) d = nextafterf(d, INFINITY);
  for (int it = 0; it < 16; it++) {
    const float p = nextafterf(d, -INFINITY);
    if (__fmul_rn(p, nrm) > thresh) d = p;
    else break;
  }
  if (!(__fmul_rn(d, nrm) > thresh) || __fmul_rn(nextafterf(d, -INFINITY), nrm) > thresh)
    return false;
  *dmin = d;
  return true;
}

template <bool ALLV, bool MUL>
__device__ __forceinline__ void count_vec_body(const float* tile, int offset, int nw1,
                                               unsigned valid, const int* s_ahead,
                                               const int* s_behind, const float* s_norm,
                                               const float* s_dmin, float thresh,
                                               unsigned* cnt) {
#pragma unroll
  for (int g = 0; g < 2; g++) {
    const int j0 = 1024 * g + 4 * threadIdx.x;
    float win[12];
    vec_window(tile, j0, offset, win);
    const unsigned vg = (valid >> (4 * g)) & 0xFu;
#pragma unroll
    for (int wi = 0; wi < VH_MAXW; wi++) {
      if (wi >= nw1) break;
      float d[4];
      vec_boxcar(tile, j0, offset, wi, s_ahead[wi], s_behind[wi], win, d);
      unsigned c = 0;
      if (MUL) {
        const float nrm = s_norm[wi];
#pragma unroll
        for (int q = 0; q < 4; q++)
          c += (ALLV || ((vg >> q) & 1u)) && (__fmul_rn(d[q], nrm) > thresh);
      } else {
        const float dm = s_dmin[wi];
#pragma unroll
        for (int q = 0; q < 4; q++) c += (ALLV || ((vg >> q) & 1u)) && (d[q] >= dm);
      }
      cnt[wi >> 1] += c << (16 * (wi & 1));
    }
  }
}

// Block (x, y): tiles [x * tpb, (x + 1) * tpb) of series y (tpb <= 8); the
// next tile's window is copied (cp.async, double buffer) while the current one
// is counted.  With group maxima (ctx.gmax, recorded by the block-RMS pass) a
// tile whose covering groups all lie below a width's bound dmin cannot hold a
// hit of that width (|d| <= group max < dmin for each of its samples, and
// the test is d >= dmin); a tile that no width can hit gets zero counts
// without being read.  Tiles with hits are appended to hb.tile_list.
__global__ void __launch_bounds__(HIT_THREADS) k_count_hits_vec(WidthCtx ctx, HitBuffers hb,
                                                                int nw1, size_t slen,
                                                                size_t span4, int tpb) {
  extern __shared__ __align__(16) float tiles[];  // [2][span4]
  __shared__ int s_ahead[VH_MAXW], s_behind[VH_MAXW];
  __shared__ float s_norm[VH_MAXW], s_dmin[VH_MAXW], s_skip[VH_MAXW];
  __shared__ int s_mul;
  __shared__ unsigned s_need;
  __shared__ unsigned red[HIT_THREADS / 32][VH_MAXW / 2];
  const size_t ser = blockIdx.y;
  const unsigned t_begin = blockIdx.x * (unsigned)tpb;
  const unsigned t_end = min(t_begin + (unsigned)tpb, hb.ntiles);
  const float thresh = ctx.thresh;
  const float* sc = ctx.scan + ser * ctx.scan_pitch;
  const bool use_gmax = ctx.gmax != nullptr && ctx.ngroups > 0 && ctx.gmax_nw >= nw1;
  if (threadIdx.x == 0) {
    s_mul = 0;
    s_need = use_gmax ? 0u : 0xFFu;
  }
  __syncthreads();
  if (threadIdx.x < (unsigned)nw1) {
    s_ahead[threadIdx.x] = ctx.winfo[threadIdx.x].ahead;
    s_behind[threadIdx.x] = ctx.winfo[threadIdx.x].behind;
    const float nrm = ctx.norm[ser * ctx.nw + threadIdx.x];
    s_norm[threadIdx.x] = nrm;
    float dm = 0.f;
    const bool ok = hit_bound(nrm, thresh, &dm);
    if (!ok) atomicOr(&s_mul, 1);
    s_dmin[threadIdx.x] = dm;
    s_skip[threadIdx.x] = ok ? dm : -1.f;  // -1: never skipped (maxima are >= 0)
  }
  if (t_begin >= t_end) return;  // uniform
  const unsigned ntb = t_end - t_begin;
  if (use_gmax) {
    __syncthreads();
    for (unsigned idx = threadIdx.x; idx < ntb * (unsigned)nw1; idx += blockDim.x) {
      const unsigned ti = idx / (unsigned)nw1, wi = idx - ti * (unsigned)nw1;
      const size_t i0 = (size_t)(t_begin + ti) * HIT_TILE;
      const size_t g_lo = i0 / ctx.gsize, g_hi = (i0 + HIT_TILE - 1) / ctx.gsize;
      bool need = true;
      if (g_hi < ctx.ngroups) {
        // bit patterns of non-negative floats (or NaN, which wins and keeps
        // the tile) order as unsigned
        const float* gm = ctx.gmax + (ser * (size_t)ctx.gmax_nw + wi) * ctx.ngroups;
        unsigned mk = 0;
        for (size_t g = g_lo; g <= g_hi; g++) mk = max(mk, __float_as_uint(gm[g]));
        need = !(__uint_as_float(mk) < s_skip[wi]);
      }
      if (need) atomicOr(&s_need, 1u << ti);
    }
    __syncthreads();
    // skipped tiles: zero counts (read by the scans and the write pass)
    for (unsigned idx = threadIdx.x; idx < ntb * (unsigned)nw1; idx += blockDim.x) {
      const unsigned ti = idx / (unsigned)nw1, wi = idx - ti * (unsigned)nw1;
      if (!((s_need >> ti) & 1u))
        hb.tile_cnt[(ser * ctx.nw + wi) * hb.ntiles + t_begin + ti] = 0;
    }
  }
  unsigned rest = s_need & ((1u << ntb) - 1u);
  if (!rest) return;  // uniform
  const int offset = ctx.offset;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned t = t_begin + (unsigned)(__ffs(rest) - 1);
  rest &= rest - 1u;
  int bi = 0;
  vec_prefetch(sc, (size_t)t * HIT_TILE, tiles, span4, slen);
  for (;;) {
    float* tile = tiles + (size_t)bi * span4;
    // the previous tile is counted and its reduction slots are read
    __syncthreads();
    const bool more = rest != 0u;
    unsigned tn = 0;
    if (more) {
      tn = t_begin + (unsigned)(__ffs(rest) - 1);
      rest &= rest - 1u;
      vec_prefetch(sc, (size_t)tn * HIT_TILE, tiles + (size_t)(bi ^ 1) * span4, span4, slen);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const size_t i0 = (size_t)t * HIT_TILE;
    bool allv;
    const unsigned valid = vec_valid(ctx, i0, &allv);
    unsigned cnt[VH_MAXW / 2];
#pragma unroll
    for (int p = 0; p < VH_MAXW / 2; p++) cnt[p] = 0;
    if (s_mul) {
      if (allv) count_vec_body<true, true>(tile, offset, nw1, valid, s_ahead, s_behind, s_norm, s_dmin, thresh, cnt);
      else count_vec_body<false, true>(tile, offset, nw1, valid, s_ahead, s_behind, s_norm, s_dmin, thresh, cnt);
    } else {
      if (allv) count_vec_body<true, false>(tile, offset, nw1, valid, s_ahead, s_behind, s_norm, s_dmin, thresh, cnt);
      else count_vec_body<false, false>(tile, offset, nw1, valid, s_ahead, s_behind, s_norm, s_dmin, thresh, cnt);
    }
#pragma unroll
    for (int p = 0; p < VH_MAXW / 2; p++) {
      if (2 * p >= nw1) break;
      unsigned c = cnt[p];
#pragma unroll
      for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
      if (lane == 0) red[warp][p] = c;
    }
    __syncthreads();
    unsigned tot = 0;
    if (threadIdx.x < (unsigned)nw1) {
      const int wi = threadIdx.x;
      for (int k = 0; k < HIT_THREADS / 32; k++) tot += (red[k][wi >> 1] >> (16 * (wi & 1))) & 0xFFFFu;
      const size_t sw = ser * ctx.nw + wi;
      hb.tile_cnt[sw * hb.ntiles + t] = tot;
      if (tot) atomicAdd(&hb.sw_cnt[sw], tot);
    }
    if (__syncthreads_or(tot != 0u) && threadIdx.x == 0 && hb.tile_list)
      hb.tile_list[atomicAdd(hb.tile_list_n, 1u)] = (unsigned)(ser * hb.ntiles + t);
    if (!more) break;
    t = tn;
    bi ^= 1;
  }
}


__device__ __forceinline__ void write_hits_vec_tile(const WidthCtx& ctx, const HitBuffers& hb,
                                                    int nw1, size_t slen, size_t span4,
                                                    float* tile, unsigned* wsum, size_t ser,
                                                    unsigned t) {
  unsigned any = 0;
  for (int wi = 0; wi < nw1; wi++) any |= hb.tile_cnt[(ser * ctx.nw + wi) * hb.ntiles + t];
  if (!any) return;  // uniform across the block
  const size_t i0 = (size_t)t * HIT_TILE;
  const VecTile vt = vec_stage(ctx, ctx.scan + ser * ctx.scan_pitch, i0, tile, span4, slen);
  const float thresh = ctx.thresh;
  const int offset = ctx.offset;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float win0[12], win1[12];
  vec_window(tile, 4 * threadIdx.x, offset, win0);
  vec_window(tile, 1024 + 4 * threadIdx.x, offset, win1);
  for (int wi = 0; wi < nw1; wi++) {
    const size_t sw = ser * ctx.nw + wi;
    if (hb.tile_cnt[sw * hb.ntiles + t] == 0) continue;  // uniform across the block
    const WidthInfo& w = ctx.winfo[wi];
    const float nrm = ctx.norm[sw];
    float v0[4], v1[4];
    vec_boxcar(tile, 4 * threadIdx.x, offset, wi, w.ahead, w.behind, win0, v0);
    vec_boxcar(tile, 1024 + 4 * threadIdx.x, offset, wi, w.ahead, w.behind, win1, v1);
    unsigned f = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      v0[q] = __fmul_rn(v0[q], nrm);
      v1[q] = __fmul_rn(v1[q], nrm);
      if (((vt.valid >> q) & 1u) && v0[q] > thresh) f |= 1u << q;
      if (((vt.valid >> (4 + q)) & 1u) && v1[q] > thresh) f |= 1u << (4 + q);
    }
    // hits in index order: all of run group 0 (samples 0..1023) by thread,
    // then group 1; one block exclusive scan of (count0 | count1 << 16)
    const unsigned c = (unsigned)__popc(f & 0xFu) | ((unsigned)__popc(f >> 4) << 16);
    unsigned x = c;
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, x, dd);
      if (lane >= dd) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    unsigned pre = 0, tot = 0;
    for (int k = 0; k < HIT_THREADS / 32; k++) {
      const unsigned ws = wsum[k];
      pre += (k < warp) ? ws : 0u;
      tot += ws;
    }
    __syncthreads();
    pre += x - c;  // exclusive, both halves
    const unsigned base = hb.sw_off[sw] + hb.tile_off[sw * hb.ntiles + t];
    const unsigned p0 = base + (pre & 0xFFFFu);
    const unsigned p1 = base + (tot & 0xFFFFu) + (pre >> 16);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      if ((f >> q) & 1u) {
        const unsigned pos = p0 + __popc(f & ((1u << q) - 1u));
        if (pos < hb.cap) {
          hb.ind[pos] = (unsigned)(i0 + 4 * threadIdx.x + q);
          hb.val[pos] = v0[q];
          hb.sw[pos] = (unsigned)sw;
        }
      }
      if ((f >> (4 + q)) & 1u) {
        const unsigned pos = p1 + __popc((f >> 4) & ((1u << q) - 1u));
        if (pos < hb.cap) {
          hb.ind[pos] = (unsigned)(i0 + 1024 + 4 * threadIdx.x + q);
          hb.val[pos] = v1[q];
          hb.sw[pos] = (unsigned)sw;
        }
      }
    }
  }
}

// Block (x, y): tile x of series y; or, with hb.list_valid, the tiles listed
// by the count pass (the only ones with hits), strided over the blocks.
__global__ void __launch_bounds__(HIT_THREADS) k_write_hits_vec(WidthCtx ctx, HitBuffers hb,
                                                                int nw1, size_t slen,
                                                                size_t span4) {
  extern __shared__ __align__(16) float tile[];
  __shared__ unsigned wsum[HIT_THREADS / 32];
  if (!hb.list_valid) {
    write_hits_vec_tile(ctx, hb, nw1, slen, span4, tile, wsum, blockIdx.y, blockIdx.x);
    return;
  }
  const unsigned n = *hb.tile_list_n;
  for (unsigned idx = blockIdx.x; idx < n; idx += gridDim.x) {
    const unsigned e = hb.tile_list[idx];
    write_hits_vec_tile(ctx, hb, nw1, slen, span4, tile, wsum, e / hb.ntiles, e % hb.ntiles);
    __syncthreads();  // the staged tile is reused by the next item
  }
}

// Vector kernels apply when the offset is a multiple of 4 (>= 4), the widths
// are 1, 2, 4, ... and at most VH_MAXW of them are unscrunched.
static bool vec_hits_ok(const WidthCtx& ctx, int nw1) {
  if (nw1 < 1 || nw1 > VH_MAXW || ctx.offset < 4 || (ctx.offset & 3) || (ctx.scan_pitch & 3) ||
      (reinterpret_cast<uintptr_t>(ctx.scan) & 15) || ctx.stride >= 0xFFFFFFFFull)
    return false;
  for (int wi = 0; wi < nw1; wi++) {
    const WidthInfo& w = ctx.host_winfo[wi];
    if (w.width != (1 << wi)) return false;
    if (w.ahead != (w.width - 1) / 2 + 1 || w.behind != w.width / 2) return false;
    if (wi >= 3 && (((w.ahead | w.behind) & 3) != 0)) return false;
  }
  return true;
}

cudaError_t count_hits(const WidthCtx& ctx, HitBuffers& hb, unsigned ntiles, cudaStream_t s) {
  hb.ntiles = ntiles;
  hb.list_valid = false;
  cudaError_t e = cudaMemsetAsync(hb.sw_cnt, 0, ((size_t)ctx.nser * ctx.nw + 1) * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  // unscrunched widths share one staged window per tile
  int nw1 = 0;
  while (nw1 < ctx.nw && ctx.host_winfo[nw1].ts == 1) nw1++;
  const size_t smem = (HIT_TILE + 2 * (size_t)ctx.offset + 2) * sizeof(float);
  const size_t span4 = (HIT_TILE + 2 * (size_t)ctx.offset + 2 + 3) & ~(size_t)3;
  const size_t slen = ctx.scan_len;
  if (vec_hits_ok(ctx, nw1) && 2 * span4 * sizeof(float) <= 200 * 1024) {
    if ((e = raise_smem_limit(k_count_hits_vec, 2 * span4 * sizeof(float))) != cudaSuccess)
      return e;
    if (hb.tile_list) {
      if ((e = cudaMemsetAsync(hb.tile_list_n, 0, sizeof(unsigned), s)) != cudaSuccess) return e;
      hb.list_valid = true;
    }
    // about 8 consecutive tiles per block (at most 8), spread evenly
    const unsigned nbx = (ntiles + 7) / 8;
    const unsigned tpb = (ntiles + nbx - 1) / nbx;
    k_count_hits_vec<<<dim3((ntiles + tpb - 1) / tpb, ctx.nser), HIT_THREADS,
                       2 * span4 * sizeof(float), s>>>(ctx, hb, nw1, slen, span4, (int)tpb); note_launch();
  } else if (nw1 > 0 && smem <= 200 * 1024) {
    if ((e = raise_smem_limit(k_count_hits_multi, smem)) != cudaSuccess) return e;
    k_count_hits_multi<<<dim3(ntiles, ctx.nser), HIT_THREADS, smem, s>>>(ctx, hb, nw1, slen); note_launch();
  } else {
    nw1 = 0;
  }
  if (nw1 < ctx.nw) {
    k_count_hits<<<dim3(ntiles, ctx.nw - nw1, ctx.nser), HIT_THREADS, 0, s>>>(ctx, hb, nw1); note_launch();
  }
  return cudaGetLastError();
}

cudaError_t scan_hit_counts(const WidthCtx& ctx, HitBuffers& hb, cudaStream_t s) {
  size_t rows = (size_t)ctx.nser * ctx.nw;
  k_scan_tiles<<<(unsigned)((rows + 3) / 4), 128, 0, s>>>(hb.tile_cnt, hb.tile_off, hb.ntiles,
                                                          rows); note_launch();
  return cudaGetLastError();
}

cudaError_t write_hits(const WidthCtx& ctx, HitBuffers& hb, cudaStream_t s) {
  int nw1 = 0;
  while (nw1 < ctx.nw && ctx.host_winfo[nw1].ts == 1) nw1++;
  const size_t smem = (HIT_TILE + 2 * (size_t)ctx.offset + 2) * sizeof(float);
  const size_t span4 = (HIT_TILE + 2 * (size_t)ctx.offset + 2 + 3) & ~(size_t)3;
  const size_t slen = ctx.scan_len;
  if (vec_hits_ok(ctx, nw1) && span4 * sizeof(float) <= 200 * 1024) {
    if (cudaError_t e = raise_smem_limit(k_write_hits_vec, span4 * sizeof(float)))
      return e;
    // the listed tiles (count pass), strided over a grid of 8 blocks per SM;
    // else every tile once
    const size_t ntile_all = (size_t)hb.ntiles * ctx.nser;
    const dim3 grid = hb.list_valid ? dim3((unsigned)std::min<size_t>(ntile_all, 148 * 8))
                                    : dim3(hb.ntiles, ctx.nser);
    k_write_hits_vec<<<grid, HIT_THREADS, span4 * sizeof(float), s>>>(ctx, hb, nw1, slen,
                                                                      span4); note_launch();
  } else if (nw1 > 0 && smem <= 200 * 1024) {
    if (cudaError_t e = raise_smem_limit(k_write_hits_multi, smem)) return e;
    k_write_hits_multi<<<dim3(hb.ntiles, ctx.nser), HIT_THREADS, smem, s>>>(ctx, hb, nw1, slen); note_launch();
  } else {
    nw1 = 0;
  }
  if (nw1 < ctx.nw) {
    k_write_hits<<<dim3(hb.ntiles, ctx.nw - nw1, ctx.nser), HIT_THREADS, 0, s>>>(ctx, hb, nw1); note_launch();
  }
  return cudaGetLastError();
}

// ===========================================================================
// Device-wide exclusive scan of unsigned values (3 phases).
// ===========================================================================
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ unsigned block_exclusive_scan(unsigned v, unsigned* total) {
  __shared__ unsigned ws[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    unsigned y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    unsigned w = (lane < (int)(blockDim.x >> 5)) ? ws[lane] : 0u;
    unsigned z = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      unsigned y = __shfl_up_sync(0xffffffffu, z, d);
      if (lane >= d) z += y;
    }
    ws[lane] = z - w;
    if (lane == 31 && total) *total = z;
  }
  __syncthreads();
  unsigned r = ws[warp] + x - v;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles_u32(const unsigned* __restrict__ in,
                                                                 unsigned* __restrict__ out,
                                                                 size_t n,
                                                                 unsigned* __restrict__ sums) {
  const size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
  unsigned v[SCAN_ITEMS];
  unsigned t = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    v[k] = (base + k < n) ? in[base + k] : 0u;
    t += v[k];
  }
  __shared__ unsigned tot;
  unsigned pre = block_exclusive_scan(t, &tot);
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    if (base + k < n) out[base + k] = pre;
    pre += v[k];
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_add(unsigned* __restrict__ out, size_t n,
                                                           const unsigned* __restrict__ sums_off) {
  const size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
  unsigned a = sums_off[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++)
    if (base + k < n) out[base + k] += a;
}

size_t scan_tmp_words(size_t n) {
  size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  size_t nb2 = (nb + SCAN_TILE - 1) / SCAN_TILE;
  return 2 * nb + 2 * nb2 + 8;
}

cudaError_t scan_u32(const unsigned* in, unsigned* out, size_t n, unsigned* total, unsigned* tmp,
                     cudaStream_t s) {
  if (n == 0) return cudaMemsetAsync(total, 0, sizeof(unsigned), s);
  size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  unsigned* sums = tmp;
  unsigned* sums_off = tmp + nb;
  k_scan_tiles_u32<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, out, n, sums); note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (nb == 1) {
    cudaMemsetAsync(sums_off, 0, sizeof(unsigned), s);
    return cudaMemcpyAsync(total, sums, sizeof(unsigned), cudaMemcpyDeviceToDevice, s);
  }
  // recursive scan of the block sums
  e = scan_u32(sums, sums_off, nb, total, tmp + 2 * nb, s);
  if (e != cudaSuccess) return e;
  k_scan_add<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(out, n, sums_off); note_launch();
  return cudaGetLastError();
}

// ===========================================================================
// Giants (find_giants.cu:194-316, pipeline.cu:755-775)
// ===========================================================================
// 1 when hit k (of nhits) starts a giant: the first hit of its (series,
// width), or one farther than the width's merge distance from the previous.
__device__ __forceinline__ unsigned giant_head_of(const WidthCtx& ctx, const HitBuffers& hb,
                                                  size_t k) {
  const unsigned sw = hb.sw[k];
  unsigned h = 1;
  if (k > 0 && hb.sw[k - 1] == sw) {
    const WidthInfo& w = ctx.winfo[sw % ctx.nw];
    // not_nearby: b > a + max_dist  (find_giants.cu:79-87)
    h = ((unsigned long long)hb.ind[k] > (unsigned long long)hb.ind[k - 1] + w.merge_dist) ? 1u : 0u;
  }
  return h;
}

__global__ void k_giant_heads(WidthCtx ctx, HitBuffers hb, unsigned nhits, unsigned* head) {
  size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nhits) return;
  head[k] = giant_head_of(ctx, hb, k);
}

// Hit k's share of its giant: the first maximum (larger value wins, ties to
// the smaller hit position), begin, end, filter and DM key.  Giants at or
// beyond gcap are not written (the device-count form's capacity).
__device__ __forceinline__ void giant_reduce_at(const WidthCtx& ctx, const HitBuffers& hb,
                                                size_t k, unsigned nhits, const GiantBuffers& gb,
                                                unsigned gcap) {
  const bool live = k < nhits;
  const int lane = threadIdx.x & 31;
  unsigned g = 0xFFFFFFFFu;
  unsigned long long key = 0;
  if (live) {
    g = gb.gid[k] + gb.head[k] - 1u;  // inclusive count of heads - 1
    key = ((unsigned long long)float_key(hb.val[k]) << 32) |
          (unsigned long long)(0xFFFFFFFFu - (unsigned)k);
  }
  // a giant's hits are consecutive: reduce each run inside the warp, then one
  // atomic per run (max is order-independent, so the result is the same)
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const unsigned long long ok = __shfl_down_sync(0xffffffffu, key, off);
    const unsigned og = __shfl_down_sync(0xffffffffu, g, off);
    if (lane + off < 32 && og == g && ok > key) key = ok;
  }
  const unsigned gp = __shfl_up_sync(0xffffffffu, g, 1);
  if (!live || g >= gcap) return;
  if (lane == 0 || gp != g) atomicMax(&gb.key[g], key);
  unsigned sw = hb.sw[k];
  const WidthInfo& w = ctx.winfo[sw % ctx.nw];
  bool is_head = gb.head[k] != 0;
  bool is_last = (k + 1 == nhits) || gb.head[k + 1] != 0;
  unsigned long long scr = (unsigned long long)w.scr;
  if (is_head) gb.begin[g] = ((unsigned long long)hb.ind[k] + w.rel_off) * scr;
  if (is_last) gb.end[g] = ((unsigned long long)hb.ind[k] + 1ull + w.rel_off) * scr;
  if (is_head) {
    // DM key: units (beams searched independently) are kept dm_key_gap > dm_tol
    // apart so clustering never links two units
    const unsigned ser = sw / ctx.nw;
    gb.filter[g] = w.filter_idx;
    gb.dm[g] = (int)((ser / ctx.dms_per_unit) * ctx.dm_key_gap + ctx.dm_offset +
                     ser % ctx.dms_per_unit);
  }
}

__global__ void k_giant_reduce(WidthCtx ctx, HitBuffers hb, unsigned nhits, GiantBuffers gb) {
  giant_reduce_at(ctx, hb, (size_t)blockIdx.x * blockDim.x + threadIdx.x, nhits, gb,
                  0xFFFFFFFFu);
}

__device__ __forceinline__ void giant_finish_at(const HitBuffers& hb, size_t g,
                                                const GiantBuffers& gb, const WidthInfo* winfo,
                                                int nw) {
  unsigned long long key = gb.key[g];
  unsigned k = 0xFFFFFFFFu - (unsigned)(key & 0xFFFFFFFFull);
  const WidthInfo& w = winfo[hb.sw[k] % nw];
  gb.peak[g] = hb.val[k];
  gb.ind[g] = ((unsigned long long)hb.ind[k] + w.rel_off) * (unsigned long long)w.scr;
}

__global__ void k_giant_finish(HitBuffers hb, unsigned ngiants, GiantBuffers gb,
                               const WidthInfo* winfo, int nw) {
  size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngiants) return;
  giant_finish_at(hb, g, gb, winfo, nw);
}

__global__ void k_giant_place(GiantBuffers src, unsigned n, int dm_key_gap,
                              const unsigned* __restrict__ first,
                              const unsigned* __restrict__ dst_base, GiantBuffers dst) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned u = (unsigned)src.dm[i] / (unsigned)dm_key_gap;
  const unsigned j = dst_base[u] + (i - first[u]);
  dst.peak[j] = src.peak[i];
  dst.ind[j] = src.ind[i];
  dst.begin[j] = src.begin[i];
  dst.end[j] = src.end[i];
  dst.filter[j] = src.filter[i];
  dst.dm[j] = src.dm[i];
}

cudaError_t giant_place(const GiantBuffers& src, unsigned n, int dm_key_gap,
                        const unsigned* first, const unsigned* dst_base, GiantBuffers& dst,
                        cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_giant_place<<<(n + 255) / 256, 256, 0, s>>>(src, n, dm_key_gap, first, dst_base, dst);
  note_launch();
  return cudaGetLastError();
}

cudaError_t giant_heads(const WidthCtx& ctx, const HitBuffers& hb, unsigned nhits,
                        GiantBuffers& gb, cudaStream_t s) {
  if (nhits == 0) return cudaSuccess;
  k_giant_heads<<<(nhits + 255) / 256, 256, 0, s>>>(ctx, hb, nhits, gb.head); note_launch();
  return cudaGetLastError();
}

cudaError_t giant_fill(const WidthCtx& ctx, const HitBuffers& hb, unsigned nhits,
                       unsigned ngiants, GiantBuffers& gb, cudaStream_t s) {
  if (nhits == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(gb.key, 0, (size_t)ngiants * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  k_giant_reduce<<<(nhits + 255) / 256, 256, 0, s>>>(ctx, hb, nhits, gb); note_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_giant_finish<<<(ngiants + 255) / 256, 256, 0, s>>>(hb, ngiants, gb, ctx.winfo, ctx.nw); note_launch();
  return cudaGetLastError();
}

// ===========================================================================
// Clustering (label_candidate_clusters.cu:141-197,203-394)
//
// The reference's neighbour sweep labels[i] = min(labels[i], labels[j]) over
// coincident j, run sequentially, gives every giant the smallest index
// reachable from it through a chain of coincident giants with decreasing
// indices (a coincident j > i still holds its own, larger, label when i is
// swept).  That value is the unique fixed point of
//   lab[i] = min(i, min_{j < i coincident} lab[j]),
// which these sweeps reach from lab[i] = i with atomicMin updates in any
// order; the final chain trace of the reference is then the identity.
// ===========================================================================
constexpr int CL_TILE = 128;
constexpr int CL_YBLOCKS = 8;  // chunks of earlier giants per window, about

__global__ void k_cluster_init(int* label, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) label[i] = i;
}

// Block (x, y): giants [x*CL_TILE, +CL_TILE) against the y-th chunk of
// `jchunk` earlier giants inside their DM window.  The chunk is the window
// bound over CL_YBLOCKS (at least 128), so every tile's window is spread over
// about that many blocks: short scans for small windows, and a grid that
// stays near tiles x CL_YBLOCKS for large ones.
// The sweep of block (blockIdx.x, blockIdx.y) over the first n giants.
__device__ __forceinline__ void cluster_sweep_block(const ClusterArgs& a, const GiantBuffers& gb,
                                                    const int n, unsigned* changed,
                                                    const int jchunk) {
  __shared__ unsigned s_samp[CL_TILE], s_beam[CL_TILE];
  __shared__ int s_f[CL_TILE], s_dm[CL_TILE], s_lab[CL_TILE];
  const int i_first = blockIdx.x * CL_TILE;
  const int i = i_first + threadIdx.x;
  const int i_last = min(i_first + CL_TILE, n) - 1;
  if ((long long)blockIdx.y * jchunk > (long long)i_last) return;  // uniform: past the tile
  // giants are in ascending DM order: the first candidate neighbour is the
  // first giant within dm_tol of the tile's smallest DM
  const int dm_first = gb.dm[i_first];
  int lo = 0, hi = i_first;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if ((long long)gb.dm[mid] + (long long)a.dm_tol < (long long)dm_first) lo = mid + 1;
    else hi = mid;
  }
  const long long jb = (long long)lo + (long long)blockIdx.y * jchunk;
  if (jb > (long long)i_last) return;  // uniform: this chunk lies past the tile
  const int j_begin = (int)jb;
  const int j_end = (int)min((long long)j_begin + jchunk, (long long)i_last + 1);
  // sample indices fit 31 bits (checked by the host); the test below is
  // are_coincident_beam (are_coincident.cuh:47-68): same beam, time within
  // time_tol x the wider boxcar (a power of two), filter and DM within tolerance.
  // A giant's beam is computed once, when it is staged.
  unsigned si = 0, bi = 0;
  int fi = 0, di = 0, best = 0x7FFFFFFF;
  if (i < n) {
    si = (unsigned)gb.ind[i];
    bi = (unsigned)(gb.ind[i] / a.nsamps_beam);
    fi = gb.filter[i];
    di = gb.dm[i];
    best = gb.label[i];
  }
  const int start_best = best;
  const unsigned ftol = (unsigned)min(a.filter_tol, 0x7FFFFFFFull);
  const unsigned dtol = (unsigned)min(a.dm_tol, 0x7FFFFFFFull);
  for (int j0 = j_begin; j0 < j_end; j0 += CL_TILE) {
    const int j = j0 + threadIdx.x;
    __syncthreads();
    if (j < j_end) {
      const unsigned long long sj = gb.ind[j];
      s_samp[threadIdx.x] = (unsigned)sj;
      s_beam[threadIdx.x] = (unsigned)(sj / a.nsamps_beam);
      s_f[threadIdx.x] = gb.filter[j];
      s_dm[threadIdx.x] = gb.dm[j];
      s_lab[threadIdx.x] = *((volatile int*)&gb.label[j]);
    }
    __syncthreads();
    if (i < n) {
      const int jn = min(min(CL_TILE, j_end - j0), i - j0);  // only j < i
      for (int jj = 0; jj < jn; jj++) {
        const unsigned sj = s_samp[jj];
        const int fj = s_f[jj];
        const unsigned dt = sj > si ? sj - si : si - sj;
        const unsigned long long tt = a.time_tol << max(fi, fj);
        const bool coinc = s_beam[jj] == bi && (unsigned long long)dt <= tt &&
                           (unsigned)abs(fj - fi) <= ftol &&
                           (unsigned)abs(s_dm[jj] - di) <= dtol;
        if (coinc && s_lab[jj] < best) best = s_lab[jj];
      }
    }
  }
  if (i < n && best < start_best) {
    int old = atomicMin(&gb.label[i], best);
    if (best < old) *changed = 1u;
  }
}

__global__ void __launch_bounds__(CL_TILE) k_cluster_sweep(ClusterArgs a, GiantBuffers gb,
                                                           unsigned* changed, int jchunk) {
  cluster_sweep_block(a, gb, a.ngiants, changed, jchunk);
}

// Path jumping: lab[i] is reachable from i, so anything reachable from lab[i]
// is too; taking lab[lab[i]] keeps every label on the same fixed point.
__global__ void k_cluster_jump(int* label, int n, unsigned* changed) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int l = label[i];
  int ll = *((volatile int*)&label[l]);
  if (ll < l) {
    atomicMin(&label[i], ll);
    *changed = 1u;
  }
}

cudaError_t cluster_init(GiantBuffers& gb, int n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_cluster_init<<<(n + 255) / 256, 256, 0, s>>>(gb.label, n); note_launch();
  return cudaGetLastError();
}

cudaError_t cluster_sweep(const ClusterArgs& a, GiantBuffers& gb, unsigned* changed,
                          cudaStream_t s) {
  if (a.ngiants == 0) return cudaSuccess;
  // a window holds at most the unit's giants (plus the tile's own)
  const long long wmax = (long long)(a.max_unit_giants > 0 ? a.max_unit_giants : a.ngiants) +
                         CL_TILE;
  long long chunk = (wmax + CL_YBLOCKS - 1) / CL_YBLOCKS;
  chunk = std::max<long long>(128, (chunk + 127) / 128 * 128);
  const long long ny = (std::min<long long>(wmax, a.ngiants) + chunk - 1) / chunk;
  dim3 grid((a.ngiants + CL_TILE - 1) / CL_TILE, (unsigned)std::max<long long>(ny, 1));
  k_cluster_sweep<<<grid, CL_TILE, 0, s>>>(a, gb, changed, (int)chunk); note_launch();
  k_cluster_jump<<<(a.ngiants + 255) / 256, 256, 0, s>>>(gb.label, a.ngiants, changed); note_launch();
  return cudaGetLastError();
}

// ===========================================================================
// Merge (merge_candidates.cu:74-134): groups in ascending label order; per
// group the first member with the largest peak, members summed; DM gathered.
// ===========================================================================
__global__ void k_root_flags(const int* label, int n, unsigned* flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = (label[i] == i) ? 1u : 0u;
}

__global__ void k_merge_reduce(GiantBuffers gb, int n, const unsigned* root_off,
                               unsigned long long* gkey, unsigned long long* members) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned g = root_off[gb.label[i]];
  unsigned long long key = ((unsigned long long)float_key(gb.peak[i]) << 32) |
                           (unsigned long long)(0xFFFFFFFFu - (unsigned)i);
  atomicMax(&gkey[g], key);
  atomicAdd(&members[g], 1ull);
}

__global__ void k_merge_emit(GiantBuffers gb, int dm_key_gap, const unsigned* ngroups,
                             const unsigned long long* gkey, const unsigned long long* members,
                             const float* dm_list, GroupRow* rows) {
  unsigned g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= *ngroups) return;
  unsigned i = 0xFFFFFFFFu - (unsigned)(gkey[g] & 0xFFFFFFFFull);
  GroupRow r;
  r.peak = gb.peak[i];
  r.ind = gb.ind[i];
  r.begin = gb.begin[i];
  r.end = gb.end[i];
  r.filter = (unsigned long long)gb.filter[i];
  const int key = gb.dm[i];
  r.dm_ind = (unsigned long long)(key % dm_key_gap);
  r.unit = (unsigned long long)(key / dm_key_gap);
  r.members = members[g];
  r.dm = dm_list[key % dm_key_gap];
  rows[g] = r;
}

// First giant of each unit: giants are ordered by DM key, and unit u's keys
// lie in [u * dm_key_gap, (u + 1) * dm_key_gap).  offs[u] for u = 0..units.
__global__ void k_unit_offsets(const int* __restrict__ dm, int n, int dm_key_gap, int units,
                               unsigned* offs) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u > units) return;
  const long long target = (long long)u * dm_key_gap;
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if ((long long)dm[mid] < target) lo = mid + 1;
    else hi = mid;
  }
  offs[u] = (unsigned)lo;
}

cudaError_t unit_giant_offsets(const GiantBuffers& gb, int n, int dm_key_gap, int units,
                               unsigned* offs, cudaStream_t s) {
  k_unit_offsets<<<(units + 1 + 127) / 128, 128, 0, s>>>(gb.dm, n, dm_key_gap, units, offs);
  note_launch();
  return cudaGetLastError();
}

cudaError_t merge_groups(const GiantBuffers& gb, int n, int dm_key_gap, const float* dm_list,
                         unsigned* root_flag,
                         unsigned* root_off, unsigned* nroots, unsigned* scan_tmp,
                         unsigned long long* gkey, GroupRow* rows, cudaStream_t s) {
  if (n == 0) return cudaMemsetAsync(nroots, 0, sizeof(unsigned), s);
  k_root_flags<<<(n + 255) / 256, 256, 0, s>>>(gb.label, n, root_flag); note_launch();
  cudaError_t e = scan_u32(root_flag, root_off, (size_t)n, nroots, scan_tmp, s);
  if (e != cudaSuccess) return e;
  // gkey: [n] keys followed by [n] member counts
  unsigned long long* members = gkey + n;
  if ((e = cudaMemsetAsync(gkey, 0, 2 * (size_t)n * sizeof(unsigned long long), s)) != cudaSuccess)
    return e;
  k_merge_reduce<<<(n + 255) / 256, 256, 0, s>>>(gb, n, root_off, gkey, members); note_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // emit for every possible group index; rows beyond nroots are never read
  k_merge_emit<<<(n + 255) / 256, 256, 0, s>>>(gb, dm_key_gap, nroots, gkey, members, dm_list,
                                               rows); note_launch();
  return cudaGetLastError();
}

// ===========================================================================
// Device-count forms of the giant, clustering and merge stages, for a gulp
// captured as a CUDA graph.  The hit and giant totals stay in device words
// that the kernels read; grids are sized by capacities fixed when the graph
// is captured and every kernel clamps to them.  A total above its capacity
// is seen by the host after the gulp, which then searches the gulp again on
// the host-sized path, so a clamped result is never reported.
// ===========================================================================
__device__ __forceinline__ unsigned clamp_count(const unsigned* n, unsigned cap) {
  const unsigned v = *n;
  return v < cap ? v : cap;
}

// head[k] for every k < hcap (0 past the hit count, so that a scan over the
// capacity counts the giants)
__global__ void k_giant_heads_dev(WidthCtx ctx, HitBuffers hb, const unsigned* nhits,
                                  unsigned hcap, unsigned* head) {
  const unsigned n = clamp_count(nhits, hcap);
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < hcap;
       k += (size_t)gridDim.x * blockDim.x)
    head[k] = k < n ? giant_head_of(ctx, hb, k) : 0u;
}

__global__ void k_giant_reduce_dev(WidthCtx ctx, HitBuffers hb, const unsigned* nhits,
                                   unsigned hcap, GiantBuffers gb, unsigned gcap) {
  giant_reduce_at(ctx, hb, (size_t)blockIdx.x * blockDim.x + threadIdx.x,
                  clamp_count(nhits, hcap), gb, gcap);
}

__global__ void k_giant_finish_dev(HitBuffers hb, const unsigned* ngiants, unsigned gcap,
                                   GiantBuffers gb, const WidthInfo* winfo, int nw) {
  const unsigned n = clamp_count(ngiants, gcap);
  for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
       g += (size_t)gridDim.x * blockDim.x)
    giant_finish_at(hb, g, gb, winfo, nw);
}

__global__ void k_unit_offsets_dev(const int* __restrict__ dm, const unsigned* ngiants,
                                   unsigned gcap, int dm_key_gap, int units, unsigned* offs) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u > units) return;
  const int n = (int)clamp_count(ngiants, gcap);
  const long long target = (long long)u * dm_key_gap;
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if ((long long)dm[mid] < target) lo = mid + 1;
    else hi = mid;
  }
  offs[u] = (unsigned)lo;
}

// geo[0] = giant count (clamped), geo[1] = the sweep's chunk of earlier
// giants per block (the host form's rule in cluster_sweep, from the largest
// unit's giant count)
__global__ void k_cluster_geom(const unsigned* __restrict__ offs, int units,
                               const unsigned* ngiants, unsigned gcap, int* geo) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const unsigned n = clamp_count(ngiants, gcap);
  unsigned max_unit = 0;
  for (int u = 0; u < units; u++) max_unit = max(max_unit, offs[u + 1] - offs[u]);
  const long long wmax = (long long)(max_unit > 0 ? max_unit : n) + CL_TILE;
  long long chunk = (wmax + CL_YBLOCKS - 1) / CL_YBLOCKS;
  chunk = max(128ll, (chunk + 127) / 128 * 128);
  geo[0] = (int)n;
  geo[1] = (int)chunk;
}

__global__ void k_cluster_init_dev(int* label, const int* geo) {
  const int n = geo[0];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    label[i] = i;
}

// Sweep `which` (0, 1) of pair `pair`: nothing to do once the previous
// pair's second sweep changed no label (the fixed point is reached).
__global__ void __launch_bounds__(CL_TILE) k_cluster_sweep_dev(ClusterArgs a, GiantBuffers gb,
                                                               const int* geo, unsigned* flags,
                                                               int pair, int which) {
  if (pair > 0 && *((volatile unsigned*)&flags[2 * pair - 1]) == 0u) return;
  const int n = geo[0];
  if ((long long)blockIdx.x * CL_TILE >= (long long)n) return;
  cluster_sweep_block(a, gb, n, &flags[2 * pair + which], geo[1]);
}

__global__ void k_cluster_jump_dev(int* label, const int* geo, unsigned* flags, int pair,
                                   int which) {
  if (pair > 0 && *((volatile unsigned*)&flags[2 * pair - 1]) == 0u) return;
  const int n = geo[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int l = label[i];
  const int ll = *((volatile int*)&label[l]);
  if (ll < l) {
    atomicMin(&label[i], ll);
    flags[2 * pair + which] = 1u;
  }
}

__global__ void k_root_flags_dev(const int* label, const int* geo, unsigned gcap,
                                 unsigned* flag) {
  const int n = geo[0];
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < gcap; i += gridDim.x * blockDim.x)
    flag[i] = ((int)i < n && label[i] == (int)i) ? 1u : 0u;
}

__global__ void k_merge_reduce_dev(GiantBuffers gb, const int* geo, const unsigned* root_off,
                                   unsigned long long* gkey, unsigned long long* members) {
  const int n = geo[0];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned g = root_off[gb.label[i]];
    const unsigned long long key = ((unsigned long long)float_key(gb.peak[i]) << 32) |
                                   (unsigned long long)(0xFFFFFFFFu - (unsigned)i);
    atomicMax(&gkey[g], key);
    atomicAdd(&members[g], 1ull);
  }
}

static unsigned grid_for(size_t n, unsigned threads) {
  return (unsigned)std::max<size_t>(1, std::min<size_t>((n + threads - 1) / threads, 148 * 32));
}

cudaError_t giants_dev(const WidthCtx& ctx, const HitBuffers& hb, const unsigned* nhits,
                       unsigned hcap, GiantBuffers& gb, unsigned gcap, unsigned* ngiants,
                       unsigned* scan_tmp, cudaStream_t s) {
  k_giant_heads_dev<<<grid_for(hcap, 256), 256, 0, s>>>(ctx, hb, nhits, hcap, gb.head);
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if ((e = scan_u32(gb.head, gb.gid, hcap, ngiants, scan_tmp, s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(gb.key, 0, (size_t)gcap * sizeof(unsigned long long), s)) !=
      cudaSuccess)
    return e;
  // one thread per hit slot: the warp reduction needs whole runs in a warp
  k_giant_reduce_dev<<<(unsigned)((hcap + 255) / 256), 256, 0, s>>>(ctx, hb, nhits, hcap, gb,
                                                                     gcap);
  note_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_giant_finish_dev<<<grid_for(gcap, 256), 256, 0, s>>>(hb, ngiants, gcap, gb, ctx.winfo,
                                                         ctx.nw);
  note_launch();
  return cudaGetLastError();
}

cudaError_t cluster_merge_dev(const ClusterArgs& a, GiantBuffers& gb, unsigned gcap,
                              const unsigned* ngiants, int units, int dm_key_gap,
                              unsigned* unit_off, int* geo, unsigned* flags, int pairs,
                              const float* dm_list, unsigned* root_flag, unsigned* root_off,
                              unsigned* nroots, unsigned* scan_tmp, unsigned long long* gkey,
                              GroupRow* rows, cudaStream_t s) {
  k_unit_offsets_dev<<<(units + 1 + 127) / 128, 128, 0, s>>>(gb.dm, ngiants, gcap, dm_key_gap,
                                                             units, unit_off);
  note_launch();
  k_cluster_geom<<<1, 32, 0, s>>>(unit_off, units, ngiants, gcap, geo);
  note_launch();
  k_cluster_init_dev<<<grid_for(gcap, 256), 256, 0, s>>>(gb.label, geo);
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(flags, 0, 2 * (size_t)pairs * sizeof(unsigned), s)) != cudaSuccess)
    return e;
  // the sweep grid of the host form at the capacity: tiles x CL_YBLOCKS
  // (chunks past a tile's window return at once)
  const dim3 sgrid((gcap + CL_TILE - 1) / CL_TILE, CL_YBLOCKS);
  for (int p = 0; p < pairs; p++)
    for (int w = 0; w < 2; w++) {
      k_cluster_sweep_dev<<<sgrid, CL_TILE, 0, s>>>(a, gb, geo, flags, p, w);
      note_launch();
      k_cluster_jump_dev<<<(gcap + 255) / 256, 256, 0, s>>>(gb.label, geo, flags, p, w);
      note_launch();
    }
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_root_flags_dev<<<grid_for(gcap, 256), 256, 0, s>>>(gb.label, geo, gcap, root_flag);
  note_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = scan_u32(root_flag, root_off, gcap, nroots, scan_tmp, s)) != cudaSuccess) return e;
  unsigned long long* members = gkey + gcap;
  if ((e = cudaMemsetAsync(gkey, 0, 2 * (size_t)gcap * sizeof(unsigned long long), s)) !=
      cudaSuccess)
    return e;
  k_merge_reduce_dev<<<grid_for(gcap, 256), 256, 0, s>>>(gb, geo, root_off, gkey, members);
  note_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_merge_emit<<<(gcap + 255) / 256, 256, 0, s>>>(gb, dm_key_gap, nroots, gkey, members,
                                                    dm_list, rows);
  note_launch();
  return cudaGetLastError();
}

// ===========================================================================
// RFI mask (clean_filterbank_rfi.cu:447-506)
//   mask[t] = |x[t]| > tol  OR, for some width w in 1,2,..,boxcar_max with
//   t in [off, count+1-boxcar_max+off): a flagged j in [t-behind, t+ahead),
//   where j in [off, count+1-boxcar_max+off) is flagged when
//   |boxcar_w(j-off) * (1/sqrt(w))| > tol  (off = boxcar_max/2).
// ===========================================================================
// Width norm 1/sqrt(w) of clean_filterbank_rfi.cu:476-477: sqrtf in float,
// the reciprocal in double, rounded to float (each step correctly rounded, as
// on the host).
__device__ __forceinline__ float rfi_width_norm(int w) {
  return __double2float_rn(__ddiv_rn(1.0, (double)__fsqrt_rn(__int2float_rn(w))));
}

__global__ void k_rfi_flags(const float* __restrict__ scan, size_t count, int bmax, int nwid,
                            float tol, unsigned char* __restrict__ flags) {
  size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  const int off = bmax / 2;
  const size_t nf = count + 1 - (size_t)bmax;
  unsigned char f = 0;
  if (j >= (size_t)off && j < (size_t)off + nf) {
    size_t k = j - off;
    for (int wi = 0; wi < nwid; wi++) {
      int w = 1 << wi;
      int ahead = (w - 1) / 2 + 1, behind = w / 2;
      float v = __fsub_rn(scan[off + ahead + k], scan[off - behind + k]);
      v = __fmul_rn(v, rfi_width_norm(w));
      if (fabsf(v) > tol) f |= (unsigned char)(1u << wi);
    }
  }
  flags[j] = f;
}

__global__ void k_rfi_mask(const float* __restrict__ x, size_t count, int bmax, int nwid,
                           float tol, const unsigned char* __restrict__ flags, int* __restrict__ mask) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const int off = bmax / 2;
  const size_t nf = count + 1 - (size_t)bmax;
  int m = fabsf(x[t]) > tol;
  if (!m && t >= (size_t)off && t < (size_t)off + nf) {
    for (int wi = 0; wi < nwid && !m; wi++) {
      int w = 1 << wi;
      int ahead = (w - 1) / 2 + 1, behind = w / 2;
      for (size_t j = t - behind; j < t + ahead; j++) {
        if (flags[j] & (1u << wi)) { m = 1; break; }
      }
    }
  }
  mask[t] = m;
}

cudaError_t rfi_mask(const float* x, const float* scan, size_t count, size_t boxcar_max,
                     float rfi_tol, int* mask, int* fmask, cudaStream_t s) {
  int nwid = 0;
  for (size_t w = 1; w <= boxcar_max && nwid < 8; w *= 2) nwid++;
  // one flag bit per width (boxcar_max <= 128 keeps them in a byte)
  if (boxcar_max > 128) return cudaErrorInvalidValue;
  unsigned char* flags = reinterpret_cast<unsigned char*>(fmask + 32);
  unsigned nb = (unsigned)((count + 255) / 256);
  k_rfi_flags<<<nb, 256, 0, s>>>(scan, count, (int)boxcar_max, nwid, rfi_tol, flags); note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_rfi_mask<<<nb, 256, 0, s>>>(x, count, (int)boxcar_max, nwid, rfi_tol, flags, mask); note_launch();
  return cudaGetLastError();
}

}  // namespace hdb
