// kernels_fb.cu -- filterbank-side kernels: layout change, zero-DM series,
// RFI zapping and brute-force dedispersion.
//
// Filterbank layouts:
//   TF  (input, as the reference receives it): spectrum t at in + t*nchans,
//       one byte per channel (8-bit data).
//   FT  (device working copy): channel c at ft + c*pitch, one byte per sample,
//       pitch a multiple of 64 bytes with zero padding past nsamps so the
//       dedispersion tiles can be fetched with 16-byte-aligned bulk copies.
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace hdb {

static unsigned long long g_launches = 0;
void note_launch() { __atomic_add_fetch(&g_launches, 1ull, __ATOMIC_RELAXED); }
unsigned long long launch_count() { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }
void add_launches(long long n) {
  __atomic_add_fetch(&g_launches, (unsigned long long)n, __ATOMIC_RELAXED);
}

cudaError_t raise_smem_limit(const void* func, size_t bytes) {
  static std::mutex m;
  static std::map<std::pair<int, const void*>, size_t> limit;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(m);
  size_t& cur = limit[{dev, func}];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

// ---------------------------------------------------------------------------
// TF -> FT byte transpose, 128 samples x 128 channels per block through
// shared memory.  The tile holds 128 sample rows of 32 channel words; word w
// of row t sits at column w ^ (((t >> 2) ^ (t & 3)) & 31), so the row-wise
// stores of the load phase (a warp stores four consecutive rows at once in
// the 16-byte form) and the sample-wise loads of the store phase (lane l
// reads rows 4l..4l+3 of one column) all hit 32 distinct banks.  A thread turns four
// samples x four channels into four output words with byte permutes.  Rows
// of whole 16-byte words are loaded 16 bytes at a time.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int tp_col(int t, int w) { return w ^ (((t >> 2) ^ (t & 3)) & 31); }

__global__ void __launch_bounds__(256) k_transpose_tf_ft(const uint8_t* __restrict__ in,
                                                         size_t nsamps, int nchans,
                                                         uint8_t* __restrict__ out,
                                                         size_t pitch, size_t out_unit) {
  __shared__ uint32_t tile[128 * 32];
  // blockIdx.z: unit (independent filterbank) of a batch
  in += (size_t)blockIdx.z * nsamps * (size_t)nchans;
  out += (size_t)blockIdx.z * out_unit;
  const size_t t0 = (size_t)blockIdx.x * 128;
  const int c0 = blockIdx.y * 128;
  const int nwords = nchans >> 2;
  const int w0 = c0 >> 2;
  if ((nchans & 15) == 0 && (reinterpret_cast<uintptr_t>(in) & 15) == 0) {
    // thread: 16-byte chunk q of rows r, r + 32, r + 64, r + 96
    const int q = threadIdx.x & 7, r0 = threadIdx.x >> 3;
    uint4 v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int r = r0 + 32 * k;
      const size_t t = t0 + r;
      v[k] = make_uint4(0u, 0u, 0u, 0u);
      if (t < nsamps && w0 + 4 * q < nwords)
        v[k] = *reinterpret_cast<const uint4*>(in + t * nchans + (size_t)(w0 + 4 * q) * 4);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int r = r0 + 32 * k;
      tile[r * 32 + tp_col(r, 4 * q)] = v[k].x;
      tile[r * 32 + tp_col(r, 4 * q + 1)] = v[k].y;
      tile[r * 32 + tp_col(r, 4 * q + 2)] = v[k].z;
      tile[r * 32 + tp_col(r, 4 * q + 3)] = v[k].w;
    }
  } else {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t v[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
      const size_t t = t0 + warp + 8 * k;
      v[k] = 0u;
      if (t < nsamps && w0 + lane < nwords)
        v[k] = reinterpret_cast<const uint32_t*>(in + t * nchans)[w0 + lane];
    }
#pragma unroll
    for (int k = 0; k < 16; k++) {
      const int r = warp + 8 * k;
      tile[r * 32 + tp_col(r, lane)] = v[k];
    }
  }
  __syncthreads();
  // warp: channel words wsel = warp, warp + 8, ...; lane: samples 4l .. 4l+3
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t t = t0 + 4 * lane;
  for (int ws = warp; ws < 32; ws += 8) {
    if (4 * ws + c0 >= nchans) break;
    uint32_t a[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int r = 4 * lane + j;
      a[j] = tile[r * 32 + tp_col(r, ws)];
    }
    // 4 x 4 byte transpose: o[b] = byte b of a[0..3]
    const uint32_t lo01 = __byte_perm(a[0], a[1], 0x5140), lo23 = __byte_perm(a[2], a[3], 0x5140);
    const uint32_t hi01 = __byte_perm(a[0], a[1], 0x7362), hi23 = __byte_perm(a[2], a[3], 0x7362);
    const uint32_t o[4] = {__byte_perm(lo01, lo23, 0x5410), __byte_perm(lo01, lo23, 0x7632),
                           __byte_perm(hi01, hi23, 0x5410), __byte_perm(hi01, hi23, 0x7632)};
    if (t < nsamps) {
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const int c = c0 + 4 * ws + b;
        if (c < nchans) reinterpret_cast<uint32_t*>(out + (size_t)c * pitch + t)[0] = o[b];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Packed TF -> byte FT rows for NB = 1, 2, 4 and 16 bits per sample.  A
// spectrum is C * NB / 32 little-endian 32-bit words; channel c is the NB-bit
// field at bit (c mod (32 / NB)) * NB of word c / (32 / NB) (the order of the
// reference's writer and cleaning functor: Formats/giant_maker.C:385-392,
// Pipeline/clean_filterbank_rfi.cu:86-90).  NB < 8 unpacks into one byte
// plane; NB = 16 splits each sample into its low byte (plane `out`) and high
// byte (plane `out + hi_off`), dedispersed separately and combined as
// lo + 256 hi (exact integer sums).  128 x 128 tiles through shared memory.
// ---------------------------------------------------------------------------
template <int NB>
__global__ void __launch_bounds__(256) k_unpack_tf_ft(const uint32_t* __restrict__ in,
                                                      size_t nsamps, int nchans,
                                                      uint8_t* __restrict__ out, size_t pitch,
                                                      size_t out_unit, size_t hi_off) {
  constexpr int CPW = 32 / NB;                 // channels per word
  constexpr int WPR = 128 / CPW;               // words per tile row
  constexpr uint32_t MASK = (NB == 32) ? 0xFFFFFFFFu : ((1u << NB) - 1u);
  __shared__ uint16_t vals[128][130];          // [t][channel]
  const size_t row_words = (size_t)nchans * NB / 32;
  in += (size_t)blockIdx.z * nsamps * row_words;
  out += (size_t)blockIdx.z * out_unit;
  const size_t t0 = (size_t)blockIdx.x * 128;
  const int c0 = blockIdx.y * 128;
  const size_t w0 = (size_t)c0 / CPW;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int r = warp; r < 128; r += 8) {
    const size_t t = t0 + r;
    for (int w = lane; w < WPR; w += 32) {
      uint32_t v = 0;
      if (t < nsamps && w0 + w < row_words) v = in[t * row_words + w0 + w];
#pragma unroll
      for (int k = 0; k < CPW; k++) vals[r][w * CPW + k] = (uint16_t)((v >> (k * NB)) & MASK);
    }
  }
  __syncthreads();
  for (int cr = warp; cr < 128; cr += 8) {
    const int c = c0 + cr;
    if (c >= nchans) break;
    const size_t t = t0 + 4 * lane;
    if (t >= nsamps) continue;
    uint32_t lo = 0, hi = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const uint32_t v = vals[4 * lane + j][cr];
      lo |= (v & 0xFFu) << (8 * j);
      hi |= (v >> 8) << (8 * j);
    }
    reinterpret_cast<uint32_t*>(out + (size_t)c * pitch + t)[0] = lo;
    if (NB == 16) reinterpret_cast<uint32_t*>(out + hi_off + (size_t)c * pitch + t)[0] = hi;
  }
}

// rows x n floats (pitch apart): lo = RN(lo + 256 hi), both exact integer sums
__global__ void k_combine_planes(float* __restrict__ lo, const float* __restrict__ hi,
                                 size_t pitch, size_t n, size_t rows) {
  const size_t total = rows * n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / n, k = i - r * n;
    const size_t at = r * pitch + k;
    lo[at] = __uint2float_rn(__float2uint_rn(lo[at]) + 256u * __float2uint_rn(hi[at]));
  }
}

// ---------------------------------------------------------------------------
// Zero-DM series: s[t] = (float) sum_c in[t][c]  (dedisp at DM 0, all channels;
// Pipeline/clean_filterbank_rfi.cu:361-397).  One warp per spectrum.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_dm0_sum(const uint8_t* __restrict__ in, size_t nsamps,
                                                 int nchans, float* __restrict__ s) {
  size_t t = (size_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (t >= nsamps) return;
  const uint32_t* row = reinterpret_cast<const uint32_t*>(in + t * nchans);
  unsigned acc = 0;
  for (int w = lane; w < (nchans >> 2); w += 32) acc = __dp4a(row[w], 0x01010101u, acc);
#pragma unroll
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) s[t] = (float)(int)acc;
}

// ---------------------------------------------------------------------------
// Broadband zapping (Pipeline/clean_filterbank_rfi.cu:33-113,197-234).
// ---------------------------------------------------------------------------
// Robert Jenkins' 32-bit integer mix.
__device__ __forceinline__ uint32_t mix32(uint32_t a) {
  a = (a + 0x7ed55d16u) + (a << 12);
  a = (a ^ 0xc761c23cu) ^ (a >> 19);
  a = (a + 0x165667b1u) + (a << 5);
  a = (a + 0xd3a2646cu) ^ (a << 9);
  a = (a + 0xfd7046c5u) + (a << 3);
  a = (a ^ 0xb55a4f09u) ^ (a >> 16);
  return a;
}

// Park-Miller minimal standard (a = 48271, m = 2^31 - 1) and Thrust's integer
// distribution: a double in [lo, hi + 1) from (x - 1) / (2^31 - 2), truncated.
__device__ __forceinline__ uint32_t minstd_next(uint32_t& s) {
  s = (uint32_t)((48271ull * (unsigned long long)s) % 2147483647ull);
  return s;
}
__device__ __forceinline__ uint32_t uniform_uint(uint32_t& s, uint32_t lo, uint32_t hi) {
  double a = (double)lo;
  double b = __dadd_rn((double)hi, 1.0);
  double u = (double)(minstd_next(s) - 1u);
  u = __ddiv_rn(u, 2147483646.0);
  double r = __dadd_rn(__dmul_rn(u, __dsub_rn(b, a)), a);
  return __double2uint_rz(r);
}

__device__ uint32_t zap_word(const uint32_t* __restrict__ win, const int* __restrict__ mask,
                             unsigned i, unsigned t, unsigned c, unsigned stride, unsigned ns,
                             unsigned r) {
  uint32_t s = mix32(i) % 2147483647u;
  if (s == 0) s = 1;
  uint32_t result = 0;
#pragma unroll 1
  for (unsigned k = 0; k < 32; k += 8) {
    unsigned min_t = t > r ? t - r : 0;
    unsigned max_t = t < ns - 1 - r ? t + r : ns - 1;
    unsigned nt = uniform_uint(s, min_t, max_t);
    int attempts = 0;
    while (mask[nt] && ++attempts < 11) nt = uniform_uint(s, min_t, max_t);
    uint32_t v = (win[nt * stride + c] >> k) & 0xFFu;
    result |= v << k;
  }
  return result;
}

// Zap masked spectra and write the result channel-major (FT), and optionally
// time-major (TF) for callers that want the cleaned filterbank back.
__global__ void __launch_bounds__(256) k_zap_to_ft(const uint8_t* __restrict__ in, size_t nsamps,
                                                   int nchans, const int* __restrict__ mask,
                                                   unsigned max_resample_dist,
                                                   uint8_t* __restrict__ out_ft, size_t pitch,
                                                   uint8_t* __restrict__ out_tf) {
  __shared__ uint32_t tile[128][33];
  const size_t t0 = (size_t)blockIdx.x * 128;
  const int c0 = blockIdx.y * 128;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned stride = (unsigned)(nchans >> 2);
  const uint32_t* win = reinterpret_cast<const uint32_t*>(in);
  for (int r = warp; r < 128; r += 8) {
    size_t t = t0 + r;
    unsigned w = (unsigned)(c0 >> 2) + lane;
    uint32_t v = 0;
    if (t < nsamps && w < stride) {
      if (mask[t]) {
        unsigned i = (unsigned)t * stride + w;
        v = zap_word(win, mask, i, (unsigned)t, w, stride, (unsigned)nsamps, max_resample_dist);
      } else {
        v = win[t * stride + w];
      }
      if (out_tf) reinterpret_cast<uint32_t*>(out_tf)[t * stride + w] = v;
    }
    tile[r][lane] = v;
  }
  if (!out_ft) return;
  __syncthreads();
  for (int cr = warp; cr < 128; cr += 8) {
    int c = c0 + cr;
    if (c >= nchans) break;
    int wsel = cr >> 2, bsel = cr & 3;
    uint32_t o = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      uint32_t v = tile[4 * lane + j][wsel];
      o |= ((v >> (8 * bsel)) & 0xFFu) << (8 * j);
    }
    size_t t = t0 + 4 * lane;
    if (t < nsamps) reinterpret_cast<uint32_t*>(out_ft + (size_t)c * pitch + t)[0] = o;
  }
}

// ---------------------------------------------------------------------------
// Narrow-band RFI: the branch of Pipeline/clean_filterbank_rfi.cu:303-351 that
// the reference disables (measure_bandpass.cu:45-275 and
// zap_narrow_rfi_functor, clean_filterbank_rfi.cu:114-193).  The data are cut
// into stretches of baseline_length / dt spectra per filterbank (unit); each
// stretch gets its own bandpass and band deviation from 3125 spectra drawn
// with thrust::default_random_engine(123456), and its bytes are zapped
// against them.
// ---------------------------------------------------------------------------
constexpr int NB_SPECTRA = 3125;

// spectrum draws of each stretch, in order (measure_bandpass.cu:95-108)
__global__ void k_nb_indices(const unsigned* __restrict__ len, int nstretch,
                             unsigned* __restrict__ idx) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nstretch) return;
  uint32_t st = 123456u;
  for (int i = 0; i < NB_SPECTRA; i++)
    idx[(size_t)g * NB_SPECTRA + i] = uniform_uint(st, 0u, len[g] - 1u);
}

// spectra[g][i][c] = (float) fb[(start[g] + idx[g][i]) * C + c]
__global__ void k_nb_gather(const uint8_t* __restrict__ fb, int C,
                            const unsigned long long* __restrict__ start,
                            const unsigned* __restrict__ idx, size_t total,
                            float* __restrict__ out) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t gi = e / C;
    const int c = (int)(e % C);
    const size_t g = gi / NB_SPECTRA;
    out[e] = (float)fb[(size_t)(start[g] + idx[gi]) * C + c];
  }
}

// one level of the recursive median: out[g][a][c] = median of in[g][5a..5a+4][c]
__global__ void k_nb_scrunch5(const float* __restrict__ in, int C, int count_in, int nstretch,
                              float* __restrict__ out) {
  const int count_out = count_in / 5;
  const size_t total = (size_t)nstretch * count_out * C;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % C);
    const size_t r = e / C;
    const size_t a = r % count_out, g = r / count_out;
    const float* b = in + ((size_t)g * count_in + 5 * a) * C + c;
    out[e] = med5(b[0], b[C], b[2 * (size_t)C], b[3 * (size_t)C], b[4 * (size_t)C]);
  }
}

// median_filter5_kernel (median_filter.cu:99-124): window shrunk at the ends
__device__ __forceinline__ float nb_filter5(const float* in, unsigned count, unsigned i) {
  if (i > 1 && i < count - 2) return med5(in[i - 2], in[i - 1], in[i], in[i + 1], in[i + 2]);
  if (i == 0) return med3(in[i], in[i + 1], in[i + 2]);
  if (i == 1) return med4(in[i - 1], in[i], in[i + 1], in[i + 2]);
  if (i == count - 1) return med3(in[i], in[i - 1], in[i - 2]);
  return med4(in[i + 1], in[i], in[i - 1], in[i - 2]);
}

// measure_bandpass.cu:141-163 / 220-245 on v[g] (C values, scaled first by
// `scale` unless it is 1): scrunch by 5, 5-wide median, mean of neighbours
// (thrust::adjacent_difference), stretch to C/5*5 and extrapolate the rest.
// One block per stretch; tmp[g] holds C/5 values.
__global__ void k_nb_smooth(float* __restrict__ v, float* __restrict__ tmp, int C, float scale) {
  float* x = v + (size_t)blockIdx.x * C;
  const unsigned n5 = (unsigned)C / 5;
  float* t = tmp + (size_t)blockIdx.x * (n5 + 1);
  if (scale != 1.f) {
    for (int i = threadIdx.x; i < C; i += blockDim.x) x[i] = __fmul_rn(x[i], scale);
    __syncthreads();
  }
  for (unsigned j = threadIdx.x; j < n5; j += blockDim.x)
    t[j] = med5(x[5 * j], x[5 * j + 1], x[5 * j + 2], x[5 * j + 3], x[5 * j + 4]);
  __syncthreads();
  for (unsigned j = threadIdx.x; j < n5; j += blockDim.x) x[j] = nb_filter5(t, n5, j);
  __syncthreads();
  for (unsigned j = threadIdx.x; j < n5; j += blockDim.x)
    t[j] = j == 0 ? x[0] : __fmul_rn(0.5f, __fadd_rn(x[j], x[j - 1]));
  // for some channel counts (1140, 2220, ...) the last stretched sample lands
  // just past the last input with a fraction above 1e-5 and reads t[n5] (the
  // reference reads past its vector there): defined as 0
  if (threadIdx.x == 0) t[n5] = 0.f;
  __syncthreads();
  const float step = __fdiv_rn((float)(n5 - 1), (float)(n5 * 5 - 1));
  for (unsigned j = threadIdx.x; j < n5 * 5; j += blockDim.x) x[j] = stretch_at(t, j, step);
  __syncthreads();
  if (threadIdx.x == 0)
    for (unsigned i = n5 * 5; i < (unsigned)C; i++)
      x[i] = __fsub_rn(__fmul_rn(2.f, x[i - 1]), x[i - 2]);
}

// spectra[g][i][c] = |spectra[g][i][c] - bandpass[g][c]|
__global__ void k_nb_absdev(float* __restrict__ sp, const float* __restrict__ bp, int C,
                            size_t total) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t g = e / ((size_t)NB_SPECTRA * C);
    sp[e] = fabsf(__fsub_rn(sp[e], bp[g * C + e % C]));
  }
}

// rms[g] = the (C/2)-th smallest of mad[g] (std::nth_element), by ranks
__global__ void k_nb_rms(const float* __restrict__ mad, int C, float* __restrict__ rms) {
  const float* m = mad + (size_t)blockIdx.x * C;
  const int k = C / 2;
  for (int i = threadIdx.x; i < C; i += blockDim.x) {
    const float x = m[i];
    int lt = 0, le = 0;
    for (int j = 0; j < C; j++) {
      lt += m[j] < x;
      le += m[j] <= x;
    }
    if (lt <= k && k < le) rms[blockIdx.x] = x;  // equal values only
  }
}

// zap_narrow_rfi_functor over each spectrum's words in order (one thread per
// spectrum; draws read the spectrum as earlier words left it, the sequential
// semantics of the functor's in-place reads).  Bandpass entry and draw range
// use channel w + k as the reference does; the hash takes the word's index
// within its filterbank.
__global__ void k_nb_zap(uint32_t* __restrict__ data, size_t nsamps, int units, int C,
                         size_t nsmooth, int nsub, const float* __restrict__ bp,
                         const float* __restrict__ rms, float rfi_tol, unsigned max_dist) {
  const size_t tg = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tg >= nsamps * (size_t)units) return;
  const size_t u = tg / nsamps, tl = tg % nsamps;
  const size_t g = u * nsub + tl / nsmooth;
  const float* b = bp + g * C;
  const float thresh = __fmul_rn(rfi_tol, rms[g]);
  const unsigned stride = (unsigned)C / 4, nch = (unsigned)C;
  uint32_t* row = data + tg * stride;
  for (unsigned w = 0; w < stride; w++) {
    const unsigned i = (unsigned)(tl * stride + w);
    uint32_t word = row[w];
    uint32_t st = mix32(i) % 2147483647u;
    if (st == 0) st = 1;
    bool any = false;
    for (unsigned k = 0; k < 4; k++) {
      const unsigned c = w + k;
      const uint32_t val = (word >> (k * 8)) & 0xFFu;
      if (fabsf(__fsub_rn(__uint2float_rn(val), b[c])) > thresh) {
        any = true;
        const unsigned min_c = c > max_dist ? c - max_dist : 0;
        const unsigned max_c = c < nch - 1 - max_dist ? c + max_dist : nch - 1;
        unsigned nc = uniform_uint(st, min_c, max_c);
        uint32_t nv = (row[nc / 4] >> ((nc % 4) * 8)) & 0xFFu;
        int attempts = 0;
        while (fabsf(__fsub_rn(__uint2float_rn(nv), b[nc])) > thresh && ++attempts < 11) {
          nc = uniform_uint(st, min_c, max_c);
          nv = (row[nc / 4] >> ((nc % 4) * 8)) & 0xFFu;
        }
        word &= ~(0xFFu << (k * 8));
        word |= nv << (k * 8);
      }
    }
    if (any) row[w] = word;
  }
}

// ---------------------------------------------------------------------------
// Brute-force dedispersion.
//
//   out[d][t] = (float) sum_{c active} in[c][t + delay[d][c]],  t < nout
//
// CTA = DB = 2*NW DMs x TB = 128*K*G samples, NW consumer warps + 1 producer
// warp.  The producer walks the active channels in stages of CH: for each
// stage it tabulates the byte offset of every (DM, channel) pair in shared
// memory and issues one 1-D bulk async copy (TMA, cp.async.bulk) per channel
// row segment [t0 + min_d delay - align, +rowb) into a ring of NST stage
// buffers, signalling a `full` mbarrier; consumer warps release a buffer
// through an `empty` mbarrier (one arrival per warp).  There is no block-wide
// barrier in the main loop, so warps drift freely within the ring.
//
// Warp w owns DMs 2w and 2w+1.  In each of G groups of 32*K words, lane l
// owns the K consecutive output words (4K samples) starting at word K*l.  A
// (DM, channel) term reads the K+1 row words that cover the lane's window
// shifted by the delay, and realigns each output word with a funnel shift.
// Because K is odd, the 32 lanes' j-th loads (word K*l + j) fall in 32
// distinct banks: every shared load is one wavefront, and a term costs
// 4 (K+1) / (4 K) bytes of shared-memory bandwidth per sample (2 at K = 1,
// 1.33 at K = 3, 1.2 at K = 5).  Each realigned word is split into two
// 16-bit lane pairs (even/odd samples); two channels are summed per 3-input
// add, so one add accumulates four sample-channel terms.  The 16-bit lanes
// are drained into 32-bit sums after at most 257 channels (255 * 257 =
// 65535), so the sums are exact.  Every mbarrier wait is bounded; a wait that
// gives up sets bit 0 of a.err and the warp leaves its loop.
//
// Pipe balance: the shifts, byte permutes and 3-input adds all issue to the
// ALU pipe, which bounds the kernel, while the FMA pipe idles.  The odd-byte
// sums are therefore accumulated with integer multiply-adds by a.one (= 1,
// unknown to the compiler), which issue to the FMA pipe; and the producer
// tabulates, per (DM, channel), the shared-memory word index of the row
// segment and the realignment shift, so the consumers spend no ALU work on
// addressing.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t mad_u32(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

// CTAs per SM the register budget allows: per lane about 12 registers per
// owned output word (two DMs x {2 packed, 4 drained} sums; 8 with the
// compact drain) plus ~48 others.
constexpr int dd_regs(int k, int g, bool a16) { return (a16 ? 8 : 12) * k * g + 48; }
constexpr int dd_min_blocks(int nw, int k, int g, bool a16) {
  return (65536 / ((nw + 1) * 32 * dd_regs(k, g, a16))) < 1
             ? 1
             : (65536 / ((nw + 1) * 32 * dd_regs(k, g, a16))) > 3
                   ? 3
                   : (65536 / ((nw + 1) * 32 * dd_regs(k, g, a16)));
}

// A16 (at most 511 active channels): the sums drained after the first 256 or
// 257 channels stay packed as two 16-bit lane pairs (each <= 257 * 255 =
// 65535), and the remaining < 257 channels are added to them in 32 bits when
// the output is written; 8 rather than 12 registers per output word, so
// more CTAs fit an SM.
template <int NW, int K, int G, int CH, int NST, bool A16>
__global__ void __launch_bounds__((NW + 1) * 32, dd_min_blocks(NW, K, G, A16))
    k_dedisp(DedispArgs a) {
  static_assert(K % 2 == 1, "odd K keeps the strided shared loads conflict-free");
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr int DB = 2 * NW;
  constexpr int TB = 128 * K * G;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + NST;
  // [NST][DB*CH] {word index of the (DM, channel) row segment in `rows`,
  // realignment shift in bits}
  int2* s_off = reinterpret_cast<int2*>(smem + 128);
  uint8_t* rows = smem + 128 + NST * DB * CH * sizeof(int2);  // [NST][CH][rowb]
  const int dblk = blockIdx.x;
  const size_t t0 = (size_t)blockIdx.y * TB;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int d_lo = dblk * DB;
  const int* __restrict__ bmin = a.blk_min + (size_t)dblk * a.nchans;
  const int nstage = (a.nact + CH - 1) / CH;
  const size_t C = (size_t)a.nchans;

  if (threadIdx.x == 0) {
    for (int b = 0; b < NST; b++) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], NW);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == NW) {
    // ---------------- producer ----------------
    // blockIdx.z selects the unit (an independent filterbank of the batch)
    const uint8_t* __restrict__ in = a.in + (size_t)blockIdx.z * a.in_unit;
    int issued = 0;
    for (int st = 0; st < nstage; st++) {
      const int buf = st % NST;
      if (st >= NST) {
        if (!mbar_wait(&empty[buf], (uint32_t)(((st / NST) - 1) & 1), a.wait_limit)) {
          if (lane == 0) atomicOr(a.err, 1u);
          break;
        }
      }
      // error-path test: the last stage is never copied (nor announced), so
      // its `full` phase never completes and the consumers' wait gives up
      if (a.withhold_last && st == nstage - 1) break;
      const int k0 = st * CH;
      const int nk = min(CH, a.nact - k0);
      int2* off = s_off + buf * DB * CH;
      for (int e = lane; e < DB * CH; e += 32) {
        const int k = e % CH;
        if (k < nk) {
          const int c = a.chans[k0 + k];
          const int d = min(d_lo + e / CH, a.dm_count - 1);
          const size_t lo = (t0 + (size_t)bmin[c]) & ~(size_t)15;
          const int o = (int)(t0 + (size_t)a.delays[(size_t)d * C + c] - lo);
          off[e] = make_int2(((buf * CH + k) * a.rowb + o) >> 2, (o & 3) * 8);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_expect_tx(&full[buf], (uint32_t)(nk * a.rowb));
      __syncwarp();
      if (lane < nk) {
        const int c = a.chans[k0 + lane];
        const size_t lo = (t0 + (size_t)bmin[c]) & ~(size_t)15;
        bulk_g2s(rows + (size_t)(buf * CH + lane) * a.rowb, in + (size_t)c * a.in_pitch + lo,
                 (uint32_t)a.rowb, &full[buf]);
      }
      issued = st + 1;
    }
    // let every copy this CTA issued land before the warp exits
    for (int st = (issued > NST ? issued - NST : 0); st < issued; st++)
      mbar_wait(&full[st % NST], (uint32_t)((st / NST) & 1), a.wait_limit);
    return;
  }

  // ---------------- consumers ----------------
  // pk[..][0] sums the raw words (bytes b0..b3 of 4 samples) modulo 2^32 and
  // pk[..][1] the odd bytes (b1, b3) in two 16-bit lanes.  With at most 257
  // channels between drains every byte-lane sum is <= 65535, so
  // raw - (odd << 8) = E0 + 2^16 E2 exactly: the even-byte sums.
  constexpr int W = K * G;  // output words per lane and DM
  constexpr int NA = A16 ? 2 : 4;
  uint32_t pk[2][W][2];
  // drained sums: samples 0..3 in 32 bits, or (A16) {even, odd} lane pairs
  uint32_t acc[2][W][NA];
#pragma unroll
  for (int d = 0; d < 2; d++)
#pragma unroll
    for (int w = 0; w < W; w++) {
      pk[d][w][0] = pk[d][w][1] = 0;
#pragma unroll
      for (int q = 0; q < NA; q++) acc[d][w][q] = 0;
    }
  auto drain = [&]() {
#pragma unroll
    for (int d = 0; d < 2; d++)
#pragma unroll
      for (int w = 0; w < W; w++) {
        const uint32_t odd = pk[d][w][1];
        const uint32_t even = pk[d][w][0] - (odd << 8);
        if constexpr (A16) {
          // only drain before the last: the accumulators are still zero
          acc[d][w][0] = even;
          acc[d][w][1] = odd;
        } else {
          acc[d][w][0] += even & 0xFFFFu;
          acc[d][w][2] += even >> 16;
          acc[d][w][1] += odd & 0xFFFFu;
          acc[d][w][3] += odd >> 16;
        }
        pk[d][w][0] = pk[d][w][1] = 0;
      }
  };
  // first word of this lane in group 0; group g adds 32*K*g words
  const int lw = K * lane;

  int nsum = 0;
  bool failed = false;
  for (int st = 0; st < nstage; st++) {
    const int buf = st % NST;
    if (!mbar_wait(&full[buf], (uint32_t)((st / NST) & 1), a.wait_limit)) {
      if (lane == 0) atomicOr(a.err, 1u);
      failed = true;
      break;
    }
    const int k0 = st * CH;
    const int nk = min(CH, a.nact - k0);
    const int2* off = s_off + buf * DB * CH + (2 * warp) * CH;
    const uint32_t* rows32 = reinterpret_cast<const uint32_t*>(rows);
    const uint32_t one = a.one;
    int k = 0;
    for (; k + 1 < nk; k += 2) {
#pragma unroll
      for (int d = 0; d < 2; d++) {
        const int2 oa = off[d * CH + k];
        const int2 ob = off[d * CH + k + 1];
        const uint32_t* pa = rows32 + (oa.x + lw);
        const uint32_t* pb = rows32 + (ob.x + lw);
#pragma unroll
        for (int g = 0; g < G; g++) {
          uint32_t wa[K + 1], wb[K + 1];
#pragma unroll
          for (int j = 0; j <= K; j++) {
            wa[j] = pa[32 * K * g + j];
            wb[j] = pb[32 * K * g + j];
          }
#pragma unroll
          for (int j = 0; j < K; j++) {
            const uint32_t xa = __funnelshift_r(wa[j], wa[j + 1], oa.y);
            const uint32_t xb = __funnelshift_r(wb[j], wb[j + 1], ob.y);
            pk[d][K * g + j][0] += xa + xb;
            pk[d][K * g + j][1] = mad_u32(__byte_perm(xb, 0u, 0x4341), one,
                                          mad_u32(__byte_perm(xa, 0u, 0x4341), one,
                                                  pk[d][K * g + j][1]));
          }
        }
      }
      nsum += 2;
      if (nsum >= 256) { drain(); nsum = 0; }
    }
    if (k < nk) {
#pragma unroll
      for (int d = 0; d < 2; d++) {
        const int2 oa = off[d * CH + k];
        const uint32_t* pa = rows32 + (oa.x + lw);
#pragma unroll
        for (int g = 0; g < G; g++) {
          uint32_t wa[K + 1];
#pragma unroll
          for (int j = 0; j <= K; j++) wa[j] = pa[32 * K * g + j];
#pragma unroll
          for (int j = 0; j < K; j++) {
            const uint32_t xa = __funnelshift_r(wa[j], wa[j + 1], oa.y);
            pk[d][K * g + j][0] += xa;
            pk[d][K * g + j][1] = mad_u32(__byte_perm(xa, 0u, 0x4341), one, pk[d][K * g + j][1]);
          }
        }
      }
      nsum += 1;
      if (nsum >= 256) { drain(); nsum = 0; }
    }
    __syncwarp();
    if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];"
                                :: "r"(smem_addr(&empty[buf])) : "memory");
  }
  if (failed) return;
  if constexpr (!A16) drain();
  float* __restrict__ out = a.out + (size_t)blockIdx.z * a.out_unit;
#pragma unroll
  for (int d = 0; d < 2; d++) {
    int dd = d_lo + 2 * warp + d;
    if (dd >= a.dm_count) continue;
    float* o = out + (size_t)dd * a.out_pitch;
#pragma unroll
    for (int g = 0; g < G; g++)
#pragma unroll
      for (int j = 0; j < K; j++) {
        const int w = K * g + j;
        size_t t = t0 + 4 * (32 * K * g + lw + j);
        uint32_t s0, s1, s2, s3;
        if constexpr (A16) {
          const uint32_t odd = pk[d][w][1];
          const uint32_t even = pk[d][w][0] - (odd << 8);
          s0 = (even & 0xFFFFu) + (acc[d][w][0] & 0xFFFFu);
          s2 = (even >> 16) + (acc[d][w][0] >> 16);
          s1 = (odd & 0xFFFFu) + (acc[d][w][1] & 0xFFFFu);
          s3 = (odd >> 16) + (acc[d][w][1] >> 16);
        } else {
          s0 = acc[d][w][0];
          s1 = acc[d][w][1];
          s2 = acc[d][w][2];
          s3 = acc[d][w][3];
        }
        float4 v = make_float4((float)s0, (float)s1, (float)s2, (float)s3);
        if (t + 3 < a.nout) {
          *reinterpret_cast<float4*>(o + t) = v;
        } else {
          if (t < a.nout) o[t] = v.x;
          if (t + 1 < a.nout) o[t + 1] = v.y;
          if (t + 2 < a.nout) o[t + 2] = v.z;
        }
      }
  }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
cudaError_t launch_transpose_tf_ft(const uint8_t* in, size_t nsamps, int nchans, uint8_t* out,
                                   size_t pitch, cudaStream_t s, size_t units, size_t out_unit) {
  if (units < 1 || units > 65535) return cudaErrorInvalidValue;
  dim3 grid((unsigned)((nsamps + 127) / 128), (unsigned)((nchans + 127) / 128), (unsigned)units);
  k_transpose_tf_ft<<<grid, 256, 0, s>>>(in, nsamps, nchans, out, pitch, out_unit); note_launch();
  return cudaGetLastError();
}

cudaError_t launch_unpack_tf_ft(const uint8_t* in, size_t nsamps, int nchans, int nbits,
                                uint8_t* out, size_t pitch, cudaStream_t s, size_t units,
                                size_t out_unit, size_t hi_off) {
  if (units < 1 || units > 65535 || nchans < 1 || ((size_t)nchans * nbits) % 32 ||
      (reinterpret_cast<uintptr_t>(in) & 3) || pitch % 4)
    return cudaErrorInvalidValue;
  dim3 grid((unsigned)((nsamps + 127) / 128), (unsigned)((nchans + 127) / 128), (unsigned)units);
  const uint32_t* w = reinterpret_cast<const uint32_t*>(in);
  switch (nbits) {
    case 1: k_unpack_tf_ft<1><<<grid, 256, 0, s>>>(w, nsamps, nchans, out, pitch, out_unit, 0); break;
    case 2: k_unpack_tf_ft<2><<<grid, 256, 0, s>>>(w, nsamps, nchans, out, pitch, out_unit, 0); break;
    case 4: k_unpack_tf_ft<4><<<grid, 256, 0, s>>>(w, nsamps, nchans, out, pitch, out_unit, 0); break;
    case 16:
      k_unpack_tf_ft<16><<<grid, 256, 0, s>>>(w, nsamps, nchans, out, pitch, out_unit, hi_off);
      break;
    default: return cudaErrorInvalidValue;
  }
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_combine_planes(float* lo, const float* hi, size_t pitch, size_t n, size_t rows,
                                  cudaStream_t s) {
  if (rows == 0 || n == 0) return cudaSuccess;
  const size_t total = rows * n;
  const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16);
  k_combine_planes<<<blocks, 256, 0, s>>>(lo, hi, pitch, n, rows);
  note_launch();
  return cudaGetLastError();
}

// Scrunched input of adaptive dt: the byte mean of s consecutive samples
// (rounded half up) of each channel row, zero past nsamps / s.
__global__ void __launch_bounds__(256) k_scrunch_ft(const uint8_t* __restrict__ in,
                                                    size_t in_pitch, size_t ns, int s,
                                                    uint8_t* __restrict__ out, size_t out_pitch,
                                                    size_t in_unit, size_t out_unit) {
  const size_t u = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= out_pitch) return;
  const size_t c = blockIdx.y;
  in += (size_t)blockIdx.z * in_unit + c * in_pitch;
  out += (size_t)blockIdx.z * out_unit + c * out_pitch;
  unsigned v = 0;
  if (u < ns) {
    unsigned sum = 0;
    for (int j = 0; j < s; j++) sum += in[(size_t)s * u + j];
    v = (sum + (unsigned)(s / 2)) / (unsigned)s;
  }
  out[u] = (uint8_t)v;
}

cudaError_t launch_scrunch_ft(const uint8_t* in, size_t in_pitch, size_t nsamps, int nchans,
                              int s, uint8_t* out, size_t out_pitch, size_t units,
                              size_t in_unit, size_t out_unit, cudaStream_t st) {
  if (s < 1 || units < 1 || units > 65535 || nchans < 1 || nchans > 65535)
    return cudaErrorInvalidValue;
  dim3 grid((unsigned)((out_pitch + 255) / 256), (unsigned)nchans, (unsigned)units);
  k_scrunch_ft<<<grid, 256, 0, st>>>(in, in_pitch, nsamps / (size_t)s, s, out, out_pitch,
                                      in_unit, out_unit);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_dm0_sum(const uint8_t* in, size_t nsamps, int nchans, float* out,
                           cudaStream_t s) {
  k_dm0_sum<<<(unsigned)((nsamps + 7) / 8), 256, 0, s>>>(in, nsamps, nchans, out); note_launch();
  return cudaGetLastError();
}

cudaError_t launch_zap(const uint8_t* in, size_t nsamps, int nchans, const int* mask,
                       unsigned max_resample_dist, uint8_t* out_ft, size_t pitch,
                       uint8_t* out_tf, cudaStream_t s) {
  dim3 grid((unsigned)((nsamps + 127) / 128), (unsigned)((nchans + 127) / 128));
  k_zap_to_ft<<<grid, 256, 0, s>>>(in, nsamps, nchans, mask, max_resample_dist, out_ft, pitch,
                                   out_tf); note_launch();
  return cudaGetLastError();
}

// Scratch layout of the narrow-band stage (bytes, 256-aligned pieces).
struct NbLayout {
  size_t idx, start, len, s1, s2, s3, s4, s5, bp, mad, tmp, rms, total;
};
static NbLayout nb_layout(size_t nstretch, int C) {
  NbLayout L{};
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = o;
    o += (bytes + 255) / 256 * 256;
    return at;
  };
  const size_t n = nstretch;
  L.idx = take(n * NB_SPECTRA * sizeof(unsigned));
  L.start = take(n * sizeof(unsigned long long));
  L.len = take(n * sizeof(unsigned));
  L.s1 = take(n * NB_SPECTRA * C * sizeof(float));
  L.s2 = take(n * (NB_SPECTRA / 5) * C * sizeof(float));
  L.s3 = take(n * (NB_SPECTRA / 25) * C * sizeof(float));
  L.s4 = take(n * (NB_SPECTRA / 125) * C * sizeof(float));
  L.s5 = take(n * (NB_SPECTRA / 625) * C * sizeof(float));
  L.bp = take(n * C * sizeof(float));
  L.mad = take(n * C * sizeof(float));
  L.tmp = take(n * (C / 5 + 1) * sizeof(float));
  L.rms = take(n * sizeof(float));
  L.total = o;
  return L;
}

size_t narrow_band_stretches(size_t nsamps, float dt, float baseline_length) {
  const size_t nsmooth = (size_t)(baseline_length / (1 * dt));
  return nsmooth ? (nsamps + nsmooth - 1) / nsmooth : 0;
}

size_t narrow_band_scratch_bytes(size_t units, size_t nsamps, int nchans, float dt,
                                 float baseline_length) {
  return nb_layout(units * narrow_band_stretches(nsamps, dt, baseline_length), nchans).total;
}

cudaError_t narrow_band(uint8_t* tf, size_t units, size_t nsamps, int nchans, float dt,
                        float baseline_length, float rfi_tol, void* scratch, cudaStream_t s) {
  const size_t nsmooth = (size_t)(baseline_length / (1 * dt));
  const int C = nchans;
  if (nsmooth == 0 || C % 4 != 0 || C < 20 || units == 0) return cudaErrorInvalidValue;
  if (nsamps * (size_t)(C / 4) >= 0xFFFFFFFFull) return cudaErrorInvalidValue;
  const size_t nsub = (nsamps + nsmooth - 1) / nsmooth;
  const size_t ns = units * nsub;
  const NbLayout L = nb_layout(ns, C);
  uint8_t* base = static_cast<uint8_t*>(scratch);
  auto F = [&](size_t off) { return reinterpret_cast<float*>(base + off); };
  unsigned* idx = reinterpret_cast<unsigned*>(base + L.idx);
  unsigned long long* start = reinterpret_cast<unsigned long long*>(base + L.start);
  unsigned* len = reinterpret_cast<unsigned*>(base + L.len);
  std::vector<unsigned long long> h_start(ns);
  std::vector<unsigned> h_len(ns);
  for (size_t u = 0; u < units; u++)
    for (size_t g = 0; g < nsub; g++) {
      h_start[u * nsub + g] = u * nsamps + g * nsmooth;
      h_len[u * nsub + g] = (unsigned)std::min(nsmooth, nsamps - g * nsmooth);
    }
  cudaError_t e = cudaMemcpyAsync(start, h_start.data(), ns * sizeof(unsigned long long),
                                  cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(len, h_len.data(), ns * sizeof(unsigned), cudaMemcpyHostToDevice, s);
  // both copies read host vectors that go out of scope: finish them here
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  auto blocks = [](size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); };
  k_nb_indices<<<(unsigned)((ns + 63) / 64), 64, 0, s>>>(len, (int)ns, idx); note_launch();
  const size_t tot1 = ns * NB_SPECTRA * (size_t)C;
  k_nb_gather<<<blocks(tot1), 256, 0, s>>>(tf, C, start, idx, tot1, F(L.s1)); note_launch();
  // bandpass: recursive median, smoothing
  const size_t lev[6] = {L.s1, L.s2, L.s3, L.s4, L.s5, L.bp};
  int count = NB_SPECTRA;
  for (int l = 0; l < 5; l++, count /= 5) {
    k_nb_scrunch5<<<blocks(ns * (count / 5) * (size_t)C), 256, 0, s>>>(F(lev[l]), C, count,
                                                                      (int)ns, F(lev[l + 1]));
    note_launch();
  }
  k_nb_smooth<<<(unsigned)ns, 256, 0, s>>>(F(L.bp), F(L.tmp), C, 1.f); note_launch();
  // band deviation: |spectra - bandpass|, recursive median, x 1.4826, smoothing
  k_nb_absdev<<<blocks(tot1), 256, 0, s>>>(F(L.s1), F(L.bp), C, tot1); note_launch();
  const size_t lev2[6] = {L.s1, L.s2, L.s3, L.s4, L.s5, L.mad};
  count = NB_SPECTRA;
  for (int l = 0; l < 5; l++, count /= 5) {
    k_nb_scrunch5<<<blocks(ns * (count / 5) * (size_t)C), 256, 0, s>>>(F(lev2[l]), C, count,
                                                                       (int)ns, F(lev2[l + 1]));
    note_launch();
  }
  k_nb_smooth<<<(unsigned)ns, 256, 0, s>>>(F(L.mad), F(L.tmp), C, 1.4826f); note_launch();
  k_nb_rms<<<(unsigned)ns, 256, 0, s>>>(F(L.mad), C, F(L.rms)); note_launch();
  const size_t nspec = units * nsamps;
  k_nb_zap<<<(unsigned)((nspec + 127) / 128), 128, 0, s>>>(
      reinterpret_cast<uint32_t*>(tf), nsamps, (int)units, C, nsmooth, (int)nsub, F(L.bp),
      F(L.rms), rfi_tol, (unsigned)(C / 60));
  note_launch();
  return cudaGetLastError();
}

namespace {
constexpr int DD_NST = 3;
// Shared memory of a variant: DB = dm_block DMs, `ch` channel rows per stage.
size_t dd_smem(int dm_block, int ch, int rowb) {
  return 128 + (size_t)DD_NST * dm_block * ch * sizeof(int2) + (size_t)DD_NST * ch * rowb;
}
template <int NW, int K, int G, int CH>
cudaError_t launch_dd(const DedispArgs& a, cudaStream_t s) {
  // the compact drain holds two 257-channel chunks at most
  auto kern = a.nact <= 511 ? k_dedisp<NW, K, G, CH, DD_NST, true>
                            : k_dedisp<NW, K, G, CH, DD_NST, false>;
  const size_t smem = dd_smem(2 * NW, CH, a.rowb);
  cudaError_t e = raise_smem_limit(kern, smem);
  if (e != cudaSuccess) return e;
  const int DB = 2 * NW, TB = 128 * K * G;
  dim3 grid((unsigned)((a.dm_count + DB - 1) / DB), (unsigned)((a.nout + TB - 1) / TB),
            (unsigned)a.units);
  kern<<<grid, (NW + 1) * 32, smem, s>>>(a); note_launch();
  return cudaGetLastError();
}
template <int NW, int K, int G>
cudaError_t launch_rows(const DedispArgs& a, int rows, cudaStream_t s) {
  switch (rows) {
    case 16: return launch_dd<NW, K, G, 16>(a, s);
    case 8: return launch_dd<NW, K, G, 8>(a, s);
    case 4: return launch_dd<NW, K, G, 4>(a, s);
    case 2: return launch_dd<NW, K, G, 2>(a, s);
    case 1: return launch_dd<NW, K, G, 1>(a, s);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace

// Channel rows per stage (16, 8, 4, 2 or 1): the most that keep three CTAs on
// an SM (72 KB each), else two (110 KB), else one (200 KB).  More rows per
// stage spread the per-stage waits and hand-offs over more channels.  Rows are long when few
// channels cover a wide DM range (a DM block's delay span is long).  The
// sums are exact integers, so the choice does not change the result.
int dedisp_rows_per_stage(int dm_block, int rowb) {
  for (size_t cap : {(size_t)72 * 1024, (size_t)110 * 1024, (size_t)200 * 1024})
    for (int ch = 16; ch >= 1; ch /= 2)
      if (dd_smem(dm_block, ch, rowb) <= cap) return ch;
  return 0;
}

size_t dedisp_smem_bytes(int dm_block, int rows, int rowb) {
  return dd_smem(dm_block, rows, rowb);
}

cudaError_t launch_dedisp(const DedispArgs& a, const DedispTile& t, cudaStream_t s) {
  if (a.units < 1 || a.units > 65535) return cudaErrorInvalidValue;
  // {dm_block, time_block} -> consumer warps NW = dm_block / 2, words per
  // lane K, groups G with time_block = 128 K G (kDedispTiles)
#define HDB_DD_TILE(DBk, NWk, Kk, Gk) \
  if (t.dm_block == DBk && t.time_block == 128 * Kk * Gk) return launch_rows<NWk, Kk, Gk>(a, t.rows, s);
  HDB_DD_TILE(8, 4, 1, 8)
  HDB_DD_TILE(8, 4, 5, 1)
  HDB_DD_TILE(8, 4, 3, 2)
  HDB_DD_TILE(8, 4, 3, 3)
  HDB_DD_TILE(8, 4, 5, 2)
  HDB_DD_TILE(16, 8, 1, 4)
  HDB_DD_TILE(16, 8, 3, 1)
  HDB_DD_TILE(16, 8, 5, 1)
  HDB_DD_TILE(16, 8, 3, 2)
  HDB_DD_TILE(32, 16, 1, 2)
  HDB_DD_TILE(32, 16, 3, 1)
#undef HDB_DD_TILE
  return cudaErrorInvalidValue;
}

}  // namespace hdb
