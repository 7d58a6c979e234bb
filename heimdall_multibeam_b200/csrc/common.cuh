// common.cuh -- device helpers shared by the search kernels.
//
// All kernels are compiled with -fmad=false: every float expression that has a
// counterpart in the reference (Pipeline/*.cu) rounds exactly as written there,
// so results are bit-identical to the reference's own stage code run on the
// host (Thrust's sequential/OpenMP backend).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hdb {

// ---- selection networks (Pipeline/median_filter.cu:21-75) ----------------
// The reference picks the middle element(s) with comparison trees; any exact
// selection yields the same value for non-NaN input.
#define HDB_CSWAP(x, y) do { if ((y) < (x)) { float t_ = (x); (x) = (y); (y) = t_; } } while (0)

__device__ __forceinline__ float med3(float a, float b, float c) {
  HDB_CSWAP(a, b);
  HDB_CSWAP(b, c);
  HDB_CSWAP(a, b);
  return b;
}

__device__ __forceinline__ float med4(float a, float b, float c, float d) {
  HDB_CSWAP(a, b);
  HDB_CSWAP(c, d);
  HDB_CSWAP(a, c);
  HDB_CSWAP(b, d);
  return __fmul_rn(0.5f, __fadd_rn(b, c));
}

__device__ __forceinline__ float med5(float a, float b, float c, float d, float e) {
  float t;
  HDB_CSWAP(a, b);
  HDB_CSWAP(c, d);
  if (c < a) { t = a; a = c; c = t; t = b; b = d; d = t; }
  a = e;
  HDB_CSWAP(a, b);
  if (c < a) { t = a; a = c; c = t; t = b; b = d; d = t; }
  return (c < b) ? c : b;
}

// Median of 5 by min/max: drop the smallest and the largest of a..d (the
// larger of the pair minima and the smaller of the pair maxima remain), then
// take the median of those two and e.  Equal to med5 for NaN-free input (both
// select the middle value); callers use it only where NaN is excluded.
__device__ __forceinline__ float med5_mm(float a, float b, float c, float d, float e) {
  const float lo = fmaxf(fminf(a, b), fminf(c, d));
  const float hi = fminf(fmaxf(a, b), fmaxf(c, d));
  return fmaxf(fminf(lo, hi), fminf(fmaxf(lo, hi), e));
}

// Order-preserving 32-bit key of a float (larger float -> larger key).
__device__ __forceinline__ uint32_t float_key(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  return __uint_as_float(u);
}

// float -> unsigned truncation with NaN -> 0 (the conversion the reference's
// `unsigned int j = x;` performs on both host and device).
__device__ __forceinline__ unsigned f2u(float x) {
  return (x != x) ? 0u : __float2uint_rz(x);
}

// Pipeline/median_filter.cu:451-479, one output of linear_stretch.
// The reference tests `frac > 1e-5` with frac a float promoted to double.
// 1e-5f (9.9999997e-06) lies below 1e-5 and the next float above it lies above
// 1e-5, so `frac > 1e-5f` in float selects exactly the same values.
constexpr float kStretchEps = 1e-5f;

__device__ __forceinline__ float stretch_at(const float* in, unsigned i, float step) {
  float x = __fmul_rn(__uint2float_rn(i), step);
  unsigned j = f2u(x);
  float fr = __fsub_rn(x, __uint2float_rn(j));
  float add = (fr > kStretchEps) ? __fmul_rn(fr, __fsub_rn(in[j + 1], in[j])) : 0.f;
  return __fadd_rn(in[j], add);
}

// Pipeline/median_filter.cu:481-519, one output of linear_stretch_beam
// (i is the global output index across beams, beam = i / out_count_beam).
__device__ __forceinline__ float stretch_beam_at(const float* in, unsigned i, float step,
                                                 unsigned long long beam) {
  float x = __fmul_rn(__uint2float_rn(i), step);
  float fb = __ull2float_rn(beam);
  unsigned k = f2u(__fadd_rn(x, fb));
  float o = __fadd_rn(__fsub_rn(x, __uint2float_rn(k)), fb);
  float add = (o > kStretchEps) ? __fmul_rn(o, __fsub_rn(in[k + 1], in[k])) : 0.f;
  return __fadd_rn(in[k], add);
}

// ---- bounded mbarrier helpers (TMA bulk-copy staging) --------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count));
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// 1-D bulk async copy global -> shared, completion signalled on `bar`.
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

// Waits for phase `parity` of `bar`; gives up after max_iter polls and
// returns false (the caller records an error and leaves the kernel).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t max_iter) {
  uint32_t a = smem_addr(bar);
  for (uint32_t it = 0; it < max_iter; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done) : "r"(a), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace hdb
