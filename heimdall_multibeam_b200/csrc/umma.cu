// umma.cu -- BF16 GEMM on the fifth-generation tensor cores (tcgen05.mma with
// FP32 accumulators in tensor memory) for the classifier's training.
//
//   D[m][n] = sum_k A[m][k] B[n][k]      A: M x K, B: N x K, both K-major
//   C(m, n) = (accumulate ? C(m, n) : 0) + D[m][n],  C(m, n) = C[m*scm + n*scn]
//
// A CTA owns tiles of 128 rows of D (the M of one tcgen05.mma) by Npad
// columns (N rounded up to 16, at most 128), looping over tiles (persistent;
// grid = min(tiles, 2 per SM)).  K runs in blocks of 64 through a ring of
// shared-memory stages that TMA fills from 2-D tensor maps, one box of
// 8 K-elements x rows per 8-wide K chunk, no swizzle: a box lands as the rows'
// 16-byte core-matrix slices in order, which is the K-major no-swizzle layout
// tcgen05 reads (stride between 8-row groups SBO = 128 B, between the two
// K halves of an MMA LBO = rows x 16 B).  Rows and K past the matrix are
// zero-filled by TMA.
//
// Warps 0-3: epilogue (each reads its 32 TMEM lanes with tcgen05.ld and
// stores its rows); warp 4: TMA producer (one thread); warp 5: allocates the
// TMEM (two accumulator buffers, so a tile's MMAs overlap the previous
// tile's epilogue) and one thread issues the MMAs (K = 16 each) and commits
// them to mbarriers.  Every mbarrier wait is bounded: a wait that gives up
// sets *err, and the kernel drains its copies and MMAs in flight (again
// bounded) and frees its TMEM before returning.
//
// Split-K (K ranges per tile column of the grid): each split writes its
// partial tile to a workspace and k_umma_reduce adds the splits in order, so
// the result does not depend on scheduling.
#include <algorithm>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <mutex>

#include "common.cuh"
#include "internal.h"

namespace hdb {
namespace {

constexpr int UM_BM = 128;     // rows per tile (tcgen05 M)
constexpr int UM_BK = 64;      // K per stage
constexpr int UM_ST = 4;       // stages
constexpr int UM_THREADS = 192;
constexpr uint32_t UM_WAIT = 1u << 24;

struct UmmaArgs {
  int M, N, K, Npad;
  int mtiles, splits;   // tiles = mtiles x splits
  int kblocks;          // K blocks of one split (the last split may have fewer)
  int kblocks_total;
  float* C;             // output (splits == 1) or workspace [splits][M][Npad]
  long long scm, scn;
  int accumulate;
  unsigned* err;
};

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];"
      :: "r"(smem_addr(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar)) : "memory");
}

// shared-memory matrix descriptor: K-major, no swizzle (layout type 0),
// version 1, start/LBO/SBO in 16-byte units
__device__ __forceinline__ uint64_t umma_desc(const void* p, uint32_t lbo, uint32_t sbo) {
  const uint64_t a = smem_addr(p);
  return ((a >> 4) & 0x3FFFull) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
      :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum) : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
      :: "r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(UM_THREADS, 1)
    k_umma_gemm(const __grid_constant__ CUtensorMap map_a,
                const __grid_constant__ CUtensorMap map_b, UmmaArgs g) {
  extern __shared__ __align__(1024) uint8_t um_smem[];
  // [stage][A: 8 chunks x 128 rows x 16 B][B: 8 chunks x Npad rows x 16 B]
  uint8_t* base = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(um_smem) + 1023) & ~(uintptr_t)1023);
  const uint32_t a_chunk = UM_BM * 16, b_chunk = (uint32_t)g.Npad * 16;
  const uint32_t a_bytes = 8 * a_chunk, stage_bytes = a_bytes + 8 * b_chunk;
  uint64_t* full = reinterpret_cast<uint64_t*>(base + UM_ST * stage_bytes);
  uint64_t* empty = full + UM_ST;
  uint64_t* tfull = empty + UM_ST;   // [2] accumulator ready
  uint64_t* tempty = tfull + 2;      // [2] accumulator read out
  uint64_t* drain = tempty + 2;      // MMAs in flight after a failed wait
  uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t ncols = (uint32_t)(2 * g.Npad <= 32 ? 32 : 2 * g.Npad <= 64 ? 64
                                    : 2 * g.Npad <= 128 ? 128 : 256);
  if (threadIdx.x == 0) {
    for (int s = 0; s < UM_ST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);
    }
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_addr(tslot)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const int ntiles = g.mtiles * g.splits;
  const int kb = g.kblocks;

  if (warp == 4) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int mt = tile % g.mtiles, sp = tile / g.mtiles;
        const int k0 = sp * kb * UM_BK;
        const int nb = min(kb, g.kblocks_total - sp * kb);
        for (int b = 0; b < nb && ok; b++, it++) {
          const int s = it % UM_ST;
          if (it >= UM_ST &&
              !mbar_wait(&empty[s], (uint32_t)(((it / UM_ST) - 1) & 1), UM_WAIT)) {
            atomicOr(g.err, 1u);
            ok = false;
            break;
          }
          const int kk = k0 + b * UM_BK;
          // the K chunks of 8 that the block's MMAs (K = 16 each) read; a
          // chunk past K is zero-filled by TMA
          const int nch = 2 * min(4, (g.K - kk + 15) / 16);
          mbar_expect_tx(&full[s], (uint32_t)nch * (a_chunk + b_chunk));
          uint8_t* st = base + (size_t)s * stage_bytes;
          for (int c = 0; c < nch; c++) {
            tma_load_2d(st + c * a_chunk, &map_a, kk + 8 * c, mt * UM_BM, &full[s]);
            tma_load_2d(st + a_bytes + c * b_chunk, &map_b, kk + 8 * c, 0, &full[s]);
          }
        }
      }
      // every copy issued must land before the thread leaves
      for (int j = (it > UM_ST ? it - UM_ST : 0); j < it; j++)
        mbar_wait(&full[j % UM_ST], (uint32_t)((j / UM_ST) & 1), UM_WAIT);
    }
  } else if (warp == 5) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) |
                             ((uint32_t)(g.Npad >> 3) << 17) | ((uint32_t)(UM_BM >> 4) << 24);
      int it = 0, t = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, t++) {
        const int sp = tile / g.mtiles;
        const int buf = t & 1;
        const uint32_t dacc = tmem + (uint32_t)(buf * g.Npad);
        // the epilogue has read this buffer's previous tile
        if (t >= 2 && !mbar_wait(&tempty[buf], (uint32_t)(((t / 2) - 1) & 1), UM_WAIT)) {
          atomicOr(g.err, 2u);
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int k0 = sp * kb * UM_BK;
        const int nb = min(kb, g.kblocks_total - sp * kb);
        uint32_t accum = 0;
        for (int b = 0; b < nb; b++, it++) {
          const int s = it % UM_ST;
          if (!mbar_wait(&full[s], (uint32_t)((it / UM_ST) & 1), UM_WAIT)) {
            atomicOr(g.err, 4u);
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const int kk = k0 + b * UM_BK;
          const int nstep = min(4, (g.K - kk + 15) / 16);
          const uint8_t* st = base + (size_t)s * stage_bytes;
          for (int j = 0; j < nstep; j++) {
            const uint64_t ad = umma_desc(st + 2 * j * a_chunk, a_chunk, 128);
            const uint64_t bd = umma_desc(st + a_bytes + 2 * j * b_chunk, b_chunk, 128);
            umma_bf16(dacc, ad, bd, idesc, accum);
            accum = 1;
          }
          umma_commit(&empty[s]);  // the stage is free once these MMAs complete
        }
        if (!ok) break;
        umma_commit(&tfull[buf]);
      }
      if (!ok) {
        // let the MMAs already issued complete before the TMEM is freed
        umma_commit(drain);
        mbar_wait(drain, 0, UM_WAIT);
      }
    }
  } else {
    // ---------------- epilogue (warps 0-3, TMEM lanes 32w..32w+31) ----------------
    int t = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, t++) {
      const int mt = tile % g.mtiles, sp = tile / g.mtiles;
      const int buf = t & 1;
      if (!mbar_wait(&tfull[buf], (uint32_t)((t / 2) & 1), UM_WAIT)) {
        if (lane == 0) atomicOr(g.err, 8u);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int m = mt * UM_BM + warp * 32 + lane;
      for (int c0 = 0; c0 < g.Npad; c0 += 16) {
        uint32_t r[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(buf * g.Npad + c0), r);
        if (m < g.M) {
          if (g.splits == 1) {
            for (int j = 0; j < 16; j++) {
              const int n = c0 + j;
              if (n < g.N) {
                float* c = g.C + (long long)m * g.scm + (long long)n * g.scn;
                const float v = __uint_as_float(r[j]);
                *c = g.accumulate ? __fadd_rn(*c, v) : v;
              }
            }
          } else {
            float* w = g.C + ((size_t)sp * g.M + m) * g.Npad + c0;
            for (int j = 0; j < 16; j++) w[j] = __uint_as_float(r[j]);
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[buf]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 5) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(ncols)
                 : "memory");
  }
}

// C(m, n) = (accumulate ? C(m, n) : 0) + sum over splits s of W[s][m][n], in
// split order
__global__ void k_umma_reduce(const float* __restrict__ ws, int splits, int M, int N, int Npad,
                              float* __restrict__ C, long long scm, long long scn,
                              int accumulate) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)M * N) return;
  const int m = (int)(i / N), n = (int)(i % N);
  float v = 0.f;
  for (int s = 0; s < splits; s++) v = __fadd_rn(v, ws[((size_t)s * M + m) * Npad + n]);
  float* c = C + (long long)m * scm + (long long)n * scn;
  *c = accumulate ? __fadd_rn(*c, v) : v;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 2-D map of a K-major BF16 matrix (rows x K, row pitch ld elements), boxes of
// 8 elements x box_rows
bool make_map(CUtensorMap* map, const void* ptr, long long rows, long long K, long long ld,
              int box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {8, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

}  // namespace

size_t umma_workspace_floats(int M, int N, int K, int splits) {
  if (splits <= 1) return 0;
  const int Npad = (N + 15) / 16 * 16;
  return (size_t)splits * M * Npad;
}

cudaError_t umma_gemm(int M, int N, int K, const void* A, long long lda, const void* B,
                      long long ldb, float* C, long long scm, long long scn, int accumulate,
                      int splits, float* ws, unsigned* err, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0) return cudaSuccess;
  if (!err) return cudaErrorInvalidValue;
  // operand rows 16-byte aligned, K in whole 8-element chunks of the map
  if (N > 128 || (K % 8) || (lda % 8) || (ldb % 8) ||
      (reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15))
    return cudaErrorNotSupported;
  const int Npad = (N + 15) / 16 * 16;
  const int kblocks_total = (K + UM_BK - 1) / UM_BK;
  splits = std::max(1, std::min(splits, kblocks_total));
  const int kb = (kblocks_total + splits - 1) / splits;
  splits = (kblocks_total + kb - 1) / kb;
  if (splits > 1 && !ws) return cudaErrorInvalidValue;
  CUtensorMap ma, mb;
  if (!make_map(&ma, A, M, K, lda, UM_BM) || !make_map(&mb, B, N, K, ldb, Npad))
    return cudaErrorNotSupported;
  UmmaArgs g{};
  g.M = M;
  g.N = N;
  g.K = K;
  g.Npad = Npad;
  g.mtiles = (M + UM_BM - 1) / UM_BM;
  g.splits = splits;
  g.kblocks = kb;
  g.kblocks_total = kblocks_total;
  g.C = splits > 1 ? ws : C;
  g.scm = scm;
  g.scn = scn;
  g.accumulate = accumulate;
  g.err = err;
  const size_t stage = (size_t)8 * UM_BM * 16 + (size_t)8 * Npad * 16;
  const size_t smem = 1024 + UM_ST * stage + 8 * (2 * UM_ST + 5) + 16;
  cudaError_t e = raise_smem_limit(k_umma_gemm, smem);
  if (e != cudaSuccess) return e;
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = g.mtiles * splits;
  const int grid = std::min(ntiles, 2 * sms);
  k_umma_gemm<<<grid, UM_THREADS, smem, s>>>(ma, mb, g);
  note_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (splits > 1) {
    const size_t n = (size_t)M * N;
    k_umma_reduce<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(ws, splits, M, N, Npad, C, scm,
                                                               scn, accumulate);
    note_launch();
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace hdb
