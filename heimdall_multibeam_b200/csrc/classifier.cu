// classifier.cu -- the learned candidate classifier: a two-branch CNN over a
// candidate's DM-time patch (64 x 64) and frequency-time patch (64 x 256),
// trained and evaluated by BF16 tensor-core GEMMs with FP32 accumulation.
//
// Network (175 666 parameters):
//   branch A (DM-time, 1 x 64 x 64) and branch B (freq-time, 1 x 64 x 256),
//   each: conv3x3(1->8) ReLU maxpool2, conv3x3(8->16) ReLU maxpool2,
//         conv3x3(16->32) ReLU maxpool2   -> A: 32x8x8, B: 32x8x32
//   concat (10240) -> FC 16 ReLU -> FC 2 -> softmax (class 1 = pulse)
// Convolutions run as implicit GEMMs over an im2col matrix: forward
// (W x col), backward-data (W^T x dOut, then col2im) and backward-weights
// (dOut x col^T, split over the pixel dimension).  Every GEMM takes BF16
// operands (weights rounded from FP32 master copies, activations stored in
// BF16) and accumulates in FP32 with mma.sync m16n8k16.  Adam updates the
// FP32 master weights.  Activation layout: [channel][batch][row][col].
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "heimdall_b200.h"
#include "internal.h"

namespace hdb {
namespace clf {

using bf16 = __nv_bfloat16;

// ===========================================================================
// BF16 GEMM, FP32 accumulation: C(m, n) (+)= sum_k A(m, k) B(k, n) with
// element strides A(m, k) = A[m*sam + k*sak], B(k, n) = B[k*sbk + n*sbn],
// C(m, n) = C[m*scm + n*scn].  Block tile 32 x 64 x 32, 4 warps of 16 x 32.
// blockIdx.z splits K into chunks of kchunk; with more than one split the
// partial sums are added atomically (C must hold the initial value).
// ===========================================================================
constexpr int GBM = 32, GBN = 64, GBK = 32, GPAD = 8;

struct GemmArgs {
  int M, N, K;
  const bf16* A;
  long long sam, sak;
  const bf16* B;
  long long sbk, sbn;
  float* C;
  long long scm, scn;
  int accumulate;  // add to C (single split) instead of overwriting
  int kchunk;      // K per blockIdx.z
};

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(128) k_gemm_bf16(GemmArgs g) {
  __shared__ __align__(16) bf16 As[GBM][GBK + GPAD];  // [m][k]
  __shared__ __align__(16) bf16 Bs[GBN][GBK + GPAD];  // [n][k]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = blockIdx.y * GBM, n0 = blockIdx.x * GBN;
  const int kb = blockIdx.z * g.kchunk;
  const int ke = min(g.K, kb + g.kchunk);
  const int wm = (warp & 1) * 16, wn = (warp >> 1) * 32;
  const int gr = lane >> 2, tq = lane & 3;
  float acc[4][4];
#pragma unroll
  for (int j = 0; j < 4; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  const bf16 zero = __float2bfloat16(0.f);
  for (int k0 = kb; k0 < ke; k0 += GBK) {
    // tiles, zero outside the matrix; the faster index follows the unit stride
    for (int e = tid; e < GBM * GBK; e += 128) {
      int m, k;
      if (g.sak == 1) { m = e / GBK; k = e % GBK; } else { k = e / GBM; m = e % GBM; }
      const int gm = m0 + m, gk = k0 + k;
      As[m][k] = (gm < g.M && gk < ke) ? g.A[gm * g.sam + gk * g.sak] : zero;
    }
    for (int e = tid; e < GBN * GBK; e += 128) {
      int n, k;
      if (g.sbn == 1) { k = e / GBN; n = e % GBN; } else { n = e / GBK; k = e % GBK; }
      const int gn = n0 + n, gk = k0 + k;
      Bs[n][k] = (gn < g.N && gk < ke) ? g.B[gk * g.sbk + gn * g.sbn] : zero;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GBK; kk += 16) {
      uint32_t a[4];
      a[0] = *reinterpret_cast<const uint32_t*>(&As[wm + gr][kk + 2 * tq]);
      a[1] = *reinterpret_cast<const uint32_t*>(&As[wm + gr + 8][kk + 2 * tq]);
      a[2] = *reinterpret_cast<const uint32_t*>(&As[wm + gr][kk + 2 * tq + 8]);
      a[3] = *reinterpret_cast<const uint32_t*>(&As[wm + gr + 8][kk + 2 * tq + 8]);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        uint32_t b[2];
        b[0] = *reinterpret_cast<const uint32_t*>(&Bs[wn + 8 * j + gr][kk + 2 * tq]);
        b[1] = *reinterpret_cast<const uint32_t*>(&Bs[wn + 8 * j + gr][kk + 2 * tq + 8]);
        mma_bf16(acc[j], a, b);
      }
    }
    __syncthreads();
  }
  const bool split = gridDim.z > 1;
#pragma unroll
  for (int j = 0; j < 4; j++) {
#pragma unroll
    for (int h = 0; h < 4; h++) {
      const int m = m0 + wm + gr + (h >> 1) * 8;
      const int n = n0 + wn + 8 * j + 2 * tq + (h & 1);
      if (m < g.M && n < g.N) {
        float* c = g.C + m * g.scm + n * g.scn;
        if (split) atomicAdd(c, acc[j][h]);
        else *c = g.accumulate ? *c + acc[j][h] : acc[j][h];
      }
    }
  }
}

cudaError_t gemm(const GemmArgs& a0, int splits, cudaStream_t s) {
  GemmArgs a = a0;
  if (a.M <= 0 || a.N <= 0 || a.K <= 0) return cudaSuccess;
  splits = std::max(1, std::min(splits, (a.K + GBK - 1) / GBK));
  a.kchunk = ((a.K + splits - 1) / splits + GBK - 1) / GBK * GBK;
  splits = (a.K + a.kchunk - 1) / a.kchunk;
  dim3 grid((unsigned)((a.N + GBN - 1) / GBN), (unsigned)((a.M + GBM - 1) / GBM), (unsigned)splits);
  if (grid.y > 65535 || grid.z > 65535) return cudaErrorInvalidValue;
  k_gemm_bf16<<<grid, 128, 0, s>>>(a); note_launch();
  return cudaGetLastError();
}

// ===========================================================================
// Elementwise and layout kernels
// ===========================================================================
__global__ void k_to_bf16(const float* __restrict__ in, bf16* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16(in[i]);
}

// network input: patch values (in units of the row's robust deviation)
// limited to +-kInputClip, so that very bright rows do not saturate training
constexpr float kInputClip = 16.f;
__global__ void k_input_bf16(const float* __restrict__ in, bf16* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16(fminf(fmaxf(in[i], -kInputClip), kInputClip));
}

// weights [co][k] (k < kw) -> BF16 [co][kp], zero columns kw..kp-1
__global__ void k_weights_bf16(const float* __restrict__ w, int co, int kw, int kp,
                               bf16* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= co * kp) return;
  const int o = i / kp, k = i % kp;
  out[i] = __float2bfloat16(k < kw ? w[o * kw + k] : 0.f);
}

// im2col of a 3x3, pad-1 convolution: in [ci][b][h][w] -> col [kp][b*h*w]
// (row ci*9 + ky*3 + kx; rows >= ci*9 are zero)
__global__ void k_im2col3(const bf16* __restrict__ in, int ci, int nb, int h, int w, int kp,
                          bf16* __restrict__ col) {
  const size_t P = (size_t)nb * h * w;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P * kp) return;
  const int r = (int)(i / P);
  const size_t p = i % P;
  bf16 v = __float2bfloat16(0.f);
  if (r < ci * 9) {
    const int c = r / 9, ky = (r % 9) / 3, kx = r % 3;
    const int x = (int)(p % w), y = (int)((p / w) % h);
    const size_t b = p / ((size_t)w * h);
    const int yy = y + ky - 1, xx = x + kx - 1;
    if (yy >= 0 && yy < h && xx >= 0 && xx < w)
      v = in[(((size_t)c * nb + b) * h + yy) * w + xx];
  }
  col[i] = v;
}

// im2col in K-major order for the tensor-core GEMM: colT [b*h*w][kp], the kp
// taps of one output pixel contiguous (the same values as k_im2col3)
__global__ void k_im2col3_t(const bf16* __restrict__ in, int ci, int nb, int h, int w, int kp,
                            bf16* __restrict__ colT) {
  const size_t P = (size_t)nb * h * w;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P * kp) return;
  const size_t p = i / kp;
  const int r = (int)(i % kp);
  bf16 v = __float2bfloat16(0.f);
  if (r < ci * 9) {
    const int c = r / 9, ky = (r % 9) / 3, kx = r % 3;
    const int x = (int)(p % w), y = (int)((p / w) % h);
    const size_t b = p / ((size_t)w * h);
    const int yy = y + ky - 1, xx = x + kx - 1;
    if (yy >= 0 && yy < h && xx >= 0 && xx < w)
      v = in[(((size_t)c * nb + b) * h + yy) * w + xx];
  }
  colT[i] = v;
}

// col2im: dcol [kp][b*h*w] (FP32) -> din [ci][b][h][w], summing the 9 taps
// that read each input pixel
__global__ void k_col2im3(const float* __restrict__ dcol, int ci, int nb, int h, int w,
                          float* __restrict__ din) {
  const size_t P = (size_t)nb * h * w;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P * ci) return;
  const int c = (int)(i / P);
  const size_t p = i % P;
  const int x = (int)(p % w), y = (int)((p / w) % h);
  const size_t bo = (p / ((size_t)w * h)) * (size_t)w * h;
  float sum = 0.f;
#pragma unroll
  for (int ky = 0; ky < 3; ky++)
#pragma unroll
    for (int kx = 0; kx < 3; kx++) {
      // output pixel (y - ky + 1, x - kx + 1) read this input through tap (ky, kx)
      const int yo = y - ky + 1, xo = x - kx + 1;
      if (yo >= 0 && yo < h && xo >= 0 && xo < w)
        sum += dcol[(size_t)(c * 9 + ky * 3 + kx) * P + bo + (size_t)yo * w + xo];
    }
  din[i] = sum;
}

// conv output [co][b][h][w] (FP32) + bias -> ReLU -> 2x2 max pool ->
// act [co][b][h/2][w/2] (BF16), arg = position of the maximum (0..3)
__global__ void k_bias_relu_pool(const float* __restrict__ z, const float* __restrict__ bias,
                                 int co, int nb, int h, int w, bf16* __restrict__ act,
                                 unsigned char* __restrict__ arg) {
  const int h2 = h / 2, w2 = w / 2;
  const size_t n = (size_t)co * nb * h2 * w2;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x2 = (int)(i % w2), y2 = (int)((i / w2) % h2);
  const size_t cb = i / ((size_t)w2 * h2);  // c * nb + b
  const int c = (int)(cb / nb);
  const float* zp = z + cb * (size_t)h * w;
  float best = -INFINITY;
  int bi = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const float v = fmaxf(zp[(size_t)(2 * y2 + (q >> 1)) * w + 2 * x2 + (q & 1)] + bias[c], 0.f);
    if (v > best) { best = v; bi = q; }
  }
  act[i] = __float2bfloat16(best);
  arg[i] = (unsigned char)bi;
}

// backward of bias/ReLU/pool: dact [co][b][h/2][w/2] (FP32) -> dz [co][b][h][w]
// (BF16, the next GEMM's operand), and the bias gradient
__global__ void k_pool_relu_back(const float* __restrict__ dact, const bf16* __restrict__ act,
                                 const unsigned char* __restrict__ arg, int co, int nb, int h,
                                 int w, bf16* __restrict__ dz, float* __restrict__ dbias) {
  const int h2 = h / 2, w2 = w / 2;
  const size_t n = (size_t)co * nb * h * w;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  float v = 0.f;
  int c = -1;
  if (i < n) {
    const int x = (int)(i % w), y = (int)((i / w) % h);
    const size_t cb = i / ((size_t)w * h);
    c = (int)(cb / nb);
    const size_t j = (cb * h2 + y / 2) * w2 + x / 2;
    const int q = (y & 1) * 2 + (x & 1);
    if (y / 2 < h2 && x / 2 < w2 && arg[j] == q && __bfloat162float(act[j]) > 0.f) v = dact[j];
    dz[i] = __float2bfloat16(v);
  }
  (void)c;
  (void)dbias;
}

// bias gradient of the same layer: dbias[c] += the sum over c's pixels of the
// pre-activation gradient, one block per channel, in a fixed order (each
// thread's strided partial, then a fixed tree), so every run gives the same
// bits
__global__ void __launch_bounds__(256) k_bias_grad(const float* __restrict__ dact,
                                                   const bf16* __restrict__ act,
                                                   const unsigned char* __restrict__ arg,
                                                   int nb, int h, int w,
                                                   float* __restrict__ dbias) {
  __shared__ float part[256];
  const int c = blockIdx.x;
  const int h2 = h / 2, w2 = w / 2;
  const size_t per = (size_t)nb * h * w;
  float acc = 0.f;
  for (size_t k = threadIdx.x; k < per; k += blockDim.x) {
    const size_t i = (size_t)c * per + k;
    const int x = (int)(i % w), y = (int)((i / w) % h);
    const size_t cb = i / ((size_t)w * h);
    const size_t j = (cb * h2 + y / 2) * w2 + x / 2;
    const int q = (y & 1) * 2 + (x & 1);
    if (y / 2 < h2 && x / 2 < w2 && arg[j] == q && __bfloat162float(act[j]) > 0.f)
      acc = __fadd_rn(acc, dact[j]);
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) part[threadIdx.x] = __fadd_rn(part[threadIdx.x], part[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) dbias[c] = __fadd_rn(dbias[c], part[0]);
}

// pooled activations of both branches -> x [b][10240] (A: 2048, B: 8192)
__global__ void k_flatten(const bf16* __restrict__ a, const bf16* __restrict__ bb, int nb,
                          bf16* __restrict__ x) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nb * 10240) return;
  const int n = (int)(i / 10240), f = (int)(i % 10240);
  if (f < 2048) {
    const int c = f / 64, s = f % 64;  // A: 32 x (8 x 8)
    x[i] = a[((size_t)c * nb + n) * 64 + s];
  } else {
    const int g = f - 2048, c = g / 256, s = g % 256;  // B: 32 x (8 x 32)
    x[i] = bb[((size_t)c * nb + n) * 256 + s];
  }
}

__global__ void k_unflatten(const float* __restrict__ dx, int nb, float* __restrict__ da,
                            float* __restrict__ db) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nb * 10240) return;
  const int n = (int)(i / 10240), f = (int)(i % 10240);
  if (f < 2048) {
    const int c = f / 64, s = f % 64;
    da[((size_t)c * nb + n) * 64 + s] = dx[i];
  } else {
    const int g = f - 2048, c = g / 256, s = g % 256;
    db[((size_t)c * nb + n) * 256 + s] = dx[i];
  }
}

// FC1 bias + ReLU: z1 [16][b] -> h [b][16] (FP32)
__global__ void k_fc1_act(const float* __restrict__ z1, const float* __restrict__ b1, int nb,
                          float* __restrict__ h) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb * 16) return;
  const int n = i / 16, o = i % 16;
  h[i] = fmaxf(z1[o * nb + n] + b1[o], 0.f);
}

// FC2, softmax, cross-entropy and their backward, FC2 weight/bias gradients,
// the FC1 pre-activation gradient dz1 [16][b] (BF16) and its bias gradient.
// One thread per sample; w2 [2][16], b2 [2].
// The per-sample terms of the loss and of the FC2/FC1-bias gradients go to
// hs [b][18] (loss / nb, dL/dl1, the 16 dz) and k_head_reduce sums them over
// the batch in sample order.
constexpr int kHeadTerms = 18;
__global__ void k_head(const float* __restrict__ h, const float* __restrict__ w2,
                       const float* __restrict__ b2, const int* __restrict__ labels, int nb,
                       int backward, float* __restrict__ prob, bf16* __restrict__ dz1,
                       float* __restrict__ hs) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nb) return;
  const float* hn = h + n * 16;
  float l0 = b2[0], l1 = b2[1];
  for (int o = 0; o < 16; o++) {
    l0 += w2[o] * hn[o];
    l1 += w2[16 + o] * hn[o];
  }
  const float mx = fmaxf(l0, l1);
  const float e0 = expf(l0 - mx), e1 = expf(l1 - mx);
  const float p1 = e1 / (e0 + e1);
  prob[n] = p1;
  if (!backward) return;
  const int y = labels[n];
  const float lse = mx + logf(e0 + e1);
  float* t = hs + (size_t)n * kHeadTerms;
  t[0] = (lse - (y ? l1 : l0)) / nb;
  const float d1 = (p1 - (y ? 1.f : 0.f)) / nb;  // dL/dl1; dL/dl0 = -d1
  const float d0 = -d1;
  t[1] = d1;
  for (int o = 0; o < 16; o++) {
    const float dh = d0 * w2[o] + d1 * w2[16 + o];
    const float dz = hn[o] > 0.f ? dh : 0.f;
    dz1[o * nb + n] = __float2bfloat16(dz);
    t[2 + o] = dz;
  }
}

// loss (+= the per-sample terms), gb2, gw2 [2][16] and gb1 [16] from hs and
// h, each a sum over the samples in order (thread per output)
__global__ void k_head_reduce(const float* __restrict__ h, const float* __restrict__ hs, int nb,
                              float* __restrict__ loss, float* __restrict__ gw2,
                              float* __restrict__ gb2, float* __restrict__ gb1) {
  const int k = threadIdx.x;  // 0: loss, 1-2: gb2, 3-34: gw2, 35-50: gb1
  if (k > 50) return;
  float acc = 0.f;
  for (int n = 0; n < nb; n++) {
    const float* t = hs + (size_t)n * kHeadTerms;
    const float d1 = t[1], d0 = -d1;
    float v;
    if (k == 0) v = t[0];
    else if (k == 1) v = d0;
    else if (k == 2) v = d1;
    else if (k < 19) v = d0 * h[n * 16 + (k - 3)];
    else if (k < 35) v = d1 * h[n * 16 + (k - 19)];
    else v = t[2 + (k - 35)];
    acc = __fadd_rn(acc, v);
  }
  if (k == 0) loss[0] = __fadd_rn(loss[0], acc);
  else if (k < 3) gb2[k - 1] = __fadd_rn(gb2[k - 1], acc);
  else if (k < 35) gw2[k - 3] = __fadd_rn(gw2[k - 3], acc);
  else gb1[k - 35] = __fadd_rn(gb1[k - 35], acc);
}

// per-sample batch gather: dataset [n][len] (BF16) rows idx -> [b][len]
__global__ void k_gather(const bf16* __restrict__ src, const int* __restrict__ idx, int nb,
                         int len, bf16* __restrict__ dst) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nb * len) return;
  const int n = (int)(i / len), k = (int)(i % len);
  dst[i] = src[(size_t)idx[n] * len + k];
}

// Adam (Kingma & Ba 2015) on the FP32 master weights
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

inline unsigned nblk(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace clf

// ===========================================================================
// Fused inference: the whole network for one candidate per CTA iteration.
//
// A persistent CTA of 16 warps takes candidates in turn.  Activations live in
// shared memory as [row + 1][col + 1][channel] BF16 with a zero ring (the
// convolutions' padding).  Each 3x3 convolution is an implicit GEMM on the
// tensor cores (mma.sync m16n8k16, FP32 accumulation) with the 16 rows of an
// MMA tile = 2 image rows x 8 columns and its columns = output channels; the
// K dimension runs over taps and input channels: one tap x 16 channels
// (c_in = 16), two taps x 8 channels (c_in = 8) or the 9 taps of the single
// input channel.  Bias, ReLU and the 2x2 max-pool are applied to the
// accumulators in registers (the vertical pair sits in one thread, the
// horizontal pair in lanes 4 apart) and the pooled value is rounded to BF16
// once, as in the training path.  The last layer of each branch writes the
// flattened feature vector (10240 BF16) to shared memory; each warp then
// computes one FC1 unit (fixed lane order and shuffle tree), and thread 0 the
// FC2 logits and the softmax.  Every candidate is summed in the same order
// whatever the grid, so all scoring entry points agree bit for bit.
// ===========================================================================
namespace inf {
using namespace clf;
constexpr int kWarps = 16, kThreads = kWarps * 32;
// shared-memory regions (bytes)
// Pixels of 16 channels are stored 24 elements (48 bytes) apart, so that the
// 8 pixels of an MMA fragment load fall on distinct banks; 1 and 8 channels
// are dense.
template <int C>
__host__ __device__ constexpr int pix_stride() { return C == 16 ? 24 : C; }
constexpr int kR0 = 18 * 66 * 24 * 2;   // B input [66][258]; B pool-2 [18][66][24]; A pool-1 [34][34][8]
constexpr int kR1 = 34 * 130 * 8 * 2;   // B pool-1 [34][130][8]; A input [66][66]; A pool-2 [18][18][24]
constexpr int kF = 10240 * 2;           // flattened features
// weight fragments per layer: ksteps x (c_out / 8) x 32 lanes of uint2
constexpr int kFragL1 = 1 * 1 * 32, kFragL2 = 5 * 2 * 32, kFragL3 = 9 * 4 * 32;
constexpr int kFragBranch = kFragL1 + kFragL2 + kFragL3;
constexpr int kWF = 2 * kFragBranch * 8;
constexpr size_t kSmem = (size_t)kR0 + kR1 + kF + kWF + 256 * sizeof(float);

struct Args {
  const float* dm;   // [n][64][64] FP32 patches
  const float* ft;   // [n][64][256]
  int n;
  const float* w;    // FP32 parameters
  int off_w[2][3], off_b[2][3], off_b1, off_w2, off_b2;
  const bf16* wb1;   // FC1 weights [16][10240] BF16
  float* prob;       // [n]
};

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// weight fragment b0/b1 of k-step s, n-tile j for this lane; K order as the
// A fragments below
template <int CI>
__device__ uint2 weight_frag(const float* W, int s, int j, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int co = 8 * j + g;
  auto wk = [&](int k) -> bf16 {
    int tap, ci;
    if (CI == 16) { tap = s; ci = k; }
    else if (CI == 8) { tap = 2 * s + (k >> 3); ci = k & 7; }
    else { tap = k; ci = 0; }
    if (tap >= 9) return __float2bfloat16(0.f);
    return __float2bfloat16(W[co * (CI * 9) + ci * 9 + tap]);
  };
  uint2 r;
  r.x = pack2(wk(2 * t), wk(2 * t + 1));
  r.y = pack2(wk(2 * t + 8), wk(2 * t + 9));
  return r;
}

template <int CI, int CO>
__device__ void build_frags(const float* W, uint2* wf) {
  constexpr int KS = CI == 16 ? 9 : (CI == 8 ? 5 : 1);
  constexpr int NT = CO / 8;
  for (int e = threadIdx.x; e < KS * NT * 32; e += blockDim.x) {
    const int lane = e & 31, j = (e >> 5) % NT, s = (e >> 5) / NT;
    wf[e] = weight_frag<CI>(W, s, j, lane);
  }
}

// zero ring of a [H2 + 2][W2 + 2][C] buffer
__device__ void zero_ring(bf16* buf, int H2, int W2, int C) {
  const int Wp = W2 + 2, Hp = H2 + 2;
  const int ring = 2 * Wp + 2 * H2;  // pixels
  const bf16 z = __float2bfloat16(0.f);
  for (int e = threadIdx.x; e < ring * C; e += blockDim.x) {
    const int px = e / C, c = e % C;
    int y, x;
    if (px < Wp) { y = 0; x = px; }
    else if (px < 2 * Wp) { y = Hp - 1; x = px - Wp; }
    else { const int q = px - 2 * Wp; y = 1 + (q >> 1); x = (q & 1) ? Wp - 1 : 0; }
    buf[((size_t)y * Wp + x) * C + c] = z;
  }
}

// patch rows (FP32, global) -> BF16 [66][W + 2] with a zero ring, limited to
// +-kInputClip as the training input
__device__ void load_input(const float* __restrict__ src, int W, bf16* dst) {
  zero_ring(dst, 64, W, 1);
  const int n4 = 64 * W / 4;
  for (int e = threadIdx.x; e < n4; e += blockDim.x) {
    const float4 v = reinterpret_cast<const float4*>(src)[e];
    const int y = (4 * e) / W, x = (4 * e) % W;
    bf16* o = dst + (size_t)(y + 1) * (W + 2) + x + 1;
    o[0] = __float2bfloat16(fminf(fmaxf(v.x, -kInputClip), kInputClip));
    o[1] = __float2bfloat16(fminf(fmaxf(v.y, -kInputClip), kInputClip));
    o[2] = __float2bfloat16(fminf(fmaxf(v.z, -kInputClip), kInputClip));
    o[3] = __float2bfloat16(fminf(fmaxf(v.w, -kInputClip), kInputClip));
  }
}

// conv 3x3 (pad 1) + bias + ReLU + 2x2 max-pool of an H x W x CI image
// (pixels pix_stride<CI>() elements apart).
// out: [H/2 + 2][W/2 + 2][pix_stride<CO>()] interior, or (feat) the flattened features at
// feat[c * (H/2 * W/2) + y * W/2 + x].
template <int CI, int CO>
__device__ void conv_layer(const bf16* __restrict__ in, int H, int W, const uint2* __restrict__ wf,
                           const float* __restrict__ bias, bf16* __restrict__ out,
                           bf16* __restrict__ feat) {
  constexpr int KS = CI == 16 ? 9 : (CI == 8 ? 5 : 1);
  constexpr int NT = CO / 8;
  constexpr int PSI = pix_stride<CI>(), PSO = pix_stride<CO>();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int Wp = W + 2, W2 = W / 2, H2 = H / 2;
  const int ntx = W / 8, ntiles = H2 * ntx;
  float bia[NT][2];
#pragma unroll
  for (int j = 0; j < NT; j++) {
    bia[j][0] = bias[8 * j + 2 * t];
    bia[j][1] = bias[8 * j + 2 * t + 1];
  }
  for (int tile = warp; tile < ntiles; tile += kWarps) {
    const int ty = tile / ntx, tx = tile % ntx;
    // pixel rows of the MMA tile: row g -> (2ty, 8tx + g), row g + 8 -> (2ty + 1, 8tx + g);
    // padded index of pixel (y, x) at tap (ky, kx) = (y + ky) * Wp + x + kx
    const int p0 = (2 * ty) * Wp + 8 * tx + g;
    const int p1 = p0 + Wp;
    float acc[NT][4];
#pragma unroll
    for (int j = 0; j < NT; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
#pragma unroll
    for (int s = 0; s < KS; s++) {
      uint32_t a[4];
      if (CI == 16) {
        const int o = (s / 3) * Wp + (s % 3);
        a[0] = *reinterpret_cast<const uint32_t*>(in + (size_t)(p0 + o) * PSI + 2 * t);
        a[1] = *reinterpret_cast<const uint32_t*>(in + (size_t)(p1 + o) * PSI + 2 * t);
        a[2] = *reinterpret_cast<const uint32_t*>(in + (size_t)(p0 + o) * PSI + 2 * t + 8);
        a[3] = *reinterpret_cast<const uint32_t*>(in + (size_t)(p1 + o) * PSI + 2 * t + 8);
      } else if (CI == 8) {
        const int j0 = 2 * s, j1 = 2 * s + 1;
        const int o0 = (j0 / 3) * Wp + (j0 % 3);
        a[0] = *reinterpret_cast<const uint32_t*>(in + (size_t)(p0 + o0) * PSI + 2 * t);
        a[1] = *reinterpret_cast<const uint32_t*>(in + (size_t)(p1 + o0) * PSI + 2 * t);
        if (j1 < 9) {
          const int o1 = (j1 / 3) * Wp + (j1 % 3);
          a[2] = *reinterpret_cast<const uint32_t*>(in + (size_t)(p0 + o1) * PSI + 2 * t);
          a[3] = *reinterpret_cast<const uint32_t*>(in + (size_t)(p1 + o1) * PSI + 2 * t);
        } else {
          a[2] = a[3] = 0u;
        }
      } else {
        // K = tap; taps 2t, 2t + 1 and (t = 0 only) tap 8
        const int ta = 2 * t, tb = 2 * t + 1;
        const int oa = (ta / 3) * Wp + (ta % 3), ob = (tb / 3) * Wp + (tb % 3);
        a[0] = pack2(in[p0 + oa], in[p0 + ob]);
        a[1] = pack2(in[p1 + oa], in[p1 + ob]);
        const bf16 z = __float2bfloat16(0.f);
        const int o8 = 2 * Wp + 2;
        a[2] = t == 0 ? pack2(in[p0 + o8], z) : 0u;
        a[3] = t == 0 ? pack2(in[p1 + o8], z) : 0u;
      }
#pragma unroll
      for (int j = 0; j < NT; j++) {
        const uint2 b = wf[(s * NT + j) * 32 + lane];
        const uint32_t bb[2] = {b.x, b.y};
        mma_bf16(acc[j], a, bb);
      }
    }
    // epilogue: c0 (row g, co 2t), c1 (row g, co 2t+1), c2/c3 the same for row g + 8
    const int py = ty, px = 4 * tx + (g >> 1);
#pragma unroll
    for (int j = 0; j < NT; j++) {
      float m0 = fmaxf(fmaxf(acc[j][0] + bia[j][0], 0.f), fmaxf(acc[j][2] + bia[j][0], 0.f));
      float m1 = fmaxf(fmaxf(acc[j][1] + bia[j][1], 0.f), fmaxf(acc[j][3] + bia[j][1], 0.f));
      m0 = fmaxf(m0, __shfl_xor_sync(0xffffffffu, m0, 4));
      m1 = fmaxf(m1, __shfl_xor_sync(0xffffffffu, m1, 4));
      if ((g & 1) == 0) {
        const int co = 8 * j + 2 * t;
        if (feat) {
          feat[(size_t)co * (H2 * W2) + py * W2 + px] = __float2bfloat16(m0);
          feat[(size_t)(co + 1) * (H2 * W2) + py * W2 + px] = __float2bfloat16(m1);
        } else {
          *reinterpret_cast<uint32_t*>(out + ((size_t)(py + 1) * (W2 + 2) + px + 1) * PSO + co) =
              pack2(__float2bfloat16(m0), __float2bfloat16(m1));
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kThreads, 1) k_clf_infer(Args a) {
  extern __shared__ __align__(128) uint8_t smem[];
  bf16* r0 = reinterpret_cast<bf16*>(smem);
  bf16* r1 = reinterpret_cast<bf16*>(smem + kR0);
  bf16* feat = reinterpret_cast<bf16*>(smem + kR0 + kR1);
  uint2* wf = reinterpret_cast<uint2*>(smem + kR0 + kR1 + kF);
  float* hid = reinterpret_cast<float*>(smem + kR0 + kR1 + kF + kWF);
  // weight fragments of both branches, once per CTA
  for (int br = 0; br < 2; br++) {
    uint2* f = wf + br * kFragBranch;
    build_frags<1, 8>(a.w + a.off_w[br][0], f);
    build_frags<8, 16>(a.w + a.off_w[br][1], f + kFragL1);
    build_frags<16, 32>(a.w + a.off_w[br][2], f + kFragL1 + kFragL2);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int cand = blockIdx.x; cand < a.n; cand += gridDim.x) {
    __syncthreads();  // fragments ready / previous candidate's FC done
    // ---- branch B (freq-time, 64 x 256): features 2048.. ----
    const uint2* fB = wf + kFragBranch;
    load_input(a.ft + (size_t)cand * 16384, 256, r0);
    zero_ring(r1, 32, 128, 8);
    __syncthreads();
    conv_layer<1, 8>(r0, 64, 256, fB, a.w + a.off_b[1][0], r1, nullptr);
    __syncthreads();
    zero_ring(r0, 16, 64, pix_stride<16>());
    conv_layer<8, 16>(r1, 32, 128, fB + kFragL1, a.w + a.off_b[1][1], r0, nullptr);
    __syncthreads();
    conv_layer<16, 32>(r0, 16, 64, fB + kFragL1 + kFragL2, a.w + a.off_b[1][2], nullptr,
                       feat + 2048);
    __syncthreads();
    // ---- branch A (DM-time, 64 x 64): features 0..2047 ----
    const uint2* fA = wf;
    load_input(a.dm + (size_t)cand * 4096, 64, r1);
    zero_ring(r0, 32, 32, 8);
    __syncthreads();
    conv_layer<1, 8>(r1, 64, 64, fA, a.w + a.off_b[0][0], r0, nullptr);
    __syncthreads();
    zero_ring(r1, 16, 16, pix_stride<16>());
    conv_layer<8, 16>(r0, 32, 32, fA + kFragL1, a.w + a.off_b[0][1], r1, nullptr);
    __syncthreads();
    conv_layer<16, 32>(r1, 16, 16, fA + kFragL1 + kFragL2, a.w + a.off_b[0][2], nullptr, feat);
    __syncthreads();
    // ---- FC1: warp o computes hidden unit o ----
    {
      const int o = warp;
      const uint4* wrow = reinterpret_cast<const uint4*>(a.wb1 + (size_t)o * 10240);
      const uint4* x = reinterpret_cast<const uint4*>(feat);
      float sum = 0.f;
      for (int i = lane; i < 10240 / 8; i += 32) {
        const uint4 wv = wrow[i], xv = x[i];
        const uint32_t wa[4] = {wv.x, wv.y, wv.z, wv.w}, xa[4] = {xv.x, xv.y, xv.z, xv.w};
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const float2 wf2 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&wa[q]));
          const float2 xf2 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&xa[q]));
          sum = __fadd_rn(sum, __fmul_rn(wf2.x, xf2.x));
          sum = __fadd_rn(sum, __fmul_rn(wf2.y, xf2.y));
        }
      }
#pragma unroll
      for (int off = 16; off; off >>= 1) sum = __fadd_rn(sum, __shfl_xor_sync(0xffffffffu, sum, off));
      if (lane == 0) hid[o] = fmaxf(sum + a.w[a.off_b1 + o], 0.f);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const float* w2 = a.w + a.off_w2;
      const float* b2 = a.w + a.off_b2;
      float l0 = b2[0], l1 = b2[1];
      for (int o = 0; o < 16; o++) {
        l0 += w2[o] * hid[o];
        l1 += w2[16 + o] * hid[o];
      }
      const float mx = fmaxf(l0, l1);
      const float e0 = expf(l0 - mx), e1 = expf(l1 - mx);
      a.prob[cand] = e1 / (e0 + e1);
    }
  }
}
}  // namespace inf

// ===========================================================================
// Candidate patches (Applications/candidate_profiler.C)
// ===========================================================================
// DM-time: row r = DM trial dm - 32 + r (zero outside 0..D-1), column t = the
// width-w boxcar sum starting at first + t, first = ind - 32 - w/2 (0 if
// ind <= 32 + w/2), from the series' prefix sums S: S[first+t+w] - S[first+t]
// (zero when it would read past S[len]); gen_dm_time_plot:232-415 with
// do_filter (its boxcar spans scanned[t + w/2 + (w-1)/2 + 1] - scanned[t]).
__global__ void k_patch_dm(const float* __restrict__ scan, size_t scan_pitch, size_t len,
                           const PatchJob* __restrict__ jobs, float* __restrict__ out) {
  const PatchJob jb = jobs[blockIdx.x];
  const unsigned w = 1u << jb.filter;
  const long long first = (jb.ind > 32u + w / 2) ? (long long)jb.ind - 32 - w / 2 : 0;
  float* o = out + (size_t)blockIdx.x * 4096;
  for (int e = threadIdx.x; e < 4096; e += blockDim.x) {
    const int r = e / 64, t = e % 64;
    const int d = jb.dm - 32 + r;
    float v = 0.f;
    const long long a = first + t, b = a + w;
    if (d >= 0 && d < jb.ndm && b <= (long long)len) {
      const float* S = scan + (size_t)(jb.series0 + d) * scan_pitch;
      v = __fsub_rn(S[b], S[a]);
    }
    o[e] = v;
  }
}

// Freq-time: gen_freq_time_plot:136-230 on the undispersed filterbank (TF
// bytes): 64 sub-bands of fs = nchans/64 channels x 256 bins of ts samples
// from first; each pixel the float sum, time outer and channel inner, of
// x / 255 * 255 divided by ts * fs; samples outside the gulp read as 0.
// x / 255 * 255 comes from a 256-entry table of the same rounded operations;
// rows outside the gulp are skipped (they add +0 to a sum that is >= +0, which
// leaves it unchanged).  Grid: x = candidate, y = 64 groups of 4 time bins;
// block = 4 bins x 64 sub-bands, so a warp reads 32 adjacent sub-bands of one
// row.
__global__ void __launch_bounds__(256) k_patch_ft(const uint8_t* __restrict__ tf, size_t nsamps,
                                                  int nchans, const PatchJob* __restrict__ jobs,
                                                  float* __restrict__ out) {
  __shared__ float lut[256];
  lut[threadIdx.x] = __fmul_rn(__fdiv_rn((float)threadIdx.x, 255.f), 255.f);
  __syncthreads();
  const PatchJob jb = jobs[blockIdx.x];
  const int fs = nchans / 64;
  const int cs = threadIdx.x & 63;
  const int ti = blockIdx.y * 4 + (threadIdx.x >> 6);
  const uint8_t* fb = tf + (size_t)jb.unit * nsamps * nchans + (size_t)cs * fs;
  const long long t0 = jb.ft_first + (long long)ti * jb.ft_ts;
  const long long lo = t0 > 0 ? t0 : 0;
  const long long end = t0 + (long long)jb.ft_ts;
  const long long hi = end < (long long)nsamps ? end : (long long)nsamps;
  float sum = 0.f;
  for (long long t = lo; t < hi; t++) {
    const uint8_t* row = fb + (size_t)t * nchans;
    for (int f = 0; f < fs; f++) sum = __fadd_rn(sum, lut[row[f]]);
  }
  const float npix = (float)((size_t)jb.ft_ts * (size_t)fs);
  out[(size_t)blockIdx.x * 16384 + cs * 256 + ti] = __fdiv_rn(sum, npix);
}

// k-th smallest (0-based) of v[lo..hi) in shared memory, by ranks
__device__ float warp_kth(const float* v, int lo, int hi, int k) {
  const int lane = threadIdx.x & 31;
  float found = 0.f;
  bool have = false;
  for (int i = lo + lane; i < hi; i += 32) {
    const float x = v[i];
    int lt = 0, le = 0;
    for (int j = lo; j < hi; j++) {
      lt += v[j] < x;
      le += v[j] <= x;
    }
    if (lt <= k && k < le) { found = x; have = true; }
  }
  const unsigned m = __ballot_sync(0xffffffffu, have);
  return __shfl_sync(0xffffffffu, found, m ? __ffs(m) - 1 : 0);
}

// normalise_series_array (candidate_profiler.C:88-134) on rows of n values,
// one warp per row.  A row whose deviation is zero becomes zero for the
// classifier's patches (zero_flat); the profiler keeps the reference's
// arithmetic there (a division by zero: NaN or +-inf).
template <bool ZERO_FLAT>
__global__ void k_normalise_rows_t(float* __restrict__ data, int n, size_t nrows, size_t pitch,
                                   int rows_per_group, size_t group_pitch) {
  extern __shared__ float nr_smem[];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t row = (size_t)blockIdx.x * (blockDim.x >> 5) + wib;
  float* v = nr_smem + (size_t)wib * 2 * n;  // [n] values, [n] scratch
  float* a = v + n;
  if (row >= nrows) return;  // whole warp
  // rows come in groups (e.g. the trials of one candidate's plot)
  float* x = data + (row / rows_per_group) * group_pitch + (row % rows_per_group) * pitch;
  for (int j = lane; j < n; j += 32) v[j] = x[j];
  __syncwarp();
  const float m1 = warp_kth(v, 0, n / 2, n / 4);
  const float m2 = warp_kth(v, n / 2, n, n / 4);
  const double gradient = (double)__fdiv_rn(__fsub_rn(m2, m1), (float)(n / 2));
  const float median0 = (float)((double)m1 - gradient * (double)(n / 4));
  for (int j = lane; j < n; j += 32) {
    const float base = (float)((double)median0 + (double)j * gradient);
    const float y = __fsub_rn(v[j], base);
    v[j] = y;
    a[j] = fabsf(y);
  }
  __syncwarp();
  const float mad = warp_kth(a, 0, n, n / 2);
  const float stddev = (float)((double)mad * 1.4826);
  const float val = (float)(1.0 / (double)stddev);
  for (int j = lane; j < n; j += 32)
    x[j] = (!ZERO_FLAT || stddev > 0.f) ? __fmul_rn(v[j], val) : 0.f;
}

cudaError_t normalise_rows(float* data, int n, size_t nrows, size_t pitch, int rows_per_group,
                           size_t group_pitch, bool zero_flat, cudaStream_t s) {
  if (n < 2 || nrows == 0) return cudaSuccess;
  const size_t smem = 2 * (size_t)n * sizeof(float);
  // rows of up to 1024 values: four warps per block; longer: one
  const int wpb = n <= 1024 ? 4 : 1;
  if (smem * wpb > 200 * 1024) return cudaErrorInvalidValue;
  const void* fn = zero_flat ? reinterpret_cast<const void*>(k_normalise_rows_t<true>)
                             : reinterpret_cast<const void*>(k_normalise_rows_t<false>);
  cudaError_t e = raise_smem_limit(fn, smem * wpb);
  if (e != cudaSuccess) return e;
  const unsigned nb = (unsigned)((nrows + wpb - 1) / wpb);
  if (zero_flat)
    k_normalise_rows_t<true><<<nb, 32 * wpb, smem * wpb, s>>>(data, n, nrows, pitch,
                                                             rows_per_group, group_pitch);
  else
    k_normalise_rows_t<false><<<nb, 32 * wpb, smem * wpb, s>>>(data, n, nrows, pitch,
                                                              rows_per_group, group_pitch);
  note_launch();
  return cudaGetLastError();
}

cudaError_t extract_patches(const float* scan, size_t scan_pitch, size_t len, const uint8_t* tf,
                            size_t nsamps, int nchans, const PatchJob* jobs, int njobs,
                            float* dm_out, float* ft_out, cudaStream_t s) {
  if (njobs <= 0) return cudaSuccess;
  k_patch_dm<<<njobs, 256, 0, s>>>(scan, scan_pitch, len, jobs, dm_out); note_launch();
  k_patch_ft<<<dim3((unsigned)njobs, 64), 256, 0, s>>>(tf, nsamps, nchans, jobs, ft_out); note_launch();
  const size_t r1 = (size_t)njobs * 64;
  cudaError_t e = normalise_rows(dm_out, 64, r1, 64, 1, 64, true, s);
  if (e == cudaSuccess) e = normalise_rows(ft_out, 256, r1, 256, 1, 256, true, s);
  return e == cudaSuccess ? cudaGetLastError() : e;
}
}  // namespace hdb

// ===========================================================================
// The model
// ===========================================================================
using hdb::clf::bf16;

namespace {

struct ConvSpec {
  int ci, co, h, w;  // input channels, output channels, input rows, cols
  int kw() const { return ci * 9; }
  int kp() const { return (ci * 9 + 15) / 16 * 16; }
};
// branch A: 64 x 64 input; branch B: 64 x 256 input
const ConvSpec kConv[2][3] = {{{1, 8, 64, 64}, {8, 16, 32, 32}, {16, 32, 16, 16}},
                              {{1, 8, 64, 256}, {8, 16, 32, 128}, {16, 32, 16, 64}}};
constexpr int kFeat = 10240, kHid = 16;

struct DBuf {
  void* p = nullptr;
  size_t cap = 0;
  ~DBuf() { if (p) cudaFree(p); }
  template <class T> T* as() { return reinterpret_cast<T*>(p); }
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = hdb::dev_malloc(&p, std::max<size_t>(bytes, 256));
    if (e == cudaSuccess) cap = std::max<size_t>(bytes, 256);
    return e;
  }
};

}  // namespace

struct hd_classifier_t {
  int device = 0;
  cudaStream_t stream = nullptr;
  // flat FP32 parameters: per conv layer W [co][ci*9] then b [co], branch A
  // then B, then W1 [16][10240], b1 [16], W2 [2][16], b2 [2]
  size_t off_w[2][3], off_b[2][3], off_w1, off_b1, off_w2, off_b2, nparam;
  DBuf w, g, m, v;          // parameters, gradients, Adam moments
  DBuf wb_conv[2][3], wb1;  // BF16 weight copies
  bool bf16_stale = true;   // the FP32 weights changed since the BF16 copies
  long long step = 0;
  // per-batch work buffers
  int cap_batch = 0;
  DBuf in[2], col, z, act[2][3], arg[2][3], dz, dcol, dact_a[2], dact_b[2], x, z1, h, dz1,
      dx, prob, loss, labels, idx, hs;
  DBuf tc_ws, tc_err;               // tensor-core GEMM: split-K workspace, error word
  DBuf data_dm, data_ft, data_lab;  // resident training set
  DBuf stage_dm, stage_ft, sprob;    // scoring: host patches staged in FP32, scores
  int nsm = 0;
  size_t data_n = 0;
  cudaEvent_t ev[2] = {};  // around the last scoring call, on `stream`
  float score_ms = 0.f;

  ~hd_classifier_t() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

using namespace hdb::clf;

#define CK(x)                                               \
  do {                                                      \
    cudaError_t e_ = (x);                                   \
    if (e_ != cudaSuccess) return e_;                       \
  } while (0)

cudaError_t alloc_batch(hd_classifier c, int nb) {
  if (nb <= c->cap_batch) return cudaSuccess;
  size_t maxcol = 0, maxz = 0;
  for (int br = 0; br < 2; br++)
    for (int l = 0; l < 3; l++) {
      const ConvSpec& s = kConv[br][l];
      const size_t P = (size_t)nb * s.h * s.w;
      maxcol = std::max(maxcol, (size_t)s.kp() * P);
      maxz = std::max(maxz, (size_t)s.co * P);
      CK(c->act[br][l].ensure((size_t)s.co * P / 4 * sizeof(bf16)));
      CK(c->arg[br][l].ensure((size_t)s.co * P / 4));
    }
  CK(c->in[0].ensure((size_t)nb * 64 * 64 * sizeof(bf16)));
  CK(c->in[1].ensure((size_t)nb * 64 * 256 * sizeof(bf16)));
  CK(c->col.ensure(maxcol * sizeof(bf16)));
  CK(c->dcol.ensure(maxcol * sizeof(float)));
  CK(c->z.ensure(maxz * sizeof(float)));
  CK(c->dz.ensure(maxz * sizeof(bf16)));
  for (int br = 0; br < 2; br++) {
    CK(c->dact_a[br].ensure(maxz / 4 * sizeof(float)));
    CK(c->dact_b[br].ensure(maxz / 4 * sizeof(float)));
  }
  CK(c->x.ensure((size_t)nb * kFeat * sizeof(bf16)));
  CK(c->dx.ensure((size_t)nb * kFeat * sizeof(float)));
  CK(c->z1.ensure((size_t)nb * kHid * sizeof(float)));
  CK(c->h.ensure((size_t)nb * kHid * sizeof(float)));
  CK(c->dz1.ensure((size_t)nb * kHid * sizeof(bf16)));
  CK(c->prob.ensure((size_t)nb * sizeof(float)));
  CK(c->hs.ensure((size_t)nb * kHeadTerms * sizeof(float)));
  CK(c->loss.ensure(sizeof(float)));
  CK(c->labels.ensure((size_t)nb * sizeof(int)));
  CK(c->idx.ensure((size_t)nb * sizeof(int)));
  c->cap_batch = nb;
  return cudaSuccess;
}

cudaError_t refresh_bf16(hd_classifier c) {
  if (!c->bf16_stale) return cudaSuccess;
  c->bf16_stale = false;
  cudaStream_t s = c->stream;
  float* w = c->w.as<float>();
  for (int br = 0; br < 2; br++)
    for (int l = 0; l < 3; l++) {
      const ConvSpec& sp = kConv[br][l];
      CK(c->wb_conv[br][l].ensure((size_t)sp.co * sp.kp() * sizeof(bf16)));
      k_weights_bf16<<<nblk((size_t)sp.co * sp.kp()), 256, 0, s>>>(
          w + c->off_w[br][l], sp.co, sp.kw(), sp.kp(), c->wb_conv[br][l].as<bf16>()); hdb::note_launch();
    }
  CK(c->wb1.ensure((size_t)kHid * kFeat * sizeof(bf16)));
  k_to_bf16<<<nblk((size_t)kHid * kFeat), 256, 0, s>>>(w + c->off_w1, c->wb1.as<bf16>(),
                                                       (size_t)kHid * kFeat); hdb::note_launch();
  return cudaGetLastError();
}

// C(m, n) (+)= sum_k A[m*lda + k] B[n*ldb + k] on the tcgen05 tensor cores
// (umma_gemm): both operands K-major; split K over `splits` CTAs per tile
// column, the splits added in order through c->tc_ws.
cudaError_t tc_gemm(hd_classifier c, int M, int N, int K, const bf16* A, long long lda,
                    const bf16* B, long long ldb, float* C, long long scm, long long scn,
                    int accumulate, int splits) {
  const size_t ws = hdb::umma_workspace_floats(M, N, K, splits);
  CK(c->tc_ws.ensure(std::max<size_t>(ws, 1) * sizeof(float)));
  CK(c->tc_err.ensure(sizeof(unsigned)));
  return hdb::umma_gemm(M, N, K, A, lda, B, ldb, C, scm, scn, accumulate, splits,
                        c->tc_ws.as<float>(), c->tc_err.as<unsigned>(), c->stream);
}

// Forward over the batch already in c->in[]; with backward, accumulates the
// gradients of the mean cross-entropy into c->g (which the caller zeroes).
cudaError_t run_batch(hd_classifier c, int nb, bool backward) {
  cudaStream_t s = c->stream;
  float* w = c->w.as<float>();
  float* g = c->g.as<float>();
  CK(refresh_bf16(c));
  // ---- forward ----
  for (int br = 0; br < 2; br++) {
    const bf16* cur = c->in[br].as<bf16>();
    for (int l = 0; l < 3; l++) {
      const ConvSpec& sp = kConv[br][l];
      const size_t P = (size_t)nb * sp.h * sp.w;
      // z [co][P] = W [co][kp] x col: on the tensor cores as z^T [P][co] =
      // colT [P][kp] x W^T, M = P pixels, N = co, K = kp
      k_im2col3_t<<<nblk(P * sp.kp()), 256, 0, s>>>(cur, sp.ci, nb, sp.h, sp.w, sp.kp(),
                                                     c->col.as<bf16>()); hdb::note_launch();
      CK(tc_gemm(c, (int)P, sp.co, sp.kp(), c->col.as<bf16>(), sp.kp(),
                 c->wb_conv[br][l].as<bf16>(), sp.kp(), c->z.as<float>(), 1, (long long)P, 0,
                 1));
      k_bias_relu_pool<<<nblk(P / 4 * sp.co), 256, 0, s>>>(
          c->z.as<float>(), w + c->off_b[br][l], sp.co, nb, sp.h, sp.w,
          c->act[br][l].as<bf16>(), c->arg[br][l].as<unsigned char>()); hdb::note_launch();
      cur = c->act[br][l].as<bf16>();
    }
  }
  k_flatten<<<nblk((size_t)nb * kFeat), 256, 0, s>>>(c->act[0][2].as<bf16>(),
                                                     c->act[1][2].as<bf16>(), nb,
                                                     c->x.as<bf16>()); hdb::note_launch();
  // z1 [16][b] = W1 x x: z1^T [b][16] = x [b][10240] x W1^T, K split over 64
  CK(tc_gemm(c, nb, kHid, kFeat, c->x.as<bf16>(), kFeat, c->wb1.as<bf16>(), kFeat,
             c->z1.as<float>(), 1, nb, 0, 64));
  k_fc1_act<<<nblk((size_t)nb * kHid), 256, 0, s>>>(c->z1.as<float>(), w + c->off_b1, nb,
                                                    c->h.as<float>()); hdb::note_launch();
  if (backward) CK(cudaMemsetAsync(c->loss.p, 0, sizeof(float), s));
  k_head<<<nblk(nb, 128), 128, 0, s>>>(c->h.as<float>(), w + c->off_w2, w + c->off_b2,
                                       c->labels.as<int>(), nb, backward ? 1 : 0,
                                       c->prob.as<float>(), c->dz1.as<bf16>(),
                                       c->hs.as<float>()); hdb::note_launch();
  if (!backward) return cudaGetLastError();
  k_head_reduce<<<1, 64, 0, s>>>(c->h.as<float>(), c->hs.as<float>(), nb, c->loss.as<float>(),
                                 g + c->off_w2, g + c->off_b2, g + c->off_b1); hdb::note_launch();
  // ---- backward ----
  {
    // dW1 [16][10240] += dz1 [16][b] x x [b][10240]
    GemmArgs ga{kHid, kFeat, nb, c->dz1.as<bf16>(), nb, 1, c->x.as<bf16>(), kFeat, 1,
                g + c->off_w1, kFeat, 1, 1, 0};
    CK(gemm(ga, 1, s));
    // dx [b][10240] = dz1^T x W1
    GemmArgs gd{kFeat, nb, kHid, c->wb1.as<bf16>(), 1, kFeat, c->dz1.as<bf16>(), nb, 1,
                c->dx.as<float>(), 1, kFeat, 0, 0};
    CK(gemm(gd, 1, s));
  }
  k_unflatten<<<nblk((size_t)nb * kFeat), 256, 0, s>>>(c->dx.as<float>(), nb,
                                                       c->dact_a[0].as<float>(),
                                                       c->dact_a[1].as<float>()); hdb::note_launch();
  for (int br = 0; br < 2; br++) {
    float* dcur = c->dact_a[br].as<float>();   // gradient of this layer's pooled output
    float* dnext = c->dact_b[br].as<float>();  // gradient of its input
    for (int l = 2; l >= 0; l--) {
      const ConvSpec& sp = kConv[br][l];
      const size_t P = (size_t)nb * sp.h * sp.w;
      k_pool_relu_back<<<nblk(P * sp.co), 256, 0, s>>>(
          dcur, c->act[br][l].as<bf16>(), c->arg[br][l].as<unsigned char>(), sp.co, nb, sp.h,
          sp.w, c->dz.as<bf16>(), g + c->off_b[br][l]); hdb::note_launch();
      k_bias_grad<<<sp.co, 256, 0, s>>>(dcur, c->act[br][l].as<bf16>(),
                                        c->arg[br][l].as<unsigned char>(), nb, sp.h, sp.w,
                                        g + c->off_b[br][l]); hdb::note_launch();
      // the layer's input again, as im2col (recomputed rather than stored)
      const bf16* lin = l == 0 ? c->in[br].as<bf16>() : c->act[br][l - 1].as<bf16>();
      k_im2col3<<<nblk(P * sp.kp()), 256, 0, s>>>(lin, sp.ci, nb, sp.h, sp.w, sp.kp(),
                                                   c->col.as<bf16>()); hdb::note_launch();
      // dW [co][kw] += dz [co][P] x col^T; the padded columns kw..kp are dropped
      // by writing into a [co][kp] scratch is avoided: N = kw with row stride kw
      // on the tensor cores as dW^T [kw][co] += col [kw][P] x dz^T: M = kw
      // taps, N = co, K = P pixels split over the SMs; the splits are added
      // in order (the same gradient every run)
      const int splits = (int)std::min<size_t>(296, (P + 8191) / 8192);
      CK(tc_gemm(c, sp.kw(), sp.co, (int)P, c->col.as<bf16>(), (long long)P, c->dz.as<bf16>(),
                 (long long)P, g + c->off_w[br][l], 1, sp.kw(), 1, splits));
      if (l > 0) {
        // dcol [kp][P] = W^T x dz, then col2im into the previous layer's output gradient
        GemmArgs gd{sp.kp(), (int)P, sp.co, c->wb_conv[br][l].as<bf16>(), 1, sp.kp(),
                    c->dz.as<bf16>(), (long long)P, 1, c->dcol.as<float>(), (long long)P, 1, 0, 0};
        CK(gemm(gd, 1, s));
        k_col2im3<<<nblk(P * sp.ci), 256, 0, s>>>(c->dcol.as<float>(), sp.ci, nb, sp.h, sp.w,
                                                 dnext); hdb::note_launch();
        std::swap(dcur, dnext);
      }
    }
  }
  return cudaGetLastError();
}

cudaError_t upload_patches(hd_classifier c, const float* dm, const float* ft, int nb) {
  cudaStream_t s = c->stream;
  // host floats -> device BF16 through a temporary FP32 copy in dcol
  CK(c->dcol.ensure((size_t)nb * 16384 * sizeof(float)));
  CK(cudaMemcpyAsync(c->dcol.p, dm, (size_t)nb * 4096 * sizeof(float), cudaMemcpyHostToDevice, s));
  k_input_bf16<<<nblk((size_t)nb * 4096), 256, 0, s>>>(c->dcol.as<float>(), c->in[0].as<bf16>(),
                                                       (size_t)nb * 4096); hdb::note_launch();
  CK(cudaMemcpyAsync(c->dcol.p, ft, (size_t)nb * 16384 * sizeof(float), cudaMemcpyHostToDevice, s));
  k_input_bf16<<<nblk((size_t)nb * 16384), 256, 0, s>>>(c->dcol.as<float>(), c->in[1].as<bf16>(),
                                                        (size_t)nb * 16384); hdb::note_launch();
  return cudaGetLastError();
}

// The fused inference kernel over n device FP32 patch pairs -> d_prob.
cudaError_t infer(hd_classifier c, const float* d_dm, const float* d_ft, size_t n, float* d_prob) {
  cudaStream_t s = c->stream;
  if (n > 0x7FFFFFFFull) return cudaErrorInvalidValue;
  CK(refresh_bf16(c));
  if (c->nsm == 0) {
    CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device));
    CK(cudaFuncSetAttribute(hdb::inf::k_clf_infer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)hdb::inf::kSmem));
  }
  hdb::inf::Args a{};
  a.dm = d_dm;
  a.ft = d_ft;
  a.n = (int)n;
  a.w = c->w.as<float>();
  for (int br = 0; br < 2; br++)
    for (int l = 0; l < 3; l++) {
      a.off_w[br][l] = (int)c->off_w[br][l];
      a.off_b[br][l] = (int)c->off_b[br][l];
    }
  a.off_b1 = (int)c->off_b1;
  a.off_w2 = (int)c->off_w2;
  a.off_b2 = (int)c->off_b2;
  a.wb1 = c->wb1.as<bf16>();
  a.prob = d_prob;
  const unsigned grid = (unsigned)std::min<size_t>(n, (size_t)c->nsm);
  hdb::inf::k_clf_infer<<<grid, hdb::inf::kThreads, hdb::inf::kSmem, s>>>(a); hdb::note_launch();
  return cudaGetLastError();
}

// Scores of n patch pairs (device FP32, or host FP32 staged in chunks); after
// `after` (an event on another stream, or null) when the patches come from
// that stream.  Device time between the events ev[0] and ev[1].
constexpr size_t kStageChunk = 2048;
cudaError_t score_batches(hd_classifier c, const float* dm, const float* ft, size_t n,
                          bool on_device, cudaEvent_t after, float* scores) {
  cudaStream_t s = c->stream;
  if (after) CK(cudaStreamWaitEvent(s, after, 0));
  CK(cudaEventRecord(c->ev[0], s));
  if (on_device) {
    CK(c->sprob.ensure(n * sizeof(float)));
    CK(infer(c, dm, ft, n, c->sprob.as<float>()));
    CK(cudaMemcpyAsync(scores, c->sprob.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
  } else {
    const size_t ch = std::min(n, kStageChunk);
    CK(c->stage_dm.ensure(ch * 4096 * sizeof(float)));
    CK(c->stage_ft.ensure(ch * 16384 * sizeof(float)));
    CK(c->sprob.ensure(ch * sizeof(float)));
    for (size_t i0 = 0; i0 < n; i0 += ch) {
      // the staging buffers are reused by the next chunk, whose copies are
      // ordered after this chunk's kernel on the same stream
      const size_t k = std::min(ch, n - i0);
      CK(cudaMemcpyAsync(c->stage_dm.p, dm + i0 * 4096, k * 4096 * sizeof(float),
                         cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(c->stage_ft.p, ft + i0 * 16384, k * 16384 * sizeof(float),
                         cudaMemcpyHostToDevice, s));
      CK(infer(c, c->stage_dm.as<float>(), c->stage_ft.as<float>(), k, c->sprob.as<float>()));
      CK(cudaMemcpyAsync(scores + i0, c->sprob.p, k * sizeof(float), cudaMemcpyDeviceToHost, s));
    }
  }
  CK(cudaEventRecord(c->ev[1], s));
  CK(cudaStreamSynchronize(s));
  return cudaEventElapsedTime(&c->score_ms, c->ev[0], c->ev[1]);
}

// the tensor-core GEMM's error word: zeroed before a run, read after it
cudaError_t tc_reset(hd_classifier c) {
  CK(c->tc_err.ensure(sizeof(unsigned)));
  return cudaMemsetAsync(c->tc_err.p, 0, sizeof(unsigned), c->stream);
}
cudaError_t tc_check(hd_classifier c) {
  unsigned v = 0;
  CK(cudaMemcpy(&v, c->tc_err.p, sizeof(unsigned), cudaMemcpyDeviceToHost));
  return v ? cudaErrorLaunchTimeout : cudaSuccess;
}

hd_error to_hd(cudaError_t e) {
  if (e == cudaSuccess) return HD_NO_ERROR;
  if (e == cudaErrorMemoryAllocation) return HD_MEM_ALLOC_FAILED;
  return HD_INTERNAL_GPU_ERROR;
}

}  // namespace

extern "C" {

hd_size hd_classifier_param_count(void) {
  size_t n = 0;
  for (int br = 0; br < 2; br++)
    for (int l = 0; l < 3; l++) n += (size_t)kConv[br][l].co * kConv[br][l].kw() + kConv[br][l].co;
  return n + (size_t)kHid * kFeat + kHid + 2 * kHid + 2;
}

hd_error hd_classifier_create(hd_classifier* out, int gpu_id, unsigned long long seed) {
  if (!out) return HD_INVALID_POINTER;
  *out = nullptr;
  if (cudaSetDevice(gpu_id) != cudaSuccess) return HD_INVALID_DEVICE_INDEX;
  hd_classifier c = new (std::nothrow) hd_classifier_t();
  if (!c) return HD_MEM_ALLOC_FAILED;
  c->device = gpu_id;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev[0]) != cudaSuccess || cudaEventCreate(&c->ev[1]) != cudaSuccess) {
    delete c;
    return HD_PRIOR_GPU_ERROR;
  }
  size_t o = 0;
  for (int br = 0; br < 2; br++)
    for (int l = 0; l < 3; l++) {
      c->off_w[br][l] = o; o += (size_t)kConv[br][l].co * kConv[br][l].kw();
      c->off_b[br][l] = o; o += kConv[br][l].co;
    }
  c->off_w1 = o; o += (size_t)kHid * kFeat;
  c->off_b1 = o; o += kHid;
  c->off_w2 = o; o += 2 * kHid;
  c->off_b2 = o; o += 2;
  c->nparam = o;
  // He-normal initial weights (std sqrt(2 / fan_in)), zero conv biases
  std::vector<float> h(o, 0.f);
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  auto fill = [&](size_t off, size_t n, int fan_in) {
    const float sd = std::sqrt(2.f / (float)fan_in);
    for (size_t i = 0; i < n; i++) h[off + i] = nd(rng) * sd;
  };
  for (int br = 0; br < 2; br++)
    for (int l = 0; l < 3; l++)
      fill(c->off_w[br][l], (size_t)kConv[br][l].co * kConv[br][l].kw(), kConv[br][l].kw());
  fill(c->off_w1, (size_t)kHid * kFeat, kFeat);
  fill(c->off_w2, 2 * kHid, kHid);
  // small positive FC1 biases keep the 16 hidden units active at the start
  for (int o = 0; o < kHid; o++) h[c->off_b1 + o] = 0.1f;
  cudaError_t e = c->w.ensure(o * sizeof(float));
  if (e == cudaSuccess) e = c->g.ensure(o * sizeof(float));
  if (e == cudaSuccess) e = c->m.ensure(o * sizeof(float));
  if (e == cudaSuccess) e = c->v.ensure(o * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(c->w.p, h.data(), o * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(c->m.p, 0, o * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(c->v.p, 0, o * sizeof(float));
  if (e != cudaSuccess) {
    delete c;
    return to_hd(e);
  }
  *out = c;
  return HD_NO_ERROR;
}

void hd_classifier_destroy(hd_classifier c) {
  if (!c) return;
  cudaSetDevice(c->device);
  delete c;
}

hd_error hd_classifier_get_params(hd_classifier c, float* params, hd_size count) {
  if (!c) return HD_INVALID_PIPELINE;
  if (!params || count != c->nparam) return HD_INVALID_POINTER;
  cudaSetDevice(c->device);
  return to_hd(cudaMemcpy(params, c->w.p, c->nparam * sizeof(float), cudaMemcpyDeviceToHost));
}

hd_error hd_classifier_set_params(hd_classifier c, const float* params, hd_size count) {
  if (!c) return HD_INVALID_PIPELINE;
  if (!params || count != c->nparam) return HD_INVALID_POINTER;
  cudaSetDevice(c->device);
  c->bf16_stale = true;
  c->step = 0;
  cudaError_t e = cudaMemcpy(c->w.p, params, c->nparam * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(c->m.p, 0, c->nparam * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(c->v.p, 0, c->nparam * sizeof(float));
  return to_hd(e);
}

hd_error hd_classifier_gradients(hd_classifier c, const float* dm_time, const float* freq_time,
                                 const int* labels, hd_size n, float* grads, float* loss) {
  if (!c) return HD_INVALID_PIPELINE;
  if (!dm_time || !freq_time || !labels || n == 0 || n > 4096) return HD_INVALID_POINTER;
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  cudaError_t e = alloc_batch(c, (int)n);
  if (e == cudaSuccess) e = tc_reset(c);
  if (e == cudaSuccess) e = upload_patches(c, dm_time, freq_time, (int)n);
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->labels.p, labels, n * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->g.p, 0, c->nparam * sizeof(float), s);
  if (e == cudaSuccess) e = run_batch(c, (int)n, true);
  if (e == cudaSuccess && grads)
    e = cudaMemcpyAsync(grads, c->g.p, c->nparam * sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && loss) e = cudaMemcpyAsync(loss, c->loss.p, sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = tc_check(c);
  return to_hd(e);
}

hd_error hd_classifier_train(hd_classifier c, const float* dm_time, const float* freq_time,
                             const int* labels, hd_size n, int epochs, int batch, float lr,
                             unsigned long long seed, float* epoch_loss) {
  if (!c) return HD_INVALID_PIPELINE;
  if (!dm_time || !freq_time || !labels || n == 0 || epochs <= 0 || batch <= 0 || batch > 4096)
    return HD_INVALID_POINTER;
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  const int nb = (int)std::min<size_t>(batch, n);
  cudaError_t e = alloc_batch(c, nb);
  if (e == cudaSuccess) e = tc_reset(c);
  // the training set stays on the device in BF16
  if (e == cudaSuccess) e = c->data_dm.ensure(n * 4096 * sizeof(bf16));
  if (e == cudaSuccess) e = c->data_ft.ensure(n * 16384 * sizeof(bf16));
  if (e == cudaSuccess) e = c->data_lab.ensure(n * sizeof(int));
  if (e != cudaSuccess) return to_hd(e);
  for (size_t i0 = 0; i0 < n && e == cudaSuccess; i0 += (size_t)nb) {
    const int k = (int)std::min<size_t>(nb, n - i0);
    e = upload_patches(c, dm_time + i0 * 4096, freq_time + i0 * 16384, k);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(c->data_dm.as<bf16>() + i0 * 4096, c->in[0].p, (size_t)k * 4096 * sizeof(bf16),
                          cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(c->data_ft.as<bf16>() + i0 * 16384, c->in[1].p, (size_t)k * 16384 * sizeof(bf16),
                          cudaMemcpyDeviceToDevice, s);
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c->data_lab.p, labels, n * sizeof(int), cudaMemcpyHostToDevice, s);
  std::vector<int> order(n);
  for (size_t i = 0; i < n; i++) order[i] = (int)i;
  std::mt19937_64 rng(seed);
  std::vector<int> bidx(nb);
  for (int ep = 0; ep < epochs && e == cudaSuccess; ep++) {
    std::shuffle(order.begin(), order.end(), rng);
    double lsum = 0.0;
    int nbatches = 0;
    for (size_t i0 = 0; i0 + (size_t)nb <= n && e == cudaSuccess; i0 += (size_t)nb) {
      for (int j = 0; j < nb; j++) bidx[j] = order[i0 + j];
      e = cudaMemcpyAsync(c->idx.p, bidx.data(), nb * sizeof(int), cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) break;
      k_gather<<<nblk((size_t)nb * 4096), 256, 0, s>>>(c->data_dm.as<bf16>(), c->idx.as<int>(), nb, 4096,
                                                       c->in[0].as<bf16>()); hdb::note_launch();
      k_gather<<<nblk((size_t)nb * 16384), 256, 0, s>>>(c->data_ft.as<bf16>(), c->idx.as<int>(), nb, 16384,
                                                        c->in[1].as<bf16>()); hdb::note_launch();
      // labels of the batch (gather of one int per sample)
      {
        std::vector<int> hl(nb);
        for (int j = 0; j < nb; j++) hl[j] = labels[bidx[j]];
        e = cudaMemcpyAsync(c->labels.p, hl.data(), nb * sizeof(int), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // hl and bidx are reused
      }
      if (e == cudaSuccess) e = cudaMemsetAsync(c->g.p, 0, c->nparam * sizeof(float), s);
      if (e == cudaSuccess) e = run_batch(c, nb, true);
      if (e != cudaSuccess) break;
      c->step++;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.f - (float)std::pow(b1, (double)c->step);
      const float c2 = 1.f - (float)std::pow(b2, (double)c->step);
      c->bf16_stale = true;
      k_adam<<<nblk(c->nparam), 256, 0, s>>>(c->w.as<float>(), c->g.as<float>(), c->m.as<float>(),
                                             c->v.as<float>(), c->nparam, lr, b1, b2, 1e-8f, c1, c2); hdb::note_launch();
      float l = 0.f;
      e = cudaMemcpyAsync(&l, c->loss.p, sizeof(float), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      lsum += l;
      nbatches++;
    }
    if (epoch_loss) epoch_loss[ep] = nbatches ? (float)(lsum / nbatches) : 0.f;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = tc_check(c);
  return to_hd(e);
}

hd_error hd_classifier_score(hd_classifier c, const float* dm_time, const float* freq_time,
                             hd_size n, float* scores) {
  if (!c) return HD_INVALID_PIPELINE;
  if (!dm_time || !freq_time || !scores) return HD_INVALID_POINTER;
  if (n == 0) return HD_NO_ERROR;
  cudaSetDevice(c->device);
  return to_hd(score_batches(c, dm_time, freq_time, n, false, nullptr, scores));
}

hd_error hd_classifier_score_device(hd_classifier c, const float* d_dm_time,
                                    const float* d_freq_time, hd_size n, float* scores) {
  if (!c) return HD_INVALID_PIPELINE;
  if (!d_dm_time || !d_freq_time || !scores) return HD_INVALID_POINTER;
  if (n == 0) return HD_NO_ERROR;
  cudaSetDevice(c->device);
  return to_hd(score_batches(c, d_dm_time, d_freq_time, n, true, nullptr, scores));
}

hd_error hd_classifier_get_timing(hd_classifier c, float* ms) {
  if (!c) return HD_INVALID_PIPELINE;
  if (!ms) return HD_INVALID_POINTER;
  *ms = c->score_ms;
  return HD_NO_ERROR;
}

hd_error hd_bf16_gemm_tc(int m, int n, int k, const void* d_a, long long sam, long long sak,
                         const void* d_b, long long sbk, long long sbn, float* d_c,
                         long long scm, long long scn, int accumulate, int splits) {
  if (!d_a || !d_b || !d_c) return HD_INVALID_POINTER;
  if (sak != 1 || sbk != 1) return HD_INVALID_STRIDE;
  float* ws = nullptr;
  unsigned* err = nullptr;
  const size_t nws = hdb::umma_workspace_floats(m, n, k, splits);
  cudaError_t e = hdb::dev_malloc(&err, sizeof(unsigned));
  if (e == cudaSuccess && nws) e = hdb::dev_malloc(&ws, nws * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(err, 0, sizeof(unsigned));
  if (e == cudaSuccess)
    e = hdb::umma_gemm(m, n, k, d_a, sam, d_b, sbn, d_c, scm, scn, accumulate, splits, ws, err, 0);
  hd_error he = HD_NO_ERROR;
  if (e == cudaErrorNotSupported) he = HD_INVALID_STRIDE;
  else if (e == cudaSuccess) e = cudaDeviceSynchronize();
  unsigned v = 0;
  if (he == HD_NO_ERROR && e == cudaSuccess) {
    e = cudaMemcpy(&v, err, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && v) he = HD_INTERNAL_GPU_ERROR;
  }
  if (he == HD_NO_ERROR) he = to_hd(e);
  if (ws) cudaFree(ws);
  if (err) cudaFree(err);
  return he;
}

hd_error hd_bf16_gemm(int m, int n, int k, const void* d_a, long long sam, long long sak,
                      const void* d_b, long long sbk, long long sbn, float* d_c, long long scm,
                      long long scn, int accumulate, int splits) {
  if (!d_a || !d_b || !d_c) return HD_INVALID_POINTER;
  GemmArgs a{m, n, k, static_cast<const bf16*>(d_a), sam, sak, static_cast<const bf16*>(d_b),
             sbk, sbn, d_c, scm, scn, accumulate, 0};
  cudaError_t e = gemm(a, splits, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return to_hd(e);
}

}  // extern "C"

namespace hdb {
cudaError_t classifier_score_device(hd_classifier c, const float* d_dm, const float* d_ft,
                                    size_t n, cudaEvent_t after, float* scores) {
  if (n == 0) return cudaSuccess;
  return score_batches(c, d_dm, d_ft, n, true, after, scores);
}
int classifier_device(hd_classifier c) { return c->device; }
}  // namespace hdb
