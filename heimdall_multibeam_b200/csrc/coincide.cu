// coincide.cu -- cross-beam coincidence of candidate lists
// (Applications/Candidates.C: Candidate::is_coincident 64-77,
// CandidateChunk::compute_coincidence 236-291, write_coincident_candidates
// 293-326, operator<< 85-93).
//
// Every candidate j of beam i looks, beam by beam (k = 0, 1, ... except i),
// for the first candidate l of beam k in list order that is coincident with
// it: |sample_idx difference| <= sep_time * 2^max(filter), |filter
// difference| <= sep_filter, |dm_trial difference| <= 9999 and
// |snr_l - snr_j| / (snr_l + snr_j) <= 0.4 (float arithmetic).  Each such
// beam adds one to j's beam count; if snr_l is above the largest S/N seen so
// far, l's beam becomes j's primary beam and snr_l its max_snr.  One thread
// per candidate; the lists of all beams sit in one array grouped by beam in
// their input order.
#include <algorithm>
#include <cstdio>
#include <vector>

#include <cuda_runtime.h>

#include "heimdall_b200.h"
#include "internal.h"

namespace {

struct CoincCand {
  long long samp;
  float snr;
  unsigned filter, dm_trial, beam, group;
};

__device__ __forceinline__ bool coincident(const CoincCand& self, const CoincCand& c,
                                           unsigned sep_time, unsigned sep_filter) {
  // tol = sep_time * powf(2, max(filter)) in float, truncated to 64 bits;
  // 2^n is exact as ldexpf(1, n)
  const unsigned fmax = max(c.filter, self.filter);
  const float p2 = ldexpf(1.0f, (int)min(fmax, 127u));
  const long long tol = (long long)__fmul_rn((float)sep_time, p2);
  const long long dt = c.samp - self.samp;
  if ((dt < 0 ? -dt : dt) > tol) return false;
  const int ddm = (int)c.dm_trial - (int)self.dm_trial;
  if ((unsigned long long)(ddm < 0 ? -ddm : ddm) > 9999ull) return false;
  const int dfl = (int)c.filter - (int)self.filter;
  if ((unsigned)(dfl < 0 ? -dfl : dfl) > sep_filter) return false;
  const float r = __fdiv_rn(fabsf(__fsub_rn(c.snr, self.snr)), __fadd_rn(c.snr, self.snr));
  return r <= 0.4f;
}

__global__ void k_coincide(const CoincCand* __restrict__ c, const unsigned* __restrict__ first,
                           int nbeams, int n, unsigned sep_time, unsigned sep_filter,
                           unsigned* __restrict__ nb_out, unsigned* __restrict__ prim_out,
                           float* __restrict__ max_out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const CoincCand self = c[j];
  unsigned nb = 1, prim = self.beam;
  float best = self.snr;
  for (int k = 0; k < nbeams; k++) {
    if ((unsigned)k == self.group) continue;
    for (unsigned l = first[k]; l < first[k + 1]; l++) {
      const CoincCand o = c[l];
      if (coincident(self, o, sep_time, sep_filter)) {
        nb++;
        if (o.snr > best) {
          prim = o.beam;
          best = o.snr;
        }
        break;
      }
    }
  }
  nb_out[j] = nb;
  prim_out[j] = prim;
  max_out[j] = best;
}

hd_error to_hd(cudaError_t e) {
  if (e == cudaSuccess) return HD_NO_ERROR;
  if (e == cudaErrorMemoryAllocation) return HD_MEM_ALLOC_FAILED;
  if (e == cudaErrorInvalidDevice) return HD_INVALID_DEVICE_INDEX;
  return HD_INTERNAL_GPU_ERROR;
}

// beam-grouped order of the candidates: beam 1 first, input order within a beam
std::vector<size_t> beam_order(const hd_candidate* cands, size_t n) {
  std::vector<size_t> order(n);
  for (size_t i = 0; i < n; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t a, size_t b) { return cands[a].beam < cands[b].beam; });
  return order;
}

}  // namespace

extern "C" {

hd_error hd_coincide(const hd_candidate* cands, hd_size n, hd_size nbeams, unsigned sep_time,
                     unsigned sep_filter, int gpu_id, hd_coincidence* out) {
  if (n == 0) return HD_NO_ERROR;
  if (!cands || !out) return HD_INVALID_POINTER;
  if (nbeams == 0 || nbeams > 0x7FFFFFFF || n > 0x7FFFFFFF) return HD_INVALID_STRIDE;
  for (size_t i = 0; i < n; i++)
    if (cands[i].beam < 1 || cands[i].beam > nbeams) return HD_INVALID_STRIDE;
  if (cudaSetDevice(gpu_id) != cudaSuccess) return HD_INVALID_DEVICE_INDEX;
  const std::vector<size_t> order = beam_order(cands, n);
  std::vector<CoincCand> h(n);
  std::vector<unsigned> first(nbeams + 1, 0);
  for (size_t r = 0; r < n; r++) {
    const hd_candidate& c = cands[order[r]];
    h[r] = CoincCand{(long long)c.samp_idx, c.snr, (unsigned)c.filter, (unsigned)c.dm_trial,
                     (unsigned)c.beam, (unsigned)(c.beam - 1)};
    first[c.beam]++;
  }
  for (size_t b = 0; b < nbeams; b++) first[b + 1] += first[b];
  CoincCand* d_c = nullptr;
  unsigned *d_first = nullptr, *d_nb = nullptr, *d_prim = nullptr;
  float* d_max = nullptr;
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = hdb::dev_malloc(&d_c, n * sizeof(CoincCand));
  if (e == cudaSuccess) e = hdb::dev_malloc(&d_first, (nbeams + 1) * sizeof(unsigned));
  if (e == cudaSuccess) e = hdb::dev_malloc(&d_nb, n * sizeof(unsigned));
  if (e == cudaSuccess) e = hdb::dev_malloc(&d_prim, n * sizeof(unsigned));
  if (e == cudaSuccess) e = hdb::dev_malloc(&d_max, n * sizeof(float));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_c, h.data(), n * sizeof(CoincCand), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_first, first.data(), (nbeams + 1) * sizeof(unsigned),
                        cudaMemcpyHostToDevice, s);
  std::vector<unsigned> nb(n), prim(n);
  std::vector<float> mx(n);
  if (e == cudaSuccess) {
    k_coincide<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(d_c, d_first, (int)nbeams, (int)n,
                                                          sep_time, sep_filter, d_nb, d_prim,
                                                          d_max);
    hdb::note_launch();
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(nb.data(), d_nb, n * sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(prim.data(), d_prim, n * sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(mx.data(), d_max, n * sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(d_c);
  cudaFree(d_first);
  cudaFree(d_nb);
  cudaFree(d_prim);
  cudaFree(d_max);
  if (s) cudaStreamDestroy(s);
  if (e != cudaSuccess) return to_hd(e);
  for (size_t r = 0; r < n; r++) {
    hd_coincidence& o = out[order[r]];
    o.nbeams = nb[r];
    o.primary_beam = prim[r];
    o.max_snr = mx[r];
  }
  return HD_NO_ERROR;
}

hd_error hd_write_coincident_candidates(const char* path, const hd_candidate* cands,
                                        const hd_coincidence* co, hd_size n) {
  if (!path) return HD_INVALID_POINTER;
  if (n && (!cands || !co)) return HD_INVALID_POINTER;
  FILE* f = std::fopen(path, "w");
  if (!f) return HD_INVALID_POINTER;
  // beam by beam, input order within a beam (CandidateChunk keeps one list per beam)
  for (size_t r : beam_order(cands, n)) {
    const hd_candidate& c = cands[r];
    const hd_coincidence& o = co[r];
    std::fprintf(f, "%g\t%lld\t%g\t%u\t%u\t%g\t%u\t%lld\t%lld\t%u\t\t%u\t%g\t%u\n", c.snr,
                 (long long)c.samp_idx, c.time, (unsigned)c.filter, (unsigned)c.dm_trial, c.dm,
                 (unsigned)c.members, (long long)c.begin, (long long)c.end, o.nbeams,
                 o.primary_beam, o.max_snr, (unsigned)c.beam);
  }
  std::fclose(f);
  return HD_NO_ERROR;
}

}  // extern "C"
