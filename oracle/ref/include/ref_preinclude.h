/* Force-included into every reference translation unit of the host build.
 * It supplies what nvcc used to provide implicitly: sequence/transform
 * headers some files forget, unqualified max/min/abs, and host versions of
 * the two device intrinsics the reference calls
 * (Pipeline/label_candidate_clusters.cu:115,371). */
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <thrust/sequence.h>
#include <thrust/transform.h>
#include <thrust/functional.h>
#include <cuda_runtime_api.h>
using std::max;
using std::min;
using std::abs;
#define register
inline unsigned int atomicAdd(unsigned int* p, unsigned int v) {
  unsigned int old;
#pragma omp atomic capture
  { old = *p; *p += v; }
  return old;
}
template <class T>
inline cudaError_t cudaGetSymbolAddress(void** dev_ptr, T& symbol) {
  *dev_ptr = (void*)&symbol;
  return cudaSuccess;
}
