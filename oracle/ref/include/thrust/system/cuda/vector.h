/* Build shim: Pipeline/hd/cached_allocator.cuh:10,55,90,113 names the CUDA
 * system's tag, malloc, free and pointer.  For the host (OpenMP) build of the
 * reference these map onto the OpenMP system, so the reference's custom
 * temporary allocator keeps working unchanged. */
#pragma once
#include <thrust/system/omp/vector.h>
#include <thrust/system/omp/memory.h>
namespace thrust { namespace system { namespace cuda {
  using tag = thrust::system::omp::tag;
  using thrust::system::omp::malloc;
  using thrust::system::omp::free;
  template <typename T> using pointer = thrust::system::omp::pointer<T>;
}}}
