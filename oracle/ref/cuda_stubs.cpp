/* Host stand-ins for the CUDA runtime calls the reference's pipeline makes
 * around its Thrust stages (Pipeline/pipeline.cu:54-57,80-124), so the
 * reference stage code can run on Thrust's OpenMP backend without a GPU.
 * TEST INFRASTRUCTURE ONLY. */
#include <cuda_runtime_api.h>

extern "C" {
cudaError_t cudaGetDeviceCount(int* count) { if (count) *count = 1; return cudaSuccess; }
cudaError_t cudaSetDevice(int) { return cudaSuccess; }
cudaError_t cudaSetDeviceFlags(unsigned int) { return cudaSuccess; }
cudaError_t cudaThreadSynchronize(void) { return cudaSuccess; }
const char* cudaGetErrorString(cudaError_t) { return "host stub"; }
}
