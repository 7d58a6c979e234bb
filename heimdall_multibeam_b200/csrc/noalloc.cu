// noalloc.cu -- zero-DM RFI cleaning on caller-owned device buffers without
// any device allocation.
//
// Who needs this: callers that cannot allocate device memory while they run,
// for example a real-time ingest loop in which a cudaMalloc or cudaFree would
// synchronise the whole device and stall the other streams, or a process whose
// device memory is committed up front to a fixed budget.  For them every
// scratch buffer of the cleaning stage lives in one statically sized device
// array that is part of this library, so the call itself never allocates.
//
// Cost and limits: the array (HD_NOALLOC_SCRATCH_BYTES, about 10.6 MiB) is
// reserved on every GPU where this library's device code is loaded and stays
// reserved until the process exits.  It bounds a call to
// HD_NOALLOC_MAX_NSAMPS spectra and HD_NOALLOC_MAX_BEAMS beams.
#include <cstdio>
#include <mutex>

#include "heimdall_b200.h"
#include "internal.h"

namespace {

constexpr size_t kMaxN = HD_NOALLOC_MAX_NSAMPS;
constexpr size_t kMaxBeams = HD_NOALLOC_MAX_BEAMS;
constexpr size_t kAlign = 256;

constexpr size_t up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// Scratch layout (bytes), sized for the largest accepted call.
constexpr size_t kSeriesBytes = up((kMaxN + 64) * sizeof(float));      // zero-DM series
constexpr size_t kScanBytes = up((kMaxN + 64) * sizeof(float));        // its prefix sum
constexpr size_t kFlagBytes = up(128 + kMaxN + 512);                   // width norms + flags
constexpr size_t kRmsBytes = up((kMaxBeams + 16) * sizeof(float));     // per-beam RMS
constexpr size_t kBaseFloats = kMaxN + 64;                             // scrunched baseline
constexpr size_t kBaseBytes = up(kBaseFloats * sizeof(float));
constexpr size_t kTreeFloats = kMaxN + 8 * kMaxBeams + 1024;           // median-tree ping-pong
constexpr size_t kTreeBytes = up(kTreeFloats * sizeof(float));
constexpr size_t kErrBytes = kAlign;                                   // error word
constexpr size_t kTotal = kSeriesBytes + kScanBytes + kFlagBytes + kRmsBytes + kBaseBytes +
                          2 * kTreeBytes + kErrBytes;
static_assert(kTotal <= HD_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the stated size");

// The scratch array.  Host code must not use this name as an address: on the
// host it is only a stand-in for the symbol, so its device address is looked
// up with cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_scratch[HD_NOALLOC_SCRATCH_BYTES];

std::mutex g_mu;
unsigned char* g_dev_addr[64] = {};

// Device address of g_scratch on the current device, looked up once per
// device (the lookup is the only runtime call this set-up makes).  The
// address belongs to the device's primary context: after cudaDeviceReset the
// cached value is stale, so the entry point is not for use after a reset.
hd_error scratch_address(unsigned char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return HD_INVALID_DEVICE_INDEX;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_dev_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) return HD_PRIOR_GPU_ERROR;
    g_dev_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_dev_addr[dev];
  return HD_NO_ERROR;
}

}  // namespace

extern "C" hd_error hd_clean_filterbank_rfi_noalloc(const hd_byte* d_in, hd_size nsamps,
                                                    hd_size nchans, hd_size nbits,
                                                    hd_byte* d_out, int* d_mask, hd_float dt,
                                                    hd_float baseline_length, hd_float rfi_tol,
                                                    hd_size boxcar_max, hd_size nbeams,
                                                    void* stream, unsigned* d_status) {
  if (!d_in || !d_out || !d_mask) return HD_INVALID_POINTER;
  if (nbits != 8) return HD_INVALID_NBITS;
  if (nchans == 0 || nchans % 4 != 0 || nbeams == 0) return HD_INVALID_STRIDE;
  if (nsamps > kMaxN || nbeams > kMaxBeams) {
    fprintf(stderr,
            "hd_clean_filterbank_rfi_noalloc: %zu spectra / %zu beams exceed the fixed "
            "scratch limit of %zu spectra / %zu beams\n",
            (size_t)nsamps, (size_t)nbeams, kMaxN, kMaxBeams);
    return HD_INVALID_STRIDE;
  }
  // one flag bit per boxcar width in a byte: widths 1..128
  if (boxcar_max > 128) {
    fprintf(stderr, "hd_clean_filterbank_rfi_noalloc: boxcar_max %zu exceeds 128\n",
            (size_t)boxcar_max);
    return HD_INVALID_STRIDE;
  }
  const size_t nsmooth = (size_t)(baseline_length / (2 * dt));
  if (nsamps < boxcar_max + 1 || nsmooth / 4 >= nsamps) return HD_TOO_FEW_NSAMPS;
  const size_t stride = nsamps / nbeams;
  const size_t need_base = nbeams * hdb::baseline_samples(stride, nsmooth) + 64;
  const size_t need_tree = hdb::baseline_scratch(stride, nsmooth, nbeams);
  if (need_base > kBaseFloats || need_tree > kTreeFloats) {
    // short beams with a long baseline need more median-tree scratch per
    // spectrum than the fixed array holds
    fprintf(stderr,
            "hd_clean_filterbank_rfi_noalloc: %zu beams of %zu spectra with a %zu-spectrum "
            "baseline need %zu baseline and %zu tree floats; the fixed scratch holds %zu and "
            "%zu\n",
            (size_t)nbeams, stride, nsmooth, need_base, need_tree, kBaseFloats, kTreeFloats);
    return HD_INVALID_STRIDE;
  }

  unsigned char* base = nullptr;
  hd_error he = scratch_address(&base);
  if (he != HD_NO_ERROR) return he;
  float* x = reinterpret_cast<float*>(base);
  float* scan = reinterpret_cast<float*>(base + kSeriesBytes);
  int* flags = reinterpret_cast<int*>(base + kSeriesBytes + kScanBytes);
  float* rms = reinterpret_cast<float*>(base + kSeriesBytes + kScanBytes + kFlagBytes);
  float* bl = reinterpret_cast<float*>(base + kSeriesBytes + kScanBytes + kFlagBytes + kRmsBytes);
  unsigned char* tree = base + kSeriesBytes + kScanBytes + kFlagBytes + kRmsBytes + kBaseBytes;
  hdb::TreeScratch ws{reinterpret_cast<float*>(tree), reinterpret_cast<float*>(tree + kTreeBytes),
                      kTreeFloats};
  unsigned* err = reinterpret_cast<unsigned*>(tree + 2 * kTreeBytes);

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t spitch = (nsamps + 64 + 3) & ~(size_t)3;  // multiple of 4 floats
  // The array keeps the previous call's contents; the series (and the zero
  // the baseline stretch may read after its last sample) and the error word
  // must start at zero.
  if (cudaMemsetAsync(x, 0, spitch * sizeof(float), s) != cudaSuccess ||
      cudaMemsetAsync(err, 0, sizeof(unsigned), s) != cudaSuccess)
    return HD_INTERNAL_GPU_ERROR;
  if (hdb::launch_dm0_sum(d_in, nsamps, (int)nchans, x, s) != cudaSuccess)
    return HD_INTERNAL_GPU_ERROR;
  hdb::SeriesBatch sb{x, spitch, 1, nsamps, stride, stride, (int)nbeams};
  if (hdb::remove_baseline(sb, nsmooth, bl, ws, s) != cudaSuccess ||
      hdb::rms_beams(sb, rms, ws, s) != cudaSuccess ||
      hdb::normalise_scan(sb, rms, scan, spitch, x, s, err) != cudaSuccess ||
      hdb::rfi_mask(x, scan, nsamps, boxcar_max, rfi_tol, d_mask, flags, s) != cudaSuccess ||
      hdb::launch_zap(d_in, nsamps, (int)nchans, d_mask, (unsigned)(nsmooth / 4), nullptr, 0,
                      d_out, s) != cudaSuccess)
    return HD_INTERNAL_GPU_ERROR;
  // the error word, for a caller that reads it once the stream is done
  if (d_status &&
      cudaMemcpyAsync(d_status, err, sizeof(unsigned), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return HD_INTERNAL_GPU_ERROR;
  return HD_NO_ERROR;
}
