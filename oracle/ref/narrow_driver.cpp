/* narrow_driver.cpp -- TEST INFRASTRUCTURE ONLY: the reference's narrow-band
 * RFI branch (Pipeline/clean_filterbank_rfi.cu:303-351, which the reference
 * disables at :303) run with the reference's own code: measure_bandpass from
 * the built library, and zap_narrow_rfi_functor compiled here from
 * clean_filterbank_rfi.cu where it lies, inside a namespace of its own (the
 * file's headers are included first, so their guards keep them out of it).
 * The functor is applied to the words in index order, which fixes the
 * result of its in-place reads (with Thrust's parallel for_each it depends
 * on thread timing). */
#include <algorithm>
#include <cstddef>
#include <stdio.h>
#include <vector>

#include "hd/clean_filterbank_rfi.h"
#include "hd/remove_baseline.h"
#include "hd/get_rms.h"
#include "hd/measure_bandpass.h"
#include "hd/matched_filter.h"
#include <dedisp.h>
#include <thrust/host_vector.h>
#include <thrust/device_vector.h>
#include <thrust/random.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/constant_iterator.h>

namespace ref_cfr {
#include "clean_filterbank_rfi.cu"
}

extern "C" int ref_measure_bandpass(const unsigned char* fb, size_t nsamps, size_t nchans,
                                    float* bandpass, float* rms) {
  return (int)measure_bandpass(fb, nsamps, nchans, 8, bandpass, rms);
}

extern "C" int ref_narrow_band(unsigned char* data, size_t nsamps, size_t nchans, float dt,
                               float baseline_length, float rfi_tol) {
  typedef unsigned int WordType;
  const size_t stride = nchans * 8 / 8 / sizeof(WordType);
  const size_t max_chan_resample_dist = nchans / 60;
  const size_t nsamps_smooth = (size_t)(baseline_length / (1 * dt));
  if (nsamps_smooth == 0) return -1;
  std::vector<float> bp(nchans);
  for (size_t g = 0; g < nsamps; g += nsamps_smooth) {
    const size_t ng = std::min(nsamps_smooth, nsamps - g);
    float rms = 0;
    measure_bandpass(data + g * nchans, ng, nchans, 8, bp.data(), &rms);
    ref_cfr::zap_narrow_rfi_functor<WordType> zapit((WordType*)data, bp.data(), rfi_tol * rms,
                                                   (unsigned)stride, 8, (unsigned)nchans,
                                                   (unsigned)max_chan_resample_dist);
    for (size_t i = g * stride; i < (g + ng) * stride; i++) zapit((unsigned)i);
  }
  return 0;
}
