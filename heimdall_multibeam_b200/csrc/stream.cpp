// stream.cpp -- sigproc filterbank input and the gulp loop with overlap carry.
//
//   hd_read_sigproc_header   Formats/hd/header.h:133-198 (read_header) and
//                            Formats/SigprocFile.C:16-51
//   hd_params_from_sigproc   the data-source fields Applications/heimdall.C:
//                            103-119 copies into hd_params, with
//                            Formats/hd/DataSource.h:49-82 (mjd2utctm)
//   hd_search_sigproc_file   the gulp loop of Applications/heimdall.C:153-292
//
// The loop keeps the overlap on the device: two device buffers alternate, the
// overlap of each beam is copied device to device from the one just searched
// into the next, and only the new block crosses PCIe.  While the GPU searches
// the current gulp, a host thread reads the next block from the file into
// pinned memory (in parallel pieces) and copies it, with the overlap carry,
// into the other device buffer on a separate stream.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <string>
#include <thread>
#include <vector>

#include <sys/stat.h>
#include <unistd.h>

#include <cuda_runtime.h>

#include "heimdall_b200.h"
#include "internal.h"

namespace {

// One header string: a 4-byte length (1..79) and the characters
// (header.h:120-129).
bool read_str(FILE* f, std::string& s) {
  int len = 0;
  if (std::fread(&len, sizeof(int), 1, f) != 1) return false;
  if (len <= 0 || len >= 80) return false;
  char buf[80];
  if (std::fread(buf, 1, (size_t)len, f) != (size_t)len) return false;
  s.assign(buf, (size_t)len);
  return true;
}

template <class T>
bool read_val(FILE* f, T& v) {
  return std::fread(&v, sizeof(T), 1, f) == 1;
}

void copy_str(char* dst, const std::string& s) {
  const size_t n = std::min<size_t>(s.size(), 79);
  std::memcpy(dst, s.data(), n);
  dst[n] = '\0';
}

// Days since the start of the Julian period of a Julian day number -> civil
// date, by the integer algorithm of Fliegel and Van Flandern (Comm. ACM 11,
// 657, 1968).
void jd_to_civil(long jd, int& year, int& month, int& day) {
  long l = jd + 68569;
  const long n = 4 * l / 146097;
  l = l - (146097 * n + 3) / 4;
  const long i = 4000 * (l + 1) / 1461001;
  l = l - 1461 * i / 4 + 31;
  const long j = 80 * l / 2447;
  day = (int)(l - 2447 * j / 80);
  l = j / 11;
  month = (int)(j + 2 - 12 * l);
  year = (int)(100 * (n - 49) + i + l);
}

}  // namespace

extern "C" {

hd_error hd_read_sigproc_header(const char* path, hd_sigproc_header* h) {
  if (!path || !h) return HD_INVALID_POINTER;
  FILE* f = std::fopen(path, "rb");
  if (!f) return HD_INVALID_POINTER;
  std::memset(h, 0, sizeof(*h));
  std::string s;
  if (!read_str(f, s) || s != "HEADER_START") {
    std::fclose(f);
    return HD_UNKNOWN_ERROR;
  }
  bool want_source = false, want_raw = false, ok = true;
  for (;;) {
    if (!read_str(f, s)) {
      ok = false;
      break;
    }
    if (s == "HEADER_END") break;
    if (s == "source_name") want_source = true;
    else if (s == "rawdatafile") want_raw = true;
    else if (s == "az_start") ok = read_val(f, h->az_start);
    else if (s == "za_start") ok = read_val(f, h->za_start);
    else if (s == "src_raj") ok = read_val(f, h->src_raj);
    else if (s == "src_dej") ok = read_val(f, h->src_dej);
    else if (s == "tstart") ok = read_val(f, h->tstart);
    else if (s == "tsamp") ok = read_val(f, h->tsamp);
    else if (s == "period") ok = read_val(f, h->period);
    else if (s == "fch1") ok = read_val(f, h->fch1);
    else if (s == "foff") ok = read_val(f, h->foff);
    else if (s == "nchans") ok = read_val(f, h->nchans);
    else if (s == "telescope_id") ok = read_val(f, h->telescope_id);
    else if (s == "machine_id") ok = read_val(f, h->machine_id);
    else if (s == "data_type") ok = read_val(f, h->data_type);
    else if (s == "ibeam") ok = read_val(f, h->ibeam);
    else if (s == "nbeams") ok = read_val(f, h->nbeams);
    else if (s == "nbits") ok = read_val(f, h->nbits);
    else if (s == "barycentric") ok = read_val(f, h->barycentric);
    else if (s == "pulsarcentric") ok = read_val(f, h->pulsarcentric);
    else if (s == "nbins") ok = read_val(f, h->nbins);
    else if (s == "nsamples") ok = read_val(f, h->nsamples);
    else if (s == "nifs") ok = read_val(f, h->nifs);
    else if (s == "npuls") ok = read_val(f, h->npuls);
    else if (s == "refdm") ok = read_val(f, h->refdm);
    else if (s == "signed") ok = read_val(f, h->signed_data);
    else if (want_source) {
      copy_str(h->source_name, s);
      want_source = false;
    } else if (want_raw) {
      copy_str(h->rawdatafile, s);
      want_raw = false;
    } else {
      h->unknown_keys++;  // the reference warns and carries on
    }
    if (!ok) break;
  }
  if (!ok) {
    std::fclose(f);
    return HD_UNKNOWN_ERROR;
  }
  h->size = (int)std::ftell(f);
  if (h->nsamples == 0 && h->nchans > 0 && h->nbits > 0) {
    // header.h:190-193: the whole file's size (header included) over the
    // bytes of one spectrum
    std::fseek(f, 0, SEEK_END);
    const long long fsize = (long long)std::ftell(f);
    h->nsamples = (int)(fsize / h->nchans * 8 / h->nbits);
  }
  std::fclose(f);
  return HD_NO_ERROR;
}

long long hd_mjd_to_utc(double mjd) {
  // DataSource.h:49-82: whole seconds of the day, one second added when the
  // fraction left is below 1 (always, as written), the civil date of the
  // Julian day, and mktime in the local time zone
  const int days = (int)mjd;
  const double fdays = mjd - (double)days;
  const double seconds = fdays * 86400.0;
  int secs = (int)seconds;
  const double fracsec = seconds - (double)secs;
  if (fracsec - 1 < 0.0000001) secs++;
  int year = 0, month = 0, day = 0;
  jd_to_civil((long)days + 2400001L, year, month, day);
  struct tm t;
  std::memset(&t, 0, sizeof(t));
  t.tm_year = year - 1900;
  t.tm_mon = month - 1;
  t.tm_mday = day;
  t.tm_hour = secs / 3600;
  secs -= 3600 * t.tm_hour;
  t.tm_min = secs / 60;
  secs -= 60 * t.tm_min;
  t.tm_sec = secs;
  t.tm_isdst = -1;
  return (long long)std::mktime(&t);
}

hd_error hd_params_from_sigproc(const hd_sigproc_header* h, struct hd_params* p) {
  if (!h || !p) return HD_INVALID_POINTER;
  if (h->nchans <= 0 || h->tsamp <= 0.0) return HD_INVALID_STRIDE;
  p->nchans = (hd_size)h->nchans;
  p->dt = (hd_float)h->tsamp;
  p->f0 = (hd_float)h->fch1;
  p->df = (hd_float)h->foff;
  p->nbeams = h->nbeams > 0 ? (hd_size)h->nbeams : 1;
  if (!p->override_beam) p->beam = h->ibeam > 0 ? (hd_size)(h->ibeam - 1) : 0;
  p->utc_start = (time_t)hd_mjd_to_utc(h->tstart);
  // the data source keeps tsamp as a float and its rate as 1 / that float
  // (SigprocFile.C:38-39, DataSource.h:90)
  const float ts = (float)h->tsamp;
  const double rate = 1 / ts;
  p->spectra_per_second = (hd_size)rate;
  return HD_NO_ERROR;
}

}  // extern "C"

namespace {

// The gulp loop over nfiles files read in lockstep.  File u is unit u of
// each gulp: one file is searched with hd_execute_device, several with one
// hd_execute_beams call per gulp.  Every file has the same header fields
// that shape the search (channels, bits, sampling time, band, beams per
// file); the first short block of any file ends the loop.
hd_error search_files(hd_pipeline pl, const char* const* paths, size_t nfiles,
                      hd_size nsamps_gulp, hd_gulp_callback on_gulp, void* user,
                      hd_size* total_nsamps, hd_size* ngulps) {
  if (!pl) return HD_INVALID_PIPELINE;
  if (!paths || nfiles == 0) return HD_INVALID_POINTER;
  for (size_t u = 0; u < nfiles; u++)
    if (!paths[u]) return HD_INVALID_POINTER;
  std::vector<hd_sigproc_header> hs(nfiles);
  for (size_t u = 0; u < nfiles; u++) {
    const hd_error e = hd_read_sigproc_header(paths[u], &hs[u]);
    if (e != HD_NO_ERROR) return e;
  }
  const hd_sigproc_header& h = hs[0];
  // the sample widths hd_execute takes (packed files: see hd_execute)
  if (h.nbits != 1 && h.nbits != 2 && h.nbits != 4 && h.nbits != 8 && h.nbits != 16)
    return HD_INVALID_NBITS;
  if (((size_t)h.nchans * (size_t)h.nbits) % 32 != 0) return HD_INVALID_STRIDE;
  for (size_t u = 1; u < nfiles; u++) {
    const hd_sigproc_header& g = hs[u];
    if (g.nbits != h.nbits || g.nchans != h.nchans || g.tsamp != h.tsamp || g.fch1 != h.fch1 ||
        g.foff != h.foff || g.nbeams != h.nbeams)
      return HD_INVALID_STRIDE;
  }
  const size_t nbeams = h.nbeams > 0 ? (size_t)h.nbeams : 1;
  const size_t nbits = (size_t)h.nbits;
  const size_t stride = (size_t)h.nchans * nbits / 8;  // bytes per spectrum
  if (nsamps_gulp == 0 || nsamps_gulp % nbeams != 0) return HD_INVALID_STRIDE;
  if (cudaSetDevice(hdb::pipeline_device(pl)) != cudaSuccess) return HD_INVALID_DEVICE_INDEX;
  std::vector<FILE*> fs(nfiles, nullptr);
  for (size_t u = 0; u < nfiles; u++) {
    fs[u] = std::fopen(paths[u], "rb");
    if (!fs[u]) {
      for (FILE* f : fs) if (f) std::fclose(f);
      return HD_INVALID_POINTER;
    }
  }

  const size_t max_overlap = hd_get_max_overlap(pl, nbeams);  // all beams of a file
  const size_t M = hd_get_max_overlap(pl, 1);  // per beam: boxcar_max + max delay
  const int dev = hdb::pipeline_device(pl);
  const size_t cap = (nsamps_gulp + max_overlap) * stride;  // one file's region
  const size_t block = nsamps_gulp * stride;
  hd_byte* d_buf[2] = {nullptr, nullptr};
  hd_byte* h_blk[2] = {nullptr, nullptr};
  cudaStream_t cs = nullptr;  // copies into the next gulp's buffer
  auto cleanup = [&]() {
    if (cs) cudaStreamSynchronize(cs);
    for (auto p : d_buf) if (p) cudaFree(p);
    for (auto p : h_blk) if (p) cudaFreeHost(p);
    if (cs) cudaStreamDestroy(cs);
    for (FILE* f : fs) std::fclose(f);
  };
  if (hdb::dev_malloc(&d_buf[0], nfiles * cap) != cudaSuccess ||
      hdb::dev_malloc(&d_buf[1], nfiles * cap) != cudaSuccess ||
      cudaMallocHost(&h_blk[0], nfiles * block) != cudaSuccess ||
      cudaMallocHost(&h_blk[1], nfiles * block) != cudaSuccess ||
      cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
    cleanup();
    return HD_MEM_ALLOC_FAILED;
  }
  // SigprocFile.C:59-68 reads up to a block of whole spectra.  Here each
  // block's bytes are read by up to 8 threads at disjoint offsets (positioned
  // reads), which a single stream read cannot keep up with at gulp sizes.
  std::vector<size_t> pos(nfiles), file_size(nfiles);
  for (size_t u = 0; u < nfiles; u++) {
    struct stat st;
    file_size[u] = fstat(fileno(fs[u]), &st) == 0 ? (size_t)st.st_size : 0;
    pos[u] = (size_t)hs[u].size;
  }
  auto read_one = [&](size_t u, hd_byte* dst) -> size_t {
    const int fd = fileno(fs[u]);
    const size_t want =
        std::min(block, file_size[u] > pos[u] ? file_size[u] - pos[u] : (size_t)0);
    const size_t nt = std::min<size_t>(8, std::max<size_t>(1, want >> 23));
    const size_t base = pos[u];
    std::atomic<bool> ok{true};
    std::vector<std::thread> th;
    for (size_t i = 0; i < nt; i++)
      th.emplace_back([&, i]() {
        size_t lo = want * i / nt;
        const size_t hi = want * (i + 1) / nt;
        while (lo < hi) {
          const ssize_t r = pread(fd, dst + lo, hi - lo, (off_t)(base + lo));
          if (r <= 0) {
            ok = false;
            return;
          }
          lo += (size_t)r;
        }
      });
    for (auto& t : th) t.join();
    pos[u] += want;
    return ok ? want / stride : 0;  // a read error ends the loop
  };
  // the next block of every file into h_blk[hb] (file u at u * block), up
  // to 16 files at a time; the fewest whole spectra any file gave
  auto read_blocks = [&](int hb_) -> size_t {
    std::vector<size_t> got(nfiles, 0);
    const size_t nw = std::min<size_t>(16, nfiles);
    if (nw == 1) {
      got[0] = read_one(0, h_blk[hb_]);
    } else {
      std::vector<std::thread> th;
      for (size_t i = 0; i < nw; i++)
        th.emplace_back([&, i]() {
          for (size_t u = i; u < nfiles; u += nw) got[u] = read_one(u, h_blk[hb_] + u * block);
        });
      for (auto& t : th) t.join();
    }
    size_t least = block / stride;
    for (size_t u = 0; u < nfiles; u++) least = std::min(least, got[u]);
    return least;
  };
  // heimdall.C:209-265: the next gulp of file u holds, beam by beam, the
  // last `ov` spectra of that beam's region in the gulp just searched
  // (per_beam spectra each, in d_buf[from]) followed by the beam's part of
  // the file's new block (pinned h_blk[hb_new]).  The searched buffer is
  // only read.
  auto stage_next = [&](int from, int hb_new, size_t per_beam, size_t ov) -> bool {
    const int to_buf = from ^ 1;
    const size_t done_pb = per_beam - ov;
    const size_t next_pb = ov + nsamps_gulp / nbeams;
    for (size_t u = 0; u < nfiles; u++) {
      hd_byte* dst = d_buf[to_buf] + u * cap;
      const hd_byte* src = d_buf[from] + u * cap;
      const hd_byte* blk = h_blk[hb_new] + u * block;
      for (size_t b = 0; b < nbeams && ov > 0; b++)
        if (cudaMemcpyAsync(dst + b * next_pb * stride, src + (b * per_beam + done_pb) * stride,
                            ov * stride, cudaMemcpyDeviceToDevice, cs) != cudaSuccess)
          return false;
      for (size_t b = 0; b < nbeams; b++) {
        const size_t lo = b * nsamps_gulp / nbeams;
        const size_t hi = (b + 1) * nsamps_gulp / nbeams;
        if (cudaMemcpyAsync(dst + (ov + b * next_pb) * stride, blk + lo * stride,
                            (hi - lo) * stride, cudaMemcpyHostToDevice, cs) != cudaSuccess)
          return false;
      }
    }
    return true;
  };

  // the first block of every file is searched as it is (overlap 0)
  size_t nsamps_read = read_blocks(0);
  int cur = 0, hb = 0;
  size_t overlap = 0;      // per beam
  size_t total = 0;        // samples per beam searched so far
  size_t gulps = 0;
  std::vector<hd_candidate> cands;
  std::vector<const hd_byte*> units(nfiles);
  std::vector<hd_error> statuses(nfiles);
  hd_error result = HD_NO_ERROR;
  bool stop = nsamps_read < nsamps_gulp;  // a short first block is never searched
  // the first blocks land at the start of each file's region of buffer 0
  for (size_t u = 0; u < nfiles && !stop; u++)
    if (cudaMemcpyAsync(d_buf[0] + u * cap, h_blk[0] + u * block, block, cudaMemcpyHostToDevice,
                        cs) != cudaSuccess) {
      cleanup();
      return HD_MEM_COPY_FAILED;
    }
  while (nsamps_read && !stop) {
    // this gulp's spectra are in d_buf[cur]
    if (cudaStreamSynchronize(cs) != cudaSuccess) {
      result = HD_MEM_COPY_FAILED;
      break;
    }
    const size_t to_process = nsamps_gulp + overlap * nbeams;
    const size_t per_beam = to_process / nbeams;
    // the overlap this search leaves: hd_execute sets nsamps_processed =
    // nsamps - nbeams * M before any kernel runs (0 below that)
    const size_t ov_pred = to_process >= nbeams * M ? M : per_beam;
    // while the GPU searches this gulp, a host thread reads the next blocks
    // and stages the next gulp (overlap carry and new blocks) on the copy stream
    size_t next_read = 0;
    bool staged = false;
    std::thread reader([&]() {
      next_read = read_blocks(hb ^ 1);
      if (next_read < nsamps_gulp || cudaSetDevice(dev) != cudaSuccess) return;
      staged = stage_next(cur, hb ^ 1, per_beam, ov_pred);
    });
    hd_size processed = 0;
    hd_error e;
    if (nfiles == 1) {
      e = hd_execute_device(pl, d_buf[cur], to_process, nbits, total, nbeams, &processed);
    } else {
      for (size_t u = 0; u < nfiles; u++) units[u] = d_buf[cur] + u * cap;
      e = hd_execute_beams(pl, units.data(), nfiles, to_process, nbits, total, nbeams, nullptr, 1,
                           statuses.data(), &processed);
    }
    reader.join();
    if (e != HD_NO_ERROR && e != HD_TOO_MANY_EVENTS) {
      result = e;
      break;
    }
    gulps++;
    hd_size n = 0;
    hd_get_candidates(pl, nullptr, &n);
    cands.resize(n);
    if (n) hd_get_candidates(pl, cands.data(), &n);
    if (on_gulp) on_gulp(user, cands.data(), n, (hd_size)total);
    overlap = (to_process - processed) / nbeams;
    total += processed / nbeams;
    nsamps_read = next_read;
    hb ^= 1;
    // a short block ends the search (heimdall.C:269-272,285-287)
    if (nsamps_read < nsamps_gulp) break;
    if (!staged || overlap != ov_pred) {
      // the staging did not happen or assumed another overlap: place the
      // next gulp again once the copy stream is idle
      if (cudaStreamSynchronize(cs) != cudaSuccess || !stage_next(cur, hb, per_beam, overlap)) {
        result = HD_MEM_COPY_FAILED;
        break;
      }
    }
    cur ^= 1;
  }
  cleanup();
  if (total_nsamps) *total_nsamps = total;
  if (ngulps) *ngulps = gulps;
  return result;
}

}  // namespace

extern "C" {

hd_error hd_search_sigproc_file(hd_pipeline pl, const char* path, hd_size nsamps_gulp,
                                hd_gulp_callback on_gulp, void* user, hd_size* total_nsamps,
                                hd_size* ngulps) {
  if (!pl) return HD_INVALID_PIPELINE;
  if (!path) return HD_INVALID_POINTER;
  return search_files(pl, &path, 1, nsamps_gulp, on_gulp, user, total_nsamps, ngulps);
}

hd_error hd_search_sigproc_files(hd_pipeline pl, const char* const* paths, hd_size nfiles,
                                 hd_size nsamps_gulp, hd_gulp_callback on_gulp, void* user,
                                 hd_size* total_nsamps, hd_size* ngulps) {
  return search_files(pl, paths, nfiles, nsamps_gulp, on_gulp, user, total_nsamps, ngulps);
}

}  // extern "C"
