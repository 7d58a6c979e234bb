// params.cpp -- defaults, command-line parsing and error strings of the hd_*
// interface (Pipeline/default_params.C:10-66, Pipeline/parse_command_line.C:
// 23-188, Pipeline/error.C:15-59).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "heimdall_b200.h"

extern "C" {

void hd_set_default_params(hd_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->verbosity = 0;
  p->sigproc_file = nullptr;
  p->yield_cpu = false;
  p->nsamps_gulp = 262144;
  p->dm_gulp_size = 2048;
  p->baseline_length = 2.0f;
  p->beam = 0;
  p->nbeams = 1;
  p->override_beam = false;
  p->nchans = 1024;
  p->dt = 64e-6f;
  p->f0 = 1581.804688f;
  p->df = -.390625f;
  p->dm_min = 0.0f;
  p->dm_max = 1000.0f;
  p->dm_tol = 1.25f;
  p->dm_pulse_width = 40;
  p->dm_nbits = 32;
  // adaptive time resolution, as the reference defaults
  p->use_scrunching = true;
  p->scrunch_tol = 1.15f;
  p->rfi_tol = 5.0f;
  p->rfi_min_beams = 8;
  p->boxcar_max = 4096;
  p->detect_thresh = 6.0f;
  p->cand_sep_time = 3;
  p->cand_sep_filter = 3;
  p->cand_sep_dm = 200;
  p->cand_rfi_dm_cut = 1;  // 1.5 stored in an integer field, as in the reference
  p->max_giant_rate = 0;
  p->min_tscrunch_width = 4096;
  p->num_channel_zaps = 0;
  p->channel_zaps = nullptr;
  p->coincidencer_host = nullptr;
  p->coincidencer_port = -1;
  p->beam_count = 13;
  p->gpu_id = 0;
  p->utc_start = 0;
  p->spectra_per_second = 0;
  p->output_dir = ".";
}

void hd_print_usage(void) {
  hd_params p;
  hd_set_default_params(&p);
  printf("Usage: heimdall [options]\n");
  printf("    -k  key                  use PSRDADA hexidecimal key\n");
  printf("    -vVgG                    increase verbosity level\n");
  printf("    -yield_cpu               TBA\n");
  printf("    -gpu_id ID               run on specified GPU\n");
  printf("    -nsamps_gulp num         number of samples to be read at a time [%zu]\n",
         (size_t)p.nsamps_gulp);
  printf("    -baseline_length num     TBA\n");
  printf("    -beam ##                 over-ride beam number\n");
  printf("    -nbeams ##               give number of beams [def 1]\n");
  printf("    -output_dir path         create all output files in specified path\n");
  printf("    -dm min max              min and max DM\n");
  printf("    -dm_tol num              smear tolerance factor between DM trials [%g]\n",
         (double)p.dm_tol);
  printf("    -coincidencer host:port  connect to the coincidencer on the specified host and port\n");
  printf("    -zap_chans start end     zap all channels between start and end channels inclusive\n");
  printf("    -max_giant_rate nevents  limit the maximum number of individual detections per minute to nevents\n");
  printf("    -dm_pulse_width num      expected minimum pulse width [default %g]\n",
         (double)p.dm_pulse_width);
  printf("    -dm_nbits num            number of bits in dedispersed time series\n");
  printf("    -scrunching              use adaptive dm-dependent time scrunching\n");
  printf("    -scrunching_tol num      TBA\n");
  printf("    -rfi_tol num             TBA\n");
  printf("    -rfi_min_beams num       TBA\n");
  printf("    -boxcar_max num          TBA\n");
  printf("    -min_tscrunch_width num  vary between high quality (large value) and high performance (low value)\n");
}

static char* dup_str(const char* s) {
  size_t n = std::strlen(s) + 1;
  char* d = static_cast<char*>(std::malloc(n));
  if (d) std::memcpy(d, s, n);
  return d;
}

int hd_parse_command_line(int argc, char* argv[], hd_params* params) {
  size_t i = 0;
  auto is = [&](const char* f) { return std::strcmp(argv[i], f) == 0; };
  auto next = [&]() -> const char* { return (i + 1 < (size_t)argc) ? argv[++i] : "0"; };
  auto vmax = [&](int v) { if (params->verbosity < v) params->verbosity = v; };
  while (++i < (size_t)argc) {
    if (is("-h")) { hd_print_usage(); return -1; }
    if (is("-v")) vmax(1);
    else if (is("-V")) vmax(2);
    else if (is("-g")) vmax(3);
    else if (is("-G")) vmax(4);
#ifdef HAVE_PSRDADA
    else if (is("-k")) sscanf(next(), "%x", (unsigned*)&params->dada_id);
#endif
    else if (is("-f")) params->sigproc_file = dup_str(next());
    else if (is("-yield_cpu")) params->yield_cpu = atoi(next()) != 0;
    else if (is("-nsamps_gulp")) params->nsamps_gulp = atoi(next());
    else if (is("-baseline_length")) params->baseline_length = (float)atof(next());
    else if (is("-dm")) {
      params->dm_min = (float)atof(next());
      params->dm_max = (float)atof(next());
    }
    else if (is("-dm_tol")) params->dm_tol = (float)atof(next());
    else if (is("-dm_pulse_width")) params->dm_pulse_width = (float)atof(next());
    else if (is("-dm_nbits")) params->dm_nbits = atoi(next());
    else if (is("-gpu_id")) params->gpu_id = atoi(next());
    else if (is("-scrunching")) params->use_scrunching = atoi(next()) != 0;
    else if (is("-scrunch_tol")) params->scrunch_tol = (float)atof(next());
    else if (is("-rfi_tol")) params->rfi_tol = (float)atof(next());
    else if (is("-rfi_min_beams")) params->rfi_min_beams = atoi(next());
    else if (is("-boxcar_max")) params->boxcar_max = atoi(next());
    else if (is("-detect_thresh")) params->detect_thresh = (float)atof(next());
    else if (is("-beam")) {
      params->beam = (hd_size)(atoi(next()) - 1);
      params->override_beam = true;
    }
    else if (is("-nbeams")) params->nbeams = atoi(next());
    else if (is("-beam_count")) params->beam_count = atoi(next());
    else if (is("-cand_sep_time")) params->cand_sep_time = atoi(next());
    else if (is("-cand_sep_filter")) params->cand_sep_filter = atoi(next());
    else if (is("-cand_sep_dm_trial")) params->cand_sep_dm = atoi(next());
    else if (is("-cand_rfi_dm_cut")) params->cand_rfi_dm_cut = (hd_size)atof(next());
    else if (is("-max_giant_rate")) params->max_giant_rate = (float)atof(next());
    else if (is("-output_dir")) params->output_dir = dup_str(next());
    else if (is("-min_tscrunch_width")) params->min_tscrunch_width = atoi(next());
    else if (is("-coincidencer")) {
      std::string a = next();
      size_t c = a.find(':');
      std::string host = a.substr(0, c);
      std::string port = c == std::string::npos ? "" : a.substr(c + 1);
      params->coincidencer_host = dup_str(host.c_str());
      params->coincidencer_port = atoi(port.c_str());
    }
    else if (is("-zap_chans")) {
      unsigned iz = params->num_channel_zaps;
      hd_range_t* z = static_cast<hd_range_t*>(
          std::realloc(params->channel_zaps, sizeof(hd_range_t) * (iz + 1)));
      if (!z) return -1;
      params->channel_zaps = z;
      params->num_channel_zaps = iz + 1;
      z[iz].start = atoi(next());
      z[iz].end = atoi(next());
    }
    else fprintf(stderr, "WARNING: Unknown parameter '%s'\n", argv[i]);
  }
  if (params->sigproc_file == nullptr) {
#ifdef HAVE_PSRDADA
    if (params->dada_id != 0) return 0;
#endif
    fprintf(stderr, "ERROR: no input mechanism specified\n");
    hd_print_usage();
    return -1;
  }
  return 0;
}

const char* hd_get_error_string(hd_error error) {
  switch (error) {
    case HD_NO_ERROR: return "No error";
    case HD_MEM_ALLOC_FAILED: return "Memory allocation failed";
    case HD_MEM_COPY_FAILED: return "Memory copy failed";
    case HD_INVALID_DEVICE_INDEX: return "Invalid device index";
    case HD_DEVICE_ALREADY_SET: return "Device is already set and cannot be changed";
    case HD_INVALID_PIPELINE: return "Invalid pipeline";
    case HD_INVALID_POINTER: return "Invalid pointer";
    case HD_INVALID_STRIDE: return "Invalid stride";
    case HD_INVALID_NBITS: return "Invalid nbits";
    case HD_TOO_FEW_NSAMPS: return "No. samples < maximum delay";
    case HD_PRIOR_GPU_ERROR: return "Prior GPU error.";
    case HD_INTERNAL_GPU_ERROR: return "Internal GPU error. Please contact the author(s).";
    case HD_TOO_MANY_EVENTS: return "Too many events";
    case HD_UNKNOWN_ERROR: return "Unknown error. Please contact the author(s).";
    default: return "Invalid error code";
  }
}

}  // extern "C"
