// sigproc_dump.cpp -- test infrastructure: prints, as one JSON object, the
// header the reference's own reader gets from a sigproc file
// (Formats/hd/header.h:133-198, read_header) and the reference's MJD -> Unix
// time conversion (Formats/hd/DataSource.h:49-82, mjd2utctm) for the MJDs
// given after the file name.  Built from the reference's headers where they
// lie (oracle/Makefile, target ref); only the tests run it.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>

#include "hd/header.h"
#include "hd/DataSource.h"

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  std::ifstream f(argv[1], std::ios::binary);
  SigprocHeader h;
  const bool ok = read_header(f, h);
  std::printf("{\"ok\": %s, \"source_name\": \"%s\", \"rawdatafile\": \"%s\", ", ok ? "true" : "false",
              h.source_name.c_str(), h.rawdatafile.c_str());
  std::printf("\"az_start\": %.17g, \"za_start\": %.17g, \"src_raj\": %.17g, \"src_dej\": %.17g, ",
              h.az_start, h.za_start, h.src_raj, h.src_dej);
  std::printf("\"tstart\": %.17g, \"tsamp\": %.17g, \"period\": %.17g, \"fch1\": %.17g, ", h.tstart,
              h.tsamp, h.period, h.fch1);
  std::printf("\"foff\": %.17g, \"refdm\": %.17g, ", h.foff, h.refdm);
  std::printf("\"nchans\": %d, \"telescope_id\": %d, \"machine_id\": %d, \"data_type\": %d, ",
              h.nchans, h.telescope_id, h.machine_id, h.data_type);
  std::printf("\"ibeam\": %d, \"nbeams\": %d, \"nbits\": %d, \"barycentric\": %d, ", h.ibeam,
              h.nbeams, h.nbits, h.barycentric);
  std::printf("\"pulsarcentric\": %d, \"nbins\": %d, \"nsamples\": %d, \"nifs\": %d, ",
              h.pulsarcentric, h.nbins, h.nsamples, h.nifs);
  std::printf("\"npuls\": %d, \"signed_data\": %d, \"size\": %d, \"utc\": [", h.npuls,
              (int)h.signed_data, ok ? h.size : -1);
  for (int i = 2; i < argc; i++)
    std::printf("%s%lld", i > 2 ? ", " : "", (long long)DataSource::mjd2utctm(std::atof(argv[i])));
  std::printf("]}\n");
  return 0;
}
