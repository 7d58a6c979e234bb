// coinc_driver.cpp -- test infrastructure: runs the reference's own
// coincidencer logic (Applications/Candidates.C: CandidateChunk reading
// .cand files, compute_coincidence, write_coincident_candidates) on the
// files given.  Usage: coinc_ref nbeams sep_time sep_filter file...
// The _all.cand file goes to the current directory, named after the first
// file's UTC prefix, as the reference writes it.
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "hd/Candidates.h"

int main(int argc, char** argv) {
  if (argc < 5) return 2;
  const unsigned nbeams = (unsigned)std::atoi(argv[1]);
  const unsigned sep_time = (unsigned)std::atoi(argv[2]);
  const unsigned sep_filter = (unsigned)std::atoi(argv[3]);
  CandidateChunk chunk(nbeams, argc, 4, argv);
  chunk.compute_coincidence(sep_time, sep_filter);
  chunk.write_coincident_candidates();
  return 0;
}
