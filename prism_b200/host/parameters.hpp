// Configuration of a PRISM run: the reference's prism_context and flag parser
// (include/utils/parameters.hpp:8-60, src/utils/parameters.cu), restated over
// the prism_b200 C ABI.  Same flags, defaults and file-name conventions:
//   -i <path>   original data            -z [path]  compress (default <in>.prisma)
//   -x [path]   decompress (default <cmp>.out)      -f / -d float / double
//   -1 nx | -2 nx ny | -3 nx ny nz (x fastest)      -A eb | -R rel_eb
//   -prog       negabinary planes for progressive retrieval
//   -errors -K e1 .. eK   progressive targets       --report time,cr
// Differences: errors are reported and returned instead of exit(); -4 and
// -PW_R are rejected (the reference documents -4 but never parses it and
// leaves PW_REL unimplemented).
#pragma once
#include <stdint.h>
#include <string>
#include <vector>

enum prism_dtype_e { F4 = 4, F8 = 8 };
enum prism_mode_e { ABS = 0, REL = 1 };
enum btype_e { NB = 0, SM = 1 };

struct interpolation_parameters {
  double alpha{1.75};
  double beta{4.0};
  bool use_md[4]{true, true, true, true};
  bool use_natural[4]{false, false, false, false};
  bool reverse[4]{false, false, false, false};
};

struct prism_context {
  double eb{0.0};
  double rel_eb{0.0};
  int ndim{-1};
  uint32_t x{1}, y{1}, z{1};
  uint64_t size{1};
  bool isComp{false};
  bool isDecomp{false};
  prism_dtype_e dtype{F4};
  prism_mode_e error_mode{REL};
  std::string oriFilePath, cmpFilePath, decFilePath;
  int compMode{0};
  bool report_time{false};
  bool report_cr{false};
  btype_e bt{SM};
  std::vector<double> target_ebs;
  interpolation_parameters intp_param;
};
using context = prism_context;

void usage();
// returns 0 on success, nonzero (and prints why) on a bad command line
int parse_argv(prism_context* config, int argc, char** argv);
