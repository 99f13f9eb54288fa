// Run configuration of the PRISM C++ interface: prism_context, the
// interpolation parameters and the flag parser
// (include/utils/parameters.hpp:8-60 of the reference), with the reference's
// field names and types so that code filling or reading a prism_context
// compiles unchanged.
//
// Flags: -i <path> original data; -z [path] compress (default <in>.prisma);
// -x [path] decompress (default <cmp>.out); -f / -d float / double;
// -1 nx | -2 nx ny | -3 nx ny nz (x fastest); -A eb | -R rel_eb; -prog
// negabinary planes; -errors -K e1 .. eK progressive targets;
// --report time,cr.  The library refuses -cubic natural (it computes the
// default cubic only) and rejects -4 (parsed by no reference code path).
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "err.hpp"
#include "traits.hpp"

struct interpolation_parameters {
  double alpha{1.75};
  double beta{4.0};
  bool use_md[4];
  bool use_natural[4];
  bool reverse[4];
  uint8_t auto_tuning{3};
  interpolation_parameters()
      : use_md{true, true, true, true}, use_natural{false, false, false, false}, reverse{false, false, false, false} {}
};

typedef struct prism_context {
  double eb{0.0};
  double rel_eb{0.0};
  double pw_rel_eb{0.0};
  uint32_t radius{0};
  int ndim{-1};
  uint32_t x{1}, y{1}, z{1}, w{1};
  uint32_t size{1};
  bool isComp{false};
  bool isDecomp{false};
  prism_dtype dtype{F4};
  prism_mode error_mode{REL};
  std::string oriFilePath;
  std::string cmpFilePath;
  std::string decFilePath;
  int blocks_num{1};
  int levels{15};
  int bitgroups{8};
  int compMode{0};
  bool report_time{false};
  bool report_cr{false};
  size_t loaded_size{0};
  btype bt{SM};
  std::vector<double> target_ebs;
  interpolation_parameters intp_param;
  // plane range [begin[i], end[i]) of each level selected by the progressive
  // steps so far; parse_argv allocates them in managed memory (readable on
  // the host, writable with cudaMemset) and sets them to zero
  int* begin{nullptr};
  int* end{nullptr};
} context;

void usage();
// Parses the command line into config; a malformed line prints the reason
// and ends the process (as the reference does).
void parse_argv(prism_context* config, int argc, char** argv);
// The same, returning 0 on success and nonzero (after printing why) instead
// of ending the process.
int prism_parse_argv(prism_context* config, int argc, char** argv);
