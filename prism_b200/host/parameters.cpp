// Flag parsing for the prism CLI (restates src/utils/parameters.cu:9-234).
#include "parameters.hpp"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <stdexcept>

void usage() {
  std::cout << R"(
Options:
  -i <path> : Path to binary input file containing the original data
  -x <path> : Path to decompressed binary output file (optional)
  -z <path> : Path to compressed binary output/input file (optional)
  -f : single precision (float type)
  -d : double precision (double type)
  -1 <nx> : Dimensions for 1D array a[nx]
  -2 <nx> <ny> : Dimensions for 2D array a[ny][nx]
  -3 <nx> <ny> <nz> : Dimensions for 3D array a[nz][ny][nx]
  -A [errorBound] : Absolute error bound
  -R [errorBound] : Relative error bound
  --report [time,cr] : output the compression ratio/time
  -prog : Enable progressive compression/decompression
  -errors -<nums> <error_1> <error_2> ... : Perform progressive decompression multiple times with gradually decreasing error bounds
Examples:
  ./prism -i [oriFilePath] -f -3 [dim_x] [dim_y] [dim_z] -R [errorBound] -z [cmpFilePath] -x [decFilePath] --report time,cr
  ./prism -i [oriFilePath] -d -3 [dim_x] [dim_y] [dim_z] -R [errorBound] -z [cmpFilePath] -x [decFilePath] -prog -errors -2 1e-1 1e-2
)" << std::endl;
}

// default paths and consistency (parameters.cu:33-63)
static int check(prism_context* c) {
  if (c->ndim == -1) { std::cerr << "dim must be specified." << std::endl; return 1; }
  if (c->report_cr && c->oriFilePath.empty()) { std::cerr << "input file path must be specified." << std::endl; return 1; }
  if (c->isComp) {
    if (c->oriFilePath.empty()) { std::cerr << "input file path must be specified." << std::endl; return 1; }
    if (c->cmpFilePath.empty()) c->cmpFilePath = c->oriFilePath + ".prisma";
  }
  if (c->isDecomp) {
    if (c->oriFilePath.empty() && c->cmpFilePath.empty()) {
      std::cerr << "compressed file path must be specified." << std::endl;
      return 1;
    }
    if (c->decFilePath.empty()) {
      if (!c->cmpFilePath.empty()) c->decFilePath = c->cmpFilePath + ".out";
      else {
        c->cmpFilePath = c->oriFilePath + ".prisma";
        c->decFilePath = c->oriFilePath + ".prisma.out";
      }
    }
  }
  if (!c->isComp && !c->isDecomp) {
    printf("Please set the compression/decompression\n");
    usage();
  }
  return 0;
}

int prism_parse_argv(prism_context* c, int argc, char** argv) {
  if (argc == 1) usage();
  try {
    for (int i = 1; i < argc; ++i) {
      const char* a = argv[i];
      if (!strcmp(a, "-h")) { usage(); exit(0); }
      else if (!strcmp(a, "-f")) c->dtype = F4;
      else if (!strcmp(a, "-d")) c->dtype = F8;
      else if (!strcmp(a, "-A")) { c->error_mode = ABS; if (i + 1 < argc) c->eb = std::stod(argv[++i]); }
      else if (!strcmp(a, "-R")) { c->error_mode = REL; if (i + 1 < argc) c->rel_eb = std::stod(argv[++i]); }
      else if (!strcmp(a, "-z")) { c->isComp = true; if (i + 1 < argc && argv[i + 1][0] != '-') c->cmpFilePath = argv[++i]; }
      else if (!strcmp(a, "-x")) { c->isDecomp = true; if (i + 1 < argc && argv[i + 1][0] != '-') c->decFilePath = argv[++i]; }
      else if (!strcmp(a, "-i")) { if (i + 1 < argc) c->oriFilePath = argv[++i]; }
      else if (!strcmp(a, "-1")) {
        c->ndim = 1;
        if (i + 1 < argc) c->x = (uint32_t)std::stoi(argv[++i]); else usage();
      } else if (!strcmp(a, "-2")) {
        c->ndim = 2;
        if (i + 2 < argc) { c->x = (uint32_t)std::stoi(argv[i + 1]); c->y = (uint32_t)std::stoi(argv[i + 2]); i += 2; }
        else usage();
      } else if (!strcmp(a, "-3")) {
        c->ndim = 3;
        if (i + 3 < argc) {
          c->x = (uint32_t)std::stoi(argv[i + 1]); c->y = (uint32_t)std::stoi(argv[i + 2]);
          c->z = (uint32_t)std::stoi(argv[i + 3]); i += 3;
        } else usage();
      } else if (!strcmp(a, "-errors")) {
        c->compMode = 1;
        if (i + 1 >= argc) { std::cerr << "Number of error bounds not specified." << std::endl; return 1; }
        int k = std::stoi(argv[++i] + 1);
        c->target_ebs.resize(k);
        for (int j = 0; j < k; ++j) {
          if (i + 1 >= argc) { std::cerr << "Not enough error bounds provided." << std::endl; return 1; }
          c->target_ebs[j] = std::stod(argv[++i]);
        }
      } else if (!strcmp(a, "--report")) {
        if (i + 1 >= argc) { std::cerr << "Error: missing argument after --report" << std::endl; return 0; }
        std::stringstream ss(argv[++i]);
        std::string tok;
        while (std::getline(ss, tok, ',')) {
          if (tok == "time") c->report_time = true;
          else if (tok == "cr") c->report_cr = true;
          else std::cerr << "Warning: unknown report option: " << tok << std::endl;
        }
      } else if (!strcmp(a, "-prog")) c->bt = NB;
      else if (!strcmp(a, "-cubic")) {
        // The reference's hidden test flag switches its sweeps to the natural
        // cubic (parameters.cu:199-204).  The library computes the default
        // cubic only, so the flag is refused rather than ignored: ignoring it
        // would write files that differ from the reference's.
        if (i + 1 < argc && !strcmp(argv[++i], "natural")) {
          std::cerr << "Error: -cubic natural is not supported (default cubic only)" << std::endl;
          return 1;
        }
      } else if (!strcmp(a, "-md")) {
        if (i + 1 < argc) {
          if (!strcmp(argv[i + 1], "true")) for (bool& v : c->intp_param.use_md) v = true;
          else if (!strcmp(argv[i + 1], "false")) for (bool& v : c->intp_param.use_md) v = false;
          ++i;
        }
      } else if (!strcmp(a, "-reverse")) {
        for (bool& v : c->intp_param.reverse) v = true;
      } else {
        printf("Error: Unrecognized option '%s'.\n", a);
        return 1;
      }
    }
  } catch (const std::exception& e) {
    std::cerr << "bad number in the command line: " << e.what() << std::endl;
    return 1;
  }
  c->size = c->x * c->y * c->z * c->w;
  // the progressive plane ranges (parameters.cu:161-164): managed memory, so
  // the host reads them and callers may still clear them with cudaMemset
  if (!c->begin && cudaMallocManaged(&c->begin, 4 * sizeof(int)) != cudaSuccess) {
    std::cerr << "cannot allocate the plane ranges" << std::endl;
    return 1;
  }
  if (!c->end && cudaMallocManaged(&c->end, 4 * sizeof(int)) != cudaSuccess) {
    std::cerr << "cannot allocate the plane ranges" << std::endl;
    return 1;
  }
  for (int i = 0; i < 4; ++i) c->begin[i] = c->end[i] = 0;
  return check(c);
}

void parse_argv(prism_context* c, int argc, char** argv) {
  if (prism_parse_argv(c, argc, argv)) std::exit(1);
}
