// CUDA error check of the PRISM C++ interface (include/utils/err.hpp): prints
// the failing call and ends the process, as callers of the reference expect.
// The library itself reports failures as prism::Error exceptions and C
// status codes instead.
#pragma once
#include <cstdlib>
#include <iostream>
#define CHECK_CUDA(call)                                                                     \
  do {                                                                                       \
    cudaError_t check_cuda_err_ = (call);                                                    \
    if (check_cuda_err_ != cudaSuccess) {                                                    \
      std::cerr << "[CUDA ERROR] " << __FILE__ << ":" << __LINE__ << " - "                   \
                << cudaGetErrorString(check_cuda_err_) << std::endl;                         \
      std::exit(EXIT_FAILURE);                                                               \
    }                                                                                        \
  } while (0)
