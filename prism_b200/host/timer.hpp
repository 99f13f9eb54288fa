// Event timer of the PRISM C++ interface (include/utils/timer.hpp): start()
// records on a stream, stop() records, waits and returns milliseconds.
#pragma once
#include <cuda_runtime.h>

struct GPUTimer {
  cudaEvent_t beg, end;
  GPUTimer() {
    cudaEventCreate(&beg);
    cudaEventCreate(&end);
  }
  ~GPUTimer() {
    cudaEventDestroy(beg);
    cudaEventDestroy(end);
  }
  GPUTimer(const GPUTimer&) = delete;
  GPUTimer& operator=(const GPUTimer&) = delete;
  void start(void* stream) { cudaEventRecord(beg, (cudaStream_t)stream); }
  double stop(void* stream) {
    cudaEventRecord(end, (cudaStream_t)stream);
    cudaEventSynchronize(end);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, beg, end);
    return ms;
  }
};
