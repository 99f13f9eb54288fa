// C++ drop-in for the reference's prism::Compressor<T,E> pipeline
// (include/compressor.hpp:35-83) on top of the prism_b200 C ABI.
//
// Buffers are device pointers owned by the caller; a Compressor owns the
// device workspace (prism_handle).  The pipeline methods keep the reference's
// names: compress_pipeline / decompress_pipeline /
// decompress_progressive_pipeline.  Errors throw prism::Error instead of
// exiting the process.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <array>
#include <stdexcept>
#include <string>

#include "parameters.hpp"
#include "prism_b200.h"

namespace prism {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

template <typename T>
class Compressor {
 public:
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "float or double");
  size_t len{0};
  uint64_t total_compressed_size{0};
  std::array<bool, 4> use_md{}, reverse{};
  double time_total{0.0};  // ms, device time of the last pipeline call

  Compressor() {
    int rc = prism_create(&h_);
    if (rc) throw Error(rc, "prism_create failed");
  }
  ~Compressor() {
    if (prog_) prism_progressive_close(prog_);
    prism_destroy(h_);
  }
  Compressor(const Compressor&) = delete;
  Compressor& operator=(const Compressor&) = delete;

  void init(const prism_context* c) {
    cfg_ = *c;
    len = (size_t)c->x * c->y * c->z;
  }
  uint64_t max_compressed_size() const { return prism_max_container_size(cfg_.x, cfg_.y, cfg_.z, sizeof(T)); }

  // d_in: device field; d_out: device buffer of max_compressed_size() bytes
  void compress_pipeline(const T* d_in, uint8_t* d_out, cudaStream_t stream) {
    uint8_t flags[8];
    double bound = cfg_.error_mode == REL ? cfg_.rel_eb : cfg_.eb;
    Timer t(stream);
    check(prism_compress(h_, d_in, sizeof(T), cfg_.x, cfg_.y, cfg_.z, cfg_.error_mode, bound,
                         cfg_.bt == NB, d_out, max_compressed_size(), &total_compressed_size, flags, stream));
    time_total = t.stop();
    for (int i = 0; i < 4; ++i) { use_md[i] = flags[i]; reverse[i] = flags[4 + i]; }
  }

  void decompress_pipeline(const uint8_t* d_cont, uint64_t size, T* d_out, cudaStream_t stream) {
    double bound = cfg_.error_mode == REL ? cfg_.rel_eb : cfg_.eb;
    Timer t(stream);
    check(prism_decompress(h_, d_cont, size, sizeof(T), cfg_.x, cfg_.y, cfg_.z, cfg_.error_mode, bound, d_out,
                           stream));
    time_total = t.stop();
  }

  // One progressive step; the first call opens the resident state.  d_values
  // is refined in place (the first step overwrites it).
  void decompress_progressive_pipeline(const uint8_t* d_cont, uint64_t size, T* d_values, double target_error,
                                       cudaStream_t stream) {
    double bound = cfg_.error_mode == REL ? cfg_.rel_eb : cfg_.eb;
    if (!prog_) check(prism_progressive_open(h_, d_cont, size, sizeof(T), cfg_.x, cfg_.y, cfg_.z, cfg_.error_mode,
                                             bound, &prog_));
    Timer t(stream);
    check(prism_progressive_step(prog_, target_error, d_values, stream));
    time_total = t.stop();
    check(prism_progressive_state(prog_, nullptr, nullptr, nullptr, nullptr));  // device-side errors of the step
  }
  // The step out of place, with the reference's argument pair (output_old,
  // output_new): d_old holds the previous step's values (nullptr on the first
  // step) and d_new receives the refined ones.
  void decompress_progressive_pipeline(const uint8_t* d_cont, uint64_t size, const T* d_old, T* d_new,
                                       double target_error, cudaStream_t stream) {
    double bound = cfg_.error_mode == REL ? cfg_.rel_eb : cfg_.eb;
    if (!prog_) check(prism_progressive_open(h_, d_cont, size, sizeof(T), cfg_.x, cfg_.y, cfg_.z, cfg_.error_mode,
                                             bound, &prog_));
    Timer t(stream);
    check(prism_progressive_step_into(prog_, target_error, d_old, d_new, stream));
    time_total = t.stop();
    check(prism_progressive_state(prog_, nullptr, nullptr, nullptr, nullptr));
  }
  void progressive_state(int begin[4], int end[4], int* maxlevel, uint64_t* loaded = nullptr) const {
    prism_progressive_state(prog_, begin, end, maxlevel, loaded);
  }

 private:
  struct Timer {
    cudaEvent_t a, b;
    cudaStream_t s;
    explicit Timer(cudaStream_t st) : s(st) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, s);
    }
    double stop() {
      float ms = 0;
      cudaEventRecord(b, s);
      cudaEventSynchronize(b);
      cudaEventElapsedTime(&ms, a, b);
      return ms;
    }
    ~Timer() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  };
  void check(int rc) {
    if (rc) throw Error(rc, std::string("prism_b200: ") + prism_last_error(h_));
  }
  prism_handle* h_{nullptr};
  prism_prog* prog_{nullptr};
  prism_context cfg_{};
};

}  // namespace prism
