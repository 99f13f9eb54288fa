// The PRISM pipeline class, source-compatible with the reference's
// prism::Compressor<T,E> and prism::StatBuffer<T> (include/compressor.hpp:
// 10-90): same template parameters, public members and method signatures,
// implemented over the prism_b200 C ABI (include/prism_b200.h) on the
// sm_100a kernels.  A reference caller recompiles against these headers and
// links libprism_b200 (and this directory's io.cpp, compressor.cpp,
// parameters.cpp, prism.cpp).
//
// Differences a caller can see: failures throw prism::Error instead of ending
// the process; the intermediate buffers qc, bp and compressed_data are sized
// for this library's kernels (compressed_data holds the largest possible
// container, the reference's 4n + 32 bytes can overflow); begin/end are the
// prism_context arrays in managed memory; the stage times are CUDA-event
// times of this library's stages.
#pragma once
#include <array>
#include <cstddef>

#include "io.hpp"
#include "parameters.hpp"
#include "prism_b200.h"
#include "timer.hpp"

namespace prism {

// minimum and maximum of the device array data[0, len): result[0], result[1]
template <typename T>
void extrema_scan(T* data, size_t len, T* result);

template <typename T>
struct StatBuffer : Buffer {
  double minVal{0.0}, maxVal{0.0}, range{1.0};
  StatBuffer() : Buffer() {}
  template <typename... Dim>
  StatBuffer(prism_dtype dtype, Dim... args) : Buffer(dtype, args...) {}

  // REL mode: the range max - min of the field on the device
  double findMinMax() {
    T result[2];
    extrema_scan<T>(reinterpret_cast<T*>(d), len, result);
    minVal = result[0];
    maxVal = result[1];
    range = maxVal - minVal;
    return range;
  }
};

template <typename T, typename E>
class Compressor {
 public:
  size_t len;
  size_t bytes_;
  int radius;
  int align{0};
  int HEADERSIZE{0};  // container trailer bytes
  double range{1.0};  // REL range read from a container's trailer
  double time_pred{0.0}, time_bitplane{0.0}, time_encode{0.0};
  double itime_pred{0.0}, itime_bitplane{0.0}, itime_decode{0.0}, itime_enum{0.0};
  inBuffer* qc{nullptr};                // level-major quantisation codes
  inBuffer* ap{nullptr};                // anchors
  Buffer* compressed_data{nullptr};     // the container
  Buffer* profiling_errors{nullptr};    // auto-tune error sums
  olBuffer<T>* ol{nullptr};
  Bitplane* bp{nullptr};                // bit planes
  uint8_t* compressed_bp{nullptr};
  int *begin{nullptr}, *end{nullptr};   // the prism_context plane ranges
  size_t compressed_lossless_size{0};
  size_t total_compressed_size{0};
  std::array<std::array<size_t, 32>, 4> compressedSize_bp{};  // cumulative bytes per plane, [3 - level][plane]
  size_t* compressedSize_bp_d{nullptr};                        // the same on the device

  Compressor() {}
  ~Compressor();
  Compressor(const Compressor&) = delete;
  Compressor& operator=(const Compressor&) = delete;

  void init(prism_context* config);
  void compute_align();
  // input -> compressed_data (total_compressed_size bytes); the auto-tune
  // decisions go to config->intp_param
  void compress_pipeline(context* config, StatBuffer<T>* input, void* stream);
  void compress_predict(context* config, StatBuffer<T>* input, void* stream);
  void compress_merge(context* config, double input_range, void* stream);

  // compressed_data (its `bytes` = the container's size) -> output
  void decompress_pipeline(context* config, StatBuffer<T>* output, void* stream);
  template <int init_ap>
  void decompress_scatter(context* config, void* stream);
  void decompress_predict(context* config, StatBuffer<T>* output, void* stream);

  // one progressive step from the planes in [config->begin, config->end) to
  // those targetError needs: output_new = the refinement of output_old
  // (lastError == 0: the first step, output_old unused)
  void decompress_progressive_pipeline(context* config, StatBuffer<T>* output_old, StatBuffer<T>* output_new,
                                       double targetError, double lastError, void* stream);
  void decompress_progressive_predict(context* config, StatBuffer<T>* output_old, StatBuffer<T>* output_new,
                                      void* stream);

  // planes selected by the last progressive step (dataloader.cu:11)
  int maxlevel{4};

 private:
  prism_handle* h_{nullptr};
  prism_context* cfg_{nullptr};
  size_t cap_{0};  // device bytes of compressed_data
  uint8_t flags_[8]{};
  void check(int rc, const char* what);
  void read_trailer(context* config, bool anchors, void* stream);
};

extern template class Compressor<float, i4>;
extern template class Compressor<double, i4>;

}  // namespace prism
