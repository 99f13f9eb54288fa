// prism::Compressor<T,E> over the prism_b200 C ABI.  The pipelines follow
// src/compressor.cu:77-226 of the reference: the same container, the same
// trailer parse (decompress_scatter), the same progressive step
// (strategy on the prism_context plane ranges, decode of the selected planes,
// inverse shuffle, reconstruction of the delta added to the previous
// values); the work runs in the library's kernels.
#include "compressor.hpp"

#include <cstring>
#include <string>
#include <type_traits>

namespace prism {

namespace {

void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(PRISM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// a device-only buffer (the library's intermediates have no host copy)
template <class B>
B* device_buffer(prism_dtype dtype, size_t elems) {
  B* b = new B();
  b->dtype = dtype;
  b->tsize = dtype % 10;
  b->len = elems;
  b->lx = (uint32_t)elems;
  b->ndim = 1;
  b->bytes = b->tsize * elems;
  if (b->bytes) {
    cuda_ok(cudaMalloc(&b->d, b->bytes), "cudaMalloc");
    cuda_ok(cudaMemset(b->d, 0, b->bytes), "cudaMemset");
  }
  return b;
}

// stage order of prism_stage_times
enum { kExtrema, kAutotune, kPredict, kShuffle, kEncode, kTrailer, kStrategy, kDecode, kInverse, kReconstruct, kStages };

}  // namespace

template <typename T>
void extrema_scan(T* data, size_t len, T* result) {
  prism_handle* h = nullptr;
  int rc = prism_create(&h);
  if (rc) throw Error(rc, "prism_create failed");
  double mm[2] = {0, 0};
  rc = prism_extrema_minmax(h, data, (int)sizeof(T), len, mm, nullptr);
  std::string msg = rc ? prism_last_error(h) : "";
  prism_destroy(h);
  if (rc) throw Error(rc, "extrema_scan: " + msg);
  result[0] = (T)mm[0];
  result[1] = (T)mm[1];
}
template void extrema_scan<float>(float*, size_t, float*);
template void extrema_scan<double>(double*, size_t, double*);

template <typename T, typename E>
void Compressor<T, E>::check(int rc, const char* what) {
  if (rc) throw Error(rc, std::string(what) + ": " + (h_ ? prism_last_error(h_) : ""));
}

template <typename T, typename E>
Compressor<T, E>::~Compressor() {
  delete qc;
  delete ap;
  delete ol;
  delete bp;
  delete compressed_data;
  delete profiling_errors;
  if (compressedSize_bp_d) cudaFree(compressedSize_bp_d);
  if (h_) prism_destroy(h_);
}

template <typename T, typename E>
void Compressor<T, E>::init(prism_context* config) {
  static_assert(std::is_same<E, i4>::value, "quantisation codes are int32 (i4), as in the reference's build");
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "float or double fields");
  cfg_ = config;
  const uint32_t x = config->x, y = config->y, z = config->z;
  radius = (int)config->radius;
  len = (size_t)x * y * z;
  bytes_ = len * sizeof(T);
  if (!h_) check(prism_create(&h_), "prism_create");
  auto div = [](uint32_t l, uint32_t s) { return (l - 1) / s + 1; };
  qc = device_buffer<inBuffer>(I4, prism_code_buffer_len(x, y, z));
  ap = new inBuffer(config->dtype, 0, div(x, BLOCK_SIZE), div(y, BLOCK_SIZE), div(z, BLOCK_SIZE));
  ol = new olBuffer<T>(config->dtype, 0, 0);
  const size_t cap = prism_max_container_size(x, y, z, (int)sizeof(T));
  const size_t ref_cap = 4 * len + 32;  // the reference's container buffer
  compressed_data = new Buffer(U1, 0, (uint32_t)0);
  compressed_data->bytes = cap > ref_cap ? cap : ref_cap;
  cuda_ok(cudaMallocHost(&compressed_data->h, compressed_data->bytes), "cudaMallocHost");
  cuda_ok(cudaMalloc(&compressed_data->d, compressed_data->bytes), "cudaMalloc");
  compressed_data->len = compressed_data->bytes;
  compressed_data->lx = (uint32_t)compressed_data->bytes;
  cap_ = compressed_data->bytes;
  profiling_errors = new Buffer(config->dtype, 0, 18, 1, 1);
  bp = new Bitplane((int)x, (int)y, (int)z);
  HEADERSIZE = (int)prism_trailer_size(x, y, z, (int)sizeof(T));
  begin = config->begin;
  end = config->end;
  cuda_ok(cudaMalloc(&compressedSize_bp_d, sizeof(size_t) * 4 * 32), "cudaMalloc");
  compute_align();
}

template <typename T, typename E>
void Compressor<T, E>::compute_align() {
  align = (int)(bp->aligned_size / 4 - len);  // padding codes of the plane layout
}

template <typename T, typename E>
void Compressor<T, E>::compress_pipeline(context* config, StatBuffer<T>* input, void* stream) {
  const int mode = config->error_mode == REL ? 1 : 0;
  const double bound = mode ? config->rel_eb : config->eb;
  if (config->report_time) check(prism_profile(h_, 1), "prism_profile");
  uint64_t size = 0;
  GPUTimer t;
  t.start(stream);
  check(prism_compress(h_, input->d, (int)sizeof(T), config->x, config->y, config->z, mode, bound,
                       config->bt == NB ? 1 : 0, compressed_data->d, cap_, &size, flags_, stream),
        "compress_pipeline");
  const double total = t.stop(stream);
  total_compressed_size = size;
  compressed_lossless_size = size - HEADERSIZE;
  for (int i = 0; i < 4; ++i) {
    config->intp_param.use_md[i] = flags_[i] != 0;
    config->intp_param.reverse[i] = flags_[4 + i] != 0;
  }
  // the cumulative plane sizes, as compress_merge leaves them
  const uint8_t* tr = static_cast<const uint8_t*>(compressed_data->d) + compressed_lossless_size;
  cuda_ok(cudaMemcpy(compressedSize_bp_d, tr + 16, 1024, cudaMemcpyDeviceToDevice), "csbp");
  cuda_ok(cudaMemcpy(&compressedSize_bp[0][0], tr + 16, 1024, cudaMemcpyDeviceToHost), "csbp");
  if (config->report_time) {
    double ms[kStages];
    int counts[kStages];
    {
      const int got = prism_stage_times(h_, ms, counts, kStages, 1);  // the number of stages, or an error
      check(got < 0 ? got : 0, "prism_stage_times");
    }
    check(prism_profile(h_, 0), "prism_profile");
    time_pred = ms[kExtrema] + ms[kAutotune] + ms[kPredict];
    time_bitplane = ms[kShuffle];
    time_encode = ms[kEncode] + ms[kTrailer];
  } else {
    time_pred = total;
    time_bitplane = time_encode = 0.0;
  }
}

template <typename T, typename E>
void Compressor<T, E>::compress_predict(context* config, StatBuffer<T>* input, void* stream) {
  double errors[15];
  GPUTimer t;
  t.start(stream);
  check(prism_autotune(h_, input->d, (int)sizeof(T), config->x, config->y, config->z, errors, flags_, stream),
        "autotune");
  const bool rel = config->error_mode == REL;
  const double eb = rel ? config->rel_eb * input->range : config->eb;
  check(prism_predict(h_, input->d, (int)sizeof(T), config->x, config->y, config->z, eb, rel ? config->rel_eb : 0.0,
                      flags_, static_cast<int32_t*>(qc->d), ap->d, stream),
        "compress_predict");
  time_pred = t.stop(stream);
  for (int i = 0; i < 4; ++i) {
    config->intp_param.use_md[i] = flags_[i] != 0;
    config->intp_param.reverse[i] = flags_[4 + i] != 0;
  }
  T err[18] = {};
  for (int i = 0; i < 15; ++i) err[i] = (T)errors[i];
  std::memcpy(profiling_errors->h, err, sizeof(err));
  cuda_ok(cudaMemcpy(profiling_errors->d, err, sizeof(err), cudaMemcpyHostToDevice), "errors");
}

// trailer after the lossless stream (compressor.cu:139-151)
template <typename T, typename E>
void Compressor<T, E>::compress_merge(context* config, double input_range, void* stream) {
  total_compressed_size = compressed_lossless_size + HEADERSIZE;
  uint8_t* tr = static_cast<uint8_t*>(compressed_data->d) + compressed_lossless_size;
  uint8_t hdr[16];
  for (int i = 0; i < 4; ++i) {
    hdr[i] = config->intp_param.use_md[i];
    hdr[4 + i] = config->intp_param.reverse[i];
  }
  std::memcpy(hdr + 8, &input_range, 8);
  cudaStream_t st = (cudaStream_t)stream;
  cuda_ok(cudaMemcpyAsync(tr, hdr, 16, cudaMemcpyHostToDevice, st), "trailer");
  cuda_ok(cudaMemcpyAsync(tr + 16, compressedSize_bp_d, 1024, cudaMemcpyDeviceToDevice, st), "trailer");
  cuda_ok(cudaMemcpyAsync(tr + 1040, ap->d, ap->bytes, cudaMemcpyDeviceToDevice, st), "trailer");
  cuda_ok(cudaStreamSynchronize(st), "trailer");
}

// parse the trailer of the container in compressed_data (`bytes` = its
// size): flags into config->intp_param, the range, the plane sizes, and the
// anchors when INIT_AP (compressor.cu:192-210); without INIT_AP the anchors
// are zero, as the progressive steps after the first need them
template <typename T, typename E>
template <int init_ap>
void Compressor<T, E>::decompress_scatter(context* config, void* stream) {
  total_compressed_size = compressed_data->bytes;
  if (total_compressed_size < (size_t)HEADERSIZE + 8) throw Error(PRISM_ERR_CORRUPT, "container shorter than its trailer");
  compressed_lossless_size = total_compressed_size - HEADERSIZE;
  const uint8_t* tr = static_cast<const uint8_t*>(compressed_data->d) + compressed_lossless_size;
  cudaStream_t st = (cudaStream_t)stream;
  uint8_t hdr[16];
  cuda_ok(cudaMemcpyAsync(hdr, tr, 16, cudaMemcpyDeviceToHost, st), "trailer");
  cuda_ok(cudaMemcpyAsync(&compressedSize_bp[0][0], tr + 16, 1024, cudaMemcpyDeviceToHost, st), "trailer");
  cuda_ok(cudaMemcpyAsync(compressedSize_bp_d, tr + 16, 1024, cudaMemcpyDeviceToDevice, st), "trailer");
  if (init_ap == 1) cuda_ok(cudaMemcpyAsync(ap->d, tr + 1040, ap->bytes, cudaMemcpyDeviceToDevice, st), "trailer");
  else cuda_ok(cudaMemsetAsync(ap->d, 0, ap->bytes, st), "trailer");
  cuda_ok(cudaStreamSynchronize(st), "trailer");
  for (int i = 0; i < 4; ++i) {
    config->intp_param.use_md[i] = hdr[i] != 0;
    config->intp_param.reverse[i] = hdr[4 + i] != 0;
    flags_[i] = hdr[i];
    flags_[4 + i] = hdr[4 + i];
  }
  std::memcpy(&range, hdr + 8, 8);
}

template <typename T, typename E>
void Compressor<T, E>::decompress_pipeline(context* config, StatBuffer<T>* output, void* stream) {
  decompress_scatter<1>(config, stream);
  const int mode = config->error_mode == REL ? 1 : 0;
  if (mode) config->eb = config->rel_eb * range;
  if (config->report_time) check(prism_profile(h_, 1), "prism_profile");
  GPUTimer t;
  t.start(stream);
  check(prism_decompress(h_, compressed_data->d, total_compressed_size, (int)sizeof(T), config->x, config->y,
                         config->z, mode, mode ? config->rel_eb : config->eb, output->d, stream),
        "decompress_pipeline");
  const double total = t.stop(stream);
  if (config->report_time) {
    double ms[kStages];
    int counts[kStages];
    {
      const int got = prism_stage_times(h_, ms, counts, kStages, 1);  // the number of stages, or an error
      check(got < 0 ? got : 0, "prism_stage_times");
    }
    check(prism_profile(h_, 0), "prism_profile");
    itime_decode = ms[kDecode];
    itime_bitplane = ms[kInverse];
    itime_pred = ms[kReconstruct];
  } else {
    itime_pred = total;
  }
}

template <typename T, typename E>
void Compressor<T, E>::decompress_predict(context* config, StatBuffer<T>* output, void* stream) {
  const bool rel = config->error_mode == REL;
  GPUTimer t;
  t.start(stream);
  check(prism_reconstruct(h_, static_cast<const int32_t*>(qc->d), ap->d, (int)sizeof(T), config->x, config->y,
                          config->z, config->eb, rel ? config->rel_eb : 0.0, flags_, maxlevel, nullptr, output->d,
                          stream),
        "decompress_predict");
  itime_pred = t.stop(stream);
}

template <typename T, typename E>
void Compressor<T, E>::decompress_progressive_predict(context* config, StatBuffer<T>* output_old,
                                                      StatBuffer<T>* output_new, void* stream) {
  const bool rel = config->error_mode == REL;
  GPUTimer t;
  t.start(stream);
  check(prism_reconstruct(h_, static_cast<const int32_t*>(qc->d), ap->d, (int)sizeof(T), config->x, config->y,
                          config->z, config->eb, rel ? config->rel_eb : 0.0, flags_, maxlevel, output_old->d,
                          output_new->d, stream),
        "decompress_progressive_predict");
  itime_pred = t.stop(stream);
}

template <typename T, typename E>
void Compressor<T, E>::decompress_progressive_pipeline(context* config, StatBuffer<T>* output_old,
                                                       StatBuffer<T>* output_new, double targetError,
                                                       double lastError, void* stream) {
  const bool first = lastError == 0;
  if (first) decompress_scatter<1>(config, stream);
  else decompress_scatter<0>(config, stream);
  if (config->error_mode == REL) {
    config->eb = config->rel_eb * range;
    targetError *= range;
  }
  if (!begin || !end) throw Error(PRISM_ERR_ARG, "prism_context begin/end not allocated (parse_argv allocates them)");
  // the plane ranges live in managed memory that callers may clear with
  // cudaMemset on any stream
  cuda_ok(cudaDeviceSynchronize(), "plane ranges");
  int b[4], e[4];
  std::memcpy(b, begin, sizeof(b));
  std::memcpy(e, end, sizeof(e));
  uint64_t csbp[128];
  std::memcpy(csbp, &compressedSize_bp[0][0], sizeof(csbp));
  GPUTimer t;
  t.start(stream);
  check(prism_find_strategy(h_, csbp, config->eb, targetError, b, e, &maxlevel, stream), "findStrategy");
  itime_enum = t.stop(stream);
  std::memcpy(begin, b, sizeof(b));
  std::memcpy(end, e, sizeof(e));
  t.start(stream);
  check(prism_lossless_decode(h_, static_cast<const uint8_t*>(compressed_data->d), config->x, config->y, config->z, b,
                              e, static_cast<uint8_t*>(bp->d), stream),
        "lossless_decode_progressive");
  itime_decode = t.stop(stream);
  t.start(stream);
  check(prism_inverse_bitshuffle(h_, static_cast<const uint8_t*>(bp->d), config->x, config->y, config->z, 1, b, e,
                                 static_cast<int32_t*>(qc->d), stream),
        "inverse_bitshuffle_progressive");
  itime_bitplane = t.stop(stream);
  if (first) decompress_predict(config, output_new, stream);
  else decompress_progressive_predict(config, output_old, output_new, stream);
}

template class Compressor<float, i4>;
template class Compressor<double, i4>;
template void Compressor<float, i4>::decompress_scatter<0>(context*, void*);
template void Compressor<float, i4>::decompress_scatter<1>(context*, void*);
template void Compressor<double, i4>::decompress_scatter<0>(context*, void*);
template void Compressor<double, i4>::decompress_scatter<1>(context*, void*);

}  // namespace prism
