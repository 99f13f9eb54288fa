// The PRISM flows (restates src/prism.cu:9-192 and the report helpers of
// include/utils/analyze.hpp:5-159 of the reference) over prism::Compressor
// and prism::StatBuffer: compress a field file into a container file,
// decompress a container, or refine a progressive container step by step
// through the -errors targets, with the same files, defaults and printed
// lines.  The error statistics of --report cr run on the GPU
// (prism_statistics) instead of host loops, and a progressive run keeps its
// container on the device across steps instead of reloading the file.
#include "prism.hpp"

#include <cmath>
#include <cstdio>
#include <iostream>
#include <array>
#include <memory>

#include "compressor.hpp"

namespace {

template <typename T, int DECOMP, int PROGRESSIVE>
void print_result(size_t n, size_t total_compressed_size, double t_enum, double t_pred, double t_plane,
                  double t_lossless) {
  const double total_bytes = (double)n * sizeof(T);
  auto gbs = [&](double ms) { return total_bytes / 1024 / 1024 / 1024 / ms * 1000; };
  printf("\n  \033[1m%-12s %-12s %-20s\033[0m\n", "type", "time (ms)", "throughtput (GB/s)");
  if (DECOMP) {
    if (PROGRESSIVE) printf("  %-12s %-12f %-10.4f\n", "loadStrategy", t_enum, gbs(t_enum));
    printf("  %-12s %-12f %-10.4f\n", "ipredict", t_pred, gbs(t_pred));
    printf("  %-12s %-12f %-10.4f\n", "ibitplane", t_plane, gbs(t_plane));
    printf("  %-12s %-12f %-10.4f\n", "ilossless", t_lossless, gbs(t_lossless));
    const double total = t_pred + t_plane + t_lossless + (PROGRESSIVE ? t_enum : 0.0);
    printf("  \033[1m%-12s\033[0m %-12f %-10.4f\n\n", "itotal", total, gbs(total));
  } else {
    printf("  %-12s %-12f %-10.4f\n", "predict", t_pred, gbs(t_pred));
    printf("  %-12s %-12f %-10.4f\n", "bitplane", t_plane, gbs(t_plane));
    printf("  %-12s %-12f %-10.4f\n", "lossless", t_lossless, gbs(t_lossless));
    const double total = t_pred + t_plane + t_lossless;
    printf("  \033[1m%-12s\033[0m %-12f %-10.4f\n\n", "total", total, gbs(total));
    printf("  compression ratio: %lf\n", total_bytes / total_compressed_size);
    printf("--------------------------------------\n");
  }
}

// error statistics of a reconstruction against the original, both on the
// device (statistic, analyze.hpp:5-73)
template <typename T>
void statistic(const T* d_ori, const T* d_dat, size_t n, void* stream) {
  prism_handle* h = nullptr;
  if (prism_create(&h)) return;
  double s[7];
  uint64_t idx = 0;
  if (prism_statistics(h, d_ori, d_dat, sizeof(T), n, s, &idx, stream) == PRISM_OK) {
    printf("  Max_E  = %.15lf, idx = %d\n", s[0], (int)idx);
    printf("  Max_RE = %G\n", s[1]);
    printf("  PSNR = %.7lf, NRMSE = %.10G\n", s[2], s[3]);
  } else {
    std::cerr << "statistics failed: " << prism_last_error(h) << std::endl;
  }
  prism_destroy(h);
}

// bytes of the planes the last step selected, added to the running total
// (calculate_accumulate_size, analyze.hpp:118-159): the per-plane size is the
// difference of consecutive cumulative sizes, across levels at plane 0
void accumulate_size(size_t& loaded, size_t n, int tsize, const int* begin, const int* end,
                     const std::array<std::array<size_t, 32>, 4>& cum) {
  const double total_bytes = (double)n * tsize;
  size_t step = 0;
  for (int l = 0; l < 4; ++l)
    for (int b = begin[l]; b < end[l]; ++b) {
      const size_t prev = b > 0 ? cum[l][b - 1] : (l > 0 ? cum[l - 1][31] : 0);
      step += cum[l][b] - prev;
    }
  loaded += step;
  printf("  Data Chunk: %zu (%lf%%)\n", step, 100.0 * step / total_bytes);
  printf("  Total Retrieved size: %zu (%lf%%)\n", loaded, 100.0 * loaded / total_bytes);
  printf("  Bit rate: %lf\n", 8.0 * tsize * loaded / total_bytes);
  printf("--------------------------------------\n");
}

template <typename T>
void compress(prism_context* c, cudaStream_t st) {
  auto input = std::make_unique<prism::StatBuffer<T>>(c->dtype, 0, c->x, c->y, c->z);
  input->template load_fromfile<ori_File>(c->oriFilePath);
  input->H2D();
  if (c->error_mode == REL) c->eb = c->rel_eb * input->findMinMax();
  if (!c->isComp) return;
  if (c->report_time) {  // warm up
    prism::Compressor<T, i4> tmp;
    tmp.init(c);
    tmp.compress_pipeline(c, input.get(), st);
  }
  prism::Compressor<T, i4> cmp;
  cmp.init(c);
  cmp.compress_pipeline(c, input.get(), st);
  cmp.compressed_data->unload_tofile(c->cmpFilePath, (long long)cmp.total_compressed_size,
                                     prism::typetofile::deviceTofile);
  if (c->report_time)
    print_result<T, 0, 0>(cmp.len, cmp.total_compressed_size, cmp.itime_enum, cmp.time_pred, cmp.time_bitplane,
                          cmp.time_encode);
}

template <typename T>
void decompress(prism_context* c, cudaStream_t st) {
  const size_t n = (size_t)c->x * c->y * c->z;
  if (c->report_time) {  // warm up
    prism::StatBuffer<T> out(c->dtype, 0, c->x, c->y, c->z);
    prism::Compressor<T, i4> tmp;
    tmp.init(c);
    tmp.compressed_data->template load_fromfile<cmp_File>(c->cmpFilePath);
    tmp.compressed_data->H2D();
    tmp.decompress_pipeline(c, &out, st);
  }
  prism::Compressor<T, i4> dec;
  dec.init(c);
  dec.compressed_data->template load_fromfile<cmp_File>(c->cmpFilePath);
  dec.compressed_data->H2D();
  prism::StatBuffer<T> out(c->dtype, 0, c->x, c->y, c->z);
  dec.decompress_pipeline(c, &out, st);
  out.unload_tofile(c->decFilePath, prism::typetofile::deviceTofile);
  if (c->report_time)
    print_result<T, 1, 0>(n, dec.total_compressed_size, dec.itime_enum, dec.itime_pred, dec.itime_bitplane,
                          dec.itime_decode);
  if (c->report_cr) {
    prism::StatBuffer<T> ori(c->dtype, 0, c->x, c->y, c->z);
    ori.template load_fromfile<ori_File>(c->oriFilePath);
    ori.H2D();
    statistic<T>(static_cast<const T*>(ori.d), static_cast<const T*>(out.d), n, st);
  }
}

template <typename T>
void progressive(prism_context* c, cudaStream_t st) {
  const size_t n = (size_t)c->x * c->y * c->z;
  std::unique_ptr<prism::StatBuffer<T>> ori;
  if (c->report_cr) {
    ori = std::make_unique<prism::StatBuffer<T>>(c->dtype, 0, c->x, c->y, c->z);
    ori->template load_fromfile<ori_File>(c->oriFilePath);
    ori->H2D();
  }
  prism::Compressor<T, i4> dec;
  dec.init(c);
  dec.compressed_data->template load_fromfile<cmp_File>(c->cmpFilePath);
  dec.compressed_data->H2D();
  auto cur = std::make_unique<prism::StatBuffer<T>>(c->dtype, 0, c->x, c->y, c->z);
  auto prev = std::make_unique<prism::StatBuffer<T>>(c->dtype, 0, c->x, c->y, c->z);
  if (c->report_time) {  // warm up, then start over from no planes
    dec.decompress_progressive_pipeline(c, nullptr, cur.get(), c->target_ebs[0], 0, st);
    CHECK_CUDA(cudaMemset(c->begin, 0, 4 * sizeof(int)));
    CHECK_CUDA(cudaMemset(c->end, 0, 4 * sizeof(int)));
  }
  size_t loaded = dec.ap->bytes;
  for (size_t i = 0; i < c->target_ebs.size(); ++i) {
    std::swap(prev, cur);
    dec.decompress_progressive_pipeline(c, prev.get(), cur.get(), c->target_ebs[i], i ? c->target_ebs[i - 1] : 0.0,
                                        st);
    if (c->report_time)
      print_result<T, 1, 1>(n, dec.total_compressed_size, dec.itime_enum, dec.itime_pred, dec.itime_bitplane,
                            dec.itime_decode);
    if (c->report_cr) {
      statistic<T>(static_cast<const T*>(ori->d), static_cast<const T*>(cur->d), n, st);
      CHECK_CUDA(cudaDeviceSynchronize());
      accumulate_size(loaded, n, (int)sizeof(T), c->begin, c->end, dec.compressedSize_bp);
    }
  }
  cur->unload_tofile(c->decFilePath, prism::typetofile::deviceTofile);
}

template <typename T>
void run(prism_context* c, cudaStream_t st) {
  if (c->isComp) compress<T>(c, st);
  if (c->isDecomp) {
    if (c->compMode && !c->target_ebs.empty()) progressive<T>(c, st);
    else decompress<T>(c, st);
  }
}

}  // namespace

int prism_initialize(prism_context* config) {
  cudaStream_t st;
  if (cudaStreamCreate(&st) != cudaSuccess) {
    std::cerr << "cannot create a CUDA stream" << std::endl;
    return 2;
  }
  int rc = 0;
  try {
    if (config->dtype == PRISM_TYPE_DOUBLE) run<double>(config, st);
    else run<float>(config, st);
  } catch (const prism::Error& e) {
    std::cerr << e.what() << std::endl;
    rc = 2;
  }
  cudaStreamDestroy(st);
  return rc;
}

void initialize(prism_context* config) {
  if (prism_initialize(config)) std::exit(EXIT_FAILURE);
}
