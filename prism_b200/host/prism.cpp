// CLI flows over the C++ Compressor (restates src/prism.cu:9-192 and the
// report helpers of include/utils/analyze.hpp:5-159).
#include "prism.hpp"

#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <vector>

#include "compressor.hpp"

namespace {

bool read_file(const std::string& path, std::vector<char>& buf, size_t min_bytes) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) { std::cerr << "Failed to open file: " << path << std::endl; return false; }
  size_t len = (size_t)f.tellg();
  if (len < min_bytes) { std::cerr << "File read incomplete or corrupted: " << path << std::endl; return false; }
  buf.resize(len);
  f.seekg(0);
  f.read(buf.data(), (std::streamsize)len);
  return true;
}

bool write_file(const std::string& path, const void* p, size_t n) {
  std::ofstream f(path, std::ios::binary);
  if (!f) { std::cerr << "can't open file" << std::endl; return false; }
  f.write((const char*)p, (std::streamsize)n);
  return true;
}

// statistic (analyze.hpp:5-73) on the GPU: max error, max relative error,
// PSNR, NRMSE of d_dat against d_ori (both on the device)
template <typename T>
void statistic(prism_handle* h, const T* d_ori, const T* d_dat, size_t n, cudaStream_t st) {
  double s[7];
  uint64_t idx = 0;
  if (prism_statistics(h, d_ori, d_dat, sizeof(T), n, s, &idx, st) != PRISM_OK) {
    std::cerr << "statistics failed: " << prism_last_error(h) << std::endl;
    return;
  }
  printf("  Max_E  = %.15lf, idx = %d\n", s[0], (int)idx);
  printf("  Max_RE = %G\n", s[1]);
  printf("  PSNR = %.7lf, NRMSE = %.10G\n", s[2], s[3]);
}

void print_time(const char* what, size_t bytes, double ms) {
  printf("\n  %-12s %-12s %-20s\n", "type", "time (ms)", "throughtput (GB/s)");
  printf("  %-12s %-12f %-10.4f\n", what, ms, 1.0 * bytes / 1024 / 1024 / 1024 / ms * 1000);
}

template <typename T>
int run(prism_context* c) {
  cudaStream_t st;
  cudaStreamCreate(&st);
  const size_t n = c->size, bytes = n * sizeof(T);
  prism::Compressor<T> comp;
  comp.init(c);
  T* d_data = nullptr;
  uint8_t* d_cont = nullptr;
  cudaMalloc(&d_data, bytes);
  cudaMalloc(&d_cont, comp.max_compressed_size());
  std::vector<char> ori;
  T* d_ori = nullptr;  // original on the device for --report cr
  prism_handle* stat_h = nullptr;
  if (c->report_cr) {
    cudaMalloc(&d_ori, bytes);
    prism_create(&stat_h);
  }
  auto upload_ori = [&]() {
    if (d_ori && !ori.empty()) cudaMemcpy(d_ori, ori.data(), bytes, cudaMemcpyHostToDevice);
  };
  try {
    if (c->isComp) {
      if (!read_file(c->oriFilePath, ori, bytes)) return 1;
      cudaMemcpy(d_data, ori.data(), bytes, cudaMemcpyHostToDevice);
      if (c->report_time) comp.compress_pipeline(d_data, d_cont, st);  // warm up
      comp.compress_pipeline(d_data, d_cont, st);
      std::vector<char> out(comp.total_compressed_size);
      cudaMemcpy(out.data(), d_cont, out.size(), cudaMemcpyDeviceToHost);
      if (!write_file(c->cmpFilePath, out.data(), out.size())) return 1;
      std::cout << "compressed file written: " << c->cmpFilePath << '\n';
      if (c->report_time) {
        print_time("total", bytes, comp.time_total);
        printf("\n  compression ratio: %lf\n--------------------------------------\n",
               1.0 * bytes / comp.total_compressed_size);
      }
    }
    if (c->isDecomp) {
      std::vector<char> cont;
      if (!read_file(c->cmpFilePath, cont, 0)) return 1;
      cudaMemcpy(d_cont, cont.data(), cont.size(), cudaMemcpyHostToDevice);
      if (c->report_cr && ori.empty() && !read_file(c->oriFilePath, ori, bytes)) return 1;
      upload_ori();
      std::vector<T> host(n);
      if (c->compMode && !c->target_ebs.empty()) {
        cudaMemset(d_data, 0, bytes);
        for (size_t i = 0; i < c->target_ebs.size(); ++i) {
          comp.decompress_progressive_pipeline(d_cont, cont.size(), d_data, c->target_ebs[i], st);
          if (c->report_time) print_time("itotal", bytes, comp.time_total);
          if (c->report_cr) {
            statistic<T>(stat_h, d_ori, d_data, n, st);
            int b[4], e[4], ml;
            uint64_t loaded = 0;
            comp.progressive_state(b, e, &ml, &loaded);
            // calculate_accumulate_size (analyze.hpp:118-159)
            printf("  Planes loaded per level: %d %d %d %d\n", e[0], e[1], e[2], e[3]);
            printf("  Total Retrieved size: %llu (%lf%%)\n", (unsigned long long)loaded, 100.0 * loaded / bytes);
            printf("  Bit rate: %lf\n--------------------------------------\n", sizeof(T) * 8.0 * loaded / bytes);
          }
        }
      } else {
        comp.decompress_pipeline(d_cont, cont.size(), d_data, st);
        if (c->report_time) print_time("itotal", bytes, comp.time_total);
      }
      cudaMemcpy(host.data(), d_data, bytes, cudaMemcpyDeviceToHost);
      if (!write_file(c->decFilePath, host.data(), bytes)) return 1;
      std::cout << "decompressed file written: " << c->decFilePath << '\n';
      if (c->report_cr && !(c->compMode && !c->target_ebs.empty())) statistic<T>(stat_h, d_ori, d_data, n, st);
    }
  } catch (const prism::Error& e) {
    std::cerr << e.what() << std::endl;
    return 2;
  }
  cudaFree(d_data);
  cudaFree(d_cont);
  if (d_ori) cudaFree(d_ori);
  if (stat_h) prism_destroy(stat_h);
  cudaStreamDestroy(st);
  return 0;
}

}  // namespace

int initialize(prism_context* config) {
  return config->dtype == F4 ? run<float>(config) : run<double>(config);
}
