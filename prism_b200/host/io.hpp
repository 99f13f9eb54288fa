// Host/device buffers of the PRISM C++ interface (include/utils/io.hpp of
// the reference): a Buffer owns a device allocation and a pinned host copy of
// the same size; StatBuffer (compressor.hpp) adds the field's range.  Names,
// members and methods are the reference's; failures throw prism::Error
// instead of ending the process.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "parameters.hpp"

namespace prism {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

enum class typetofile { hostTofile, deviceTofile };

typedef struct Buffer {
  prism_dtype dtype{U1};
  int tsize{1}, ndim{-1};
  size_t len{1}, bytes{1};
  uint32_t lx{1}, ly{1}, lz{1};
  size_t sty{1}, stz{1};  // strides of y and z in elements
  int align{0};           // extra bytes past len * tsize
  void* d{nullptr};
  void* h{nullptr};

  Buffer() {}
  virtual ~Buffer();
  Buffer(const Buffer&) = delete;
  Buffer& operator=(const Buffer&) = delete;
  // dims x, y, z (x fastest); allocates bytes = tsize * len + align on the
  // device (zeroed) and as pinned host memory
  template <typename... Dim>
  Buffer(prism_dtype type, int align_, Dim... args) : dtype(type), align(align_) {
    const uint32_t dims[] = {static_cast<uint32_t>(args)..., 1u, 1u, 1u};
    lx = sizeof...(Dim) >= 1 ? dims[0] : 1;
    ly = sizeof...(Dim) >= 2 ? dims[1] : 1;
    lz = sizeof...(Dim) >= 3 ? dims[2] : 1;
    ndim = lz > 1 ? 3 : (ly > 1 ? 2 : 1);
    tsize = dtype % 10;
    len = (size_t)lx * ly * lz;
    sty = lx;
    stz = (size_t)lx * ly;
    bytes = tsize * len + align;
    allocate(bytes);
  }

  // reads the file into the host copy: the original field must hold at least
  // `bytes` bytes; a container sets `bytes` to the file's length
  template <itype file_type>
  void load_fromfile(const std::string filename);
  void unload_tofile(const std::string filename, typetofile tf = typetofile::hostTofile);
  void unload_tofile(const std::string filename, long long numBytes, typetofile tf = typetofile::hostTofile);
  void H2D(long long numBytes = -1);
  void D2H(long long numBytes = -1);
  void H2D_cudaasync(void* stream, long long numBytes = -1);
  void D2H_cudaasync(void* stream, long long numBytes = -1);

  template <typename D>
  D len3() const { return D(lx, ly, lz); }
  template <typename D>
  D st3() const { return D(1, sty, stz); }

 protected:
  void allocate(size_t n);
} inBuffer;

// The plane buffer of a field: device memory of the plane-buffer size
// (host plane strides, io.hpp:104-132 of the reference) and its geometry.
struct Bitplane : Buffer {
  int* aligned_strides_d{nullptr};
  size_t aligned_len{1}, ori_size{1}, aligned_size{1};
  int strides[4]{0, 0, 0, 0};
  int aligned_strides[4]{0, 0, 0, 0};
  int prefix_nums[4]{0, 0, 0, 0};
  int compressed_size[4][32]{};
  Bitplane(int x, int y, int z);
};

// Outlier buffer: allocated with no entries and never written by the
// reference's pipeline (compressor.cu:109); kept for interface compatibility.
template <typename T>
struct olBuffer : Buffer {
  uint32_t *d_idx{nullptr}, *h_idx{nullptr};
  uint32_t* d_num{nullptr};
  uint32_t h_num{0};
  olBuffer() {}
  template <typename... Dim>
  olBuffer(prism_dtype dtype, Dim... args) : Buffer(dtype, args...) {}
};

}  // namespace prism
