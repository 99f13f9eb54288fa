// Buffer methods (restates the behaviour of src/utils/io.cu of the
// reference: pinned host copies, blocking and asynchronous transfers, file
// load and store with the same messages).
#include "io.hpp"

#include <fstream>
#include <iostream>

#include "prism_b200.h"

namespace prism {

static void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(PRISM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void Buffer::allocate(size_t n) {
  if (n == 0) return;
  cuda_ok(cudaMallocHost(&h, n), "cudaMallocHost");
  cuda_ok(cudaMalloc(&d, n), "cudaMalloc");
  cuda_ok(cudaMemset(d, 0, n), "cudaMemset");
}

Buffer::~Buffer() {
  if (d) cudaFree(d);
  if (h) cudaFreeHost(h);
}

template <itype file_type>
void Buffer::load_fromfile(const std::string filename) {
  std::ifstream file(filename, std::ios::binary | std::ios::ate);
  if (!file) throw Error(PRISM_ERR_ARG, "Failed to open file: " + filename);
  const size_t length = (size_t)file.tellg();
  file.seekg(0, std::ios::beg);
  if (file_type == ori_File) {
    if (length < bytes)
      throw Error(PRISM_ERR_ARG, "File read incomplete or corrupted: " + filename + " holds " +
                                     std::to_string(length) + " bytes, expected " + std::to_string(bytes));
  } else {
    // a container: the buffer takes the file's length; the device copy must
    // be large enough for it
    if (length > bytes && d) throw Error(PRISM_ERR_ARG, "container larger than the buffer: " + filename);
    bytes = length;
  }
  if (h) cudaFreeHost(h);
  h = nullptr;
  cuda_ok(cudaMallocHost(&h, length ? length : 1), "cudaMallocHost");
  file.read(reinterpret_cast<char*>(h), (std::streamsize)bytes);
}

void Buffer::unload_tofile(const std::string filename, typetofile tf) {
  if (tf == typetofile::deviceTofile) D2H();
  std::ofstream out(filename, std::ios::binary);
  if (!out) {
    std::cerr << "can't open file" << std::endl;
    return;
  }
  out.write(reinterpret_cast<char*>(h), (std::streamsize)bytes);
  std::cout << "decompressed file written: " << filename << '\n';
}

void Buffer::unload_tofile(const std::string filename, long long numBytes, typetofile tf) {
  if (tf == typetofile::deviceTofile) D2H(numBytes);
  std::ofstream out(filename, std::ios::binary);
  if (!out) {
    std::cerr << "can't open file" << std::endl;
    return;
  }
  std::cout << "compressed file written: " << filename << '\n';
  out.write(reinterpret_cast<char*>(h), numBytes);
}

void Buffer::D2H(long long numBytes) {
  cuda_ok(cudaMemcpy(h, d, numBytes < 0 ? bytes : (size_t)numBytes, cudaMemcpyDeviceToHost), "D2H");
}
void Buffer::D2H_cudaasync(void* stream, long long numBytes) {
  cuda_ok(cudaMemcpyAsync(h, d, numBytes < 0 ? bytes : (size_t)numBytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream),
          "D2H");
}
void Buffer::H2D(long long numBytes) {
  cuda_ok(cudaMemcpy(d, h, numBytes < 0 ? bytes : (size_t)numBytes, cudaMemcpyHostToDevice), "H2D");
}
void Buffer::H2D_cudaasync(void* stream, long long numBytes) {
  cuda_ok(cudaMemcpyAsync(d, h, numBytes < 0 ? bytes : (size_t)numBytes, cudaMemcpyHostToDevice, (cudaStream_t)stream),
          "H2D");
}

template void Buffer::load_fromfile<ori_File>(const std::string);
template void Buffer::load_fromfile<cmp_File>(const std::string);

Bitplane::Bitplane(int x, int y, int z) {
  dtype = U1;
  tsize = 1;
  lx = (uint32_t)x;
  ly = (uint32_t)y;
  lz = (uint32_t)z;
  len = (size_t)x * y * z;
  ndim = lz > 1 ? 3 : (ly > 1 ? 2 : 1);
  ori_size = len * 4;
  aligned_size = prism_plane_buffer_size(lx, ly, lz);
  aligned_len = aligned_size / 4;
  bytes = aligned_size + 64;  // the decoder and shuffles address a little past the last plane
  cuda_ok(cudaMalloc(&d, bytes), "cudaMalloc");
  cuda_ok(cudaMemset(d, 0, bytes), "cudaMemset");
}

}  // namespace prism
