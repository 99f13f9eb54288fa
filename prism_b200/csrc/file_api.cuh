// Container files (prism_file_* in prism_b200.h).  Included at the end of
// prism_b200.cu.
//
// Saving streams the device container to disk through two pinned staging
// buffers: the device-to-host copy of one piece overlaps the write of the
// previous one.  Progressive retrieval from a file reads the stream header,
// the 16-bit chunk size table and the trailer once, then per step only the
// chunks of the newly selected planes (the chunks of consecutive planes of a
// level are consecutive in the stream, so one read per level), which it copies
// into a device image of the container before running the usual progressive
// step on that image.  The reference instead reloads and copies the whole file
// for every target (src/prism.cu:131-135).
#include <cstdio>

namespace {

constexpr uint64_t kFilePiece = 64ull << 20;

struct PinnedBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMallocHost(&p, n);
    if (e == cudaSuccess) cap = n;
    return e;
  }
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
};

}  // namespace

int prism_file_save(const char* path, const void* d_container, uint64_t size, void* stream) {
  if (!path || !d_container || size == 0) return PRISM_ERR_ARG;
  FILE* fp = fopen(path, "wb");
  if (!fp) return PRISM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  PinnedBuf buf[2];
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int rc = PRISM_OK;
  const uint64_t piece = std::min(size, kFilePiece);
  for (int i = 0; i < 2 && !rc; ++i)
    if (buf[i].ensure(piece) != cudaSuccess || cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess)
      rc = PRISM_ERR_NOMEM;
  // piece k is copied into buf[k % 2]; while it lands, piece k-1 is written
  std::thread writer;
  uint64_t written = 0;
  bool write_ok = true;
  const uint8_t* src = (const uint8_t*)d_container;
  uint64_t npieces = (size + piece - 1) / piece;
  for (uint64_t k = 0; k < npieces && !rc; ++k) {
    const int b = (int)(k & 1);
    const uint64_t off = k * piece, len = std::min(piece, size - off);
    // buf[b] was last written out by the writer of piece k-2, joined already
    if (cudaMemcpyAsync(buf[b].p, src + off, len, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaEventRecord(ev[b], st) != cudaSuccess) {
      rc = PRISM_ERR_CUDA;
      break;
    }
    if (writer.joinable()) writer.join();  // piece k-1 was written while piece k copied
    if (cudaEventSynchronize(ev[b]) != cudaSuccess) {
      rc = PRISM_ERR_CUDA;
      break;
    }
    writer = std::thread([&, b, len]() {
      if (fwrite(buf[b].p, 1, len, fp) != len) write_ok = false;
      written += len;
    });
  }
  if (writer.joinable()) writer.join();
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  if (fclose(fp) != 0) write_ok = false;
  if (!rc && (!write_ok || written != size)) rc = PRISM_ERR_ARG;
  return rc;
}

struct prism_file {
  prism_handle* h = nullptr;
  FILE* fp = nullptr;
  uint64_t file_size = 0, bytes_read = 0;
  Geometry g;
  int tsize = 4, mode = 1;
  double bound = 0, range = 1;
  uint64_t csbp[128];
  std::vector<uint64_t> offs;  // byte offset of each chunk from the file start
  std::vector<uint16_t> sizes;
  uint8_t* d_image = nullptr;  // device copy of the container, filled as needed
  PinnedBuf stage;
  prism_prog* prog = nullptr;
  int begin[4] = {0, 0, 0, 0}, end[4] = {0, 0, 0, 0}, maxlevel = 4;
};

namespace {

int file_read(prism_file* f, uint64_t off, uint64_t len, void* dst) {
  if (fseeko(f->fp, (off_t)off, SEEK_SET) != 0) return PRISM_ERR_CORRUPT;
  if (fread(dst, 1, len, f->fp) != len) return PRISM_ERR_CORRUPT;
  f->bytes_read += len;
  return PRISM_OK;
}

// Read [off, off + len) of the file into the device image at the same offset.
int file_fetch(prism_file* f, uint64_t off, uint64_t len, cudaStream_t st) {
  while (len > 0) {
    const uint64_t n = std::min(len, kFilePiece);
    if (f->stage.ensure(n) != cudaSuccess) return PRISM_ERR_NOMEM;
    int rc = file_read(f, off, n, f->stage.p);
    if (rc) return rc;
    if (cudaMemcpyAsync(f->d_image + off, f->stage.p, n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return PRISM_ERR_CUDA;
    off += n;
    len -= n;
  }
  return PRISM_OK;
}

}  // namespace

int prism_file_open(prism_handle* h, const char* path, int dtype_size, uint32_t nx, uint32_t ny, uint32_t nz,
                    int mode, double bound, prism_file** out) {
  if (!h || !path || !out || (dtype_size != 4 && dtype_size != 8) || !dims_ok(nx, ny, nz) || !(bound > 0) ||
      (mode != 0 && mode != 1))
    return PRISM_ERR_ARG;
  *out = nullptr;
  prism_file* f = new (std::nothrow) prism_file();
  if (!f) return PRISM_ERR_NOMEM;
  f->h = h;
  f->tsize = dtype_size;
  f->mode = mode;
  f->bound = bound;
  make_geometry(nx, ny, nz, dtype_size, &f->g);
  const Geometry& g = f->g;
  int rc = PRISM_OK;
  f->fp = fopen(path, "rb");
  if (!f->fp) rc = PRISM_ERR_ARG;
  if (!rc && (fseeko(f->fp, 0, SEEK_END) != 0 || (f->file_size = (uint64_t)ftello(f->fp)) == 0)) rc = PRISM_ERR_CORRUPT;
  const uint64_t table = 8 + 2 * (uint64_t)g.chunks;
  if (!rc && f->file_size < table + g.header_size) rc = PRISM_ERR_CORRUPT;
  std::vector<uint8_t> head(table), trailer(g.header_size);
  if (!rc) rc = file_read(f, 0, table, head.data());
  if (!rc) rc = file_read(f, f->file_size - g.header_size, g.header_size, trailer.data());
  if (!rc) {
    f->sizes.resize(g.chunks);
    memcpy(f->sizes.data(), head.data() + 8, 2 * (size_t)g.chunks);
    f->offs.resize(g.chunks + 1);
    uint64_t at = table;
    for (int64_t i = 0; i < g.chunks; ++i) {
      f->offs[i] = at;
      at += f->sizes[i];
    }
    f->offs[g.chunks] = at;
    if (at > f->file_size - g.header_size) rc = PRISM_ERR_CORRUPT;
    memcpy(&f->range, trailer.data() + 8, 8);
    memcpy(f->csbp, trailer.data() + 16, 1024);
  }
  if (!rc && cudaMalloc(&f->d_image, f->file_size) != cudaSuccess) rc = PRISM_ERR_NOMEM;
  if (!rc && (cudaMemcpy(f->d_image, head.data(), table, cudaMemcpyHostToDevice) != cudaSuccess ||
              cudaMemcpy(f->d_image + f->file_size - g.header_size, trailer.data(), g.header_size,
                         cudaMemcpyHostToDevice) != cudaSuccess))
    rc = PRISM_ERR_CUDA;
  if (!rc) rc = prism_progressive_open(h, f->d_image, f->file_size, dtype_size, nx, ny, nz, mode, bound, &f->prog);
  if (rc) {
    prism_file_close(f);
    return rc;
  }
  *out = f;
  return PRISM_OK;
}

int prism_file_step(prism_file* f, double target_error, void* d_values, void* stream) {
  if (!f || !d_values || !(target_error > 0)) return PRISM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  // the step's plane selection (the same strategy the device step runs)
  int b[4], e[4], ml = f->maxlevel;
  for (int i = 0; i < 4; ++i) { b[i] = f->begin[i]; e[i] = f->end[i]; }
  const double eb = f->mode == 1 ? f->bound * f->range : f->bound;
  const double te = f->mode == 1 ? target_error * f->range : target_error;
  int rc = prism_find_strategy(f->h, f->csbp, eb, te, b, e, &ml, st);
  if (rc) return rc;
  // fetch the chunks of planes [b[i], e[i]) of each level (i = 3 - level)
  const Geometry& g = f->g;
  int64_t level_base = 0;
  for (int l = 3; l >= 0; --l) {
    const int i = 3 - l;
    const int64_t cpp = g.chunks_level[l] >> 5;
    if (e[i] > b[i]) {
      const int64_t c0 = level_base + b[i] * cpp, c1 = level_base + e[i] * cpp;
      rc = file_fetch(f, f->offs[c0], f->offs[c1] - f->offs[c0], st);
      if (rc) return rc;
    }
    level_base += g.chunks_level[l];
  }
  rc = prism_progressive_step(f->prog, target_error, d_values, stream);
  if (rc) return rc;
  return prism_progressive_state(f->prog, f->begin, f->end, &f->maxlevel, nullptr);
}

int prism_file_info(const prism_file* f, uint64_t* file_bytes, uint64_t* bytes_read, int end[4]) {
  if (!f) return PRISM_ERR_ARG;
  if (file_bytes) *file_bytes = f->file_size;
  if (bytes_read) *bytes_read = f->bytes_read;
  if (end)
    for (int i = 0; i < 4; ++i) end[i] = f->end[i];
  return PRISM_OK;
}

void prism_file_close(prism_file* f) {
  if (!f) return;
  if (f->prog) prism_progressive_close(f->prog);
  if (f->d_image) cudaFree(f->d_image);
  if (f->fp) fclose(f->fp);
  delete f;
}
