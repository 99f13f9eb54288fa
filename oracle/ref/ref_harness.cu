// Stage-dump harness for the reference PRISM build (test infrastructure only).
//
// Drives the reference library through its own public C++ API
// (include/compressor.hpp, InterpolationPredictor.hpp, bitplane.hpp, zbpc.hpp,
// dataloader.hpp) exactly in the order Compressor::compress_pipeline
// (src/compressor.cu:120-130), decompress_pipeline (:153-164) and
// decompress_progressive_pipeline (:166-190) use, and writes every
// intermediate buffer to a directory so the CPU oracle can be pinned stage by
// stage.  Two deliberate differences from the CLI, both to keep the run safe:
//   * REL mode computes max-min on the host instead of calling extrema_scan,
//     whose cudaFree of two uninitialised pointers (src/compressor.cu:299-300)
//     can abort the process;
//   * the quant-code buffer `qc` and the bit-plane buffer get zeroed slack
//     after their ends, because bitShuffle reads (and inverse_bitShuffle
//     writes) up to anchors+align codes past n, and for some shapes writes
//     up to ~2 KiB past the plane buffer (src/predictor/bitplane.cu:180-181,
//     203-259, 401-402).  The slack makes those accesses land in owned,
//     zeroed memory.
//
// usage: ref_harness f|d nx ny nz A|R bound SM|NB infile outdir [target ...]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "compressor.hpp"
#include "InterpolationPredictor.hpp"
#include "bitplane.hpp"
#include "zbpc.hpp"
#include "dataloader.hpp"

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { \
  fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); exit(3);} } while (0)

static void dump(const std::string& path, const void* host, size_t bytes) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) { perror(path.c_str()); exit(4); }
  fwrite(host, 1, bytes, f);
  fclose(f);
}

static void dump_dev(const std::string& path, const void* dev, size_t bytes) {
  std::vector<unsigned char> h(bytes);
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(h.data(), dev, bytes, cudaMemcpyDeviceToHost));
  dump(path, h.data(), bytes);
}

// Replace a device buffer by one with zeroed slack after its `bytes`.
static void pad_dev(void** d, size_t bytes, size_t slack_bytes) {
  CK(cudaFree(*d));
  CK(cudaMalloc(d, bytes + slack_bytes));
  CK(cudaMemset(*d, 0, bytes + slack_bytes));
}
static bool big_dumps() { return getenv("HARNESS_SMALL") == nullptr; }

template <typename T>
static int run(int argc, char** argv) {
  prism_context* cfg = new prism_context;
  cfg->dtype = sizeof(T) == 4 ? F4 : F8;
  cfg->x = atoi(argv[2]); cfg->y = atoi(argv[3]); cfg->z = atoi(argv[4]);
  cfg->ndim = cfg->z > 1 ? 3 : (cfg->y > 1 ? 2 : 1);
  cfg->size = cfg->x * cfg->y * cfg->z;
  bool rel = argv[5][0] == 'R';
  double bound = atof(argv[6]);
  cfg->bt = strcmp(argv[7], "NB") == 0 ? NB : SM;
  std::string in_path = argv[8], out = argv[9];
  std::vector<double> targets;
  for (int i = 10; i < argc; ++i) targets.push_back(atof(argv[i]));
  CK(cudaMalloc(&cfg->begin, 4 * sizeof(int)));
  CK(cudaMalloc(&cfg->end, 4 * sizeof(int)));
  CK(cudaMemset(cfg->begin, 0, 4 * sizeof(int)));
  CK(cudaMemset(cfg->end, 0, 4 * sizeof(int)));
  cudaStream_t stream;
  CK(cudaStreamCreate(&stream));
  const size_t n = cfg->size;
  const size_t slack = (n / 4 + 65536) * sizeof(int);

  auto* input = new prism::StatBuffer<T>(cfg->dtype, 0, cfg->x, cfg->y, cfg->z);
  {
    FILE* f = fopen(in_path.c_str(), "rb");
    if (!f || fread(input->h, sizeof(T), n, f) != n) { fprintf(stderr, "bad input\n"); return 5; }
    fclose(f);
  }
  input->H2D();
  const T* hin = (const T*)input->h;
  double mn = hin[0], mx = hin[0];
  for (size_t i = 1; i < n; ++i) { double v = hin[i]; mn = v < mn ? v : mn; mx = v > mx ? v : mx; }
  if (rel) {
    cfg->error_mode = REL; cfg->rel_eb = bound;
    input->minVal = mn; input->maxVal = mx; input->range = mx - mn;
    cfg->eb = cfg->rel_eb * input->range;
  } else {
    cfg->error_mode = ABS; cfg->eb = bound; cfg->rel_eb = 0;
  }
  FILE* meta = fopen((out + "/meta.txt").c_str(), "w");
  fprintf(meta, "eb %.17g\nrange %.17g\n", cfg->eb, input->range);

  // ---------------- compress, stage by stage ----------------
  auto* cmp = new prism::Compressor<T, i4>();
  cmp->init(cfg);
  pad_dev(&cmp->qc->d, cmp->qc->bytes, slack);
  pad_dev(&cmp->bp->d, cmp->bp->aligned_size, 1 << 20);
  double t = 0;
  spline_construct<T, i4, T>(input, cmp->ap, cmp->qc, cmp->bp->d, cmp->ol, cfg->eb, cfg->rel_eb,
                             cmp->radius, cfg->intp_param, cmp->profiling_errors, t, stream);
  CK(cudaStreamSynchronize(stream));
  CK(cudaGetLastError());
  dump(out + "/errors.bin", cmp->profiling_errors->h, 18 * sizeof(T));
  fprintf(meta, "use_md %d %d %d %d\nreverse %d %d %d %d\n", cfg->intp_param.use_md[0],
          cfg->intp_param.use_md[1], cfg->intp_param.use_md[2], cfg->intp_param.use_md[3],
          cfg->intp_param.reverse[0], cfg->intp_param.reverse[1], cfg->intp_param.reverse[2],
          cfg->intp_param.reverse[3]);
  fprintf(meta, "alpha %.17g\n", cfg->intp_param.alpha);
  if (big_dumps()) dump_dev(out + "/qc.bin", cmp->qc->d, cmp->qc->bytes);
  dump_dev(out + "/anchors.bin", cmp->ap->d, cmp->ap->bytes);
  if (big_dumps()) dump_dev(out + "/ectrl_tmp.bin", cmp->bp->d, cmp->bp->aligned_size);
  if (cfg->bt == SM) convert_to_bitplane<i4, SM>(cmp->qc, cmp->bp, cmp->ap->len, t, stream);
  else convert_to_bitplane<i4, NB>(cmp->qc, cmp->bp, cmp->ap->len, t, stream);
  CK(cudaStreamSynchronize(stream));
  if (big_dumps()) dump_dev(out + "/planes.bin", cmp->bp->d, cmp->bp->aligned_size);
  uint8_t* cptr = (uint8_t*)cmp->compressed_data->d;
  cmp->compressed_lossless_size =
      lossless_encode(cmp->bp, cptr, cmp->compressedSize_bp_d, input->bytes, t, stream);
  cmp->compress_merge(cfg, input->range, stream);
  CK(cudaStreamSynchronize(stream));
  CK(cudaGetLastError());
  fprintf(meta, "lossless_size %zu\ntotal_size %zu\n", cmp->compressed_lossless_size,
          cmp->total_compressed_size);
  dump_dev(out + "/cmp.bin", cmp->compressed_data->d, cmp->total_compressed_size);
  std::vector<unsigned char> container(cmp->total_compressed_size);
  CK(cudaMemcpy(container.data(), cmp->compressed_data->d, container.size(), cudaMemcpyDeviceToHost));
  delete cmp;

  auto load_container = [&](prism::Compressor<T, i4>* d) {
    d->init(cfg);
    pad_dev(&d->qc->d, d->qc->bytes, slack);
    pad_dev(&d->bp->d, d->bp->aligned_size, 1 << 20);
    d->compressed_data->bytes = container.size();
    CK(cudaMemcpy(d->compressed_data->d, container.data(), container.size(), cudaMemcpyHostToDevice));
  };

  // ---------------- full decompress ----------------
  if (cfg->bt == SM) {
    auto* dec = new prism::Compressor<T, i4>();
    load_container(dec);
    auto* outb = new prism::StatBuffer<T>(cfg->dtype, 0, cfg->x, cfg->y, cfg->z);
    dec->template decompress_scatter<1>(cfg, stream);
    CK(cudaStreamSynchronize(stream));
    if (cfg->error_mode == REL) cfg->eb = cfg->rel_eb * dec->range;
    lossless_decode(cptr = (uint8_t*)dec->compressed_data->d, dec->bp, outb->bytes, t, stream);
    CK(cudaStreamSynchronize(stream));
    if (big_dumps()) dump_dev(out + "/dec_planes.bin", dec->bp->d, dec->bp->aligned_size);
    inverse_convert_to_bitplane<i4, SM>(dec->bp, dec->qc, dec->ap->len, t, stream);
    CK(cudaStreamSynchronize(stream));
    if (big_dumps()) dump_dev(out + "/dec_qc.bin", dec->qc->d, dec->qc->bytes);
    dec->decompress_predict(cfg, outb, stream);
    CK(cudaStreamSynchronize(stream));
    CK(cudaGetLastError());
    dump_dev(out + "/dec.bin", outb->d, outb->bytes);
    delete dec;
    delete outb;
  }

  // ---------------- progressive decompress ----------------
  if (!targets.empty()) {
    prism::StatBuffer<T>* old = nullptr;
    for (size_t i = 0; i < targets.size(); ++i) {
      auto* dec = new prism::Compressor<T, i4>();
      load_container(dec);
      auto* nw = new prism::StatBuffer<T>(cfg->dtype, 0, cfg->x, cfg->y, cfg->z);
      double target = targets[i];
      double last = i == 0 ? 0 : targets[i - 1];
      // decompress_scatter<0> is not emitted by the library; <1> followed by
      // clearing the anchors is the same thing (later steps decode a delta).
      dec->template decompress_scatter<1>(cfg, stream);
      CK(cudaStreamSynchronize(stream));
      if (last != 0) CK(cudaMemset(dec->ap->d, 0, dec->ap->bytes));
      if (cfg->error_mode == REL) { cfg->eb = cfg->rel_eb * dec->range; target *= dec->range; }
      findStrategy_h<i4>(dec->compressedSize_bp_d, dec->begin, dec->end, cfg->eb, target, t, stream);
      CK(cudaStreamSynchronize(stream));
      CK(cudaDeviceSynchronize());
      int b[4], e[4], ml = -1;
      CK(cudaMemcpy(b, cfg->begin, sizeof(b), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(e, cfg->end, sizeof(e), cudaMemcpyDeviceToHost));
      CK(cudaMemcpyFromSymbol(&ml, maxlevel, sizeof(int)));
      fprintf(meta, "step %zu target %.17g begin %d %d %d %d end %d %d %d %d maxlevel %d\n", i, target,
              b[0], b[1], b[2], b[3], e[0], e[1], e[2], e[3], ml);
      cptr = (uint8_t*)dec->compressed_data->d;
      lossless_decode_progressive(cptr, dec->bp, nw->bytes, dec->begin, dec->end, t, stream);
      CK(cudaStreamSynchronize(stream));
      if (big_dumps()) dump_dev(out + "/prog" + std::to_string(i) + "_planes.bin", dec->bp->d, dec->bp->aligned_size);
      inverse_convert_to_bitplane_progressive<i4, NB>(dec->bp, dec->qc, dec->ap->len, dec->begin, dec->end, t, stream);
      CK(cudaStreamSynchronize(stream));
      if (big_dumps()) dump_dev(out + "/prog" + std::to_string(i) + "_qc.bin", dec->qc->d, dec->qc->bytes);
      if (last == 0) dec->decompress_predict(cfg, nw, stream);
      else dec->decompress_progressive_predict(cfg, old, nw, stream);
      CK(cudaStreamSynchronize(stream));
      CK(cudaGetLastError());
      dump_dev(out + "/prog" + std::to_string(i) + ".bin", nw->d, nw->bytes);
      delete dec;
      if (old) delete old;
      old = nw;
    }
    delete old;
  }
  fclose(meta);
  delete input;
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 10) {
    fprintf(stderr, "usage: %s f|d nx ny nz A|R bound SM|NB infile outdir [target ...]\n", argv[0]);
    return 2;
  }
  return argv[1][0] == 'd' ? run<double>(argc, argv) : run<float>(argc, argv);
}
