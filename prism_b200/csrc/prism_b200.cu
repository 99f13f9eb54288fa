// prism_b200 C ABI: pipeline orchestration over the sm_100a kernels.
//
// One stream, no host round trip inside a pipeline: the REL range, the
// auto-tune decisions, the per-level bounds, the chunk offsets and the output
// size all stay in device memory and the host reads back one small status
// block at the end of a call.  Device workspace is cached in the handle and
// only grows.
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "../../include/prism_b200.h"
#include "autotune.cuh"
#include "bitplane.cuh"
#include "geometry.h"
#include "predict.cuh"
#include "report.cuh"
#include "strategy.cuh"
#include "zbpc.cuh"

using namespace prism_b200;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = bytes + bytes / 8 + 256;
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  template <class U> U* as() const { return reinterpret_cast<U*>(p); }
};

// small device scratch block
struct Small {
  double range;
  double eb;
  uint64_t lossless_size;
  uint64_t padded_size;
  unsigned long long ticket;
  int error_flag;
  int pad;
  uint64_t csbp[128];
  unsigned char params[256];
  StrategyState sstate;
  StrategyBest sblk[kStrategyCells];
  double errors[16];
  double minmax[2];
  int dec_begin[4];  // progressive exact mode: the first plane whose chunks a step decodes, per level
  unsigned char params_odd[256];  // parameters of odd progressive steps (even steps: params)
};

struct HostResult {
  uint64_t padded_size;
  int error_flag;
  int pad;
  unsigned char params[256];
  double errors[16];
};

}  // namespace

// pipeline stages timed when profiling is on (prism_profile)
enum Stage { kStExtrema, kStAutotune, kStPredict, kStShuffle, kStEncode, kStTrailer, kStStrategy, kStDecode,
             kStInverse, kStReconstruct, kStCount };

// What a progressive step publishes for the host: the plane state, the
// error flag and the payload bytes of the planes loaded so far.
struct ProgMirror {
  StrategyState state;
  int err;
  uint64_t loaded;
};

struct prism_handle {
  DevBuf qc, planes, status, offs, bsum, part, wins, ranges, anchors, small, dev_in, dev_out, zero_anchors;
  DevBuf qc_odd;  // the code buffer of a progressive object's odd-numbered steps
  DevBuf ext;     // per-CTA partials of the extrema scan
  DevBuf sbatch;  // batched strategy searches: cells, inputs and states
  // Pinned host memory mapped into the device: kernels store the results the
  // host reads (sizes, flags, parameters, progressive state) straight into
  // it, so reading them waits only for the kernels, never behind other
  // device-to-host copies in flight on the copy engines.
  HostResult* host = nullptr;
  HostResult* host_dev = nullptr;  // device alias of host
  std::string err;
  int sm_count = 148;
  uint64_t launches = 0;       // kernels launched by this handle
  uint32_t prof = 0;  // bit i: time stage i
  // per stage, one event pair per launch since the last collection (steps
  // are enqueued back to back, so several launches of a stage can be pending)
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[kStCount];
  int ev_used[kStCount] = {};
  double acc_ms[kStCount] = {};
  int acc_n[kStCount] = {};
  // side stream for the edge-tile launches, which run beside the interior
  // launch (the two write disjoint tiles)
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // Progressive steps run their strategy, plan, decode and inverse shuffle on
  // `dec` so that they overlap the previous step's reconstruction: step k
  // writes its codes and parameters to slot k mod 2 (qc / qc_odd, params /
  // params_odd), whose last reader was the reconstruction of step k - 2
  // (event recon_done[slot]); the plane buffer is only touched on `dec`.
  // epoch counts the calls that use the handle's buffers; a step takes the
  // short wait only when the previous such call was the previous step of the
  // same object on the same stream.
  cudaStream_t dec = nullptr;
  cudaEvent_t dec_call = nullptr, dec_done = nullptr, recon_done[2] = {nullptr, nullptr};
  uint64_t epoch = 0, chain_epoch = 0;
  const void* chain_prog = nullptr;
  cudaStream_t chain_stream = nullptr;
  // device state slots of the progressive objects opened on this handle
  // (no allocation per open); bit i of prog_used = slot i taken
  DevBuf prog_slots;
  uint64_t prog_used = 0;
  ProgMirror* prog_host = nullptr;  // 64 mapped mirrors, one per slot
  ProgMirror* prog_host_dev = nullptr;
  // per slot: the chunk offsets of the slot's container, computed by its
  // first step and reused by the later ones
  DevBuf prog_offs[64];
  size_t zero_anchors_ready = 0;  // leading bytes of zero_anchors known to be zero
  // dimensions whose auto-tune sample windows `wins` holds (the windows
  // depend on the dimensions only; uploading them from pageable memory would
  // make the host wait for the stream at every compression)
  uint32_t wins_dims[3] = {0, 0, 0};
};

constexpr int kProgSlotBytes = 128;  // StrategyState + error flag

static cudaError_t host_mapped(size_t bytes, void** host, void** dev) {
  cudaError_t e = cudaHostAlloc(host, bytes, cudaHostAllocMapped);
  if (e != cudaSuccess) return e;
  memset(*host, 0, bytes);
  e = cudaHostGetDevicePointer(dev, *host, 0);
  if (e != cudaSuccess) {
    cudaFreeHost(*host);
    *host = nullptr;
  }
  return e;
}

// Run `interior` on st and `edge` on the handle's side stream concurrently;
// st waits for both before its next work.
template <class FI, class FE>
static cudaError_t fork_join(prism_handle* h, cudaStream_t st, bool have_interior, bool have_edge, FI interior,
                             FE edge) {
  if (!have_interior || !have_edge) {
    if (have_interior) interior(st);
    if (have_edge) edge(st);
    return cudaGetLastError();
  }
  cudaError_t e = cudaSuccess;
  if (!h->side) {
    e = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
  }
  if ((e = cudaEventRecord(h->fork, st)) != cudaSuccess) return e;
  if ((e = cudaStreamWaitEvent(h->side, h->fork, 0)) != cudaSuccess) return e;
  edge(h->side);
  if ((e = cudaEventRecord(h->join, h->side)) != cudaSuccess) return e;
  interior(st);
  if ((e = cudaStreamWaitEvent(st, h->join, 0)) != cudaSuccess) return e;
  return cudaGetLastError();
}

static void prof_begin(prism_handle* h, int stage, cudaStream_t st) {
  if (!((h->prof >> stage) & 1u)) return;
  auto& v = h->ev[stage];
  if (h->ev_used[stage] == (int)v.size()) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess) return;
    if (cudaEventCreate(&b) != cudaSuccess) {
      cudaEventDestroy(a);
      return;
    }
    v.emplace_back(a, b);
  }
  cudaEventRecord(v[h->ev_used[stage]].first, st);
  h->ev_used[stage] += 1;
}
static void prof_end(prism_handle* h, int stage, cudaStream_t st) {
  if (!((h->prof >> stage) & 1u) || h->ev_used[stage] == 0) return;
  cudaEventRecord(h->ev[stage][h->ev_used[stage] - 1].second, st);
}
// fold the recorded stage times into the accumulators (waits for them)
static void prof_collect(prism_handle* h) {
  for (int i = 0; i < kStCount; ++i) {
    for (int k = 0; k < h->ev_used[i]; ++k) {
      float ms = 0;
      const auto& e = h->ev[i][k];
      if (cudaEventSynchronize(e.second) == cudaSuccess && cudaEventElapsedTime(&ms, e.first, e.second) == cudaSuccess) {
        h->acc_ms[i] += ms;
        h->acc_n[i] += 1;
      }
    }
    h->ev_used[i] = 0;
  }
}

// A progressive retrieval in flight.  Its plane state and error flag live in
// device memory, so steps are enqueued back to back without waiting; the
// host copy of the state is refreshed when a caller asks for it.
struct prism_prog {
  prism_handle* h;
  const uint8_t* cont;
  uint64_t size;
  int tsize;
  Geometry g;
  int mode;
  double bound;
  int steps;
  StrategyState state;          // host copy, valid when !pending
  StrategyState* d_state = nullptr;
  int* d_err = nullptr;         // chunk errors of every step so far
  int slot = -1;                // slot in the handle's state block, or -1 (own allocation)
  bool offs_ready = false;      // the slot's chunk offsets hold this container's
  ProgMirror* mirror = nullptr;      // mapped host copy written by each step
  ProgMirror* mirror_dev = nullptr;
  uint64_t loaded = 0;          // host copy, valid when !pending
  cudaEvent_t done = nullptr;   // recorded after the last enqueued step
  bool pending = false;
  bool exact = false;           // later steps decode the chunks of plane begin - 1 as well
};

static int fail(prism_handle* h, int code, const char* what, cudaError_t e = cudaSuccess) {
  if (h) {
    h->err = what;
    if (e != cudaSuccess) {
      h->err += ": ";
      h->err += cudaGetErrorString(e);
    }
  }
  return code;
}

#define CK(call)                                                   \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return fail(h, PRISM_ERR_CUDA, #call, e_); \
  } while (0)

#define CKA(call)                                                    \
  do {                                                               \
    cudaError_t e_ = (call);                                         \
    if (e_ != cudaSuccess) return fail(h, PRISM_ERR_NOMEM, #call, e_); \
  } while (0)

static bool dims_ok(uint32_t nx, uint32_t ny, uint32_t nz) {
  return nx >= 1 && ny >= 1 && nz >= 1 && (uint64_t)nx * ny * nz >= 2;
}

// code buffer: level-major codes plus the slack the reference's shuffle reads
static uint64_t qc_len(const Geometry& g) {
  int64_t end0 = (int64_t)g.n + g.align_dev;
  int64_t last = g.sh_grid * (int64_t)kChunk + 64;
  return g.anchors + (uint64_t)std::max(end0, last) + 64;
}

static Small* small(prism_handle* h) {
  ++h->epoch;
  return h->small.as<Small>();
}

// Raise a kernel's dynamic shared-memory limit, once per device.
template <auto Kernel>
static cudaError_t smem_limit(int bytes) {
  static std::mutex m;
  static bool done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  std::lock_guard<std::mutex> lock(m);
  if (!done[dev]) {
    e = cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    done[dev] = true;
  }
  return cudaSuccess;
}

// The tile kernels run as two launches: interior tiles (part 0) and the tiles
// on the field's last slabs (part 1), on two streams.
template <class T>
static int launch_predict(prism_handle* h, const T* in, const Geometry& g, const PredParams<T>* pp, T* anchors,
                          int32_t* qc, cudaStream_t st) {
  const int smem = compress_smem_bytes<T>();
  constexpr auto k0 = predict_compress_kernel<T, 0>;
  constexpr auto k1 = predict_compress_kernel<T, 1>;
  CK(smem_limit<k0>(smem));
  CK(smem_limit<k1>(smem));
  uint64_t n0 = tiles_in_part(g, 0), n1 = tiles_in_part(g, 1);
  CK(fork_join(
      h, st, n0 > 0, n1 > 0, [&](cudaStream_t s) { k0<<<(unsigned)n0, kPredThreads, smem, s>>>(in, g, pp, anchors, qc); },
      [&](cudaStream_t s) { k1<<<(unsigned)n1, kPredThreads, smem, s>>>(in, g, pp, anchors, qc); }));
  h->launches += (n0 > 0) + (n1 > 0);
  return PRISM_OK;
}

template <class T, bool PROG>
static int launch_reconstruct(prism_handle* h, const int32_t* qc, const T* anchors, const Geometry& g,
                              const PredParams<T>* pp, const T* old, T* out, cudaStream_t st) {
  const int smem0 = recon_smem_bytes<T>(), smem1 = recon_smem_bytes<T>();
  constexpr auto k0 = reconstruct_kernel<T, PROG, 0>;
  constexpr auto k1 = reconstruct_kernel<T, PROG, 1>;
  CK(smem_limit<k0>(smem0));
  CK(smem_limit<k1>(smem1));
  uint64_t n0 = tiles_in_part(g, 0), n1 = tiles_in_part(g, 1);
  CK(fork_join(
      h, st, n0 > 0, n1 > 0,
      [&](cudaStream_t s) { k0<<<(unsigned)n0, kPredThreads, smem0, s>>>(qc, anchors, g, pp, old, out); },
      [&](cudaStream_t s) { k1<<<(unsigned)n1, kPredThreads, smem1, s>>>(qc, anchors, g, pp, old, out); }));
  h->launches += (n0 > 0) + (n1 > 0);
  return PRISM_OK;
}

static int ensure_common(prism_handle* h, const Geometry& g) {
  ++h->epoch;
  CKA(h->qc.ensure(qc_len(g) * sizeof(int32_t)));
  CKA(h->planes.ensure(g.aligned_size + 64));
  CKA(h->status.ensure((size_t)g.chunks * sizeof(unsigned long long)));
  CKA(h->offs.ensure((size_t)g.chunks * sizeof(int64_t) + 64));
  CKA(h->bsum.ensure(((size_t)g.chunks / kScanItems + 2) * sizeof(int64_t)));
  CKA(h->anchors.ensure(g.anchors * 8 + 64));
  CKA(h->small.ensure(sizeof(Small)));
  return PRISM_OK;
}

template <class T>
static const PredParams<T>* params_ptr(prism_handle* h) {
  return reinterpret_cast<const PredParams<T>*>(small(h)->params);
}

// ---- stage launchers ----

// per_sm: extrema CTAs per SM (four fill an SM; two, with 16-byte loads, still
// keep the copy bandwidth and leave room for the auto-tune beside them)
template <class T>
static int launch_extrema(prism_handle* h, const T* in, uint64_t n, cudaStream_t st, int per_sm = 4) {
  int blocks = (int)std::min<uint64_t>((n + kExtThreads - 1) / kExtThreads, (uint64_t)h->sm_count * per_sm);
  CKA(h->ext.ensure(sizeof(T) * 2 * blocks));
  prof_begin(h, kStExtrema, st);
  extrema_kernel<T><<<blocks, kExtThreads, 0, st>>>(in, n, h->ext.as<T>());
  extrema_final_kernel<T><<<1, 32, 0, st>>>(h->ext.as<T>(), blocks, &small(h)->range, small(h)->minmax);
  prof_end(h, kStExtrema, st);
  h->launches += 2;
  CK(cudaGetLastError());
  return PRISM_OK;
}

__global__ void set_double_kernel(double* p, double v) { *p = v; }

static double alpha_of(double r);

// the auto-tune's error sums over the sample windows (no dependence on the
// error bound, so it can run beside the extrema scan)
template <class T>
static int launch_autotune(prism_handle* h, const T* in, const Geometry& g, cudaStream_t st) {
  std::vector<SampleWindow> wins = sample_grid(g.nx, g.ny, g.nz);
  const int nwin = (int)wins.size();
  CKA(h->part.ensure(sizeof(T) * 15 * std::max(nwin, 1) + 64));
  if (nwin > 0) {
    if (h->wins_dims[0] != g.nx || h->wins_dims[1] != g.ny || h->wins_dims[2] != g.nz) {
      CKA(h->wins.ensure(sizeof(SampleWindow) * nwin));
      CK(cudaMemcpyAsync(h->wins.p, wins.data(), sizeof(SampleWindow) * nwin, cudaMemcpyHostToDevice, st));
      h->wins_dims[0] = g.nx;
      h->wins_dims[1] = g.ny;
      h->wins_dims[2] = g.nz;
    }
    prof_begin(h, kStAutotune, st);
    autotune_kernel<T><<<dim3(nwin, 6), kAttThreads, 0, st>>>(in, g, h->wins.as<SampleWindow>(), h->part.as<T>());
    prof_end(h, kStAutotune, st);
    h->launches += 1;
  }
  CK(cudaGetLastError());
  return PRISM_OK;
}

// the decisions and per-level parameters from the sums (or forced flags) and
// the range
template <class T>
static int launch_params(prism_handle* h, const Geometry& g, int mode, double bound, double rel_for_alpha,
                         const uint8_t* force_flags_dev, cudaStream_t st) {
  const double alpha = alpha_of(rel_for_alpha);  // InterpolationPredictor.cu:2248-2271
  Small* s = small(h);
  if (!force_flags_dev) {
    const int nwin = (int)sample_grid(g.nx, g.ny, g.nz).size();
    params_kernel<T><<<1, 32, 0, st>>>(mode, bound, &s->range, alpha, h->part.as<T>(), nwin, nullptr, 4,
                                       reinterpret_cast<PredParams<T>*>(s->params),
                                       reinterpret_cast<T*>(s->errors), &s->eb);
  } else {
    params_kernel<T><<<1, 32, 0, st>>>(mode, bound, &s->range, alpha, nullptr, 0, force_flags_dev, 4,
                                       reinterpret_cast<PredParams<T>*>(s->params), nullptr, &s->eb);
  }
  h->launches += 1;
  CK(cudaGetLastError());
  return PRISM_OK;
}

template <class T>
static int launch_autotune_params(prism_handle* h, const T* in, const Geometry& g, int mode, double bound,
                                  double rel_for_alpha, const uint8_t* force_flags_dev, cudaStream_t st) {
  if (!force_flags_dev) {
    const int rc = launch_autotune<T>(h, in, g, st);
    if (rc) return rc;
  }
  return launch_params<T>(h, g, mode, bound, rel_for_alpha, force_flags_dev, st);
}

static double alpha_of(double r) {
  const double a1 = 2.0, a2 = 1.75, a3 = 1.5, a4 = 1.25, a5 = 1;
  const double e1 = 1e-1, e2 = 1e-2, e3 = 1e-3, e4 = 1e-4, e5 = 1e-5;
  if (r >= e1) return a1;
  if (r >= e2) return a2 + (a1 - a2) * (r - e2) / (e1 - e2);
  if (r >= e3) return a3 + (a2 - a3) * (r - e3) / (e2 - e3);
  if (r >= e4) return a4 + (a3 - a4) * (r - e4) / (e3 - e4);
  if (r >= e5) return a5 + (a4 - a5) * (r - e5) / (e4 - e5);
  return a5;
}

// zero the code slots the predictor never writes but the shuffle reads
static int zero_code_padding(prism_handle* h, const Geometry& g, cudaStream_t st) {
  int32_t* qc = h->qc.as<int32_t>();
  uint64_t c3 = g.grid[2] - g.grid[3], c2 = g.grid[1] - g.grid[2], c1 = g.grid[0] - g.grid[1];
  uint64_t c0 = g.n - g.grid[0];
  uint64_t segs[4][2] = {{g.anchors + c3, g.lm_prefix[2]},
                         {g.lm_prefix[2] + c2, g.lm_prefix[1]},
                         {g.lm_prefix[1] + c1, g.lm_prefix[0]},
                         {g.lm_prefix[0] + c0, qc_len(g)}};
  for (auto& s : segs)
    if (s[1] > s[0]) CK(cudaMemsetAsync(qc + s[0], 0, (s[1] - s[0]) * sizeof(int32_t), st));
  return PRISM_OK;
}

static int launch_bitshuffle(prism_handle* h, const int32_t* qc, const Geometry& g, int nb, uint8_t* planes,
                             cudaStream_t st) {
  int64_t start_last = (g.sh_grid - 1) * (int64_t)kChunk;
  ShufPlan plan = make_shuf_plan(g, start_last);
  RangeList rng;
  int nr = fill_ranges(g, plan, rng.r, kMaxRanges);
  prof_begin(h, kStShuffle, st);
  if (nr > 0) {
    leftover_fill_kernel<<<nr, 256, 0, st>>>(planes, qc, g, rng, nr);
    h->launches += 1;
  }
  const int32_t* codes = qc + g.anchors;
  bool last_last = last_block_lands_last(g);
  if (!last_last) shuffle_last_block_kernel<<<shuffle_last_block_grid(g), 512, 0, st>>>(codes, planes, g, nb, g.aligned_size);
  if (plan.items > 0) {
    int64_t blocks = (plan.items + kShufWarps - 1) / kShufWarps;
    bitshuffle_kernel<<<(unsigned)blocks, kShufWarps * 32, 0, st>>>(codes, planes, g, plan, nb);
  }
  if (last_last) shuffle_last_block_kernel<<<shuffle_last_block_grid(g), 512, 0, st>>>(codes, planes, g, nb, g.aligned_size);
  prof_end(h, kStShuffle, st);
  h->launches += 1 + (plan.items > 0);
  CK(cudaGetLastError());
  return PRISM_OK;
}

static int launch_inverse(prism_handle* h, const uint8_t* planes, const Geometry& g, int nb, const int* dbegin,
                          const int* dend, int32_t* qc, cudaStream_t st) {
  int64_t start_last = (g.sh_grid - 1) * (int64_t)kChunk;
  // positions from the last block on are only partly written: start from 0
  uint64_t from = g.anchors + (uint64_t)start_last;
  uint64_t to = qc_len(g);
  if (to > from) CK(cudaMemsetAsync(qc + from, 0, (to - from) * sizeof(int32_t), st));
  ShufPlan plan = make_shuf_plan(g, start_last);
  int32_t* codes = qc + g.anchors;
  prof_begin(h, kStInverse, st);
  if (plan.items > 0) {
    int64_t blocks = (plan.items + kShufWarps - 1) / kShufWarps;
    inverse_bitshuffle_kernel<<<(unsigned)blocks, kShufWarps * 32, 0, st>>>(planes, codes, g, plan, nb, dbegin, dend);
    h->launches += 1;
  }
  inverse_last_block_kernel<<<last_block_rounds(g), 512, 0, st>>>(planes, codes, g, nb, dbegin, dend, g.aligned_size);
  prof_end(h, kStInverse, st);
  h->launches += 1;
  CK(cudaGetLastError());
  return PRISM_OK;
}

// first_ticket > 0 leaves the chunks before it unencoded, so the first
// encoded chunk's look-back never sees its predecessor published: used only by
// the self-test of the bounded wait (prism_lossless_wait_selftest).
static int launch_encode(prism_handle* h, const uint8_t* planes, const Geometry& g, uint8_t* stream,
                         cudaStream_t st, int first_ticket = 0, long long spin_limit = (long long)1 << 22) {
  Small* s = small(h);
  CK(cudaMemsetAsync(h->status.p, 0, (size_t)g.chunks * sizeof(unsigned long long), st));
  CK(cudaMemsetAsync(&s->ticket, 0, sizeof(unsigned long long), st));
  // little-endian: the low byte alone makes the 64-bit ticket counter equal to first_ticket
  if (first_ticket > 0) CK(cudaMemsetAsync(&s->ticket, first_ticket, 1, st));
  CK(cudaMemsetAsync(&s->error_flag, 0, sizeof(int), st));
  size_t smem = sizeof(EncodeShared);
  CK(smem_limit<zbpc_encode_kernel>((int)smem));
  int blocks = (int)std::min<int64_t>(g.chunks, (int64_t)h->sm_count * 4);
  prof_begin(h, kStEncode, st);
  zbpc_encode_kernel<<<blocks, kZThreads, smem, st>>>(planes, g, stream, h->status.as<unsigned long long>(),
                                                      &s->ticket, s->csbp, &s->lossless_size, &s->error_flag,
                                                      spin_limit);
  zbpc_finish_kernel<<<1, 32, 0, st>>>(stream, g, &s->lossless_size, &s->padded_size);
  prof_end(h, kStEncode, st);
  h->launches += 2;
  CK(cudaGetLastError());
  return PRISM_OK;
}

// err: where chunk errors go; null = the handle's flag, reset here
// payload offset of every chunk: exclusive prefix sum of the size table
static void launch_chunk_offsets(prism_handle* h, const uint8_t* stream, const Geometry& g, int64_t* offs,
                                 cudaStream_t st) {
  const uint16_t* sizes = reinterpret_cast<const uint16_t*>(stream + 8);
  int64_t nblk = (g.chunks + kScanItems - 1) / kScanItems;
  scan_sizes_block<<<(unsigned)nblk, 1024, 0, st>>>(sizes, g.chunks, offs, h->bsum.as<int64_t>());
  scan_block_sums<<<1, 32, 0, st>>>(h->bsum.as<int64_t>(), nblk);
  scan_add<<<(unsigned)((g.chunks + 255) / 256), 256, 0, st>>>(offs, g.chunks, h->bsum.as<int64_t>());
  h->launches += 3;
}

// offs_in: chunk offsets already computed for this stream (else computed here)
static int launch_decode(prism_handle* h, const uint8_t* stream, uint64_t stream_bytes, const Geometry& g,
                         const int* dbegin, const int* dend, uint8_t* planes, cudaStream_t st, int* err = nullptr,
                         const int64_t* offs_in = nullptr) {
  Small* s = small(h);
  prof_begin(h, kStDecode, st);
  const int64_t* offs = offs_in;
  if (!offs) {
    launch_chunk_offsets(h, stream, g, h->offs.as<int64_t>(), st);
    offs = h->offs.as<int64_t>();
  }
  if (!err) {
    err = &s->error_flag;
    CK(cudaMemsetAsync(err, 0, sizeof(int), st));
  }
  size_t smem = sizeof(DecodeShared);
  CK(smem_limit<zbpc_decode_kernel>((int)smem));
  int blocks = (int)std::min<int64_t>(g.chunks, (int64_t)h->sm_count * 8);
  zbpc_decode_kernel<<<blocks, kZThreads, smem, st>>>(stream, stream_bytes, offs, g, planes, dbegin, dend, err);
  prof_end(h, kStDecode, st);
  h->launches += 1;
  CK(cudaGetLastError());
  return PRISM_OK;
}

// trailer (compress_merge, compressor.cu:139-151): use_md[4], reverse[4],
// double range, size_t comp_size_bp[4][32], anchors
template <class T>
__global__ void trailer_kernel(uint8_t* stream, const uint64_t* padded, const PredParams<T>* p, const double* range,
                               const uint64_t* csbp, const T* anchors, uint64_t nanchors) {
  uint8_t* tr = stream + *padded;
  uint64_t total = 1040 + nanchors * sizeof(T);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    uint8_t v;
    if (i < 4) v = p->use_md[i];
    else if (i < 8) v = p->reverse[i - 4];
    else if (i < 16) v = reinterpret_cast<const uint8_t*>(range)[i - 8];
    else if (i < 1040) v = reinterpret_cast<const uint8_t*>(csbp)[i - 16];
    else v = reinterpret_cast<const uint8_t*>(anchors)[i - 1040];
    tr[i] = v;
  }
}

// the results of a pipeline call, stored into the handle's mapped host block
__global__ void publish_result_kernel(const Small* __restrict__ s, HostResult* out) {
  const int t = threadIdx.x;
  if (t == 0) {
    out->padded_size = s->padded_size;
    out->error_flag = s->error_flag;
  }
  if (t < (int)sizeof(s->params)) out->params[t] = s->params[t];
  if (t < 16) out->errors[t] = s->errors[t];
}

static int finish(prism_handle* h, cudaStream_t st) {
  publish_result_kernel<<<1, 256, 0, st>>>(small(h), h->host_dev);
  h->launches += 1;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  prof_collect(h);
  if (h->host->error_flag == 1) return fail(h, PRISM_ERR_TIMEOUT, "look-back wait exceeded its limit");
  if (h->host->error_flag == 2) return fail(h, PRISM_ERR_CORRUPT, "corrupt lossless chunk");
  return PRISM_OK;
}

template <class T>
static int compress_t(prism_handle* h, const T* in, const Geometry& g, int mode, double bound, int nb,
                      uint8_t* out, uint64_t cap, uint64_t* out_size, uint8_t* flags_out, cudaStream_t st) {
  int rc = ensure_common(h, g);
  if (rc) return rc;
  uint64_t need = 8 + 2 * (uint64_t)g.chunks + g.aligned_size + 8 + g.header_size;
  if (cap < need) return fail(h, PRISM_ERR_ARG, "output capacity below prism_max_container_size");
  Small* s = small(h);
  if (mode == 1) {
    // the extrema scan (two CTAs per SM) and the auto-tune side by side
    int rc_ext = PRISM_OK, rc_att = PRISM_OK;
    CK(fork_join(
        h, st, true, true, [&](cudaStream_t x) { rc_ext = launch_extrema<T>(h, in, g.n, x, 2); },
        [&](cudaStream_t x) { rc_att = launch_autotune<T>(h, in, g, x); }));
    if (rc_ext) return rc_ext;
    if (rc_att) return rc_att;
  } else {
    set_double_kernel<<<1, 1, 0, st>>>(&s->range, 1.0);
    rc = launch_autotune<T>(h, in, g, st);
    if (rc) return rc;
  }
  rc = launch_params<T>(h, g, mode, bound, mode == 1 ? bound : 0.0, nullptr, st);
  if (rc) return rc;
  rc = zero_code_padding(h, g, st);
  if (rc) return rc;
  prof_begin(h, kStPredict, st);
  rc = launch_predict<T>(h, in, g, params_ptr<T>(h), h->anchors.as<T>(), h->qc.as<int32_t>(), st);
  if (rc) return rc;
  prof_end(h, kStPredict, st);
  rc = launch_bitshuffle(h, h->qc.as<int32_t>(), g, nb, h->planes.as<uint8_t>(), st);
  if (rc) return rc;
  rc = launch_encode(h, h->planes.as<uint8_t>(), g, out, st);
  if (rc) return rc;
  prof_begin(h, kStTrailer, st);
  trailer_kernel<T><<<64, 256, 0, st>>>(out, &s->padded_size, params_ptr<T>(h), &s->range, s->csbp,
                                        h->anchors.as<T>(), g.anchors);
  prof_end(h, kStTrailer, st);
  h->launches += 1;
  CK(cudaGetLastError());
  rc = finish(h, st);
  if (rc) return rc;
  *out_size = h->host->padded_size + g.header_size;
  if (flags_out) {
    const PredParams<T>* p = reinterpret_cast<const PredParams<T>*>(h->host->params);
    for (int l = 0; l < 4; ++l) { flags_out[l] = p->use_md[l]; flags_out[4 + l] = p->reverse[l]; }
  }
  return PRISM_OK;
}

template <class T>
static int decompress_t(prism_handle* h, const uint8_t* cont, uint64_t size, const Geometry& g, int mode,
                        double bound, T* out, cudaStream_t st) {
  int rc = ensure_common(h, g);
  if (rc) return rc;
  if (size < g.header_size + 8 + 2 * (uint64_t)g.chunks) return fail(h, PRISM_ERR_CORRUPT, "container too small");
  const uint8_t* tr = cont + (size - g.header_size);
  if (reinterpret_cast<uintptr_t>(tr) % sizeof(T))  // the anchors are read in place
    return fail(h, PRISM_ERR_ARG, "container trailer not aligned to the value type");
  Small* s = small(h);
  CK(cudaMemcpyAsync(&s->range, tr + 8, sizeof(double), cudaMemcpyDeviceToDevice, st));
  params_kernel<T><<<1, 32, 0, st>>>(mode, bound, &s->range, alpha_of(mode == 1 ? bound : 0.0), nullptr, 0, tr, 4,
                                     reinterpret_cast<PredParams<T>*>(s->params), nullptr, &s->eb);
  rc = launch_decode(h, cont, size - g.header_size, g, nullptr, nullptr, h->planes.as<uint8_t>(), st);
  if (rc) return rc;
  rc = launch_inverse(h, h->planes.as<uint8_t>(), g, 0 /*SM*/, nullptr, nullptr, h->qc.as<int32_t>(), st);
  if (rc) return rc;
  prof_begin(h, kStReconstruct, st);
  rc = launch_reconstruct<T, false>(h, h->qc.as<int32_t>(), reinterpret_cast<const T*>(tr + 1040), g,
                                    params_ptr<T>(h), nullptr, out, st);
  if (rc) return rc;
  prof_end(h, kStReconstruct, st);
  h->launches += 1;
  CK(cudaGetLastError());
  return finish(h, st);
}

// ---- exported API (C linkage comes from the declarations in prism_b200.h) ----

int prism_create(prism_handle** out) {
  if (!out) return PRISM_ERR_ARG;
  prism_handle* h = new (std::nothrow) prism_handle();
  if (!h) return PRISM_ERR_NOMEM;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = host_mapped(sizeof(HostResult), (void**)&h->host, (void**)&h->host_dev);
  if (e != cudaSuccess) {
    delete h;
    return PRISM_ERR_CUDA;
  }
  *out = h;
  return PRISM_OK;
}

void prism_destroy(prism_handle* h) {
  if (!h) return;
  DevBuf* bufs[] = {&h->qc, &h->planes, &h->status, &h->offs, &h->bsum, &h->part, &h->wins, &h->ranges,
                    &h->anchors, &h->small, &h->dev_in, &h->dev_out, &h->zero_anchors, &h->prog_slots,
                    &h->sbatch, &h->qc_odd, &h->ext};
  for (DevBuf* b : bufs) b->release();
  for (DevBuf& b : h->prog_offs) b.release();
  for (int i = 0; i < kStCount; ++i)
    for (auto& e : h->ev[i]) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
  if (h->side) cudaStreamDestroy(h->side);
  if (h->fork) cudaEventDestroy(h->fork);
  if (h->join) cudaEventDestroy(h->join);
  if (h->dec) cudaStreamDestroy(h->dec);
  for (cudaEvent_t e : {h->dec_call, h->dec_done, h->recon_done[0], h->recon_done[1]})
    if (e) cudaEventDestroy(e);
  if (h->host) cudaFreeHost(h->host);
  if (h->prog_host) cudaFreeHost(h->prog_host);
  delete h;
}

const char* prism_last_error(const prism_handle* h) { return h ? h->err.c_str() : "null handle"; }

int prism_profile(prism_handle* h, int enable) {
  if (!h) return PRISM_ERR_ARG;
  h->prof = enable ? (1u << kStCount) - 1u : 0u;
  return PRISM_OK;
}

int prism_profile_stages(prism_handle* h, uint32_t mask) {
  if (!h) return PRISM_ERR_ARG;
  h->prof = mask & ((1u << kStCount) - 1u);
  return PRISM_OK;
}

int prism_stage_times(prism_handle* h, double* ms, int* counts, int n, int reset) {
  if (!h || !ms) return PRISM_ERR_ARG;
  prof_collect(h);
  for (int i = 0; i < n && i < kStCount; ++i) {
    ms[i] = h->acc_ms[i];
    if (counts) counts[i] = h->acc_n[i];
  }
  if (reset)
    for (int i = 0; i < kStCount; ++i) { h->acc_ms[i] = 0; h->acc_n[i] = 0; }
  return kStCount;
}

uint64_t prism_launch_count(const prism_handle* h) { return h ? h->launches : 0; }

uint64_t prism_max_container_size(uint32_t nx, uint32_t ny, uint32_t nz, int dtype_size) {
  Geometry g;
  make_geometry(nx, ny, nz, dtype_size, &g);
  return 8 + 2 * (uint64_t)g.chunks + g.aligned_size + 8 + g.header_size;
}

uint64_t prism_plane_buffer_size(uint32_t nx, uint32_t ny, uint32_t nz) {
  Geometry g;
  make_geometry(nx, ny, nz, 4, &g);
  return g.aligned_size;
}

uint64_t prism_trailer_size(uint32_t nx, uint32_t ny, uint32_t nz, int dtype_size) {
  Geometry g;
  make_geometry(nx, ny, nz, dtype_size, &g);
  return g.header_size;
}

uint64_t prism_code_buffer_len(uint32_t nx, uint32_t ny, uint32_t nz) {
  Geometry g;
  make_geometry(nx, ny, nz, 4, &g);
  return qc_len(g);
}

int prism_compress(prism_handle* h, const void* d_in, int dtype_size, uint32_t nx, uint32_t ny, uint32_t nz,
                   int mode, double bound, int progressive, void* d_out, uint64_t out_capacity,
                   uint64_t* out_size, uint8_t flags_out[8], void* stream) {
  if (!h || !d_in || !d_out || !out_size) return PRISM_ERR_ARG;
  if ((dtype_size != 4 && dtype_size != 8) || !dims_ok(nx, ny, nz) || !(bound > 0) || (mode != 0 && mode != 1))
    return fail(h, PRISM_ERR_ARG, "bad dtype, dimensions, mode or bound");
  Geometry g;
  make_geometry(nx, ny, nz, dtype_size, &g);
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype_size == 4)
    return compress_t<float>(h, (const float*)d_in, g, mode, bound, progressive ? 1 : 0, (uint8_t*)d_out,
                             out_capacity, out_size, flags_out, st);
  return compress_t<double>(h, (const double*)d_in, g, mode, bound, progressive ? 1 : 0, (uint8_t*)d_out,
                            out_capacity, out_size, flags_out, st);
}

int prism_compress_host(prism_handle* h, const void* h_in, int dtype_size, uint32_t nx, uint32_t ny, uint32_t nz,
                        int mode, double bound, int progressive, void* h_out, uint64_t out_capacity,
                        uint64_t* out_size, void* stream) {
  if (!h || !h_in || !h_out || !out_size) return PRISM_ERR_ARG;
  if ((dtype_size != 4 && dtype_size != 8) || !dims_ok(nx, ny, nz)) return fail(h, PRISM_ERR_ARG, "bad dims");
  uint64_t n = (uint64_t)nx * ny * nz;
  uint64_t cap = prism_max_container_size(nx, ny, nz, dtype_size);
  cudaStream_t st = (cudaStream_t)stream;
  CKA(h->dev_in.ensure(n * dtype_size));
  CKA(h->dev_out.ensure(cap));
  CK(cudaMemcpyAsync(h->dev_in.p, h_in, n * dtype_size, cudaMemcpyHostToDevice, st));
  uint64_t size = 0;
  int rc = prism_compress(h, h->dev_in.p, dtype_size, nx, ny, nz, mode, bound, progressive, h->dev_out.p, cap,
                          &size, nullptr, stream);
  if (rc) return rc;
  if (size > out_capacity) return fail(h, PRISM_ERR_ARG, "host output buffer too small");
  CK(cudaMemcpyAsync(h_out, h->dev_out.p, size, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  *out_size = size;
  return PRISM_OK;
}

int prism_decompress(prism_handle* h, const void* d_container, uint64_t size, int dtype_size, uint32_t nx,
                     uint32_t ny, uint32_t nz, int mode, double bound, void* d_out, void* stream) {
  if (!h || !d_container || !d_out) return PRISM_ERR_ARG;
  if ((dtype_size != 4 && dtype_size != 8) || !dims_ok(nx, ny, nz) || !(bound > 0) || (mode != 0 && mode != 1))
    return fail(h, PRISM_ERR_ARG, "bad dtype, dimensions, mode or bound");
  Geometry g;
  make_geometry(nx, ny, nz, dtype_size, &g);
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype_size == 4)
    return decompress_t<float>(h, (const uint8_t*)d_container, size, g, mode, bound, (float*)d_out, st);
  return decompress_t<double>(h, (const uint8_t*)d_container, size, g, mode, bound, (double*)d_out, st);
}

int prism_decompress_host(prism_handle* h, const void* h_container, uint64_t size, int dtype_size, uint32_t nx,
                          uint32_t ny, uint32_t nz, int mode, double bound, void* h_out, void* stream) {
  if (!h || !h_container || !h_out) return PRISM_ERR_ARG;
  if ((dtype_size != 4 && dtype_size != 8) || !dims_ok(nx, ny, nz)) return fail(h, PRISM_ERR_ARG, "bad dims");
  uint64_t n = (uint64_t)nx * ny * nz;
  cudaStream_t st = (cudaStream_t)stream;
  CKA(h->dev_in.ensure(size));
  CKA(h->dev_out.ensure(n * dtype_size));
  CK(cudaMemcpyAsync(h->dev_in.p, h_container, size, cudaMemcpyHostToDevice, st));
  int rc = prism_decompress(h, h->dev_in.p, size, dtype_size, nx, ny, nz, mode, bound, h->dev_out.p, stream);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h_out, h->dev_out.p, n * dtype_size, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return PRISM_OK;
}

int prism_progressive_open(prism_handle* h, const void* d_container, uint64_t size, int dtype_size, uint32_t nx,
                           uint32_t ny, uint32_t nz, int mode, double bound, prism_prog** out) {
  if (!h || !d_container || !out) return PRISM_ERR_ARG;
  if ((dtype_size != 4 && dtype_size != 8) || !dims_ok(nx, ny, nz) || !(bound > 0) || (mode != 0 && mode != 1))
    return fail(h, PRISM_ERR_ARG, "bad dtype, dimensions, mode or bound");
  prism_prog* p = new (std::nothrow) prism_prog();
  if (!p) return PRISM_ERR_NOMEM;
  p->h = h;
  p->cont = (const uint8_t*)d_container;
  p->size = size;
  p->tsize = dtype_size;
  make_geometry(nx, ny, nz, dtype_size, &p->g);
  if (size < p->g.header_size + 8 + 2 * (uint64_t)p->g.chunks) {
    delete p;
    return fail(h, PRISM_ERR_CORRUPT, "container too small");
  }
  if ((reinterpret_cast<uintptr_t>(d_container) | (size - p->g.header_size)) & 7) {
    delete p;  // the trailer's doubles and 64-bit sizes are read in place
    return fail(h, PRISM_ERR_ARG, "container or its trailer not 8-byte aligned");
  }
  p->mode = mode;
  p->bound = bound;
  p->steps = 0;
  memset(&p->state, 0, sizeof(p->state));
  p->state.maxlevel = 4;
  static_assert(sizeof(StrategyState) + sizeof(int) <= kProgSlotBytes, "progressive slot too small");
  cudaError_t e = cudaSuccess;
  if (!h->prog_slots.p) e = h->prog_slots.ensure(64 * kProgSlotBytes);
  if (e == cudaSuccess && !h->prog_host)
    e = host_mapped(64 * sizeof(ProgMirror), (void**)&h->prog_host, (void**)&h->prog_host_dev);
  int slot = -1;
  for (int i = 0; i < 64 && e == cudaSuccess; ++i)
    if (!((h->prog_used >> i) & 1)) { slot = i; break; }
  if (e == cudaSuccess && slot >= 0) {
    h->prog_used |= 1ull << slot;
    p->slot = slot;
    p->d_state = reinterpret_cast<StrategyState*>(h->prog_slots.as<unsigned char>() + slot * kProgSlotBytes);
    p->d_err = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(p->d_state) + sizeof(StrategyState));
    p->mirror = h->prog_host + slot;
    p->mirror_dev = h->prog_host_dev + slot;
  } else if (e == cudaSuccess) {  // more than 64 open at once on one handle
    e = cudaMalloc((void**)&p->d_state, kProgSlotBytes);
    p->d_err = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(p->d_state) + sizeof(StrategyState));
    if (e == cudaSuccess) e = host_mapped(sizeof(ProgMirror), (void**)&p->mirror, (void**)&p->mirror_dev);
  }
  // the device state is initialised by the first step, on its stream
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->done, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    prism_progressive_close(p);
    return fail(h, PRISM_ERR_CUDA, "progressive state", e);
  }
  *out = p;
  return PRISM_OK;
}

// strategy_finish_kernel + params_kernel of a progressive step in one launch.
// dec_begin (exact mode, may be null): per level, the first plane whose
// chunks the step decodes: begin - 1 where the level has a plane below the
// step's range and planes in it, else begin.
template <class T>
__global__ void prog_plan_kernel(const StrategyBest* __restrict__ blk, int mode, double bound, double target,
                                 const double* __restrict__ range, StrategyState* st, double alpha,
                                 const uint8_t* __restrict__ flags, PredParams<T>* params, double* eb_out,
                                 int* dec_begin) {
  strategy_finish_warp(blk, mode, bound, target, range, st);
  if (threadIdx.x != 0) return;
  compute_params<T>(mode, bound, range, alpha, nullptr, 0, flags, 4, params, nullptr, eb_out);
  params->maxlevel = st->maxlevel;
  if (dec_begin)
    for (int i = 0; i < 4; ++i) {
      const int b = st->begin[i];
      dec_begin[i] = b > 0 && b < st->end[i] ? b - 1 : b;
    }
}

__global__ void prog_init_kernel(StrategyState* st, int* err) {
  if (threadIdx.x < 4) { st->begin[threadIdx.x] = 0; st->end[threadIdx.x] = 0; }
  if (threadIdx.x == 0) { st->maxlevel = 4; *err = 0; }
}

// the state of an object whose planes [0, end) are already reconstructed
__global__ void prog_resume_kernel(StrategyState* st, int* err, int e0, int e1, int e2, int e3) {
  if (threadIdx.x != 0) return;
  const int e[4] = {e0, e1, e2, e3};
  for (int i = 0; i < 4; ++i) { st->begin[i] = e[i]; st->end[i] = e[i]; }
  st->maxlevel = 4;
  *err = 0;
}

// The state after a step, for the host: plane ranges, error flag and the
// payload bytes of every plane loaded so far.  Steps load [previous end,
// end), so the total is planes [0, end) of each level, a difference of the
// trailer's cumulative sizes (calculate_accumulate_size, analyze.hpp:118-159,
// summed over the steps).
__global__ void prog_publish_kernel(const StrategyState* __restrict__ st, const int* __restrict__ err,
                                    const uint64_t* __restrict__ cum, ProgMirror* out) {
  if (threadIdx.x != 0) return;
  uint64_t total = 0;
  for (int i = 0; i < 4; ++i) {
    const int e = min(st->end[i], 32);
    if (e > 0) total += cum[i * 32 + e - 1] - (i > 0 ? cum[i * 32 - 1] : 0);
  }
  out->state = *st;
  out->err = *err;
  out->loaded = total;
}

template <class T>
static int progressive_step_t(prism_prog* p, double target, const T* prev, T* values, cudaStream_t st) {
  prism_handle* h = p->h;
  const Geometry& g = p->g;
  // the next step of the same object on the same stream, with no other call
  // on the handle in between (and no stage but the reconstruction timed:
  // per-stage timing runs the stages one after the other)
  const bool chained = p->steps > 0 && h->chain_prog == p && h->chain_stream == st &&
                       h->chain_epoch == h->epoch && (h->prof & ~(1u << kStReconstruct)) == 0;
  if (!h->dec) {
    // default priority: the step's strategy and decode CTAs fill the slots
    // the previous reconstruction's last wave leaves idle (a high-priority
    // stream took slots from its full waves instead, measured no faster)
    CK(cudaStreamCreateWithFlags(&h->dec, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&h->dec_call, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->dec_done, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->recon_done[0], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->recon_done[1], cudaEventDisableTiming));
  }
  cudaStream_t dst = h->dec;
  const int slot = (int)(p->steps & 1);
  if (chained) {
    // the slot's codes and parameters were last read two steps back
    CK(cudaStreamWaitEvent(dst, h->recon_done[slot], 0));
  } else {
    CK(cudaEventRecord(h->dec_call, st));
    CK(cudaStreamWaitEvent(dst, h->dec_call, 0));
  }
  int rc = ensure_common(h, g);
  if (rc) return rc;
  const size_t zbytes = g.anchors * sizeof(T) + 64;
  if (h->zero_anchors.cap < zbytes) h->zero_anchors_ready = 0;
  CKA(h->zero_anchors.ensure(zbytes));
  if (h->zero_anchors_ready < zbytes) {  // the buffer is only ever read afterwards
    CK(cudaMemsetAsync(h->zero_anchors.p, 0, h->zero_anchors.cap, st));
    h->zero_anchors_ready = h->zero_anchors.cap;
  }
  Small* s = small(h);
  const uint8_t* tr = p->cont + (p->size - g.header_size);
  const double* range = reinterpret_cast<const double*>(tr + 8);
  bool first = p->steps == 0;
  StrategyState* ds = p->d_state;
  // parameters and codes alternate between two slots, so that the next
  // step's plan and inverse shuffle can run while this step's reconstruction
  // reads its own
  PredParams<T>* params = reinterpret_cast<PredParams<T>*>(slot ? s->params_odd : s->params);
  if (slot) CKA(h->qc_odd.ensure(qc_len(g) * sizeof(int32_t)));
  int32_t* codes = slot ? h->qc_odd.as<int32_t>() : h->qc.as<int32_t>();
  // ---- on the decode stream: strategy, plan, chunk offsets, decode, state
  if (first) {  // no planes loaded, all levels, no errors
    prog_init_kernel<<<1, 32, 0, dst>>>(ds, p->d_err);
    h->launches += 1;
  }
  // strategy (findStrategy_h) from the container's cumulative plane sizes;
  // it advances the object's device state in place
  const uint64_t* csbp = reinterpret_cast<const uint64_t*>(tr + 16);
  prof_begin(h, kStStrategy, dst);
  strategy_scan_kernel<<<dim3(kStrategyGroups, 33), 256, 0, dst>>>(csbp, p->mode, p->bound, target, range, s->sblk);
  // the strategy's plane ranges, then the parameters with its maxlevel
  prog_plan_kernel<T><<<1, 32, 0, dst>>>(s->sblk, p->mode, p->bound, target, range, ds,
                                         alpha_of(p->mode == 1 ? p->bound : 0.0), tr, params, &s->eb,
                                         p->exact ? s->dec_begin : nullptr);
  prof_end(h, kStStrategy, dst);
  h->launches += 2;
  // chunk offsets: once per object when it holds a slot
  const int64_t* offs = nullptr;
  if (p->slot >= 0) {
    DevBuf& ob = h->prog_offs[p->slot];
    if (!p->offs_ready) {
      CKA(ob.ensure(((size_t)g.chunks + 1) * sizeof(int64_t)));
      launch_chunk_offsets(h, p->cont, g, ob.as<int64_t>(), dst);
      p->offs_ready = true;
    }
    offs = ob.as<int64_t>();
  }
  // chunks of planes the step does not load are written as zeros; the
  // inverse shuffle keeps planes [begin, end) of what was decoded
  rc = launch_decode(h, p->cont, p->size - g.header_size, g, p->exact ? s->dec_begin : ds->begin, ds->end,
                     h->planes.as<uint8_t>(), dst, p->d_err, offs);
  if (rc) return rc;
  // the state after the step (plane ranges, errors, bytes loaded) for the host
  prog_publish_kernel<<<1, 32, 0, dst>>>(ds, p->d_err, csbp, p->mirror_dev);
  h->launches += 1;
  rc = launch_inverse(h, h->planes.as<uint8_t>(), g, 1 /*NB*/, ds->begin, ds->end, codes, dst);
  if (rc) return rc;
  CK(cudaEventRecord(h->dec_done, dst));
  // ---- on the caller's stream: reconstruction
  CK(cudaStreamWaitEvent(st, h->dec_done, 0));
  prof_begin(h, kStReconstruct, st);
  if (first) {
    rc = launch_reconstruct<T, false>(h, codes, reinterpret_cast<const T*>(tr + 1040), g, params, nullptr, values,
                                      st);
  } else {
    rc = launch_reconstruct<T, true>(h, codes, h->zero_anchors.as<T>(), g, params, prev, values, st);
  }
  if (rc) return rc;
  prof_end(h, kStReconstruct, st);
  CK(cudaEventRecord(h->recon_done[slot], st));
  CK(cudaGetLastError());
  CK(cudaEventRecord(p->done, st));
  p->pending = true;
  p->steps++;
  h->chain_prog = p;
  h->chain_stream = st;
  h->chain_epoch = h->epoch;
  return PRISM_OK;
}

// Wait for the last enqueued step, refresh the host state and report the
// device-side errors of the steps so far.
static int progressive_sync(prism_prog* p) {
  prism_handle* h = p->h;
  if (!p->pending) return PRISM_OK;
  CK(cudaEventSynchronize(p->done));
  const volatile ProgMirror* m = p->mirror;
  for (int i = 0; i < 4; ++i) {
    p->state.begin[i] = m->state.begin[i];
    p->state.end[i] = m->state.end[i];
  }
  p->state.maxlevel = m->state.maxlevel;
  const int err = m->err;
  p->loaded = m->loaded;
  p->pending = false;
  prof_collect(h);
  if (err == 2) return fail(h, PRISM_ERR_CORRUPT, "corrupt lossless chunk");
  if (err) return fail(h, PRISM_ERR_TIMEOUT, "device wait exceeded its limit");
  return PRISM_OK;
}

int prism_progressive_step(prism_prog* p, double target_error, void* d_values, void* stream) {
  if (!p || !d_values || !(target_error > 0)) return PRISM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (p->tsize == 4) return progressive_step_t<float>(p, target_error, (const float*)d_values, (float*)d_values, st);
  return progressive_step_t<double>(p, target_error, (const double*)d_values, (double*)d_values, st);
}

int prism_progressive_step_into(prism_prog* p, double target_error, const void* d_prev, void* d_out, void* stream) {
  if (!p || !d_out || !(target_error > 0) || (!d_prev && p->steps > 0)) return PRISM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (p->tsize == 4) return progressive_step_t<float>(p, target_error, (const float*)d_prev, (float*)d_out, st);
  return progressive_step_t<double>(p, target_error, (const double*)d_prev, (double*)d_out, st);
}

int prism_progressive_resume(prism_prog* p, const int end[4], void* stream) {
  if (!p || !end) return PRISM_ERR_ARG;
  if (p->steps != 0) return fail(p->h, PRISM_ERR_ARG, "resume applies to an object before its first step");
  for (int i = 0; i < 4; ++i)
    if (end[i] < 0 || end[i] > 32) return fail(p->h, PRISM_ERR_ARG, "plane ranges are 0..32");
  cudaStream_t st = (cudaStream_t)stream;
  prism_handle* h = p->h;
  prog_resume_kernel<<<1, 32, 0, st>>>(p->d_state, p->d_err, end[0], end[1], end[2], end[3]);
  h->launches += 1;
  CK(cudaGetLastError());
  for (int i = 0; i < 4; ++i) p->state.begin[i] = p->state.end[i] = end[i];
  p->state.maxlevel = 4;
  p->steps = 1;  // the next step adds to previous values, from zero anchors
  return PRISM_OK;
}

int prism_progressive_exact(prism_prog* p, int enable) {
  if (!p) return PRISM_ERR_ARG;
  p->exact = enable != 0;
  return PRISM_OK;
}

int prism_progressive_state(const prism_prog* cp, int begin[4], int end[4], int* maxlevel, uint64_t* loaded) {
  if (!cp) return PRISM_ERR_ARG;
  prism_prog* p = const_cast<prism_prog*>(cp);  // refreshes the cached host state
  const int rc = progressive_sync(p);
  for (int i = 0; i < 4; ++i) {
    if (begin) begin[i] = p->state.begin[i];
    if (end) end[i] = p->state.end[i];
  }
  if (maxlevel) *maxlevel = p->state.maxlevel;
  if (loaded) *loaded = p->loaded;
  return rc;
}

void prism_progressive_close(prism_prog* p) {
  if (!p) return;
  if (p->pending) cudaEventSynchronize(p->done);
  if (p->slot >= 0) {
    p->h->prog_used &= ~(1ull << p->slot);
  } else {
    if (p->d_state) cudaFree(p->d_state);
    if (p->mirror) cudaFreeHost(p->mirror);
  }
  if (p->done) cudaEventDestroy(p->done);
  delete p;
}

// ---- stage entry points ----

int prism_extrema(prism_handle* h, const void* d_in, int dtype_size, uint64_t n, double* range_out, void* stream) {
  if (!h || !d_in || !range_out || n == 0) return PRISM_ERR_ARG;
  CKA(h->small.ensure(sizeof(Small)));
  cudaStream_t st = (cudaStream_t)stream;
  int rc = dtype_size == 4 ? launch_extrema<float>(h, (const float*)d_in, n, st)
                           : launch_extrema<double>(h, (const double*)d_in, n, st);
  if (rc) return rc;
  CK(cudaMemcpyAsync(range_out, &small(h)->range, sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return PRISM_OK;
}

int prism_extrema_minmax(prism_handle* h, const void* d_in, int dtype_size, uint64_t n, double minmax_out[2],
                         void* stream) {
  if (!h || !d_in || !minmax_out || n == 0 || (dtype_size != 4 && dtype_size != 8)) return PRISM_ERR_ARG;
  CKA(h->small.ensure(sizeof(Small)));
  cudaStream_t st = (cudaStream_t)stream;
  int rc = dtype_size == 4 ? launch_extrema<float>(h, (const float*)d_in, n, st)
                           : launch_extrema<double>(h, (const double*)d_in, n, st);
  if (rc) return rc;
  CK(cudaMemcpyAsync(minmax_out, small(h)->minmax, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return PRISM_OK;
}

int prism_autotune(prism_handle* h, const void* d_in, int dtype_size, uint32_t nx, uint32_t ny, uint32_t nz,
                   double* errors_out, uint8_t flags_out[8], void* stream) {
  if (!h || !d_in || !dims_ok(nx, ny, nz)) return PRISM_ERR_ARG;
  Geometry g;
  make_geometry(nx, ny, nz, dtype_size, &g);
  int rc = ensure_common(h, g);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  set_double_kernel<<<1, 1, 0, st>>>(&small(h)->range, 1.0);
  rc = dtype_size == 4 ? launch_autotune_params<float>(h, (const float*)d_in, g, 0, 1.0, 0.0, nullptr, st)
                       : launch_autotune_params<double>(h, (const double*)d_in, g, 0, 1.0, 0.0, nullptr, st);
  if (rc) return rc;
  rc = finish(h, st);
  if (rc) return rc;
  for (int k = 0; k < 15; ++k) {
    if (!errors_out) break;
    errors_out[k] = dtype_size == 4 ? (double)reinterpret_cast<const float*>(h->host->errors)[k]
                                    : h->host->errors[k];
  }
  if (flags_out) {
    const uint8_t* md = dtype_size == 4 ? reinterpret_cast<const PredParams<float>*>(h->host->params)->use_md
                                        : reinterpret_cast<const PredParams<double>*>(h->host->params)->use_md;
    const uint8_t* rv = dtype_size == 4 ? reinterpret_cast<const PredParams<float>*>(h->host->params)->reverse
                                        : reinterpret_cast<const PredParams<double>*>(h->host->params)->reverse;
    for (int l = 0; l < 4; ++l) { flags_out[l] = md[l]; flags_out[4 + l] = rv[l]; }
  }
  return PRISM_OK;
}

template <class T>
static int predict_stage_t(prism_handle* h, const T* in, const Geometry& g, double eb, double rel_eb,
                           const uint8_t* flags, int32_t* codes, T* anchors, cudaStream_t st) {
  int rc = ensure_common(h, g);
  if (rc) return rc;
  Small* s = small(h);
  CK(cudaMemcpyAsync(s->params + 200, flags, 8, cudaMemcpyHostToDevice, st));
  set_double_kernel<<<1, 1, 0, st>>>(&s->range, 1.0);
  params_kernel<T><<<1, 32, 0, st>>>(0, eb, &s->range, alpha_of(rel_eb), nullptr, 0, s->params + 200, 4,
                                     reinterpret_cast<PredParams<T>*>(s->params), nullptr, &s->eb);
  rc = launch_predict<T>(h, in, g, params_ptr<T>(h), anchors, codes, st);
  if (rc) return rc;
  return finish(h, st);
}

int prism_predict(prism_handle* h, const void* d_in, int dtype_size, uint32_t nx, uint32_t ny, uint32_t nz,
                  double eb, double rel_eb, const uint8_t flags[8], int32_t* d_codes, void* d_anchors, void* stream) {
  if (!h || !d_in || !d_codes || !d_anchors || !flags || !dims_ok(nx, ny, nz) || !(eb > 0)) return PRISM_ERR_ARG;
  Geometry g;
  make_geometry(nx, ny, nz, dtype_size, &g);
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype_size == 4)
    return predict_stage_t<float>(h, (const float*)d_in, g, eb, rel_eb, flags, d_codes, (float*)d_anchors, st);
  return predict_stage_t<double>(h, (const double*)d_in, g, eb, rel_eb, flags, d_codes, (double*)d_anchors, st);
}

template <class T>
static int reconstruct_stage_t(prism_handle* h, const int32_t* codes, const T* anchors, const Geometry& g, double eb,
                               double rel_eb, const uint8_t* flags, int maxlevel, const T* old, T* out,
                               cudaStream_t st) {
  int rc = ensure_common(h, g);
  if (rc) return rc;
  Small* s = small(h);
  CK(cudaMemcpyAsync(s->params + 200, flags, 8, cudaMemcpyHostToDevice, st));
  set_double_kernel<<<1, 1, 0, st>>>(&s->range, 1.0);
  params_kernel<T><<<1, 32, 0, st>>>(0, eb, &s->range, alpha_of(rel_eb), nullptr, 0, s->params + 200, maxlevel,
                                     reinterpret_cast<PredParams<T>*>(s->params), nullptr, &s->eb);
  rc = old ? launch_reconstruct<T, true>(h, codes, anchors, g, params_ptr<T>(h), old, out, st)
           : launch_reconstruct<T, false>(h, codes, anchors, g, params_ptr<T>(h), nullptr, out, st);
  if (rc) return rc;
  return finish(h, st);
}

int prism_reconstruct(prism_handle* h, const int32_t* d_codes, const void* d_anchors, int dtype_size, uint32_t nx,
                      uint32_t ny, uint32_t nz, double eb, double rel_eb, const uint8_t flags[8], int maxlevel,
                      const void* d_old, void* d_out, void* stream) {
  if (!h || !d_codes || !d_anchors || !d_out || !flags || !dims_ok(nx, ny, nz) || !(eb > 0)) return PRISM_ERR_ARG;
  Geometry g;
  make_geometry(nx, ny, nz, dtype_size, &g);
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype_size == 4)
    return reconstruct_stage_t<float>(h, d_codes, (const float*)d_anchors, g, eb, rel_eb, flags, maxlevel,
                                      (const float*)d_old, (float*)d_out, st);
  return reconstruct_stage_t<double>(h, d_codes, (const double*)d_anchors, g, eb, rel_eb, flags, maxlevel,
                                     (const double*)d_old, (double*)d_out, st);
}

int prism_bitshuffle(prism_handle* h, const int32_t* d_codes, uint32_t nx, uint32_t ny, uint32_t nz, int progressive,
                     uint8_t* d_planes, void* stream) {
  if (!h || !d_codes || !d_planes || !dims_ok(nx, ny, nz)) return PRISM_ERR_ARG;
  Geometry g;
  make_geometry(nx, ny, nz, 4, &g);
  int rc = ensure_common(h, g);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  rc = launch_bitshuffle(h, d_codes, g, progressive ? 1 : 0, d_planes, st);
  if (rc) return rc;
  CK(cudaStreamSynchronize(st));
  return PRISM_OK;
}

static int host_range(prism_handle* h, const int* hb, const int* he, cudaStream_t st, int** db, int** de) {
  *db = *de = nullptr;
  if (!hb) return PRISM_OK;
  Small* s = small(h);
  StrategyState tmp;
  memset(&tmp, 0, sizeof(tmp));
  for (int i = 0; i < 4; ++i) { tmp.begin[i] = hb[i]; tmp.end[i] = he[i]; }
  CK(cudaMemcpyAsync(&s->sstate, &tmp, sizeof(tmp), cudaMemcpyHostToDevice, st));
  *db = s->sstate.begin;
  *de = s->sstate.end;
  return PRISM_OK;
}

int prism_inverse_bitshuffle(prism_handle* h, const uint8_t* d_planes, uint32_t nx, uint32_t ny, uint32_t nz,
                             int progressive, const int begin[4], const int end[4], int32_t* d_codes, void* stream) {
  if (!h || !d_codes || !d_planes || !dims_ok(nx, ny, nz) || (!begin) != (!end)) return PRISM_ERR_ARG;
  Geometry g;
  make_geometry(nx, ny, nz, 4, &g);
  int rc = ensure_common(h, g);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  int *db, *de;
  rc = host_range(h, begin, end, st, &db, &de);
  if (rc) return rc;
  rc = launch_inverse(h, d_planes, g, progressive ? 1 : 0, db, de, d_codes, st);
  if (rc) return rc;
  CK(cudaStreamSynchronize(st));
  return PRISM_OK;
}

int prism_lossless_encode(prism_handle* h, const uint8_t* d_planes, uint32_t nx, uint32_t ny, uint32_t nz,
                          uint8_t* d_stream, uint64_t capacity, uint64_t* size_out, uint64_t comp_size_bp[128],
                          void* stream) {
  if (!h || !d_planes || !d_stream || !size_out || !dims_ok(nx, ny, nz)) return PRISM_ERR_ARG;
  Geometry g;
  make_geometry(nx, ny, nz, 4, &g);
  if (capacity < 8 + 2 * (uint64_t)g.chunks + g.aligned_size + 8) return fail(h, PRISM_ERR_ARG, "capacity");
  int rc = ensure_common(h, g);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  rc = launch_encode(h, d_planes, g, d_stream, st);
  if (rc) return rc;
  if (comp_size_bp) CK(cudaMemcpyAsync(comp_size_bp, small(h)->csbp, 1024, cudaMemcpyDeviceToHost, st));
  rc = finish(h, st);
  if (rc) return rc;
  *size_out = h->host->padded_size;
  return PRISM_OK;
}

int prism_lossless_wait_selftest(prism_handle* h, const uint8_t* d_planes, uint32_t nx, uint32_t ny, uint32_t nz,
                                 uint8_t* d_stream, uint64_t capacity, long long spin_limit, void* stream) {
  if (!h || !d_planes || !d_stream || !dims_ok(nx, ny, nz) || spin_limit < 1) return PRISM_ERR_ARG;
  Geometry g;
  make_geometry(nx, ny, nz, 4, &g);
  if (g.chunks < 2) return fail(h, PRISM_ERR_ARG, "the self-test needs at least two chunks");
  if (capacity < 8 + 2 * (uint64_t)g.chunks + g.aligned_size + 8) return fail(h, PRISM_ERR_ARG, "capacity");
  int rc = ensure_common(h, g);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  rc = launch_encode(h, d_planes, g, d_stream, st, 1, spin_limit);
  if (rc) return rc;
  return finish(h, st);
}

// Level-0 codes whose bits the reference's last shuffle block does not carry
// (bitplane.cu:180-181, 200-260, 379-380).  The block starts at device code
// position `start`; thread t handles positions start + base + t while
// base + t < res(t), res = tail for t > 0 and tail + align for thread 0
// (tail = n mod 16384, or 16384), and thread t writes the transposed word of
// position start + base + wp, wp = ((t & 63) << 3) + (t >> 6), when wp < res(t).
//  * Real codes from the 8-code group holding position start + tail on are
//    not transposed in full (lanes at or past tail write nothing, thread 0
//    alone goes further and writes only the four planes of its own word) and
//    the inverse does not decode the ones past tail.
//  * Positions past the end of the code space read zeros; where such a
//    position lies past its level-0 plane (byte idx / 8 >= the plane stride)
//    its zero bytes land on byte idx / 8 - stride of the next planes, i.e. on
//    the bits of level-0 codes 8b..8b+7 — when the last block's writes land
//    after the first block's (as the reference's launch orders them).
// The union of both sets, counted per level-0 code.
static int64_t lost_codes(const Geometry& g) {
  const int64_t start = (g.sh_grid - 1) * (int64_t)kChunk;
  int64_t tail = (int64_t)(g.n % kChunk);
  if (tail == 0) tail = kChunk;
  const int64_t count0 = (int64_t)(g.n - g.grid[0]), base0 = g.dprefix[0], st = g.dstride[0];
  const int64_t code_end = base0 + count0;
  std::vector<uint8_t> lost((size_t)count0, 0);
  // never transposed in full: from the 8-code group that holds position
  // start + tail on (the lanes of that group at or past tail write nothing,
  // and their words carry planes of the whole group; thread 0's extra
  // positions keep only the four planes of its own word)
  for (int64_t p = std::max(start + (tail & ~(int64_t)7), base0); p < code_end; ++p) lost[(size_t)(p - base0)] = 1;
  // zero words past the plane
  if (last_block_lands_last(g)) {
    const int64_t ares = (tail + 511) / 512 * 512, ares0 = (tail + g.align_dev + 511) / 512 * 512;
    auto mark = [&](int64_t p) {
      if (p < code_end) return;
      const int64_t idx = p - base0, b = (idx >> 3) - st;
      if (idx < 0 || b < 0) return;
      for (int64_t c = 8 * b; c < 8 * b + 8 && c < count0; ++c) lost[(size_t)c] = 1;
    };
    for (int64_t base = 0; base < std::max(ares, ares0); base += 512) {
      if (base < ares)
        for (int64_t w = 1; w < 512 && w < tail; ++w) mark(start + base + w);
      mark(start + base);
    }
  }
  int64_t cnt = 0;
  for (uint8_t v : lost) cnt += v;
  return cnt;
}

uint64_t prism_lost_codes(uint32_t nx, uint32_t ny, uint32_t nz) {
  if (!dims_ok(nx, ny, nz)) return 0;
  Geometry g;
  make_geometry(nx, ny, nz, 4, &g);
  return (uint64_t)lost_codes(g);
}

int prism_lossless_decode(prism_handle* h, const uint8_t* d_stream, uint32_t nx, uint32_t ny, uint32_t nz,
                          const int begin[4], const int end[4], uint8_t* d_planes, void* stream) {
  if (!h || !d_planes || !d_stream || !dims_ok(nx, ny, nz) || (!begin) != (!end)) return PRISM_ERR_ARG;
  Geometry g;
  make_geometry(nx, ny, nz, 4, &g);
  int rc = ensure_common(h, g);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  int *db, *de;
  rc = host_range(h, begin, end, st, &db, &de);
  if (rc) return rc;
  rc = launch_decode(h, d_stream, ~0ull, g, db, de, d_planes, st);
  if (rc) return rc;
  return finish(h, st);
}

int prism_find_strategy(prism_handle* h, const uint64_t comp_size_bp[128], double eb, double target_error,
                        int begin[4], int end[4], int* maxlevel, void* stream) {
  if (!h || !comp_size_bp || !begin || !end || !maxlevel || !(eb > 0)) return PRISM_ERR_ARG;
  CKA(h->small.ensure(sizeof(Small)));
  CKA(h->part.ensure(1024 + 64));
  cudaStream_t st = (cudaStream_t)stream;
  Small* s = small(h);
  StrategyState tmp;
  for (int i = 0; i < 4; ++i) { tmp.begin[i] = begin[i]; tmp.end[i] = end[i]; }
  tmp.maxlevel = *maxlevel;
  CK(cudaMemcpyAsync(&s->sstate, &tmp, sizeof(tmp), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(h->part.p, comp_size_bp, 1024, cudaMemcpyHostToDevice, st));
  set_double_kernel<<<1, 1, 0, st>>>(&s->range, 1.0);
  strategy_scan_kernel<<<dim3(kStrategyGroups, 33), 256, 0, st>>>(h->part.as<uint64_t>(), 0, eb, target_error,
                                                                  &s->range, s->sblk);
  strategy_finish_kernel<<<1, 32, 0, st>>>(s->sblk, 0, eb, target_error, &s->range, &s->sstate);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(&tmp, &s->sstate, sizeof(tmp), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int i = 0; i < 4; ++i) { begin[i] = tmp.begin[i]; end[i] = tmp.end[i]; }
  *maxlevel = tmp.maxlevel;
  return PRISM_OK;
}


int prism_find_strategy_batch(prism_handle* h, int n, const uint64_t* comp_size_bp, const double* eb,
                              const double* target_error, int* begin, int* end, int* maxlevel, void* stream) {
  if (!h || n < 1 || n > 65535 || !comp_size_bp || !eb || !target_error || !begin || !end || !maxlevel)
    return PRISM_ERR_ARG;
  for (int i = 0; i < n; ++i)
    if (!(eb[i] > 0)) return PRISM_ERR_ARG;
  ++h->epoch;
  cudaStream_t st = (cudaStream_t)stream;
  // device layout: cells | plane sizes | bound, target pairs | states | 1.0
  const size_t cells = (size_t)n * kStrategyCells * sizeof(StrategyBest);
  const size_t in_bytes = (size_t)n * 128 * sizeof(uint64_t) + (size_t)n * 2 * sizeof(double) +
                          (size_t)n * sizeof(StrategyState) + sizeof(double);
  CKA(h->sbatch.ensure(cells + in_bytes + 64));
  std::vector<uint8_t> host(in_bytes);
  uint8_t* q = host.data();
  memcpy(q, comp_size_bp, (size_t)n * 128 * sizeof(uint64_t));
  double* bt = reinterpret_cast<double*>(q + (size_t)n * 128 * sizeof(uint64_t));
  for (int i = 0; i < n; ++i) {
    bt[2 * i] = eb[i];
    bt[2 * i + 1] = target_error[i];
  }
  StrategyState* ss = reinterpret_cast<StrategyState*>(bt + 2 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    for (int l = 0; l < 4; ++l) {
      ss[i].begin[l] = begin[4 * i + l];
      ss[i].end[l] = end[4 * i + l];
    }
    ss[i].maxlevel = maxlevel[i];
  }
  double* one = reinterpret_cast<double*>(ss + n);
  *one = 1.0;
  uint8_t* d = h->sbatch.as<uint8_t>();
  StrategyBest* d_cells = reinterpret_cast<StrategyBest*>(d);
  uint8_t* d_in = d + cells;
  const uint64_t* d_cs = reinterpret_cast<const uint64_t*>(d_in);
  const double* d_bt = reinterpret_cast<const double*>(d_in + (size_t)n * 128 * sizeof(uint64_t));
  StrategyState* d_ss = reinterpret_cast<StrategyState*>(const_cast<double*>(d_bt) + 2 * (size_t)n);
  const double* d_one = reinterpret_cast<const double*>(d_ss + n);
  CK(cudaMemcpyAsync(d_in, host.data(), in_bytes, cudaMemcpyHostToDevice, st));
  strategy_scan_batch_kernel<<<dim3(kStrategyGroups, 33, n), 256, 0, st>>>(d_cs, d_bt, d_one, d_cells);
  strategy_finish_batch_kernel<<<n, 32, 0, st>>>(d_cells, d_bt, d_one, d_ss);
  h->launches += 2;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(ss, d_ss, (size_t)n * sizeof(StrategyState), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int i = 0; i < n; ++i) {
    for (int l = 0; l < 4; ++l) {
      begin[4 * i + l] = ss[i].begin[l];
      end[4 * i + l] = ss[i].end[l];
    }
    maxlevel[i] = ss[i].maxlevel;
  }
  return PRISM_OK;
}

// ---------------------------------------------------------------------------
// Lossless encode without any allocation (prism_lossless_encode_static).
//
// Same kernels as prism_lossless_encode, but the look-back status words, the
// chunk ticket, the error flag and the small results live in one file-scope
// device array instead of a handle's workspace, so the call allocates nothing.
// The array is shared by every call in the process on a given device: calls
// whose device work overlaps (different streams, different host threads) race
// on it and must be ordered by the caller.
namespace {

constexpr int64_t kStaticMaxChunks = 16384;  // plane buffer <= 256 MiB

struct StaticEncodeScratch {
  unsigned long long status[kStaticMaxChunks];  // zeroed by every call
  unsigned long long ticket;                    // zeroed by every call
  int error_flag;                               // zeroed by every call
  int pad;
  uint64_t csbp[128];                           // zeroed by every call
  uint64_t lossless_size;
  uint64_t padded_size;
};

}  // namespace

static __device__ __align__(256) unsigned char g_static_encode_scratch[sizeof(StaticEncodeScratch)];

namespace {

constexpr int kStaticMaxDevices = 64;

struct StaticEncodeSetup {
  bool ready = false;
  StaticEncodeScratch* scratch = nullptr;
  int sm_count = 0;
};

std::mutex g_static_setup_mutex;
StaticEncodeSetup g_static_setup[kStaticMaxDevices];

// Once per device, with that device current: look up the scratch address,
// raise the encode kernel's dynamic shared-memory limit and read the SM count.
int static_encode_setup(int dev, StaticEncodeSetup* out) {
  std::lock_guard<std::mutex> lock(g_static_setup_mutex);
  StaticEncodeSetup& s = g_static_setup[dev];
  if (!s.ready) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_static_encode_scratch) != cudaSuccess) return PRISM_ERR_CUDA;
    if (cudaFuncSetAttribute(zbpc_encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(EncodeShared)) != cudaSuccess)
      return PRISM_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return PRISM_ERR_CUDA;
    s.scratch = static_cast<StaticEncodeScratch*>(p);
    s.sm_count = sms;
    s.ready = true;
  }
  *out = s;
  return PRISM_OK;
}

}  // namespace

int prism_lossless_encode_static(const uint8_t* d_planes, uint32_t nx, uint32_t ny, uint32_t nz,
                                 uint8_t* d_stream, uint64_t capacity, uint64_t* size_out,
                                 uint64_t comp_size_bp[128], void* stream) {
  if (!d_planes || !d_stream || !size_out || !dims_ok(nx, ny, nz)) return PRISM_ERR_ARG;
  Geometry g;
  make_geometry(nx, ny, nz, 4, &g);
  if (g.chunks > kStaticMaxChunks) return PRISM_ERR_LIMIT;
  if (capacity < 8 + 2 * (uint64_t)g.chunks + g.aligned_size + 8) return PRISM_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PRISM_ERR_CUDA;
  if (dev < 0 || dev >= kStaticMaxDevices) return PRISM_ERR_ARG;
  StaticEncodeSetup setup;
  int rc = static_encode_setup(dev, &setup);
  if (rc) return rc;
  StaticEncodeScratch* s = setup.scratch;
  cudaStream_t st = (cudaStream_t)stream;
  // everything the encode kernel expects at zero, reset on the caller's stream
  if (cudaMemsetAsync(s->status, 0, (size_t)g.chunks * sizeof(unsigned long long), st) != cudaSuccess ||
      cudaMemsetAsync(&s->ticket, 0,
                      offsetof(StaticEncodeScratch, lossless_size) - offsetof(StaticEncodeScratch, ticket),
                      st) != cudaSuccess)
    return PRISM_ERR_CUDA;
  int blocks = (int)std::min<int64_t>(g.chunks, (int64_t)setup.sm_count * 4);
  zbpc_encode_kernel<<<blocks, kZThreads, sizeof(EncodeShared), st>>>(
      d_planes, g, d_stream, s->status, &s->ticket, s->csbp, &s->lossless_size, &s->error_flag, (long long)1 << 22);
  zbpc_finish_kernel<<<1, 32, 0, st>>>(d_stream, g, &s->lossless_size, &s->padded_size);
  if (cudaGetLastError() != cudaSuccess) return PRISM_ERR_CUDA;
  uint64_t padded = 0;
  int flag = 0;
  if (cudaMemcpyAsync(&padded, &s->padded_size, sizeof(padded), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(&flag, &s->error_flag, sizeof(flag), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return PRISM_ERR_CUDA;
  if (comp_size_bp && cudaMemcpyAsync(comp_size_bp, s->csbp, 1024, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return PRISM_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return PRISM_ERR_CUDA;
  if (flag == 1) return PRISM_ERR_TIMEOUT;
  *size_out = padded;
  return PRISM_OK;
}

#include "batch_api.cuh"
#include "server_api.cuh"
#include "file_api.cuh"

// ---- reconstruction error statistics (--report cr) ----
int prism_statistics(prism_handle* h, const void* d_original, const void* d_data, int dtype_size, uint64_t n,
                     double out[7], uint64_t* max_err_index, void* stream) {
  if (!h || !d_original || !d_data || !out || n == 0 || (dtype_size != 4 && dtype_size != 8)) return PRISM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int blocks = (int)std::min<uint64_t>((n + kStatThreads - 1) / kStatThreads, (uint64_t)h->sm_count * 8);
  CKA(h->part.ensure(sizeof(StatPart) * blocks + 64));
  StatPart* part = h->part.as<StatPart>();
  if (dtype_size == 4)
    stats_kernel<float><<<blocks, kStatThreads, 0, st>>>((const float*)d_original, (const float*)d_data, n, part);
  else
    stats_kernel<double><<<blocks, kStatThreads, 0, st>>>((const double*)d_original, (const double*)d_data, n, part);
  stats_final_kernel<<<1, 32, 0, st>>>(part, blocks);
  h->launches += 2;
  CK(cudaGetLastError());
  StatPart r;
  CK(cudaMemcpyAsync(&r, part, sizeof(r), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const double range = r.mx - r.mn, mse = r.l2 / (double)n;
  out[0] = r.maxe;
  out[1] = r.maxe / range;
  out[2] = 20 * log10(range) - 10 * log10(mse);
  out[3] = sqrt(mse) / range;
  out[4] = r.mn;
  out[5] = r.mx;
  out[6] = r.l2;
  if (max_err_index) *max_err_index = r.idx;
  return PRISM_OK;
}
