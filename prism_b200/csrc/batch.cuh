// Batched compression: many fields of uneven shapes in one launch per stage.
//
// Every stage of the per-field pipeline (extrema, auto-tune, parameters, code
// padding, predictor, leftover bytes, last shuffle block, bulk shuffle,
// lossless encode, stream header, trailer) runs as one launch over all fields
// of the batch.  Work items of a stage are numbered across the fields (a
// field's items follow the previous field's), and a kernel maps an item to
// its field by a binary search over the per-field item prefix.  The predictor
// and the lossless encoder are persistent kernels whose CTAs pull items from
// a device counter, so large and small fields share the GPU without a wave
// tail per field.  Every field's bytes are exactly those of the per-field
// pipeline: the same tile, shuffle and chunk code runs on each item; the
// look-back of the encoder ends at the field's first chunk because each field
// has its own status slice.
#pragma once
#include "autotune.cuh"
#include "bitplane.cuh"
#include "predict.cuh"
#include "zbpc.cuh"

namespace prism_b200 {

// Per-field device state written by the batched stages.
struct BatchState {
  double range;
  double eb;
  uint64_t lossless_size;
  uint64_t padded_size;
  int error_flag;
  int pad;
  uint64_t csbp[128];
  unsigned char params[256];  // PredParams<T>
};

// Per-field descriptor, resident in device memory.
struct BatchField {
  Geometry g;
  ShufPlan plan;
  const void* in;
  uint8_t* out;
  int32_t* qc;
  uint8_t* planes;
  void* anchors;
  unsigned long long* status;
  BatchState* st;
  int mode, nb, tsize, pad;
  double bound, alpha;
};

// Window of the auto-tuner with its field.
struct BatchWindow {
  SampleWindow w;
  int field;
  int pad;
};

// Byte range of the plane buffer the bulk shuffle leaves alone, with its field.
struct BatchRange {
  uint64_t start, len;
  int field;
  int pad;
};

// One CTA of a last-block launch: field, CTA index and CTA count of the field.
struct BatchLastCta {
  int field, cta, ncta, pad;
};

// Zero-fill segment of a code buffer.
struct BatchZero {
  int32_t* ptr;
  uint64_t len;
};

// Largest i with prefix[i] <= item (prefix has n + 1 entries, prefix[0] = 0).
__device__ __forceinline__ int find_field(const uint64_t* __restrict__ prefix, int n, uint64_t item) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

constexpr uint64_t kBatchExtSeg = 1u << 18;  // values per extrema item

// REL extrema: item = (field, segment of kBatchExtSeg values); part[item] =
// {min, max} of the segment.  `gidx` maps group entries to fields.
template <class T>
__global__ void __launch_bounds__(kExtThreads)
batch_extrema_kernel(const BatchField* __restrict__ fields, const int* __restrict__ gidx,
                     const uint64_t* __restrict__ prefix, int n, uint64_t items, T* __restrict__ part) {
  __shared__ T smin[kExtThreads], smax[kExtThreads];
  for (uint64_t item = blockIdx.x; item < items; item += gridDim.x) {
    const int e = find_field(prefix, n, item);
    const BatchField& f = fields[gidx[e]];
    const T* in = reinterpret_cast<const T*>(f.in);
    const uint64_t s0 = (item - prefix[e]) * kBatchExtSeg;
    const uint64_t s1 = min(s0 + kBatchExtSeg, f.g.n);
    T mn = in[s0], mx = in[s0];
    uint64_t i = s0 + threadIdx.x;
    for (; i + 3 * blockDim.x < s1; i += 4 * blockDim.x) {  // four loads in flight
      T v[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] = __ldg(in + i + k * blockDim.x);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        mn = v[k] < mn ? v[k] : mn;
        mx = v[k] > mx ? v[k] : mx;
      }
    }
    for (; i < s1; i += blockDim.x) {
      T v = __ldg(in + i);
      mn = v < mn ? v : mn;
      mx = v > mx ? v : mx;
    }
    smin[threadIdx.x] = mn;
    smax[threadIdx.x] = mx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) {
        T a = smin[threadIdx.x + s], b = smax[threadIdx.x + s];
        if (a < smin[threadIdx.x]) smin[threadIdx.x] = a;
        if (b > smax[threadIdx.x]) smax[threadIdx.x] = b;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) { part[2 * item] = smin[0]; part[2 * item + 1] = smax[0]; }
    __syncthreads();
  }
}

// One warp per group field: range = max - min (REL) or 1 (ABS).
template <class T>
__global__ void batch_extrema_final_kernel(const BatchField* __restrict__ fields, const int* __restrict__ gidx,
                                           const uint64_t* __restrict__ prefix, int n, const T* __restrict__ part) {
  const int e = blockIdx.x;
  if (e >= n) return;
  const BatchField& f = fields[gidx[e]];
  const int lane = threadIdx.x;
  if (f.mode != 1) {
    if (lane == 0) f.st->range = 1.0;
    return;
  }
  const uint64_t b = prefix[e], c = prefix[e + 1];
  T mn = part[2 * b], mx = part[2 * b + 1];
  for (uint64_t i = b + lane; i < c; i += 32) {
    T a = part[2 * i], d = part[2 * i + 1];
    mn = a < mn ? a : mn;
    mx = d > mx ? d : mx;
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    T a = __shfl_xor_sync(0xffffffffu, mn, d), q = __shfl_xor_sync(0xffffffffu, mx, d);
    mn = a < mn ? a : mn;
    mx = q > mx ? q : mx;
  }
  if (lane == 0) f.st->range = __dsub_rn((double)mx, (double)mn);
}

// grid (windows of the group, 6): partial[window][15] as autotune_kernel
template <class T>
__global__ void __launch_bounds__(kAttThreads)
batch_autotune_kernel(const BatchField* __restrict__ fields, const BatchWindow* __restrict__ wins,
                      T* __restrict__ partial) {
  __shared__ T win[kWinVol];
  __shared__ T red[kAttThreads];
  const BatchWindow bw = wins[blockIdx.x];
  const BatchField& f = fields[bw.field];
  autotune_window<T>(win, red, reinterpret_cast<const T*>(f.in), f.g, bw.w, blockIdx.y,
                     partial + (size_t)blockIdx.x * 15);
}

// one thread per group field: per-level bounds and auto-tune decisions
template <class T>
__global__ void batch_params_kernel(const BatchField* __restrict__ fields, const int* __restrict__ gidx,
                                    const uint64_t* __restrict__ win_prefix, int n, const T* __restrict__ partial) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const BatchField& f = fields[gidx[e]];
  const uint64_t w0 = win_prefix[e];
  compute_params<T>(f.mode, f.bound, &f.st->range, f.alpha, partial + w0 * 15, (int)(win_prefix[e + 1] - w0), nullptr,
                    4, reinterpret_cast<PredParams<T>*>(f.st->params), nullptr, &f.st->eb);
}

__global__ void batch_zero_kernel(const BatchZero* __restrict__ segs, int nseg) {
  for (int s = blockIdx.x; s < nseg; s += gridDim.x) {
    int32_t* p = segs[s].ptr;
    const uint64_t len = segs[s].len;
    for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) p[i] = 0;
  }
}

// One tile of a batch field: geometry copied to shared memory (the
// per-field kernel has it in its parameters) and read from there at each use.
template <class T, int PART>
__device__ __forceinline__ void batch_tile(CompressSmem<T>& sm, Geometry& sg, const BatchField* f, uint32_t local) {
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&f->g);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&sg);
    for (int i = threadIdx.x; i < (int)(sizeof(Geometry) / 4); i += kPredThreads) dst[i] = src[i];
  }
  __syncthreads();
  const volatile Geometry& gv = sg;
  uint32_t bi[3];
  tile_of_index<PART, volatile Geometry>(gv, local, bi);
  compress_tile<T, PART == 1, volatile Geometry>(sm, reinterpret_cast<const T*>(f->in), gv, bi,
                                                 reinterpret_cast<const PredParams<T>*>(f->st->params),
                                                 reinterpret_cast<T*>(f->anchors), f->qc);
}

// the same, out of line: keeps the persistent loop's registers separate
template <class T, int PART>
__device__ __noinline__ void batch_tile_call(CompressSmem<T>& sm, Geometry& sg, const BatchField* f, uint32_t local) {
  batch_tile<T, PART>(sm, sg, f, local);
}

// Predictor over the tiles of part PART (0 interior, 1 edge) of every group
// field, one CTA per tile.  Float edge tiles keep four CTAs per SM here (56
// registers, no spills): with the field lookup, six would spill 172 bytes a
// thread, a variant not measured in this kernel.
template <class T, int PART>
constexpr int batch_predict_min_ctas() { return sizeof(T) == 4 && PART == 0 ? 6 : 4; }

template <class T, int PART>
__global__ void __launch_bounds__(kPredThreads, batch_predict_min_ctas<T, PART>())
batch_predict_kernel(const BatchField* __restrict__ fields, const int* __restrict__ gidx,
                     const uint64_t* __restrict__ prefix, int n, uint64_t items) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(16) Geometry sg;
  const uint64_t item = blockIdx.x;
  if (item >= items) return;
  const int e = find_field(prefix, n, item);
  batch_tile<T, PART>(*reinterpret_cast<CompressSmem<T>*>(smem_raw), sg, &fields[gidx[e]],
                      (uint32_t)(item - prefix[e]));
}

// The same with persistent CTAs taking tiles from a device counter.
template <class T, int PART>
__global__ void __launch_bounds__(kPredThreads, 3)
batch_predict_persistent_kernel(const BatchField* __restrict__ fields, const int* __restrict__ gidx,
                                const uint64_t* __restrict__ prefix, int n, uint64_t items,
                                unsigned long long* __restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(16) Geometry sg;
  __shared__ unsigned long long next;
  while (true) {
    __syncthreads();  // the previous tile no longer reads shared memory
    if (threadIdx.x == 0) next = atomicAdd(counter, 1ull);
    __syncthreads();
    const uint64_t item = next;
    if (item >= items) break;
    const int e = find_field(prefix, n, item);
    batch_tile_call<T, PART>(*reinterpret_cast<CompressSmem<T>*>(smem_raw), sg, &fields[gidx[e]],
                             (uint32_t)(item - prefix[e]));
  }
}

// leftover_fill_kernel over the ranges of all fields
__global__ void batch_leftover_kernel(const BatchField* __restrict__ fields, const BatchRange* __restrict__ ranges,
                                      int nranges) {
  for (int r = blockIdx.x; r < nranges; r += gridDim.x) {
    const BatchRange br = ranges[r];
    const BatchField& f = fields[br.field];
    const Geometry& g = f.g;
    for (uint64_t o = threadIdx.x; o < br.len; o += blockDim.x) {
      const uint64_t b = br.start + o;
      const uint64_t i = b >> 2;
      uint8_t v = 0;
      if (i < g.n) {
        const uint64_t x = i % g.nx, y = (i / g.nx) % g.ny, z = i / ((uint64_t)g.nx * g.ny);
        if ((x & 15) | (y & 15) | (z & 15)) {
          const uint32_t code = (uint32_t)f.qc[level_major_index(g, x, y, z)];
          v = (uint8_t)(code >> (8 * (b & 3)));
        }
      }
      f.planes[b] = v;
    }
  }
}

// the reference's last shuffle block for a list of (field, CTA) entries
__global__ void __launch_bounds__(512)
batch_last_block_kernel(const BatchField* __restrict__ fields, const BatchLastCta* __restrict__ ctas) {
  const BatchLastCta c = ctas[blockIdx.x];
  const BatchField& f = fields[c.field];
  shuffle_last_block(f.qc + f.g.anchors, f.planes, f.g, f.nb, f.g.aligned_size, c.cta, c.ncta);
}

// bulk shuffle: one warp per 1024-code item of any field
__global__ void __launch_bounds__(kShufWarps * 32)
batch_shuffle_kernel(const BatchField* __restrict__ fields, const uint64_t* __restrict__ prefix, int n,
                     uint64_t items) {
  __shared__ uint32_t tile[kShufWarps][32][33];
  const uint64_t item = (uint64_t)blockIdx.x * kShufWarps + (threadIdx.x >> 5);
  if (item >= items) return;
  const int e = find_field(prefix, n, item);
  const BatchField& f = fields[e];
  shuffle_item(tile[threadIdx.x >> 5], f.qc + f.g.anchors, f.planes, f.g, f.plan, f.nb, (int64_t)(item - prefix[e]));
}

// persistent lossless encoder over the chunks of all fields
__global__ void __launch_bounds__(kZThreads, 4)
batch_encode_kernel(const BatchField* __restrict__ fields, const uint64_t* __restrict__ prefix, int n,
                    uint64_t items, unsigned long long* __restrict__ ticket, long long spin_limit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EncodeShared& sh = *reinterpret_cast<EncodeShared*>(smem_raw);
  while (true) {
    if (threadIdx.x == 0) sh.ticket = (long long)atomicAdd(ticket, 1ull);
    __syncthreads();
    const uint64_t item = (uint64_t)sh.ticket;
    if (item >= items) break;
    const int e = find_field(prefix, n, item);
    const BatchField& f = fields[e];
    encode_chunk(sh, f.planes, f.g, f.out, f.status, (int64_t)(item - prefix[e]), f.st->csbp, &f.st->lossless_size,
                 &f.st->error_flag, spin_limit);
  }
}

// one warp per field: stream header and padding (zbpc_finish_kernel)
__global__ void batch_finish_kernel(const BatchField* __restrict__ fields, int n) {
  const int e = blockIdx.x;
  if (e >= n) return;
  const BatchField& f = fields[e];
  const uint64_t total = 8 + 2 * (uint64_t)f.g.chunks + f.st->lossless_size;
  const uint64_t pad = (8 - total % 8) % 8;
  if (threadIdx.x < pad) f.out[total + threadIdx.x] = 0;
  if (threadIdx.x == 0) {
    const long long hdr = (long long)f.g.aligned_size;
    for (int i = 0; i < 8; ++i) f.out[i] = (uint8_t)(hdr >> (8 * i));
    f.st->padded_size = total + pad;
  }
}

constexpr uint64_t kBatchTrailerSeg = 1u << 16;  // trailer bytes per item

// trailer (trailer_kernel) in items of kBatchTrailerSeg bytes over the group
template <class T>
__global__ void batch_trailer_kernel(const BatchField* __restrict__ fields, const int* __restrict__ gidx,
                                     const uint64_t* __restrict__ prefix, int n, uint64_t items) {
  for (uint64_t item = blockIdx.x; item < items; item += gridDim.x) {
    const int e = find_field(prefix, n, item);
    const BatchField& f = fields[gidx[e]];
    const PredParams<T>* p = reinterpret_cast<const PredParams<T>*>(f.st->params);
    uint8_t* tr = f.out + f.st->padded_size;
    const uint64_t total = 1040 + f.g.anchors * sizeof(T);
    const uint64_t b0 = (item - prefix[e]) * kBatchTrailerSeg, b1 = min(b0 + kBatchTrailerSeg, total);
    const uint8_t* range = reinterpret_cast<const uint8_t*>(&f.st->range);
    const uint8_t* csbp = reinterpret_cast<const uint8_t*>(f.st->csbp);
    const uint8_t* anchors = reinterpret_cast<const uint8_t*>(f.anchors);
    for (uint64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
      uint8_t v;
      if (i < 4) v = p->use_md[i];
      else if (i < 8) v = p->reverse[i - 4];
      else if (i < 16) v = range[i - 8];
      else if (i < 1040) v = csbp[i - 16];
      else v = anchors[i - 1040];
      tr[i] = v;
    }
  }
}

// per-field results for the host: padded stream size, error flag, flags
struct BatchResult {
  uint64_t padded_size;
  int error_flag;
  uint8_t flags[8];
  int pad;
};

template <class T>
__global__ void batch_collect_kernel(const BatchField* __restrict__ fields, const int* __restrict__ gidx, int n,
                                     BatchResult* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int fi = gidx[e];
  const BatchField& f = fields[fi];
  const PredParams<T>* p = reinterpret_cast<const PredParams<T>*>(f.st->params);
  BatchResult r;
  r.padded_size = f.st->padded_size;
  r.error_flag = f.st->error_flag;
  for (int l = 0; l < 4; ++l) { r.flags[l] = p->use_md[l]; r.flags[4 + l] = p->reverse[l]; }
  r.pad = 0;
  out[fi] = r;
}

}  // namespace prism_b200
