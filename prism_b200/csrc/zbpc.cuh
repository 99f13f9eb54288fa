// ZBPC lossless coder for the bit-plane buffer, byte-exact with the
// reference (src/encoder/zbpc.cu, include/encoder/RZE.hpp,
// d_zero_elimination.hpp, d_repetition_elimination.hpp).
//
// Stream layout: int64 plane-buffer size, uint16 csize[chunks], the chunk
// payloads back to back, zero padding to 8 bytes.  Chunks are 16 KiB pieces of
// each host plane (level 3 planes 0..31 first, then levels 2, 1, 0).  A chunk
// payload is either the raw bytes (csize == osize) or
//   [nonzero bytes][RE1 bytes][RE2 bytes][RE3 bytes][4-byte bitmap][osize:u16]
// where the zero-elimination bitmap (2048 B, bit i = byte i != 0, LSB first)
// is itself repetition-eliminated three times (2048 -> 256 -> 32 -> 4 bytes;
// a byte is kept iff it differs from its predecessor, byte -1 being 0).
// An all-zero chunk is just its 2-byte osize.
//
// B200 mapping.  Encode: persistent CTAs take chunk tickets from an atomic
// counter (so every chunk's predecessors are already running), build the
// payload in shared memory with block-wide prefix sums, and find their output
// offset with a decoupled look-back over a per-chunk status word (bounded
// spin: a stuck predecessor sets an error flag instead of hanging).  Decode:
// offsets come from a scan of the size table; one CTA per chunk rebuilds the
// bitmaps from the tail and scatters the bytes (a fill-forward is an inclusive
// popcount prefix).
#pragma once
#include "geometry.h"

namespace prism_b200 {

constexpr int kZThreads = 512;
constexpr int kZWarps = kZThreads / 32;

struct ChunkLoc {
  int level;        // host level (3 = coarsest, first in the stream)
  int64_t plane;
  int64_t offset;   // chunk index within the plane
  int64_t base;     // byte offset in the plane buffer
  int osize;
  bool last_of_plane;
};

__host__ __device__ __forceinline__ ChunkLoc locate_chunk(const Geometry& g, int64_t id) {
  ChunkLoc c;
  int64_t real = id;
  int l = 3;
  while (l > 0 && real >= g.chunks_level[l]) real -= g.chunks_level[l--];
  int64_t cpp = g.chunks_level[l] >> 5;
  c.level = l;
  c.plane = real / cpp;
  c.offset = real % cpp;
  int64_t b = 0;
  for (int i = 3; i > l; --i) b += g.hastride[i] << 5;
  c.base = b + c.plane * g.hastride[l] + c.offset * kChunk;
  int64_t rem = g.hastride[l] - c.offset * kChunk;
  c.osize = (int)(rem < kChunk ? rem : kChunk);
  c.last_of_plane = c.offset == cpp - 1;
  return c;
}

// ---- block-wide helpers (512 threads) ----
__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v += t;
  }
  return v;
}

// exclusive prefix over the block; *total receives the block sum
__device__ __forceinline__ int block_excl_scan(int v, int* scratch, int* total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = warp_incl_scan(v, lane);
  if (lane == 31) scratch[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int s = lane < kZWarps ? scratch[lane] : 0;
    int si = warp_incl_scan(s, lane);
    if (lane < kZWarps) scratch[lane] = si - s;
    if (lane == kZWarps - 1) scratch[32] = si;
  }
  __syncthreads();
  int r = scratch[warp] + incl - v;
  *total = scratch[32];
  __syncthreads();
  return r;
}

struct EncodeShared {
  uint8_t in[kChunk];
  // payload staging: nonzero bytes (< osize) plus up to 2048 + 256 + 32 + 6
  // bitmap bytes before the size check can reject the encoding
  uint8_t out[kChunk + 2048 + 512];
  uint8_t bm0[2048];
  uint8_t bm1[256];
  uint8_t bm2[32];
  uint8_t bm3[4];
  int scratch[40];
  long long ticket;
  long long excl;
};

// repetition elimination of `n` (<= 2048) bitmap bytes held in shared memory:
// kept bytes go to out[pos..], flags to bmo; returns the kept count
__device__ __forceinline__ int re_encode_block(const uint8_t* bm, int n, uint8_t* out, int pos,
                                               uint8_t* bmo, int* scratch) {
  // each thread takes 4 consecutive bytes (n = 2048) or 1 byte (n <= 512)
  int per = n > kZThreads ? 4 : 1;
  int i0 = threadIdx.x * per;
  int flags = 0;
  if (i0 < n) {
    for (int k = 0; k < per; ++k) {
      int i = i0 + k;
      uint8_t prev = i == 0 ? 0 : bm[i - 1];
      flags |= (bm[i] != prev) << k;
    }
  }
  int total;
  int off = block_excl_scan(__popc(flags), scratch, &total);
  if (i0 < n) {
    for (int k = 0; k < per; ++k)
      if ((flags >> k) & 1) out[pos + off++] = bm[i0 + k];
  }
  // flags -> bitmap bytes (bit i of the whole map = flag of byte i)
  if (per == 4) {
    // 4 flags per thread, 2 threads per output byte
    uint32_t f = (uint32_t)flags;
    uint32_t other = __shfl_down_sync(0xffffffffu, f, 1);
    if ((threadIdx.x & 1) == 0 && i0 < n) bmo[i0 / 8] = (uint8_t)(f | (other << 4));
  } else {
    uint32_t bal = __ballot_sync(0xffffffffu, flags & 1);
    int lane = threadIdx.x & 31;
    if ((lane & 7) == 0 && i0 < n) bmo[i0 / 8] = (uint8_t)(bal >> lane);
  }
  __syncthreads();
  return total;
}

__global__ void __launch_bounds__(kZThreads)
zbpc_encode_kernel(const uint8_t* __restrict__ planes, Geometry g, uint8_t* __restrict__ stream,
                   unsigned long long* __restrict__ status, unsigned long long* __restrict__ ticket,
                   uint64_t* __restrict__ comp_size_bp, uint64_t* __restrict__ lossless_size,
                   int* __restrict__ error_flag, long long spin_limit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EncodeShared& sh = *reinterpret_cast<EncodeShared*>(smem_raw);
  const int tid = threadIdx.x;
  const int64_t chunks = g.chunks;
  uint16_t* sizes = reinterpret_cast<uint16_t*>(stream + 8);
  uint8_t* data_out = stream + 8 + 2 * chunks;
  while (true) {
    if (tid == 0) sh.ticket = (long long)atomicAdd(ticket, 1ull);
    __syncthreads();
    const int64_t id = sh.ticket;
    if (id >= chunks) break;
    ChunkLoc loc = locate_chunk(g, id);
    const int osize = loc.osize;
    // load (base and osize are multiples of 8)
    const uint2* src = reinterpret_cast<const uint2*>(planes + loc.base);
    uint2* dst = reinterpret_cast<uint2*>(sh.in);
    for (int i = tid; i < osize / 8; i += kZThreads) dst[i] = __ldg(src + i);
    __syncthreads();
    // zero elimination: each thread 32 bytes -> one 32-bit bitmap word
    uint32_t bits = 0;
    int b0 = tid * 32;
    if (b0 < osize) {
      const uint4* w = reinterpret_cast<const uint4*>(sh.in + b0);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        uint4 v = w[q];
        uint32_t words[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
          for (int j = 0; j < 4; ++j)
            bits |= (uint32_t)(((words[k] >> (8 * j)) & 0xFF) != 0) << (q * 16 + k * 4 + j);
      }
      if (b0 + 32 > osize) bits &= (1u << (osize - b0)) - 1u;
    }
    reinterpret_cast<uint32_t*>(sh.bm0)[tid] = bits;  // 512 words = 2048 bytes
    int nz_total;
    int off = block_excl_scan(__popc(bits), sh.scratch, &nz_total);
    for (uint32_t m = bits; m; m &= m - 1) {
      int j = __ffs(m) - 1;
      sh.out[off++] = sh.in[b0 + j];
    }
    __syncthreads();
    int csize;
    bool raw = false;
    if (nz_total == 0) {
      csize = 2;
      if (tid == 0) { sh.out[0] = (uint8_t)osize; sh.out[1] = (uint8_t)(osize >> 8); }
    } else if (nz_total + 6 >= osize) {
      raw = true;
      csize = osize;
    } else {
      int pos = nz_total;
      int c1 = re_encode_block(sh.bm0, 2048, sh.out, pos, sh.bm1, sh.scratch);
      pos += c1;
      if (pos + 6 >= osize) { raw = true; csize = osize; }
      else {
        int c2 = re_encode_block(sh.bm1, 256, sh.out, pos, sh.bm2, sh.scratch);
        pos += c2;
        int c3 = re_encode_block(sh.bm2, 32, sh.out, pos, sh.bm3, sh.scratch);
        pos += c3;
        csize = pos + 6;
        if (csize >= osize) { raw = true; csize = osize; }
        else if (tid < 4) {
          sh.out[pos + tid] = sh.bm3[tid];
          if (tid == 0) { sh.out[pos + 4] = (uint8_t)osize; sh.out[pos + 5] = (uint8_t)(osize >> 8); }
        }
      }
    }
    __syncthreads();
    // decoupled look-back: flag 1 = local size, flag 2 = inclusive prefix
    if (tid < 32) {
      const unsigned long long kAgg = 1ull << 62, kInc = 2ull << 62, kMask = (1ull << 62) - 1;
      if (id == 0) {
        if (tid == 0) { atomicExch(&status[0], kInc | (unsigned long long)csize); sh.excl = 0; }
      } else {
        if (tid == 0) atomicExch(&status[id], kAgg | (unsigned long long)csize);
        long long excl = 0;
        int64_t j = id - 1;
        long long spins = 0;
        bool done = false;
        while (!done) {
          int64_t k = j - tid;
          unsigned long long v = k >= 0 ? 0ull : kInc;
          if (k >= 0) {
            do {
              v = atomicAdd(&status[k], 0ull);
              if (v == 0) {
                if (++spins > spin_limit) { atomicExch(error_flag, 1); v = kInc; }
                else __nanosleep(64);
              }
            } while (v == 0);
          }
          unsigned inc_mask = __ballot_sync(0xffffffffu, (v >> 62) == 2);
          int stop = inc_mask ? __ffs(inc_mask) - 1 : 32;
          long long part = (tid <= stop && tid < 32) ? (long long)(v & kMask) : 0;
#pragma unroll
          for (int d = 16; d > 0; d >>= 1) part += __shfl_xor_sync(0xffffffffu, part, d);
          excl += part;
          if (inc_mask) done = true;
          else j -= 32;
        }
        if (tid == 0) {
          atomicExch(&status[id], kInc | (unsigned long long)(excl + csize));
          sh.excl = excl;
        }
      }
    }
    __syncthreads();
    const long long offs = sh.excl;
    if (tid == 0) {
      sizes[id] = (uint16_t)csize;
      if (loc.last_of_plane) comp_size_bp[(3 - loc.level) * 32 + loc.plane] = (uint64_t)(offs + csize);
      if (id == chunks - 1) *lossless_size = (uint64_t)(offs + csize);
    }
    const uint8_t* payload = raw ? sh.in : sh.out;
    uint8_t* o = data_out + offs;
    for (int i = tid; i < csize; i += kZThreads) o[i] = payload[i];
    __syncthreads();
  }
}

// stream header + zero padding once the total is known
__global__ void zbpc_finish_kernel(uint8_t* stream, Geometry g, const uint64_t* lossless_size,
                                   uint64_t* padded_size) {
  uint64_t total = 8 + 2 * (uint64_t)g.chunks + *lossless_size;
  uint64_t pad = (8 - total % 8) % 8;
  if (threadIdx.x < pad) stream[total + threadIdx.x] = 0;
  if (threadIdx.x == 0) {
    long long hdr = (long long)g.aligned_size;
    for (int i = 0; i < 8; ++i) stream[i] = (uint8_t)(hdr >> (8 * i));
    *padded_size = total + pad;
  }
}

// ---------------- decode ----------------
// exclusive scan of the uint16 size table into int64 offsets (3 kernels)
constexpr int kScanItems = 4096;

__global__ void __launch_bounds__(1024) scan_sizes_block(const uint16_t* __restrict__ sizes, int64_t n,
                                                         int64_t* __restrict__ offs, int64_t* __restrict__ block_sum) {
  __shared__ int64_t warp_tot[32];
  int64_t base = (int64_t)blockIdx.x * kScanItems + threadIdx.x * 4;
  int64_t v[4];
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) { v[k] = base + k < n ? sizes[base + k] : 0; s += v[k]; }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t incl = s;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int64_t t = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += t;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int64_t w = warp_tot[lane];
    int64_t wi = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      int64_t t = __shfl_up_sync(0xffffffffu, wi, d);
      if (lane >= d) wi += t;
    }
    warp_tot[lane] = wi - w;
    if (lane == 31) block_sum[blockIdx.x] = wi;
  }
  __syncthreads();
  int64_t run = warp_tot[warp] + incl - s;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (base + k < n) offs[base + k] = run;
    run += v[k];
  }
}

__global__ void scan_block_sums(int64_t* block_sum, int64_t nblocks) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int64_t acc = 0;
    for (int64_t i = 0; i < nblocks; ++i) { int64_t t = block_sum[i]; block_sum[i] = acc; acc += t; }
  }
}

__global__ void scan_add(int64_t* offs, int64_t n, const int64_t* block_sum) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) offs[i] += block_sum[i / kScanItems];
}

struct DecodeShared {
  uint8_t in[kChunk + 16];
  uint8_t bm0[2048];
  uint8_t bm1[256];
  uint8_t bm2[32];
  uint8_t bm3[4];
  int scratch[40];
};

// fill-forward decode of `n` bitmap bytes from `data` with flags `bm`:
// out[i] = data[rank(i) - 1] (0 when no flag yet), rank = inclusive popcount
__device__ __forceinline__ void re_decode_block(const uint8_t* data, const uint8_t* bm, int n, uint8_t* out,
                                                int* scratch) {
  int per = n > kZThreads ? 4 : 1;
  int i0 = threadIdx.x * per;
  int flags = 0;
  if (i0 < n)
    for (int k = 0; k < per; ++k) flags |= ((bm[(i0 + k) >> 3] >> ((i0 + k) & 7)) & 1) << k;
  int total;
  int rank = block_excl_scan(__popc(flags), scratch, &total);
  if (i0 < n) {
    for (int k = 0; k < per; ++k) {
      rank += (flags >> k) & 1;
      out[i0 + k] = rank > 0 ? data[rank - 1] : 0;
    }
  }
  __syncthreads();
}

__device__ __forceinline__ int popc_bytes_block(const uint8_t* b, int n, int* scratch) {
  int v = 0;
  for (int i = threadIdx.x; i < n; i += kZThreads) v += __popc(b[i]);
  int total;
  block_excl_scan(v, scratch, &total);
  return total;
}

// One CTA per chunk.  begin/end (device, may be null) select the chunks of
// host planes [begin[3-l], end[3-l]) like zbpc_decode_progressive
// (zbpc.cu:420-423).  Returns per-chunk errors through error_flag.
__global__ void __launch_bounds__(kZThreads)
zbpc_decode_kernel(const uint8_t* __restrict__ stream, uint64_t stream_bytes, const int64_t* __restrict__ offs,
                   Geometry g, uint8_t* __restrict__ planes, const int* __restrict__ begin,
                   const int* __restrict__ end, int* __restrict__ error_flag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  DecodeShared& sh = *reinterpret_cast<DecodeShared*>(smem_raw);
  const int tid = threadIdx.x;
  const int64_t chunks = g.chunks;
  const uint16_t* sizes = reinterpret_cast<const uint16_t*>(stream + 8);
  const uint8_t* data_in = stream + 8 + 2 * chunks;
  for (int64_t id = blockIdx.x; id < chunks; id += gridDim.x) {
    ChunkLoc loc = locate_chunk(g, id);
    if (begin) {
      int64_t cpp = g.chunks_level[loc.level] >> 5;
      int64_t real = loc.plane * cpp + loc.offset;
      if (real < begin[3 - loc.level] * cpp || real >= end[3 - loc.level] * cpp) continue;
    }
    const int osize = loc.osize;
    const int csize = sizes[id];
    const uint64_t at = (uint64_t)(8 + 2 * chunks + offs[id]);
    if (csize > osize || at + (uint64_t)csize > stream_bytes) {  // corrupt size table
      if (tid == 0) atomicExch(error_flag, 2);
      continue;
    }
    const uint8_t* src = data_in + offs[id];
    uint8_t* dst = planes + loc.base;
    if (csize == osize) {  // raw chunk
      for (int i = tid; i < osize; i += kZThreads) dst[i] = src[i];
      continue;
    }
    for (int i = tid; i < csize; i += kZThreads) sh.in[i] = src[i];
    __syncthreads();
    bool bad = csize < 2 || (sh.in[csize - 2] | (sh.in[csize - 1] << 8)) != osize;
    int rpos = csize - 2;
    if (!bad && rpos == 0) {  // all zero
      uint2* d2 = reinterpret_cast<uint2*>(dst);
      for (int i = tid; i < osize / 8; i += kZThreads) d2[i] = make_uint2(0, 0);
      __syncthreads();
      continue;
    }
    if (!bad && rpos < 4) bad = true;
    if (bad) {
      if (tid == 0) atomicExch(error_flag, 2);
      __syncthreads();
      continue;
    }
    rpos -= 4;
    if (tid < 4) sh.bm3[tid] = sh.in[rpos + tid];
    __syncthreads();
    int c3 = popc_bytes_block(sh.bm3, 4, sh.scratch);
    rpos -= c3;
    bool ok = rpos >= 0;
    if (ok) re_decode_block(sh.in + rpos, sh.bm3, 32, sh.bm2, sh.scratch);
    int c2 = ok ? popc_bytes_block(sh.bm2, 32, sh.scratch) : 0;
    rpos -= c2;
    ok = ok && rpos >= 0;
    if (ok) re_decode_block(sh.in + rpos, sh.bm2, 256, sh.bm1, sh.scratch);
    int c1 = ok ? popc_bytes_block(sh.bm1, 256, sh.scratch) : 0;
    rpos -= c1;
    ok = ok && rpos >= 0;
    if (ok) re_decode_block(sh.in + rpos, sh.bm1, 2048, sh.bm0, sh.scratch);
    if (!ok) {
      if (tid == 0) atomicExch(error_flag, 2);
      __syncthreads();
      continue;
    }
    // zero-elimination decode: thread t owns bytes [32t, 32t+32)
    uint32_t bits = reinterpret_cast<const uint32_t*>(sh.bm0)[tid];
    int b0 = tid * 32;
    int total;
    int rank = block_excl_scan(__popc(bits), sh.scratch, &total);
    if (b0 < osize) {
      uint32_t w[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        uint32_t v = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          int bit = q * 4 + j;
          uint32_t byte = 0;
          if ((bits >> bit) & 1) byte = sh.in[rank++];
          v |= byte << (8 * j);
        }
        w[q] = v;
      }
      int nb = osize - b0 < 32 ? osize - b0 : 32;
      if (nb == 32) {
        uint2* d2 = reinterpret_cast<uint2*>(dst + b0);
#pragma unroll
        for (int q = 0; q < 4; ++q) d2[q] = make_uint2(w[2 * q], w[2 * q + 1]);
      } else {
        for (int b = 0; b < nb; ++b) dst[b0 + b] = (uint8_t)(w[b >> 2] >> (8 * (b & 3)));
      }
    }
    if (total > rpos && tid == 0) atomicExch(error_flag, 2);
    __syncthreads();
  }
}

}  // namespace prism_b200
