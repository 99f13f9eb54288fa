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

// Chunk counts fit 32 bits (a plane buffer of 2^32 chunks would be 64 TB),
// so the plane/offset split is a 32-bit division (a 64-bit one is a long
// software sequence, run by every thread for every chunk).
__host__ __device__ __forceinline__ ChunkLoc locate_chunk(const Geometry& g, int64_t id) {
  ChunkLoc c;
  int64_t real = id;
  int l = 3;
  while (l > 0 && real >= g.chunks_level[l]) real -= g.chunks_level[l--];
  const uint32_t cpp = (uint32_t)(g.chunks_level[l] >> 5), r32 = (uint32_t)real;
  const uint32_t plane = r32 / cpp;
  c.level = l;
  c.plane = plane;
  c.offset = r32 - plane * cpp;
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

// exclusive prefix over the block; *total receives the block sum.  Two
// barriers; scratch must not be reused before the next barrier.
__device__ __forceinline__ int block_excl_scan(int v, int* scratch, int* total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = warp_incl_scan(v, lane);
  if (lane == 31) scratch[warp] = incl;
  __syncthreads();
  int w = lane < kZWarps ? scratch[lane] : 0;
  int wi = warp_incl_scan(w, lane);
  int before = __shfl_sync(0xffffffffu, wi - w, warp);
  *total = __shfl_sync(0xffffffffu, wi, kZWarps - 1);
  __syncthreads();
  return before + incl - v;
}

struct EncodeShared {
  uint8_t in[kChunk + 16];
  // payload staging: nonzero bytes (< osize) plus up to 2048 + 256 + 32 + 6
  // bitmap bytes before the size check can reject the encoding
  uint8_t out[kChunk + 2048 + 512 + 16];
  uint8_t bm0[2048];
  uint8_t bm1[256];
  uint8_t bm2[32];
  uint8_t bm3[4];
  int scratch[40];
  long long ticket;
  long long excl;
  int csz;
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

// Copy n bytes from shared memory to an arbitrarily aligned global address:
// head bytes, then aligned 32-bit words (each assembled from two aligned
// shared words), then the tail.
__device__ __forceinline__ void copy_out(uint8_t* dst, const uint8_t* src, int n) {
  const int tid = threadIdx.x;
  int head = (int)((4 - ((uintptr_t)dst & 3)) & 3);
  if (head > n) head = n;
  if (tid < head) dst[tid] = src[tid];
  const int words = (n - head) >> 2;
  uint32_t* dw = reinterpret_cast<uint32_t*>(dst + head);
  const int sh = head & 3;
  const uint32_t* sw = reinterpret_cast<const uint32_t*>(src);
  for (int w = tid; w < words; w += kZThreads) {
    if (sh == 0) {
      dw[w] = sw[w];
    } else {
      // bytes head + 4w .. +3 = words w and w+1 shifted by sh bytes
      uint32_t lo = sw[w], hi = sw[w + 1];
      dw[w] = __funnelshift_r(lo, hi, 8 * sh);
    }
  }
  const int done = head + 4 * words;
  if (tid < n - done) dst[done + tid] = src[done + tid];
}

// Encode chunk `id` of one field (status is that field's slice, so the
// look-back ends at the field's first chunk).  All 512 threads of the CTA
// call this; it ends with a barrier.
__device__ __forceinline__ void encode_chunk(EncodeShared& sh, const uint8_t* __restrict__ planes, const Geometry& g,
                                             uint8_t* __restrict__ stream, unsigned long long* __restrict__ status,
                                             const int64_t id, uint64_t* __restrict__ comp_size_bp,
                                             uint64_t* __restrict__ lossless_size, int* __restrict__ error_flag,
                                             long long spin_limit) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t chunks = g.chunks;
  uint16_t* sizes = reinterpret_cast<uint16_t*>(stream + 8);
  uint8_t* data_out = stream + 8 + 2 * chunks;
  {
    const ChunkLoc loc = locate_chunk(g, id);
    const int osize = loc.osize;
    // ---- load 32 bytes per thread (base and osize are multiples of 8) ----
    const int b0 = tid * 32;
    uint32_t wds[8];
    {
      const uint2* src = reinterpret_cast<const uint2*>(planes + loc.base + b0);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint2 v = make_uint2(0, 0);
        if (b0 + 8 * q < osize) v = __ldg(src + q);
        wds[2 * q] = v.x;
        wds[2 * q + 1] = v.y;
      }
    }
    uint4* in4 = reinterpret_cast<uint4*>(sh.in + b0);
    in4[0] = make_uint4(wds[0], wds[1], wds[2], wds[3]);
    in4[1] = make_uint4(wds[4], wds[5], wds[6], wds[7]);
    // zero elimination bitmap: bit j = byte b0 + j is nonzero
    uint32_t bits = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
      for (int j = 0; j < 4; ++j) bits |= (uint32_t)(((wds[k] >> (8 * j)) & 0xFF) != 0) << (4 * k + j);
    if (b0 + 32 > osize) bits = b0 >= osize ? 0u : bits & ((1u << (osize - b0)) - 1u);
    reinterpret_cast<uint32_t*>(sh.bm0)[tid] = bits;
    int nz_total;
    const int zoff = block_excl_scan(__popc(bits), sh.scratch, &nz_total);
    // ---- decide the encoding; build the payload in sh.out ----
    int csize;
    bool raw = false;
    if (nz_total == 0) {
      csize = 2;
      if (tid == 0) { sh.out[0] = (uint8_t)osize; sh.out[1] = (uint8_t)(osize >> 8); }
    } else if (nz_total + 6 >= osize) {
      raw = true;
      csize = osize;
    } else {
      // nonzero bytes, in order: every thread walks its 32 positions
      {
        int r = zoff;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          if ((bits >> j) & 1u) sh.out[r] = (uint8_t)(wds[j >> 2] >> (8 * (j & 3)));
          r += (bits >> j) & 1u;
        }
      }
      // RE 2048 -> 256: thread t flags bitmap bytes 4t..4t+3 (bm0 is complete
      // since the scan's barriers)
      const uint32_t cur = bits;
      const uint32_t prev_byte = tid == 0 ? 0u : (reinterpret_cast<const uint32_t*>(sh.bm0)[tid - 1] >> 24);
      uint32_t f1 = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        uint32_t byte = (cur >> (8 * k)) & 0xFF;
        uint32_t before = k == 0 ? prev_byte : ((cur >> (8 * (k - 1))) & 0xFF);
        f1 |= (uint32_t)(byte != before) << k;
      }
      int c1;
      const int r1 = block_excl_scan(__popc(f1), sh.scratch, &c1);
      if (nz_total + c1 + 6 >= osize) {
        raw = true;
        csize = osize;
      } else {
        {
          int r = nz_total + r1;
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if ((f1 >> k) & 1u) sh.out[r++] = (uint8_t)(cur >> (8 * k));
        }
        uint32_t other = __shfl_down_sync(0xffffffffu, f1, 1);
        if ((tid & 1) == 0) sh.bm1[tid >> 1] = (uint8_t)(f1 | (other << 4));
        __syncthreads();
        if (warp == 0) {
          // RE 256 -> 32: lane l flags bm1 bytes 8l..8l+7
          uint32_t f2 = 0;
          uint8_t b1[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) b1[k] = sh.bm1[8 * lane + k];
          uint8_t before = lane == 0 ? 0 : sh.bm1[8 * lane - 1];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            f2 |= (uint32_t)(b1[k] != before) << k;
            before = b1[k];
          }
          int cnt2 = __popc(f2);
          int incl2 = warp_incl_scan(cnt2, lane);
          int c2 = __shfl_sync(0xffffffffu, incl2, 31);
          int r = nz_total + c1 + incl2 - cnt2;
#pragma unroll
          for (int k = 0; k < 8; ++k)
            if ((f2 >> k) & 1u) sh.out[r++] = b1[k];
          // RE 32 -> 4: lane l flags bm2 byte l (= f2)
          uint32_t prev2 = __shfl_up_sync(0xffffffffu, f2, 1);
          if (lane == 0) prev2 = 0;
          uint32_t bal = __ballot_sync(0xffffffffu, f2 != prev2);
          int c3 = __popc(bal);
          int pos = nz_total + c1 + c2;
          if ((f2 != prev2)) sh.out[pos + __popc(bal & ((1u << lane) - 1u))] = (uint8_t)f2;
          pos += c3;
          int cs = pos + 6;
          if (lane == 0) sh.csz = cs;
          if (cs < osize) {
            if (lane < 4) sh.out[pos + lane] = (uint8_t)(bal >> (8 * lane));
            if (lane == 0) { sh.out[pos + 4] = (uint8_t)osize; sh.out[pos + 5] = (uint8_t)(osize >> 8); }
          }
        }
        __syncthreads();
        csize = sh.csz;
        if (csize >= osize) { raw = true; csize = osize; }
      }
    }
    // ---- decoupled look-back: flag 1 = local size, flag 2 = inclusive prefix ----
    if (warp == 0) {
      const unsigned long long kAgg = 1ull << 62, kInc = 2ull << 62, kMask = (1ull << 62) - 1;
      if (id == 0) {
        if (lane == 0) { atomicExch(&status[0], kInc | (unsigned long long)csize); sh.excl = 0; }
      } else {
        if (lane == 0) atomicExch(&status[id], kAgg | (unsigned long long)csize);
        long long excl = 0;
        int64_t j = id - 1;
        long long spins = 0;
        bool done = false;
        while (!done) {
          int64_t k = j - lane;
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
          long long part = lane <= stop ? (long long)(v & kMask) : 0;
#pragma unroll
          for (int d = 16; d > 0; d >>= 1) part += __shfl_xor_sync(0xffffffffu, part, d);
          excl += part;
          if (inc_mask) done = true;
          else j -= 32;
        }
        if (lane == 0) {
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
    copy_out(data_out + offs, raw ? sh.in : sh.out, csize);
    __syncthreads();
  }
}

// Persistent encoder: one CTA (512 threads, 32 bytes each) per 16 KiB chunk,
// four CTAs per SM, chunks handed out in order by a ticket counter.
__global__ void __launch_bounds__(kZThreads, 4)
zbpc_encode_kernel(const uint8_t* __restrict__ planes, Geometry g, uint8_t* __restrict__ stream,
                   unsigned long long* __restrict__ status, unsigned long long* __restrict__ ticket,
                   uint64_t* __restrict__ comp_size_bp, uint64_t* __restrict__ lossless_size,
                   int* __restrict__ error_flag, long long spin_limit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EncodeShared& sh = *reinterpret_cast<EncodeShared*>(smem_raw);
  while (true) {
    if (threadIdx.x == 0) sh.ticket = (long long)atomicAdd(ticket, 1ull);
    __syncthreads();
    const int64_t id = sh.ticket;
    if (id >= g.chunks) break;
    encode_chunk(sh, planes, g, stream, status, id, comp_size_bp, lossless_size, error_flag, spin_limit);
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
  uint8_t in[kChunk + 32];
  uint8_t bm0[2048];
  uint8_t bm1[256];
  uint8_t bm2[32];
  int scratch[40];
  int flag;
};

// Copy n <= kChunk bytes from an arbitrarily aligned global address into
// shared memory with aligned 32-bit loads; no byte past src + n - 1's word is
// read.  A thread's words are w = t + k * kZThreads (k < 8); every load is
// issued before the first store, so a chunk costs one load latency.  Each
// source word is loaded once: the word after w is the next lane's (lane 31
// loads it itself).
__device__ __forceinline__ void copy_in(uint8_t* dst, const uint8_t* src, int n) {
  constexpr int kWords = kChunk / 4 / kZThreads;
  const int shift = (int)((uintptr_t)src & 3);
  const uint32_t* a = reinterpret_cast<const uint32_t*>(src - shift);
  const int last = (shift + n - 1) >> 2;  // last source word needed
  const int lane = threadIdx.x & 31;
  uint32_t* dw = reinterpret_cast<uint32_t*>(dst);
  uint32_t lo[kWords], hi[kWords];
#pragma unroll
  for (int k = 0; k < kWords; ++k) {
    const int w = threadIdx.x + k * kZThreads;
    lo[k] = w <= last ? __ldg(a + w) : 0u;
    hi[k] = (lane == 31 && w + 1 <= last) ? __ldg(a + w + 1) : 0u;
  }
#pragma unroll
  for (int k = 0; k < kWords; ++k) {
    const int w = threadIdx.x + k * kZThreads;
    const uint32_t next = __shfl_down_sync(0xffffffffu, lo[k], 1);
    if (lane != 31) hi[k] = next;
    if (4 * w < n) dw[w] = shift ? __funnelshift_r(lo[k], hi[k], 8 * shift) : lo[k];
  }
}

// Chunk holding byte `off` of the plane buffer (host placement: level 3's 32
// planes first, each plane cut into 16 KiB chunks; chunk ids follow the
// bytes).  Offsets past the buffer map past the last chunk.
__device__ __forceinline__ int64_t chunk_of_byte(const Geometry& g, int64_t off) {
  int64_t hb = 0, cb = 0;
  for (int l = 3; l >= 0; --l) {
    const int64_t span = g.hastride[l] << 5;
    if (off < hb + span || l == 0) {
      const int64_t rel = off - hb, p = rel / g.hastride[l];
      return cb + p * (g.chunks_level[l] >> 5) + (rel - p * g.hastride[l]) / kChunk;
    }
    hb += span;
    cb += g.chunks_level[l];
  }
  return 0;
}

// Grid-stride over the chunks a decode must visit.  begin/end (device, may
// be null) select the chunks of host planes [begin[3-l], end[3-l]) like
// zbpc_decode_progressive (zbpc.cu:420-423); then per level only one range
// of chunk ids matters: the selected planes' chunks and the chunks holding
// the bytes the inverse shuffle reads for those planes at their device
// placement (which are zeroed where no selected chunk covers them).  Other
// chunks are never read, so the walk skips them.  Corrupt chunks raise
// error_flag = 2.  The payload is decoded from its tail: bitmap 4 B -> 32 B
// -> 256 B -> 2048 B (fill-forward: byte i = kept byte rank(i) - 1, rank the
// inclusive flag count), then the nonzero bytes are scattered by the
// zero-elimination bitmap.
__global__ void __launch_bounds__(kZThreads, 4)
zbpc_decode_kernel(const uint8_t* __restrict__ stream, uint64_t stream_bytes, const int64_t* __restrict__ offs,
                   Geometry g, uint8_t* __restrict__ planes, const int* __restrict__ begin,
                   const int* __restrict__ end, int* __restrict__ error_flag) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  DecodeShared& sh = *reinterpret_cast<DecodeShared*>(smem_raw);
  __shared__ int64_t range_start[4], range_len[4];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t chunks = g.chunks;
  const uint16_t* sizes = reinterpret_cast<const uint16_t*>(stream + 8);
  const uint8_t* data_in = stream + 8 + 2 * chunks;
  if (tid < 4) {
    const int l = tid;
    int64_t s = 0, e = 0;
    if (!begin) {
      e = l == 0 ? chunks : 0;  // a full decode: every chunk, once
    } else if (begin[3 - l] < end[3 - l]) {
      const int lo = begin[3 - l], hi = end[3 - l];
      int64_t cb = 0;
      for (int i = 3; i > l; --i) cb += g.chunks_level[i];
      const int64_t cpp = g.chunks_level[l] >> 5;
      s = cb + lo * cpp;
      e = cb + hi * cpp;
      const int64_t a = g.daprefix[l] + (int64_t)lo * g.dstride[l], b = g.daprefix[l] + (int64_t)hi * g.dstride[l];
      const int64_t lim = (int64_t)g.aligned_size;
      if (a < b && a < lim) {
        const int64_t f = chunk_of_byte(g, a), t = chunk_of_byte(g, (b < lim ? b : lim) - 1) + 1;
        s = f < s ? f : s;
        e = t > e ? t : e;
      }
      s = s < 0 ? 0 : (s > chunks ? chunks : s);
      e = e < s ? s : (e > chunks ? chunks : e);
    }
    range_start[l] = s;
    range_len[l] = e - s;
  }
  __syncthreads();
  const int64_t visits = range_len[0] + range_len[1] + range_len[2] + range_len[3];
  for (int64_t v = blockIdx.x; v < visits; v += gridDim.x) {
    int64_t id = v;
    int r = 0;
    while (r < 3 && id >= range_len[r]) id -= range_len[r++];
    id += range_start[r];
    const ChunkLoc loc = locate_chunk(g, id);
    if (begin) {
      int64_t cpp = g.chunks_level[loc.level] >> 5;
      int64_t real = loc.plane * cpp + loc.offset;
      if (real < begin[3 - loc.level] * cpp || real >= end[3 - loc.level] * cpp) {
        // A plane this step does not load reads as zero where the inverse
        // shuffle reads it: the inverse reads, per level l, the planes
        // [lo, hi) it selects at their device placement, bytes
        // [daprefix[l] + lo dstride[l], daprefix[l] + hi dstride[l]), which
        // can reach into the host placement of neighbouring planes.  Only the
        // part of this chunk inside those ranges is zeroed (all bounds are
        // multiples of 8); the rest is never read.
        const int64_t cb = loc.base, ce = loc.base + loc.osize;
#pragma unroll 1
        for (int l = 0; l < 4; ++l) {
          const int lo = begin[3 - l], hi = end[3 - l];
          if (lo >= hi) continue;
          const int64_t r0 = g.daprefix[l] + (int64_t)lo * g.dstride[l], r1 = g.daprefix[l] + (int64_t)hi * g.dstride[l];
          const int64_t a = cb > r0 ? cb : r0, e = ce < r1 ? ce : r1;
          for (int64_t o = a + 8 * (int64_t)tid; o < e; o += 8 * (int64_t)kZThreads)
            *reinterpret_cast<uint2*>(planes + o) = make_uint2(0, 0);
        }
        continue;
      }
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
    const int b0 = tid * 32;
    if (csize == osize) {  // raw chunk: 32 bytes per thread through shared memory
      copy_in(sh.in, src, osize);
      __syncthreads();
      if (b0 < osize) {
        const uint2* s2 = reinterpret_cast<const uint2*>(sh.in + b0);
        uint2* d2 = reinterpret_cast<uint2*>(dst + b0);
        const int nq = min(4, (osize - b0) >> 3);
        for (int q = 0; q < nq; ++q) d2[q] = s2[q];
      }
      __syncthreads();
      continue;
    }
    copy_in(sh.in, src, csize);
    if (tid == 0) sh.flag = 0;
    __syncthreads();
    bool bad = csize < 2 || (sh.in[csize - 2] | (sh.in[csize - 1] << 8)) != osize;
    if (!bad && csize == 2) {  // all zero
      if (b0 < osize) {
        uint2* d2 = reinterpret_cast<uint2*>(dst + b0);
        const int nq = min(4, (osize - b0) >> 3);
        for (int q = 0; q < nq; ++q) d2[q] = make_uint2(0, 0);
      }
      __syncthreads();
      continue;
    }
    if (!bad && csize < 6) bad = true;
    if (bad) {
      if (tid == 0) atomicExch(error_flag, 2);
      __syncthreads();
      continue;
    }
    // ---- warp 0: bm3 (4 B) -> bm2 (32 B) -> bm1 (256 B) ----
    int rpos = csize - 6;  // start of bm3
    if (warp == 0) {
      const uint32_t bm3 = (uint32_t)sh.in[rpos] | ((uint32_t)sh.in[rpos + 1] << 8) |
                           ((uint32_t)sh.in[rpos + 2] << 16) | ((uint32_t)sh.in[rpos + 3] << 24);
      const int c3 = __popc(bm3);
      const int p3 = rpos - c3;  // RE3 bytes
      // bm2 byte l = kept byte (inclusive rank of flag l) - 1, or 0
      const int rank3 = __popc(bm3 & (0xffffffffu >> (31 - lane)));
      uint32_t b2 = 0;
      if (p3 >= 0 && rank3 > 0) b2 = sh.in[p3 + rank3 - 1];
      sh.bm2[lane] = (uint8_t)b2;
      // bm2 flags 256 bits: lane l owns flags 8l..8l+7 = byte b2 of lane l
      const int cnt2 = __popc(b2);
      const int incl2 = warp_incl_scan(cnt2, lane);
      const int c2 = __shfl_sync(0xffffffffu, incl2, 31);
      const int p2 = p3 - c2;  // RE2 bytes
      int r = incl2 - cnt2;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        r += (b2 >> k) & 1u;
        sh.bm1[8 * lane + k] = (p2 >= 0 && r > 0) ? sh.in[p2 + r - 1] : 0;
      }
      if (lane == 0) {
        sh.scratch[36] = p2;
        if (p3 < 0 || p2 < 0) sh.flag = 1;
      }
    }
    __syncthreads();
    const int p2 = sh.scratch[36];
    if (sh.flag) {
      if (tid == 0) atomicExch(error_flag, 2);
      __syncthreads();
      continue;
    }
    // ---- all threads: bm1 (2048 flags) -> bm0 (2048 B); thread t owns bm0 bytes 4t..4t+3 ----
    const uint32_t f1 = (sh.bm1[tid >> 1] >> (4 * (tid & 1))) & 0xFu;
    int c1;
    int r1 = block_excl_scan(__popc(f1), sh.scratch, &c1);
    const int p1 = p2 - c1;  // RE1 bytes
    if (p1 < 0) {
      if (tid == 0) atomicExch(error_flag, 2);
      __syncthreads();
      continue;
    }
    // fill-forward: byte i = RE1 byte (rank(i) - 1), rank inclusive; rank 0 -> 0
    uint32_t bits = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      r1 += (f1 >> k) & 1u;
      bits |= (uint32_t)(r1 > 0 ? sh.in[p1 + r1 - 1] : 0) << (8 * k);
    }
    // bits = this thread's 32 zero-elimination flags (bytes b0 .. b0+31)
    int nz;
    int rank = block_excl_scan(__popc(bits), sh.scratch, &nz);
    if (b0 < osize) {
      uint32_t w[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        uint32_t v = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int bit = q * 4 + j;
          if ((bits >> bit) & 1u) v |= (uint32_t)sh.in[rank] << (8 * j);
          rank += (bits >> bit) & 1u;
        }
        w[q] = v;
      }
      uint2* d2 = reinterpret_cast<uint2*>(dst + b0);
      const int nq = min(4, (osize - b0) >> 3);
      for (int q = 0; q < nq; ++q) d2[q] = make_uint2(w[2 * q], w[2 * q + 1]);
    }
    if (nz > p1 && tid == 0) atomicExch(error_flag, 2);
    __syncthreads();
  }
}

}  // namespace prism_b200
