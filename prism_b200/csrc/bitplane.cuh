// Bit-plane shuffle: level-major int32 codes <-> 32 precision-ordered planes
// per level, bit-exact with bitplane.cu.
//
// Layout (derived from the reference's 8-lane shuffle network, bitplane.cu:
// 112-154, and checked against a lane-exact emulation of it): for level l and
// code index c in that level's segment, let g = c/8, k = c%8 and w the code
// after the sign transform (SM: a -> (a & 0x7fffffff) ^ (a >> 31); NB:
// a -> (a + 0xaaaaaaaa) ^ 0xaaaaaaaa).  Then bit 7-k of byte
// planes[daprefix[l] + p*dstride[l] + g] is bit 31-p of w.
//
// B200 mapping: one warp handles 1024 consecutive codes of one level; lane l
// owns codes 32l..32l+31, i.e. the 4-byte word at byte 4l of every plane row
// of the item.  The codes pass through a padded shared-memory tile (so that
// global accesses stay coalesced 128-byte rows) and each lane turns its 32
// codes into its 32 plane words with one in-register 32x32 bit transpose
// (about 8 instructions per code instead of a shuffle network per code).
// The inverse runs the same transpose backwards; the progressive inverse
// leaves the words of planes outside [begin, end) of each level at zero.
#pragma once
#include "geometry.h"

namespace prism_b200 {

constexpr int kShufWarps = 8;     // warps per CTA
constexpr int kShufCodes = 1024;  // codes per warp work item (128 bytes per plane)

__device__ __forceinline__ uint32_t sign_transform(int32_t code, bool nb) {
  uint32_t a = (uint32_t)code;
  if (nb) return (a + 0xaaaaaaaau) ^ 0xaaaaaaaau;
  return (a & 0x7fffffffu) ^ (uint32_t)(code >> 31);
}

__device__ __forceinline__ int32_t sign_inverse(uint32_t a, bool nb) {
  if (nb) return (int32_t)((a ^ 0xaaaaaaaau) - 0xaaaaaaaau);
  return (int32_t)((a & 0x7fffffffu) ^ (uint32_t)((int32_t)a >> 31));
}

// In-register 32x32 bit transpose: afterwards a[i] bit b = (before) a[b] bit i.
// Recursive block swap over rounds j = 16, 8, 4, 2, 1: rows r and r + j
// exchange their off-diagonal j-bit blocks (byte permutes for j = 16 and 8,
// shift + select for the rest).
template <int J>
__device__ __forceinline__ void bit_swap_round(uint32_t (&a)[32], uint32_t m) {
#pragma unroll
  for (int r = 0; r < 32; ++r) {
    if (r & J) continue;
    const uint32_t x = a[r], y = a[r + J];
    a[r] = (x & m) | ((y << J) & ~m);
    a[r + J] = ((x >> J) & m) | (y & ~m);
  }
}
__device__ __forceinline__ void bit_transpose32(uint32_t (&a)[32]) {
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    const uint32_t x = a[r], y = a[r + 16];
    a[r] = __byte_perm(x, y, 0x5410);
    a[r + 16] = __byte_perm(x, y, 0x7632);
  }
#pragma unroll
  for (int r = 0; r < 32; ++r) {
    if (r & 8) continue;
    const uint32_t x = a[r], y = a[r + 8];
    a[r] = __byte_perm(x, y, 0x6240);
    a[r + 8] = __byte_perm(x, y, 0x7351);
  }
  bit_swap_round<4>(a, 0x0F0F0F0Fu);
  bit_swap_round<2>(a, 0x33333333u);
  bit_swap_round<1>(a, 0x55555555u);
}
// Bit k of a plane word as loaded (little-endian) belongs to code
// sigma(k) = 8 (k / 8) + 7 - k % 8 of the word's 32 codes (bytes in memory
// order, most significant bit first).
__device__ __forceinline__ constexpr int plane_bit_code(int k) { return 8 * (k >> 3) + 7 - (k & 7); }

// 8x8 bit transposes of the four byte columns of eight words at once (delta
// swaps of 4-, 2- and 1-bit blocks between rows i and i + s): afterwards
// byte c of w[j] bit i = (before) w[i] bit 8c + j.
__device__ __forceinline__ void bit_transpose8x4(uint32_t (&w)[8]) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t t = ((w[i] >> 4) ^ w[i + 4]) & 0x0F0F0F0Fu;
    w[i + 4] ^= t;
    w[i] ^= t << 4;
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if (i & 2) continue;
    const uint32_t t = ((w[i] >> 2) ^ w[i + 2]) & 0x33333333u;
    w[i + 2] ^= t;
    w[i] ^= t << 2;
  }
#pragma unroll
  for (int i = 0; i < 8; i += 2) {
    const uint32_t t = ((w[i] >> 1) ^ w[i + 1]) & 0x55555555u;
    w[i + 1] ^= t;
    w[i] ^= t << 1;
  }
}


// a[i] of a 4-entry array held in kernel parameters, without the local-memory
// copy a dynamic index would force
__device__ __forceinline__ int64_t pick4(const int64_t (&a)[4], int i) {
  return i == 0 ? a[0] : (i == 1 ? a[1] : (i == 2 ? a[2] : a[3]));
}

// Work decomposition: per level a run of kShufCodes-code items.
struct ShufPlan {
  int64_t seg_start[4];   // device code index where the level starts
  int64_t proc[4];        // codes of the level that get real planes
  int64_t item_prefix[5]; // first work item of each level (level 3 first)
  int64_t items;
};

inline ShufPlan make_shuf_plan(const Geometry& g, int64_t limit) {
  ShufPlan s;
  int64_t start[4] = {g.dprefix[0], g.dprefix[1], g.dprefix[2], 0};
  int64_t end[4] = {(int64_t)g.n + g.align_dev, g.dprefix[0], g.dprefix[1], g.dprefix[2]};
  int64_t acc = 0;
  for (int k = 0; k < 4; ++k) {
    int l = 3 - k;
    s.seg_start[l] = start[l];
    int64_t e = end[l] < limit ? end[l] : limit;
    s.proc[l] = e > start[l] ? e - start[l] : 0;
    s.item_prefix[k] = acc;
    acc += (s.proc[l] + kShufCodes - 1) / kShufCodes;
  }
  s.item_prefix[4] = acc;
  s.items = acc;
  return s;
}

__device__ __forceinline__ void locate_item(const ShufPlan& s, int64_t item, int* level, int64_t* local) {
  int k = 0;
  if (item >= s.item_prefix[1]) k = 1;
  if (item >= s.item_prefix[2]) k = 2;
  if (item >= s.item_prefix[3]) k = 3;
  *level = 3 - k;
  *local = item - (k == 0 ? s.item_prefix[0] : (k == 1 ? s.item_prefix[1] : (k == 2 ? s.item_prefix[2] : s.item_prefix[3])));
}

// codes (qc + anchors, device code space) -> planes.  A warp takes 1024
// consecutive codes of one level: 32 coalesced 128-byte loads into a padded
// shared-memory tile, from which lane l takes its 32 consecutive codes
// 32l..32l+31 (in plane-bit order), one in-register 32x32 bit transpose, and
// each plane's word of lane l is its 4 bytes of the plane row: one
// contiguous 128-byte warp store per plane.
// One warp work item of the forward shuffle (tw: the warp's staging tile).
__device__ __forceinline__ void shuffle_item(uint32_t (&tw)[32][33], const int32_t* __restrict__ codes,
                                             uint8_t* __restrict__ planes, const Geometry& g, const ShufPlan& plan,
                                             int nb, int64_t item) {
  const int lane = threadIdx.x & 31;
  int level;
  int64_t local;
  locate_item(plan, item, &level, &local);
  const int64_t first = local * kShufCodes;  // within the level
  int64_t count = pick4(plan.proc, level) - first;
  if (count > kShufCodes) count = kShufCodes;
  const int32_t* src = codes + pick4(plan.seg_start, level) + first;
  // tw[it][j] = transformed code 32 it + j (0 past the end: sign_transform(0)
  // = 0); all 32 loads are issued before the first store
  {
    int32_t c[32];
#pragma unroll
    for (int it = 0; it < 32; ++it) {
      const int idx = it * 32 + lane;
      c[it] = idx < count ? __ldg(src + idx) : 0;
    }
#pragma unroll
    for (int it = 0; it < 32; ++it) tw[it][lane] = sign_transform(c[it], nb);
  }
  __syncwarp();
  uint32_t a[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) a[k] = tw[lane][plane_bit_code(k)];
  __syncwarp();  // the tile is free for the warp's next item
  bit_transpose32(a);
  // a[r] = the lane's word of plane 31 - r
  const int nbytes = (int)(count / 8);
  const int64_t stride = pick4(g.dstride, level);
  uint8_t* base = planes + pick4(g.daprefix, level) + first / 8;
  if (count == kShufCodes) {  // every item but a level's last: one word per lane and plane
#pragma unroll
    for (int r = 0; r < 32; ++r) reinterpret_cast<uint32_t*>(base + (int64_t)(31 - r) * stride)[lane] = a[r];
    return;
  }
#pragma unroll
  for (int r = 0; r < 32; ++r) {
    uint8_t* dst = base + (int64_t)(31 - r) * stride;
    const uint32_t w = a[r];
    if (4 * lane + 4 <= nbytes) {
      reinterpret_cast<uint32_t*>(dst)[lane] = w;
    } else if (4 * lane < nbytes) {
      for (int b = 4 * lane; b < nbytes; ++b) dst[b] = (uint8_t)(w >> (8 * (b & 3)));
    }
  }
}

__global__ void __launch_bounds__(kShufWarps * 32)
bitshuffle_kernel(const int32_t* __restrict__ codes, uint8_t* __restrict__ planes, Geometry g,
                  ShufPlan plan, int nb) {
  __shared__ uint32_t tile[kShufWarps][32][33];
  int64_t item = (int64_t)blockIdx.x * kShufWarps + (threadIdx.x >> 5);
  if (item >= plan.items) return;
  shuffle_item(tile[threadIdx.x >> 5], codes, planes, g, plan, nb, item);
}

// planes -> codes; begin/end (device, may be null) restrict each level to
// planes [begin[3-l], end[3-l]) exactly as the progressive inverse does.
// Rows of planes outside that range are never read.
__global__ void __launch_bounds__(kShufWarps * 32, 4)
inverse_bitshuffle_kernel(const uint8_t* __restrict__ planes, int32_t* __restrict__ codes, Geometry g,
                          ShufPlan plan, int nb, const int* __restrict__ begin, const int* __restrict__ end) {
  __shared__ __align__(16) uint32_t tile[kShufWarps][32][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t item = (int64_t)blockIdx.x * kShufWarps + warp;
  if (item >= plan.items) return;
  int level;
  int64_t local;
  locate_item(plan, item, &level, &local);
  const int64_t first = local * kShufCodes;
  int64_t count = pick4(plan.proc, level) - first;
  if (count > kShufCodes) count = kShufCodes;
  int lo = 0, hi = 32;
  if (begin) { lo = begin[3 - level]; hi = end[3 - level]; }
  int32_t* dst = codes + pick4(plan.seg_start, level) + first;
  if (lo >= hi) {  // no plane of this level selected: every code is 0 in both encodings
    for (int idx = lane; idx < count; idx += 32) dst[idx] = 0;
    return;
  }
  const int nbytes = (int)(count / 8);
  const int64_t stride = pick4(g.dstride, level);
  const uint8_t* base = planes + pick4(g.daprefix, level) + first / 8;
  uint32_t (&tw)[32][33] = tile[warp];
  const bool full = count == kShufCodes;
  // a[k] = transformed code 32 lane + plane_bit_code(k) (code bit b from
  // plane 31 - b, bit k of the lane's word)
  uint32_t a[32];
  if (full && hi - lo <= 8) {
    // At most eight planes (a refinement step): they lie in the eight code
    // bits r0..r0+7, w[i] = the lane's word of plane 31 - r0 - i, and one
    // 8x8 transpose per byte column gives every code's byte.
    const int r0 = min(32 - hi, 24);
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int p = 31 - r0 - i;
      w[i] = (p >= lo && p < hi) ? __ldg(reinterpret_cast<const uint32_t*>(base + (int64_t)p * stride) + lane) : 0u;
    }
    bit_transpose8x4(w);
#pragma unroll
    for (int k = 0; k < 32; ++k) a[k] = __byte_perm(w[k & 7], 0u, 0x4440 | (k >> 3)) << r0;
  } else {
    // a[r] = the lane's word (as loaded) of plane 31 - r
    if (full) {  // every item but a level's last: one word per lane and plane
#pragma unroll
      for (int r = 0; r < 32; ++r) {
        const int p = 31 - r;
        a[r] = (p >= lo && p < hi) ? __ldg(reinterpret_cast<const uint32_t*>(base + (int64_t)p * stride) + lane) : 0u;
      }
    } else {
#pragma unroll
      for (int r = 0; r < 32; ++r) {
        const int p = 31 - r;
        const uint8_t* src = base + (int64_t)p * stride;
        uint32_t v = 0;
        if (p >= lo && p < hi) {
          if (4 * lane + 4 <= nbytes) {
            v = __ldg(reinterpret_cast<const uint32_t*>(src) + lane);
          } else if (4 * lane < nbytes) {
            for (int b = 4 * lane; b < nbytes; ++b) v |= (uint32_t)src[b] << (8 * (b & 3));
          }
        }
        a[r] = v;
      }
    }
    bit_transpose32(a);
  }
  if (full && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
    // Out through the tile in 16-byte pieces: row l holds lane l's codes
    // 32l..32l+31, its four-code block q at block q ^ (l mod 8) (each
    // quarter-warp touches eight distinct bank groups on both sides), and
    // each warp store writes 512 consecutive bytes.
    uint32_t* tv = &tw[0][0];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      uint4 v;
      v.x = (uint32_t)sign_inverse(a[plane_bit_code(4 * q)], nb);
      v.y = (uint32_t)sign_inverse(a[plane_bit_code(4 * q + 1)], nb);
      v.z = (uint32_t)sign_inverse(a[plane_bit_code(4 * q + 2)], nb);
      v.w = (uint32_t)sign_inverse(a[plane_bit_code(4 * q + 3)], nb);
      *reinterpret_cast<uint4*>(tv + 32 * lane + 4 * (q ^ (lane & 7))) = v;
    }
    __syncwarp();
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      const int row = 4 * s + (lane >> 3);
      reinterpret_cast<uint4*>(dst)[32 * s + lane] =
          *reinterpret_cast<const uint4*>(tv + 32 * row + 4 * ((lane & 7) ^ (row & 7)));
    }
    return;
  }
  // out through the padded tile, so that the codes leave in coalesced rows
#pragma unroll
  for (int k = 0; k < 32; ++k) tw[lane][plane_bit_code(k)] = a[k];
  __syncwarp();
#pragma unroll 8
  for (int it = 0; it < 32; ++it) {
    const int idx = it * 32 + lane;
    if (idx < count) dst[idx] = sign_inverse(tw[it][lane], nb);
  }
}

// ---- the reference's last shuffle block, reproduced thread by thread ----
//
// In bitplane.cu the element count of the last block is res = align + tail,
// but `align` is a local that d_comput only updates in thread 0
// (bitplane.cu:32-57, 90-91), so thread 0 uses align + tail and every other
// thread uses tail (= n % 16384, or 16384).  The block iterates in rounds of
// 512 codes; a round's writer t stores the transposed word of position
// 8*(t&63) + (t>>6) when that index (not the position) is below its own res
// (`write_pos < res`, :246), which writes zero words past the data and skips
// some real ones.  Lanes outside the active set read 0 from their partners in
// the 8-lane network (their register holds the 0 they were initialised with).
// These kernels run that logic with CTAs of 512 threads (one 512-code round
// each, or all rounds in order in one CTA where rounds overlap) and an
// explicit shared-memory emulation of the shuffle network, so the outcome is
// fixed.

__device__ __forceinline__ uint32_t bperm(uint32_t x, uint32_t y, uint32_t s) { return __byte_perm(x, y, s); }

// one xor-shuffle/byte_perm step of the 8-lane network (bitplane.cu:112-124)
__device__ __forceinline__ uint32_t net_step(uint32_t a, uint32_t q, int lane8, int step) {
  if (step == 0) return (lane8 & 4) == 0 ? bperm(a, q, 0x3276) : bperm(a, q, 0x5410);
  if (step == 1) return (lane8 & 2) == 0 ? bperm(a, q, 0x3715) : bperm(a, q, 0x6240);
  const uint32_t mask = 0x0F0F0F0Fu;
  return (lane8 & 1) == 0 ? ((a & ~mask) | ((q >> 4) & mask)) : (((q << 4) & ~mask) | (a & mask));
}
__device__ __forceinline__ uint32_t bits_fwd(uint32_t a) {
  uint32_t q;
  q = (a ^ (a >> 3)) & 0x0A0A0A0AU; a = a ^ q ^ (q << 3);
  q = (a ^ (a >> 6)) & 0x00CC00CCU; a = a ^ q ^ (q << 6);
  q = (a ^ (a >> 12)) & 0x0000F0F0U; a = a ^ q ^ (q << 12);
  return a;
}
__device__ __forceinline__ uint32_t bits_inv(uint32_t a) {
  uint32_t q;
  q = (a ^ (a >> 12)) & 0x0000F0F0U; a = a ^ q ^ (q << 12);
  q = (a ^ (a >> 6)) & 0x00CC00CCU; a = a ^ q ^ (q << 6);
  q = (a ^ (a >> 3)) & 0x0A0A0A0AU; a = a ^ q ^ (q << 3);
  return a;
}

__device__ __forceinline__ int64_t last_res_of(const Geometry& g, int t) {
  int64_t tail = (int64_t)(g.n % kChunk);
  if (tail == 0) tail = kChunk;
  return tail + (t == 0 ? g.align_dev : 0);
}

// device position -> byte of plane 4*(c&7) (bitplane.cu:143-149)
__device__ __forceinline__ int64_t place_dev(const Geometry& g, int64_t c, int64_t* stride) {
  int level = 0;
  while (level < 3 && c < g.dprefix[level]) ++level;
  int64_t idx = c - g.dprefix[level];
  *stride = g.dstride[level];
  return (idx >> 3) + g.dstride[level] * ((idx & 7) << 2) + g.daprefix[level];
}

__device__ __forceinline__ void shuffle_last_block(const int32_t* __restrict__ codes, uint8_t* __restrict__ planes,
                                                   const Geometry& g, int nb, uint64_t limit, int cta, int ncta) {
  __shared__ uint32_t a[512];
  __shared__ uint32_t shm[512];
  __shared__ unsigned char act[512];
  const int t = threadIdx.x;
  const int64_t start = (g.sh_grid - 1) * (int64_t)kChunk;
  const int64_t res = last_res_of(g, t);
  const int64_t ares = (res + 511) / 512 * 512;
  const int64_t maxa = (last_res_of(g, 0) + 511) / 512 * 512;
  shm[t] = 0;
  // a round only reads words its own round wrote; whether rounds may run in
  // parallel is decided by the launch (shuffle_last_block_grid)
  for (int64_t base = (int64_t)cta * 512; base < maxa; base += (int64_t)ncta * 512) {
    bool part = base < ares;
    bool ac = part && base + t < res;
    act[t] = ac;
    a[t] = ac ? sign_transform(codes[start + base + t], nb) : 0u;
    __syncthreads();
    for (int step = 0; step < 3; ++step) {
      int partner = t ^ (4 >> step);
      uint32_t q = act[partner] ? a[partner] : 0u;
      uint32_t v = ac ? net_step(a[t], q, t & 7, step) : 0u;
      __syncthreads();
      a[t] = v;
      __syncthreads();
    }
    if (part) shm[t] = ac ? bits_fwd(a[t]) : 0u;
    __syncthreads();
    int wp = ((t & 63) << 3) + (t >> 6);
    if (part && wp < res) {
      uint32_t w = shm[wp];
      int64_t st;
      int64_t s = place_dev(g, start + base + wp, &st);
      uint8_t b[4] = {(uint8_t)(w >> 24), (uint8_t)(w >> 8), (uint8_t)(w >> 16), (uint8_t)w};
      for (int j = 0; j < 4; ++j) {
        uint64_t o = (uint64_t)(s + j * st);
        if (o < limit) planes[o] = b[j];
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(512)
shuffle_last_block_kernel(const int32_t* __restrict__ codes, uint8_t* __restrict__ planes, Geometry g,
                          int nb, uint64_t limit) {
  shuffle_last_block(codes, planes, g, nb, limit, blockIdx.x, gridDim.x);
}

// inverse of the last block (bitplane.cu:400-450 and :532-600): thread t
// decodes positions t, t+512, ... below its own res; lanes that left the loop
// supply 0 to the network.  begin/end (device, may be null) mask planes.
__global__ void __launch_bounds__(512)
inverse_last_block_kernel(const uint8_t* __restrict__ planes, int32_t* __restrict__ codes, Geometry g, int nb,
                          const int* __restrict__ begin, const int* __restrict__ end, uint64_t limit) {
  __shared__ uint32_t a[512];
  __shared__ unsigned char act[512];
  const int t = threadIdx.x;
  const int64_t start = (g.sh_grid - 1) * (int64_t)kChunk;
  const int64_t res = last_res_of(g, t);
  const int64_t maxr = last_res_of(g, 0);
  for (int64_t base = (int64_t)blockIdx.x * 512; base < maxr; base += (int64_t)gridDim.x * 512) {
    int64_t c = start + base + t;
    bool ac = base + t < res;
    uint32_t v = 0;
    if (ac) {
      int level = 0;
      while (level < 3 && c < g.dprefix[level]) ++level;
      int64_t st;
      int64_t s = place_dev(g, c, &st);
      int lane = (int)(((c - g.dprefix[level]) & 7) << 2);
      int lo = 0, hi = 32;
      if (begin) { lo = begin[3 - level]; hi = end[3 - level]; }
      if (lo < hi) {
        const int sh[4] = {24, 8, 16, 0};
        for (int j = 0; j < 4; ++j) {
          uint64_t o = (uint64_t)(s + j * st);
          if (lane + j >= lo && lane + j < hi && o < limit) v |= (uint32_t)planes[o] << sh[j];
        }
      }
      v = bits_inv(v);
    }
    act[t] = ac;
    a[t] = v;
    __syncthreads();
    for (int step = 0; step < 3; ++step) {
      int partner = t ^ (4 >> step);
      uint32_t q = act[partner] ? a[partner] : 0u;
      uint32_t nv = ac ? net_step(a[t], q, t & 7, step) : 0u;
      __syncthreads();
      a[t] = nv;
      __syncthreads();
    }
    if (ac) codes[c] = sign_inverse(a[t], nb);
    __syncthreads();
  }
}

// The plane buffer starts out holding the predictor's linear int32 codes (the
// reference reuses that buffer, compressor.cu:328); bytes the shuffle never
// overwrites keep them.  Byte b holds byte b%4 of the code of grid point b/4
// (0 for anchors and past n).  This fills the ranges the bulk shuffle does not
// write; the last-block kernel then overwrites what it writes.
struct ByteRange { uint64_t start, len; };
// at most 32 planes x 4 levels + the tail, passed by value (kernel parameter
// space) so that no host-to-device copy precedes the launch
constexpr int kMaxRanges = 160;
struct RangeList {
  ByteRange r[kMaxRanges];
};

__global__ void leftover_fill_kernel(uint8_t* __restrict__ planes, const int32_t* __restrict__ qc, Geometry g,
                                     const RangeList ranges, int nranges) {
  for (int r = blockIdx.x; r < nranges; r += gridDim.x) {
    ByteRange br = ranges.r[r];
    for (uint64_t o = threadIdx.x; o < br.len; o += blockDim.x) {
      uint64_t b = br.start + o;
      uint64_t i = b >> 2;
      uint8_t v = 0;
      if (i < g.n) {
        uint64_t x = i % g.nx, y = (i / g.nx) % g.ny, z = i / ((uint64_t)g.nx * g.ny);
        if ((x & 15) | (y & 15) | (z & 15)) {
          uint32_t code = (uint32_t)qc[level_major_index(g, x, y, z)];
          v = (uint8_t)(code >> (8 * (b & 3)));
        }
      }
      planes[b] = v;
    }
  }
}

// Byte ranges of the plane buffer the bulk shuffle (positions before the
// last block) does not write: per plane, from the first group the bulk kernel
// leaves to the stride end, and the tail past the device placement.
inline int fill_ranges(const Geometry& g, const ShufPlan& plan, ByteRange* out, int cap) {
  int cnt = 0;
  for (int l = 3; l >= 0; --l) {
    int64_t from = plan.proc[l] / 8;
    if (from >= g.dstride[l]) continue;
    for (int p = 0; p < 32 && cnt < cap; ++p) {
      int64_t base = g.daprefix[l] + (int64_t)p * g.dstride[l];
      out[cnt++] = ByteRange{(uint64_t)(base + from), (uint64_t)(g.dstride[l] - from)};
    }
  }
  if ((uint64_t)g.dev_total < g.aligned_size && cnt < cap)
    out[cnt++] = ByteRange{(uint64_t)g.dev_total, g.aligned_size - (uint64_t)g.dev_total};
  return cnt;
}

// Whether the reference's last block writes after the others where they
// overlap (see the oracle): with more blocks than a B200 holds at once
// (148 SMs x 4 CTAs of 512 threads) it starts after the first wave finished;
// otherwise the loop round of each side decides.
// CTAs for the last-block kernels: one per 512-code round
inline int last_block_rounds(const Geometry& g) {
  int64_t tail = (int64_t)(g.n % kChunk);
  if (tail == 0) tail = kChunk;
  return (int)((tail + g.align_dev + 511) / 512);
}

// The forward last block's rounds may run concurrently only when no two of
// them can write the same byte.  Zero words written past the data spill into
// the first bytes of the next plane; that byte range is also written by the
// block's own real codes when the block reaches back to within 1024 codes of
// a level start.  Then the rounds run in order in one CTA, as in the
// reference, and the later round's byte stands.
inline int shuffle_last_block_grid(const Geometry& g) {
  const int64_t start = (g.sh_grid - 1) * (int64_t)kChunk;
  return start >= g.dprefix[0] + 1024 ? last_block_rounds(g) : 1;
}

inline bool last_block_lands_last(const Geometry& g) {
  if (g.sh_grid > 148 * 4) return true;
  int64_t tail = (int64_t)(g.n % kChunk);
  if (tail == 0) tail = kChunk;
  int64_t it_last = (tail + 511) / 512 - 1;
  int64_t it_first = (g.dprefix[0] % kChunk) / 512;
  return it_first <= it_last;
}

}  // namespace prism_b200
