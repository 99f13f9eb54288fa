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
// B200 mapping: one warp handles 256 consecutive codes of one level.  Per 32
// codes it loads one coalesced 128-byte row, does a 32x32 bit transpose with
// five xor-shuffle rounds (lane i ends up holding bit i of all 32 codes, i.e.
// plane 31-i), and after 8 rounds each lane stores the 32 bytes of its plane.
// The inverse runs the same transpose backwards; the progressive inverse
// zeroes the lanes of planes outside [begin, end) of each level.
#pragma once
#include "geometry.h"

namespace prism_b200 {

constexpr int kShufWarps = 8;  // warps per CTA
constexpr int kShufCodes = 256;  // codes per warp work item

__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, int lane) {
  const uint32_t masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    int j = 16 >> s;
    uint32_t m = masks[s];
    uint32_t t = __shfl_xor_sync(0xffffffffu, x, j);
    x = (lane & j) ? ((x & ~m) | ((t >> j) & m)) : ((x & m) | ((t & m) << j));
  }
  return x;
}

__device__ __forceinline__ uint32_t sign_transform(int32_t code, bool nb) {
  uint32_t a = (uint32_t)code;
  if (nb) return (a + 0xaaaaaaaau) ^ 0xaaaaaaaau;
  return (a & 0x7fffffffu) ^ (uint32_t)(code >> 31);
}

__device__ __forceinline__ int32_t sign_inverse(uint32_t a, bool nb) {
  if (nb) return (int32_t)((a ^ 0xaaaaaaaau) - 0xaaaaaaaau);
  return (int32_t)((a & 0x7fffffffu) ^ (uint32_t)((int32_t)a >> 31));
}

// plane word (bit k = code k of 32) <-> the 4 plane bytes in memory order
__device__ __forceinline__ uint32_t to_plane_bytes(uint32_t w) { return __byte_perm(__brev(w), 0, 0x0123); }
__device__ __forceinline__ uint32_t from_plane_bytes(uint32_t b) { return __brev(__byte_perm(b, 0, 0x0123)); }

// Work decomposition: per level a run of 256-code items.
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
  while (k < 3 && item >= s.item_prefix[k + 1]) ++k;
  *level = 3 - k;
  *local = item - s.item_prefix[k];
}

// codes (qc + anchors, device code space) -> planes
__global__ void __launch_bounds__(kShufWarps * 32)
bitshuffle_kernel(const int32_t* __restrict__ codes, uint8_t* __restrict__ planes, Geometry g,
                  ShufPlan plan, int nb) {
  const int lane = threadIdx.x & 31;
  int64_t item = (int64_t)blockIdx.x * kShufWarps + (threadIdx.x >> 5);
  if (item >= plan.items) return;
  int level;
  int64_t local;
  locate_item(plan, item, &level, &local);
  int64_t first = local * kShufCodes;  // within the level
  int64_t count = plan.proc[level] - first;
  if (count > kShufCodes) count = kShufCodes;
  const int32_t* src = codes + plan.seg_start[level] + first;
  uint32_t words[8];
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    int idx = it * 32 + lane;
    int32_t c = idx < count ? __ldg(src + idx) : 0;
    uint32_t w = sign_transform(c, nb);
    words[it] = to_plane_bytes(warp_transpose32(w, lane));
  }
  // lane i holds plane 31 - i
  int p = 31 - lane;
  uint8_t* dst = planes + g.daprefix[level] + (int64_t)p * g.dstride[level] + first / 8;
  int nbytes = (int)(count / 8);
  if (nbytes == 32) {
    uint2* d2 = reinterpret_cast<uint2*>(dst);
#pragma unroll
    for (int q = 0; q < 4; ++q) d2[q] = make_uint2(words[2 * q], words[2 * q + 1]);
  } else {
    for (int b = 0; b < nbytes; ++b) dst[b] = (uint8_t)(words[b >> 2] >> (8 * (b & 3)));
  }
}

// planes -> codes; begin/end (device, may be null) restrict each level to
// planes [begin[3-l], end[3-l]) exactly as the progressive inverse does
__global__ void __launch_bounds__(kShufWarps * 32)
inverse_bitshuffle_kernel(const uint8_t* __restrict__ planes, int32_t* __restrict__ codes, Geometry g,
                          ShufPlan plan, int nb, const int* __restrict__ begin, const int* __restrict__ end) {
  const int lane = threadIdx.x & 31;
  int64_t item = (int64_t)blockIdx.x * kShufWarps + (threadIdx.x >> 5);
  if (item >= plan.items) return;
  int level;
  int64_t local;
  locate_item(plan, item, &level, &local);
  int64_t first = local * kShufCodes;
  int64_t count = plan.proc[level] - first;
  if (count > kShufCodes) count = kShufCodes;
  int p = 31 - lane;
  bool take = true;
  if (begin) {
    int lo = begin[3 - level], hi = end[3 - level];
    take = lo < hi && p >= lo && p < hi;
  }
  const uint8_t* src = planes + g.daprefix[level] + (int64_t)p * g.dstride[level] + first / 8;
  int nbytes = (int)(count / 8);
  uint32_t words[8];
  if (take && nbytes == 32) {
    const uint2* s2 = reinterpret_cast<const uint2*>(src);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint2 v = __ldg(s2 + q);
      words[2 * q] = v.x;
      words[2 * q + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int q = 0; q < 8; ++q) words[q] = 0;
    if (take)
      for (int b = 0; b < nbytes; ++b) words[b >> 2] |= (uint32_t)src[b] << (8 * (b & 3));
  }
  int32_t* dst = codes + plan.seg_start[level] + first;
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    uint32_t w = warp_transpose32(from_plane_bytes(words[it]), lane);
    int idx = it * 32 + lane;
    if (idx < count) dst[idx] = sign_inverse(w, nb);
  }
}

// Zero bytes the reference's last shuffle block writes past the processed
// codes (bitplane.cu:243-259: whole 512-code rounds, `write_pos < res`).
// Launched after bitshuffle_kernel so these writes land last, as in the
// reference where that block runs last.  One thread per group of 8 codes.
__global__ void shuffle_zero_tail_kernel(uint8_t* __restrict__ planes, Geometry g, int64_t zfirst,
                                         int64_t zend, uint64_t limit) {
  int64_t grp = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t c = zfirst + grp * 8;
  if (c >= zend) return;
  int level = 0;
  while (level < 3 && c < g.dprefix[level]) ++level;
  int64_t gbyte = (c - g.dprefix[level]) >> 3;
  for (int p = 0; p < 32; ++p) {
    uint64_t s = (uint64_t)(gbyte + g.dstride[level] * p + g.daprefix[level]);
    if (s < limit) planes[s] = 0;
  }
}

// Bytes the reference's shuffle never writes keep the predictor's linear
// int32 scratch (it reuses the plane buffer, compressor.cu:328): byte b is
// byte b%4 of the code of grid point b/4 (0 for anchors and b/4 >= n).
struct ByteRange { uint64_t start, len; };

__global__ void leftover_fill_kernel(uint8_t* __restrict__ planes, const int32_t* __restrict__ qc, Geometry g,
                                     const ByteRange* __restrict__ ranges, int nranges) {
  for (int r = blockIdx.x; r < nranges; r += gridDim.x) {
    ByteRange br = ranges[r];
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

// The byte ranges of [0, aligned_size) that the reference shuffle leaves
// untouched (per-plane slack, codes it never processes, the tail past the
// device placement), excluding the zero-tail bytes.
inline int leftover_ranges(const Geometry& g, const ShuffleSpan& sp, ByteRange* out, int cap) {
  int cnt = 0;
  auto push = [&](int64_t a, int64_t b) {
    if (b > a && cnt < cap) out[cnt++] = ByteRange{(uint64_t)a, (uint64_t)(b - a)};
  };
  int64_t lim_real = sp.processed < sp.end0 ? sp.processed : sp.end0;
  int64_t seg_end[4] = {sp.end0, g.dprefix[0], g.dprefix[1], g.dprefix[2]};
  int64_t seg_start[4] = {g.dprefix[0], g.dprefix[1], g.dprefix[2], 0};
  int64_t z0 = lim_real, z1 = sp.written_end > lim_real ? sp.written_end : lim_real;  // zero tail
  for (int l = 3; l >= 0; --l) {
    int64_t e = seg_end[l] < lim_real ? seg_end[l] : lim_real;
    int64_t groups = e > seg_start[l] ? (e - seg_start[l]) / 8 : 0;
    int64_t from = groups;
    if (l == 0 && z1 > z0) from = (z1 - seg_start[0]) / 8;  // zero tail covers [groups, zg1)
    for (int p = 0; p < 32; ++p) {
      int64_t base = g.daprefix[l] + (int64_t)p * g.dstride[l];
      push(base + from, base + g.dstride[l]);
    }
  }
  int64_t tail_a = g.dev_total, tail_b = (int64_t)g.aligned_size;
  if (z1 > z0) {  // plane 31 of level 0 may spill zeros past the device placement
    int64_t zs = g.daprefix[0] + 31 * g.dstride[0] + (z0 - seg_start[0]) / 8;
    int64_t ze = g.daprefix[0] + 31 * g.dstride[0] + (z1 - seg_start[0]) / 8;
    if (zs < tail_a) zs = tail_a;
    if (ze > zs) { push(tail_a, zs < tail_b ? zs : tail_b); tail_a = ze; }
  }
  push(tail_a, tail_b);
  return cnt;
}

}  // namespace prism_b200
