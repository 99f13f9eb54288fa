// Field / code / bit-plane geometry shared by host and device code.
//
// One PRISM field of nx*ny*nz values (x fastest) is cut into 16^3 tiles.  The
// stride-16 grid points are the anchors; every other point belongs to one of
// four interpolation levels (level 3 = stride 8 ... level 0 = stride 1).  Three
// layouts are derived from the dimensions alone and all three are part of the
// PRISM container format:
//
//  * level-major code order (InterpolationPredictor.cu:969-995, 2070-2085):
//    anchors first, then level 3, 2, 1, 0; each level segment padded to a
//    multiple of 8 codes;
//  * device bit-plane placement (bitplane.cu:10-53): code index space without
//    the anchors, 32 planes per level, plane stride rounded up to 8 bytes, the
//    level-0 segment sized from n (not n - anchors);
//  * host plane strides (io.hpp:104-132, io.cu:117-127): pads every level with
//    1..8 codes instead of 0..7 and defines the 16 KiB chunk table of the
//    lossless stream and the plane-buffer size.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define PRISM_HD __host__ __device__ __forceinline__
#else
#define PRISM_HD inline
#endif

namespace prism_b200 {

constexpr int kChunk = 16384;  // lossless chunk size in bytes
constexpr int kTile = 16;      // predictor tile edge
constexpr int kLevels = 4;

struct Geometry {
  uint32_t nx, ny, nz;
  uint64_t n;
  uint32_t ax, ay, az;  // anchor grid
  uint64_t anchors;
  uint64_t grid[4];      // points of the stride-2, 4, 8, 16 grids
  // level-major order
  uint64_t leaps[5][2];  // grid extent in x and x*y at each level
  uint64_t lm_prefix[5]; // first level-major slot of each level (incl. anchors)
  // device plane placement (code space excludes anchors)
  int64_t dprefix[5];    // code index where level l+1 ends / level l starts
  int64_t align_dev;
  int64_t dstride[4];    // bytes per plane
  int64_t daprefix[4];   // byte offset of each level's 32 planes
  int64_t dev_total;     // bytes covered by the device placement
  // host strides / container chunking
  int64_t align_host;
  int64_t hstride[4];
  int64_t hastride[4];   // x8
  uint64_t aligned_size; // plane buffer bytes = sum 32 * hastride
  uint64_t aligned_len;  // n + align_host
  // the reference shuffle launch (bitplane.cu:609) and its last block
  int64_t sh_grid;
  int64_t sh_res;
  int64_t chunks_level[4];
  int64_t chunks;
  uint64_t header_size;  // container trailer bytes
  int tsize;
};

PRISM_HD uint64_t cdiv_u64(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// Device plane stride of a level holding `count` codes: ((count/8-1)/8+1)*8
// with C truncating division (bitplane.cu:64-67).
PRISM_HD int64_t device_stride(int64_t count) {
  int64_t q = count / 8 - 1;
  return (q / 8 + 1) * 8;
}

inline void make_geometry(uint32_t nx, uint32_t ny, uint32_t nz, int tsize, Geometry* g) {
  g->nx = nx; g->ny = ny; g->nz = nz;
  g->tsize = tsize;
  g->n = (uint64_t)nx * ny * nz;
  g->ax = (uint32_t)cdiv_u64(nx, 16);
  g->ay = (uint32_t)cdiv_u64(ny, 16);
  g->az = (uint32_t)cdiv_u64(nz, 16);
  g->anchors = (uint64_t)g->ax * g->ay * g->az;

  uint64_t grid[4];
  uint64_t sx = nx, sy = ny, sz = nz;
  for (int level = 0; level <= 4; ++level) {
    g->leaps[level][0] = sx;
    g->leaps[level][1] = sx * sy;
    if (level < 4) {
      sx = (sx + 1) >> 1; sy = (sy + 1) >> 1; sz = (sz + 1) >> 1;
      grid[level] = sx * sy * sz;  // points of the stride-2^(level+1) grid
    }
  }
  for (int l = 0; l < 4; ++l) g->grid[l] = grid[l];
  // level-major slots: pad levels 3..1 to x8
  for (int l = 0; l < 4; ++l) g->lm_prefix[l] = grid[l];
  g->lm_prefix[4] = 0;
  uint64_t al = 0;
  for (int i = 2; i >= 0; --i) {
    al += (8 - ((g->lm_prefix[i] - g->lm_prefix[i + 1] + al) % 8)) % 8;
    g->lm_prefix[i] += al;
  }

  // device placement
  int64_t pre[5];
  for (int l = 0; l < 4; ++l) pre[l] = (int64_t)grid[l] - (int64_t)g->anchors;
  pre[4] = 0;
  int64_t align = 0;
  for (int i = 2; i >= 0; --i) {
    align += (8 - ((pre[i] - pre[i + 1] + align) % 8)) % 8;
    pre[i] += align;
  }
  align += (8 - (((int64_t)g->n - pre[0] + align) % 8)) % 8;
  for (int i = 0; i < 5; ++i) g->dprefix[i] = pre[i];
  g->align_dev = align;
  g->dstride[3] = device_stride(pre[2]);
  g->dstride[2] = device_stride(pre[1] - pre[2]);
  g->dstride[1] = device_stride(pre[0] - pre[1]);
  g->dstride[0] = device_stride((int64_t)g->n - pre[0] + align);
  g->daprefix[3] = 0;
  g->daprefix[2] = g->dstride[3] * 32;
  g->daprefix[1] = g->dstride[2] * 32 + g->daprefix[2];
  g->daprefix[0] = g->dstride[1] * 32 + g->daprefix[1];
  g->dev_total = g->daprefix[0] + 32 * g->dstride[0];

  // host strides (pads 1..8 codes per level)
  int64_t hp[5];
  for (int l = 0; l < 4; ++l) hp[l] = (int64_t)grid[l] - (int64_t)g->anchors;
  hp[4] = 0;
  int64_t ha = 0;
  for (int i = 2; i >= 0; --i) {
    ha += 8 - ((hp[i] - hp[i + 1] + ha) % 8);
    hp[i] += ha;
  }
  ha += 8 - (((int64_t)g->n - hp[0] + ha) % 8);
  g->align_host = ha;
  g->hstride[3] = (hp[2] - hp[3]) >> 3;
  g->hstride[2] = (hp[1] - hp[2]) >> 3;
  g->hstride[1] = (hp[0] - hp[1]) >> 3;
  g->hstride[0] = ((int64_t)g->n - hp[0] + ha) >> 3;
  g->aligned_size = 0;
  g->chunks = 0;
  for (int l = 0; l < 4; ++l) {
    g->hastride[l] = ((g->hstride[l] + 7) / 8) * 8;
    g->aligned_size += (uint64_t)g->hastride[l] * 32;
    g->chunks_level[l] = ((g->hastride[l] + kChunk - 1) / kChunk) * 32;
    g->chunks += g->chunks_level[l];
  }
  g->aligned_len = g->n + (uint64_t)ha;
  g->sh_grid = (int64_t)((g->aligned_len - g->anchors - 1) / kChunk + 1);
  int64_t tmp = (int64_t)(g->n % kChunk);
  g->sh_res = g->align_dev + (tmp == 0 ? kChunk : tmp);
  g->header_size = 8 + 8 + 4 * 32 * 8 + g->anchors * (uint64_t)tsize;
}

// Level-major slot of grid point (gx, gy, gz) (InterpolationPredictor.cu:2070-2085).
PRISM_HD uint64_t level_major_index(const Geometry& g, uint64_t gx, uint64_t gy, uint64_t gz) {
  int level = 0;
  while (((gx | gy | gz) & 1) == 0 && level < 4) {
    gx >>= 1; gy >>= 1; gz >>= 1; ++level;
  }
  uint64_t gid = gx + gy * g.leaps[level][0] + gz * g.leaps[level][1];
  if (level < 4) {
    gid += g.lm_prefix[level] - ((gz + 1) >> 1) * g.leaps[level + 1][1] -
           (uint64_t)((gz & 1) == 0) * ((gy + 1) >> 1) * g.leaps[level + 1][0] -
           (uint64_t)(((gz | gy) & 1) == 0) * ((gx + 1) >> 1);
  }
  return gid;
}

}  // namespace prism_b200
