/* Oracle geometry -- TEST INFRASTRUCTURE ONLY (see prism_oracle.h).
 * Three views of the same field layout, each restated from the reference:
 *   - level-major code order     InterpolationPredictor.cu:969-995, 2070-2085
 *   - device plane placement     bitplane.cu:10-53 (d_comput)
 *   - host plane strides / size  io.hpp:104-132 (h_comput), io.cu:117-127
 */
#include "prism_oracle.h"

static uint64_t cdiv(uint64_t a, uint64_t b) { return (a - 1) / b + 1; }

/* Device plane stride of one level: ((count/8 - 1)/8 + 1) * 8 with C
 * truncating division (bitplane.cu:64-67). */
static int64_t dev_stride(int64_t count) {
  int64_t q = count / 8 - 1;
  return (q / 8 + 1) * 8;
}

void or_geometry(uint32_t nx, uint32_t ny, uint32_t nz, int tsize, or_geom* g) {
  g->nx = nx; g->ny = ny; g->nz = nz;
  g->n = (uint64_t)nx * ny * nz;
  g->ax = (uint32_t)cdiv(nx, 16); g->ay = (uint32_t)cdiv(ny, 16); g->az = (uint32_t)cdiv(nz, 16);
  g->anchors = (uint64_t)g->ax * g->ay * g->az;

  /* pre_compute (InterpolationPredictor.cu:969-995) */
  uint64_t sx = nx, sy = ny, sz = nz;
  for (int level = 0; level <= 4; ++level) {
    g->leaps[level][0] = sx;
    g->leaps[level][1] = sx * sy;
    if (level < 4) {
      sx = (sx + 1) >> 1; sy = (sy + 1) >> 1; sz = (sz + 1) >> 1;
      g->lm_prefix[level] = sx * sy * sz;
    }
  }
  g->lm_prefix[4] = 0;
  {
    uint64_t align = 0;
    for (int i = 2; i >= 0; --i) {
      align += (8 - ((g->lm_prefix[i] - g->lm_prefix[i + 1] + align) % 8)) % 8;
      g->lm_prefix[i] += align;
    }
  }

  /* d_comput (bitplane.cu:32-75) */
  /* counts of the stride-2^(l+1) grids minus the anchors (bitplane.cu:37-48) */
  int64_t pre[5];
  sx = nx; sy = ny; sz = nz;
  for (int level = 0; level < 4; ++level) {
    sx = (sx + 1) >> 1; sy = (sy + 1) >> 1; sz = (sz + 1) >> 1;
    pre[level] = (int64_t)(sx * sy * sz) - (int64_t)g->anchors;
  }
  pre[4] = 0;
  int64_t align = 0;
  for (int i = 2; i >= 0; --i) {
    align += (8 - ((pre[i] - pre[i + 1] + align) % 8)) % 8;
    pre[i] += align;
  }
  align += (8 - (((int64_t)g->n - pre[0] + align) % 8)) % 8;
  for (int i = 0; i < 5; ++i) g->dprefix[i] = pre[i];
  g->align_dev = align;
  g->dstride[3] = dev_stride(pre[2]);
  g->dstride[2] = dev_stride(pre[1] - pre[2]);
  g->dstride[1] = dev_stride(pre[0] - pre[1]);
  g->dstride[0] = dev_stride((int64_t)g->n - pre[0] + align);
  g->daprefix[3] = 0;
  g->daprefix[2] = g->dstride[3] * 32;
  g->daprefix[1] = g->dstride[2] * 32 + g->daprefix[2];
  g->daprefix[0] = g->dstride[1] * 32 + g->daprefix[1];

  /* h_comput (io.hpp:104-132): pads with 8 - x%8, i.e. 1..8 */
  int64_t hp[5];
  {
    int64_t p3 = (int64_t)g->anchors;
    sx = nx; sy = ny; sz = nz;
    for (int level = 0; level < 4; ++level) {
      sx = (sx + 1) >> 1; sy = (sy + 1) >> 1; sz = (sz + 1) >> 1;
      hp[level] = (int64_t)(sx * sy * sz) - p3;
    }
    hp[4] = 0;
  }
  int64_t ha = 0;
  for (int i = 2; i >= 0; --i) {
    ha += 8 - ((hp[i] - hp[i + 1] + ha) % 8);
    hp[i] += ha;
  }
  ha += 8 - (((int64_t)g->n - hp[0] + ha) % 8);
  for (int i = 0; i < 5; ++i) g->hprefix[i] = hp[i];
  g->align_host = ha;
  g->hstride[3] = (hp[2] - hp[3]) >> 3;
  g->hstride[2] = (hp[1] - hp[2]) >> 3;
  g->hstride[1] = (hp[0] - hp[1]) >> 3;
  g->hstride[0] = ((int64_t)g->n - hp[0] + ha) >> 3;
  g->aligned_size = 0;
  for (int l = 0; l < 4; ++l) {
    g->hastride[l] = ((g->hstride[l] + 8 - 1) / 8) * 8; /* io.cu:124 */
    g->aligned_size += (uint64_t)g->hastride[l] * 32;
  }
  g->aligned_len = g->n + (uint64_t)ha;

  /* bitShuffle launch (bitplane.cu:609) and its last block (:202-203) */
  g->sh_grid = (int64_t)((g->aligned_len - g->anchors - 1) / 16384 + 1);
  int64_t tmp = (int64_t)(g->n % 16384);
  g->sh_res = g->align_dev + (tmp == 0 ? 16384 : tmp);

  /* zbpc chunk table (zbpc.cu:176-178) */
  g->chunks = 0;
  for (int l = 0; l < 4; ++l) {
    g->chunks_level[l] = ((g->hastride[l] + 16384 - 1) / 16384) << 5;
    g->chunks += g->chunks_level[l];
  }
  /* trailer (compressor.cu:113): 8 + sizeof(double) + 4*32*8 + anchors */
  g->header_size = 8 + 8 + 4 * 32 * 8 + g->anchors * (uint64_t)tsize;
}

/* Level-major position of a grid point (InterpolationPredictor.cu:2070-2085). */
uint64_t or_level_major_index(const or_geom* g, uint64_t gx, uint64_t gy, uint64_t gz) {
  int level = 0;
  while (gx % 2 == 0 && gy % 2 == 0 && gz % 2 == 0 && level < 4) {
    gx >>= 1; gy >>= 1; gz >>= 1; level++;
  }
  uint64_t gid = gx + gy * g->leaps[level][0] + gz * g->leaps[level][1];
  if (level < 4) {
    gid += g->lm_prefix[level] - ((gz + 1) >> 1) * g->leaps[level + 1][1] -
           (uint64_t)(gz % 2 == 0) * ((gy + 1) >> 1) * g->leaps[level + 1][0] -
           (uint64_t)(gz % 2 == 0 && gy % 2 == 0) * ((gx + 1) >> 1);
  }
  return gid;
}
