/* Oracle strategy search -- TEST INFRASTRUCTURE ONLY (see prism_oracle.h).
 * Restates findStrategy_h / findOptimalStrategy / loadall
 * (src/loader/dataloader.cu:13-208) including the exact tie-breaking of the
 * per-thread scan (strict >), the per-block tree reduction over 1024 threads
 * and the grid reduction over 33 blocks (strict <, left operand kept). */
#include <math.h>
#include <string.h>
#include "prism_oracle.h"

/* cost[l][b] = ceil(2^(32-b) * (p^(11-3l) + p^(10-3l) + p^(9-3l))),
 * p = 1 for l = 0 else 1.25 (dataloader.cu:59-69).  The powers are exact
 * dyadic rationals (5^k / 4^k, k <= 11), computed here by repeated exact
 * multiplication. */
static double powk(double p, int k) {
  double r = 1.0;
  for (int i = 0; i < k; ++i) r *= p;
  return r;
}

void or_strategy_costs(uint64_t cost[4][33]) {
  for (int l = 0; l < 4; ++l)
    for (int b = 0; b < 33; ++b) {
      int shift = 32 - b;
      double err = shift == 0 ? 0 : (double)(1ULL << shift);
      double p = l == 0 ? 1.0 : 1.25;
      err *= powk(p, 4 * 3 - l * 3 - 1) + powk(p, 4 * 3 - l * 3 - 2) + powk(p, 4 * 3 - l * 3 - 3);
      cost[l][b] = (uint64_t)ceil(err);
    }
}

void or_find_strategy(const uint64_t cs[128], double eb, double target_error, int begin[4],
                      int end[4], int* maxlevel) {
  *maxlevel = 4; /* resetCounter */
  if (!(target_error * 0.954 >= eb)) { /* loadall (dataloader.cu:21-28) */
    for (int i = 0; i < 4; ++i) begin[i] = end[i];
    for (int i = 0; i < 4; ++i) end[i] = 32;
    *maxlevel = begin[0] < 32 ? 3 : begin[1] < 32 ? 2 : begin[2] < 32 ? 1 : begin[3] < 32 ? 0 : 4;
    return;
  }
  uint64_t target_cost = (uint64_t)floor(target_error * 0.954 / eb) - 1;
  uint64_t cost[4][33], vt[4][33];
  or_strategy_costs(cost);
  for (int i = 3; i >= 0; --i) { /* value table (dataloader.cu:44-57) */
    vt[i][0] = cs[i * 32 + 31];
    vt[i][32] = 0;
    for (int j = 31; j > 0; --j) vt[i][j] = cs[i * 32 + 31] - cs[i * 32 + j - 1];
  }
  static uint64_t maxv[1024];
  static int maxt[1024];
  static int rend[1024][4];
  uint64_t value_blk[65];
  int maxbid[65], target[33][4];
  memset(value_blk, 0, sizeof(value_blk));
  memset(maxbid, 0, sizeof(maxbid));
  for (int b0 = 0; b0 < 33; ++b0) {
    for (int tid = 0; tid < 1024; ++tid) {
      uint64_t best = 0;
      int r[4] = {32, 32, 32, 32};
      for (int pos = tid; pos < 33 * 33 * 33; pos += 1024) {
        int b1 = pos / (33 * 33), b2 = (pos / 33) % 33, b3 = pos % 33;
        uint64_t tc = cost[0][b0] + cost[1][b1] + cost[2][b2] + cost[3][b3];
        if (tc <= target_cost) {
          uint64_t v = vt[0][b0] + vt[1][b1] + vt[2][b2] + vt[3][b3];
          if (v > best) { r[0] = b0; r[1] = b1; r[2] = b2; r[3] = b3; best = v; }
        }
      }
      maxv[tid] = best;
      maxt[tid] = tid;
      memcpy(rend[tid], r, sizeof(r));
    }
    for (int stride = 512; stride > 0; stride >>= 1)
      for (int tid = 0; tid < stride; ++tid)
        if (maxv[tid] < maxv[tid + stride]) { maxv[tid] = maxv[tid + stride]; maxt[tid] = maxt[tid + stride]; }
    value_blk[b0] = maxv[0];
    maxbid[b0] = b0;
    memcpy(target[b0], rend[maxt[0]], sizeof(target[b0]));
  }
  for (int stride = 32; stride > 0; stride >>= 1)
    for (int tid = 0; tid < stride; ++tid)
      if (value_blk[tid] < value_blk[tid + stride]) {
        value_blk[tid] = value_blk[tid + stride];
        maxbid[tid] = maxbid[tid + stride];
      }
  const int* t = target[maxbid[0]];
  for (int i = 0; i < 4; ++i) begin[i] = end[i];
  /* dataloader.cu:298-321, evaluated in this order */
  if (begin[3] < t[3]) { end[3] = t[3]; *maxlevel = 0; } else end[3] = begin[3];
  if (begin[2] < t[2]) { end[2] = t[2]; *maxlevel = 1; } else end[2] = begin[2];
  if (begin[1] < t[1]) { end[1] = t[1]; *maxlevel = 2; } else end[1] = begin[1];
  if (begin[0] < t[0]) { end[0] = t[0]; *maxlevel = 3; } else end[0] = begin[0];
}
