// Progressive retrieval strategy (src/loader/dataloader.cu:13-208): pick, per
// level, how many leading bit planes to load so that the modelled error cost
// stays within floor(target*0.954/eb) - 1 while skipping the most bytes.
//
// The reference scans all 33^4 (b0, b1, b2, b3) combinations with 33 CTAs of
// 1024 threads; the per-thread scan (strict >), the per-block tree reduction
// (strict <, left kept) and the cross-block tree reduction define which of
// several equal-valued choices wins, so this kernel keeps exactly that
// structure.  The cross-block step runs as a second tiny kernel instead of the
// reference's spin barrier.
#pragma once
#include <stdint.h>

namespace prism_b200 {

struct StrategyState {
  int begin[4];
  int end[4];
  int maxlevel;
};

// cost[l][b] = ceil(2^(32-b) * (p^(11-3l) + p^(10-3l) + p^(9-3l))), p = 1 (l=0)
// or 1.25: the powers 5^k/4^k are exact in double, summed in the same order.
__device__ __forceinline__ uint64_t strategy_cost(int l, int b) {
  int shift = 32 - b;
  double err = shift == 0 ? 0.0 : (double)(1ull << shift);
  double p = l == 0 ? 1.0 : 1.25;
  double pw[3];
  for (int j = 0; j < 3; ++j) {
    int k = 12 - 3 * l - 1 - j;
    double r = 1.0;
    for (int i = 0; i < k; ++i) r = __dmul_rn(r, p);
    pw[j] = r;
  }
  err = __dmul_rn(err, __dadd_rn(__dadd_rn(pw[0], pw[1]), pw[2]));
  return (uint64_t)ceil(err);
}

struct StrategyBlock {
  unsigned long long value;
  int target[4];
};

// findStrategy_h (:179-208): the bound and target in absolute units
__device__ __forceinline__ void strategy_setup(int mode, double bound, double target, const double* range,
                                               bool* use_search, uint64_t* target_cost) {
  double eb = bound, te = target;
  if (mode == 1) { eb = __dmul_rn(bound, *range); te = __dmul_rn(target, *range); }
  double scaled = __dmul_rn(te, 0.954);
  *use_search = scaled >= eb;
  *target_cost = (uint64_t)floor(__ddiv_rn(scaled, eb)) - 1;
}

__global__ void __launch_bounds__(1024)
strategy_search_kernel(const uint64_t* __restrict__ cs, int mode, double bound, double target,
                       const double* __restrict__ range, StrategyBlock* __restrict__ out) {
  bool use_search;
  uint64_t target_cost;
  strategy_setup(mode, bound, target, range, &use_search, &target_cost);
  if (!use_search) return;
  __shared__ uint64_t cost[4][33];
  __shared__ uint64_t vt[4][33];
  __shared__ unsigned long long maxv[1024];
  __shared__ int maxt[1024];
  const int tid = threadIdx.x, b0 = blockIdx.x;
  if (tid < 4 * 33) {
    int l = tid / 33, b = tid % 33;
    cost[l][b] = strategy_cost(l, b);
    uint64_t top = cs[l * 32 + 31];
    vt[l][b] = b == 0 ? top : (b == 32 ? 0 : top - cs[l * 32 + b - 1]);
  }
  __syncthreads();
  unsigned long long best = 0;
  int r[4] = {32, 32, 32, 32};
  for (int pos = tid; pos < 33 * 33 * 33; pos += 1024) {
    int b1 = pos / (33 * 33), b2 = (pos / 33) % 33, b3 = pos % 33;
    uint64_t tc = cost[0][b0] + cost[1][b1] + cost[2][b2] + cost[3][b3];
    if (tc <= target_cost) {
      unsigned long long v = vt[0][b0] + vt[1][b1] + vt[2][b2] + vt[3][b3];
      if (v > best) { r[0] = b0; r[1] = b1; r[2] = b2; r[3] = b3; best = v; }
    }
  }
  maxv[tid] = best;
  maxt[tid] = tid;
  __syncthreads();
  for (int s = 512; s > 0; s >>= 1) {
    if (tid < s && maxv[tid] < maxv[tid + s]) { maxv[tid] = maxv[tid + s]; maxt[tid] = maxt[tid + s]; }
    __syncthreads();
  }
  if (tid == maxt[0]) {
    out[b0].value = maxv[0];
    for (int k = 0; k < 4; ++k) out[b0].target[k] = r[k];
  }
}

// Cross-block reduction + begin/end/maxlevel update (dataloader.cu:278-334),
// or loadall (:21-28) when the target is below the compression bound.
__global__ void strategy_finish_kernel(const StrategyBlock* __restrict__ blk, int mode, double bound,
                                       double target, const double* __restrict__ range,
                                       StrategyState* __restrict__ st) {
  if (threadIdx.x != 0) return;
  bool use_search;
  uint64_t target_cost;
  strategy_setup(mode, bound, target, range, &use_search, &target_cost);
  StrategyState s = *st;
  int maxlevel = 4;
  for (int i = 0; i < 4; ++i) s.begin[i] = s.end[i];
  if (!use_search) {
    for (int i = 0; i < 4; ++i) s.end[i] = 32;
    maxlevel = s.begin[0] < 32 ? 3 : s.begin[1] < 32 ? 2 : s.begin[2] < 32 ? 1 : s.begin[3] < 32 ? 0 : 4;
  } else {
    unsigned long long v[64];
    int bid[64];
    for (int i = 0; i < 64; ++i) { v[i] = i < 33 ? blk[i].value : 0; bid[i] = i < 33 ? i : 0; }
    for (int stride = 32; stride > 0; stride >>= 1)
      for (int t = 0; t < stride; ++t)
        if (v[t] < v[t + stride]) { v[t] = v[t + stride]; bid[t] = bid[t + stride]; }
    const int* tg = blk[bid[0]].target;
    if (s.begin[3] < tg[3]) { s.end[3] = tg[3]; maxlevel = 0; } else s.end[3] = s.begin[3];
    if (s.begin[2] < tg[2]) { s.end[2] = tg[2]; maxlevel = 1; } else s.end[2] = s.begin[2];
    if (s.begin[1] < tg[1]) { s.end[1] = tg[1]; maxlevel = 2; } else s.end[1] = s.begin[1];
    if (s.begin[0] < tg[0]) { s.end[0] = tg[0]; maxlevel = 3; } else s.end[0] = s.begin[0];
  }
  s.maxlevel = maxlevel;
  *st = s;
}

// The same on one warp (lane 0 writes the state): the 33 block maxima reduce
// by the same tree (at each stride, position t takes t + stride's entry when
// its value is strictly smaller), so ties resolve identically.
__device__ __forceinline__ void strategy_finish_warp(const StrategyBlock* __restrict__ blk, int mode, double bound,
                                                     double target, const double* __restrict__ range,
                                                     StrategyState* __restrict__ st) {
  const int lane = threadIdx.x & 31;
  bool use_search;
  uint64_t target_cost;
  strategy_setup(mode, bound, target, range, &use_search, &target_cost);
  int winner = 0;
  if (use_search) {
    unsigned long long v = blk[lane].value;
    int bid = lane;
    const unsigned long long w32 = lane == 0 ? blk[32].value : 0ull;
    if (v < w32) { v = w32; bid = 32; }
    for (int stride = 16; stride > 0; stride >>= 1) {
      const unsigned long long w = __shfl_down_sync(0xffffffffu, v, stride);
      const int wb = __shfl_down_sync(0xffffffffu, bid, stride);
      if (lane < stride && v < w) { v = w; bid = wb; }
    }
    winner = __shfl_sync(0xffffffffu, bid, 0);
  }
  if (lane != 0) return;
  StrategyState s = *st;
  int maxlevel = 4;
  for (int i = 0; i < 4; ++i) s.begin[i] = s.end[i];
  if (!use_search) {
    for (int i = 0; i < 4; ++i) s.end[i] = 32;
    maxlevel = s.begin[0] < 32 ? 3 : s.begin[1] < 32 ? 2 : s.begin[2] < 32 ? 1 : s.begin[3] < 32 ? 0 : 4;
  } else {
    const int* tg = blk[winner].target;
    if (s.begin[3] < tg[3]) { s.end[3] = tg[3]; maxlevel = 0; } else s.end[3] = s.begin[3];
    if (s.begin[2] < tg[2]) { s.end[2] = tg[2]; maxlevel = 1; } else s.end[2] = s.begin[2];
    if (s.begin[1] < tg[1]) { s.end[1] = tg[1]; maxlevel = 2; } else s.end[1] = s.begin[1];
    if (s.begin[0] < tg[0]) { s.end[0] = tg[0]; maxlevel = 3; } else s.end[0] = s.begin[0];
  }
  s.maxlevel = maxlevel;
  *st = s;
}

}  // namespace prism_b200
