// Progressive retrieval strategy (src/loader/dataloader.cu:13-208): pick, per
// level, how many leading bit planes to load so that the modelled error cost
// stays within floor(target*0.954/eb) - 1 while skipping the most bytes.
//
// The reference scans all 33^4 (b0, b1, b2, b3) combinations with 33 CTAs of
// 1024 threads; its per-thread scan (strict >), per-block tree reduction
// (strict <, left kept) and cross-block tree reduction define which of
// several equal-valued choices wins.  That choice is restated below as a
// total order on the candidates, so the scan runs as 297 CTAs (one per b0
// and group of scan rounds, filling the GPU) and a one-warp reduction
// instead of 33 CTAs and the reference's spin barrier.
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

// findStrategy_h (:179-208): the bound and target in absolute units
__device__ __forceinline__ void strategy_setup(int mode, double bound, double target, const double* range,
                                               bool* use_search, uint64_t* target_cost) {
  double eb = bound, te = target;
  if (mode == 1) { eb = __dmul_rn(bound, *range); te = __dmul_rn(target, *range); }
  double scaled = __dmul_rn(te, 0.954);
  *use_search = scaled >= eb;
  *target_cost = (uint64_t)floor(__ddiv_rn(scaled, eb)) - 1;
}

// Which candidate the reference's search returns.  Its block b0 scans, in
// thread t, the positions pos = t + 1024 k in increasing k and keeps the
// first maximum (strict >); a block then reduces its 1024 threads by the
// interleaved tree (strides 512..1, the left entry kept on ties) and the 33
// blocks reduce the same way.  Such a tree returns the maximum with ties
// resolved towards the smallest bit-reversed index, so the winner is the
// candidate of largest value (> 0, within the cost) with ties broken by
// bit-reversed b0, then bit-reversed t, then k.  That order is packed into
// `key` (larger wins), which lets any reduction order find it: here one CTA
// per b0 and group of four rounds k (297 CTAs of 256 threads, 16 candidates a
// thread), and a final warp over the 297 CTA results.
constexpr int kStrategyRounds = (33 * 33 * 33 + 1023) / 1024;  // 36
constexpr int kStrategyRoundsPerCta = 4;
constexpr int kStrategyGroups = kStrategyRounds / kStrategyRoundsPerCta;  // 9
constexpr int kStrategyCells = kStrategyGroups * 33;
static_assert(kStrategyRounds % kStrategyRoundsPerCta == 0, "whole groups of rounds");

struct StrategyBest {
  unsigned long long value;
  unsigned int key;  // (63 - brev6(b0)) << 16 | (1023 - brev10(t)) << 6 | (63 - k)
  unsigned int pad;
};

__device__ __forceinline__ unsigned strategy_brev(unsigned v, int bits) { return __brev(v) >> (32 - bits); }

__device__ __forceinline__ bool strategy_better(unsigned long long v, unsigned k, unsigned long long bv,
                                                unsigned bk) {
  return v > bv || (v == bv && k > bk);
}

// One CTA of the scan: group of rounds `group`, first-level plane count b0.
__device__ __forceinline__ void strategy_scan_cta(const uint64_t* __restrict__ cs, int mode, double bound,
                                                  double target, const double* __restrict__ range,
                                                  StrategyBest* __restrict__ out, const int group, const int b0) {
  bool use_search;
  uint64_t target_cost;
  strategy_setup(mode, bound, target, range, &use_search, &target_cost);
  if (!use_search) return;
  __shared__ uint64_t cost[4][33];
  __shared__ uint64_t vt[4][33];
  __shared__ unsigned long long wv[8];
  __shared__ unsigned wk[8];
  const int tid = threadIdx.x;
  if (tid < 4 * 33) {
    int l = tid / 33, b = tid % 33;
    cost[l][b] = strategy_cost(l, b);
    uint64_t top = cs[l * 32 + 31];
    vt[l][b] = b == 0 ? top : (b == 32 ? 0 : top - cs[l * 32 + b - 1]);
  }
  __syncthreads();
  const unsigned kb = (63u - strategy_brev((unsigned)b0, 6)) << 16;
  unsigned long long best = 0;
  unsigned bkey = 0;
#pragma unroll
  for (int r = 0; r < kStrategyRoundsPerCta; ++r) {
    const int k = group * kStrategyRoundsPerCta + r;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int t = q * 256 + tid, pos = k * 1024 + t;
      if (pos < 33 * 33 * 33) {
        const int b1 = pos / (33 * 33), b2 = (pos / 33) % 33, b3 = pos % 33;
        const uint64_t tc = cost[0][b0] + cost[1][b1] + cost[2][b2] + cost[3][b3];
        if (tc <= target_cost) {
          const unsigned long long v = vt[0][b0] + vt[1][b1] + vt[2][b2] + vt[3][b3];
          const unsigned key = kb | (1023u - strategy_brev((unsigned)t, 10)) << 6 | (63u - (unsigned)k);
          if (v > 0 && strategy_better(v, key, best, bkey)) { best = v; bkey = key; }
        }
      }
    }
  }
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    const unsigned long long ov = __shfl_xor_sync(0xffffffffu, best, d);
    const unsigned ok = __shfl_xor_sync(0xffffffffu, bkey, d);
    if (strategy_better(ov, ok, best, bkey)) { best = ov; bkey = ok; }
  }
  if (lane == 0) { wv[warp] = best; wk[warp] = bkey; }
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < 8; ++w)
      if (strategy_better(wv[w], wk[w], best, bkey)) { best = wv[w]; bkey = wk[w]; }
    StrategyBest r;
    r.value = best;
    r.key = bkey;
    r.pad = 0;
    out[b0 * kStrategyGroups + group] = r;
  }
}

__global__ void __launch_bounds__(256)
strategy_scan_kernel(const uint64_t* __restrict__ cs, int mode, double bound, double target,
                     const double* __restrict__ range, StrategyBest* __restrict__ out) {
  strategy_scan_cta(cs, mode, bound, target, range, out, blockIdx.x, blockIdx.y);
}

// Many independent searches in one launch (grid z = search): search i reads
// cumulative plane sizes cs + 128 i and the absolute bound / target
// bt[2 i], bt[2 i + 1], and writes its cells to out + kStrategyCells i.
__global__ void __launch_bounds__(256)
strategy_scan_batch_kernel(const uint64_t* __restrict__ cs, const double* __restrict__ bt,
                           const double* __restrict__ one, StrategyBest* __restrict__ out) {
  const int i = blockIdx.z;
  strategy_scan_cta(cs + 128 * (size_t)i, 0, bt[2 * i], bt[2 * i + 1], one, out + (size_t)kStrategyCells * i,
                    blockIdx.x, blockIdx.y);
}

// Reduction over the cells + begin/end/maxlevel update
// (dataloader.cu:278-334), or loadall (:21-28) when the target is below the
// compression bound; one warp, lane 0 writes the state.
__device__ __forceinline__ void strategy_finish_warp(const StrategyBest* __restrict__ cells, int mode, double bound,
                                                     double target, const double* __restrict__ range,
                                                     StrategyState* __restrict__ st) {
  const int lane = threadIdx.x & 31;
  bool use_search;
  uint64_t target_cost;
  strategy_setup(mode, bound, target, range, &use_search, &target_cost);
  int tg[4] = {32, 32, 32, 32};
  if (use_search) {
    unsigned long long best = 0;
    unsigned bkey = 0;
    constexpr int kPerLane = (kStrategyCells + 31) / 32;
    StrategyBest c[kPerLane];
#pragma unroll
    for (int m = 0; m < kPerLane; ++m) {  // all loads in flight before the compares
      const int i = lane + 32 * m;
      c[m] = i < kStrategyCells ? cells[i] : StrategyBest{0ull, 0u, 0u};
    }
#pragma unroll
    for (int m = 0; m < kPerLane; ++m)
      if (strategy_better(c[m].value, c[m].key, best, bkey)) { best = c[m].value; bkey = c[m].key; }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      const unsigned long long ov = __shfl_xor_sync(0xffffffffu, best, d);
      const unsigned ok = __shfl_xor_sync(0xffffffffu, bkey, d);
      if (strategy_better(ov, ok, best, bkey)) { best = ov; bkey = ok; }
    }
    if (best > 0) {  // otherwise every block reports its initial {32, 32, 32, 32}
      const int b0 = (int)strategy_brev(63u - ((bkey >> 16) & 63u), 6);
      const int t = (int)strategy_brev(1023u - ((bkey >> 6) & 1023u), 10);
      const int k = 63 - (int)(bkey & 63u);
      const int pos = k * 1024 + t;
      tg[0] = b0;
      tg[1] = pos / (33 * 33);
      tg[2] = (pos / 33) % 33;
      tg[3] = pos % 33;
    }
  }
  if (lane != 0) return;
  StrategyState s = *st;
  int maxlevel = 4;
  for (int i = 0; i < 4; ++i) s.begin[i] = s.end[i];
  if (!use_search) {
    for (int i = 0; i < 4; ++i) s.end[i] = 32;
    maxlevel = s.begin[0] < 32 ? 3 : s.begin[1] < 32 ? 2 : s.begin[2] < 32 ? 1 : s.begin[3] < 32 ? 0 : 4;
  } else {
    if (s.begin[3] < tg[3]) { s.end[3] = tg[3]; maxlevel = 0; } else s.end[3] = s.begin[3];
    if (s.begin[2] < tg[2]) { s.end[2] = tg[2]; maxlevel = 1; } else s.end[2] = s.begin[2];
    if (s.begin[1] < tg[1]) { s.end[1] = tg[1]; maxlevel = 2; } else s.end[1] = s.begin[1];
    if (s.begin[0] < tg[0]) { s.end[0] = tg[0]; maxlevel = 3; } else s.end[0] = s.begin[0];
  }
  s.maxlevel = maxlevel;
  *st = s;
}

__global__ void strategy_finish_kernel(const StrategyBest* __restrict__ cells, int mode, double bound,
                                       double target, const double* __restrict__ range,
                                       StrategyState* __restrict__ st) {
  strategy_finish_warp(cells, mode, bound, target, range, st);
}

// one warp per search of strategy_scan_batch_kernel
__global__ void strategy_finish_batch_kernel(const StrategyBest* __restrict__ cells, const double* __restrict__ bt,
                                             const double* __restrict__ one, StrategyState* __restrict__ st) {
  const int i = blockIdx.x;
  strategy_finish_warp(cells + (size_t)kStrategyCells * i, 0, bt[2 * i], bt[2 * i + 1], one, st + i);
}

}  // namespace prism_b200
