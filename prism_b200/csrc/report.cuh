// Error statistics of a reconstruction (statistic, analyze.hpp:5-73) on the
// GPU: max |error| with the first index reaching it, min/max of the original,
// and the sum of squared errors; PSNR, NRMSE and the max relative error
// follow on the host from these.  The error of an element is
// fabs((double)(data - original)) with the subtraction in the field's type,
// as in the reference.  Max/min and the index are exact; the squared-error
// sum is a fixed-order tree sum in double (the reference sums serially).
#pragma once
#include <stdint.h>

namespace prism_b200 {

struct StatPart {
  double maxe;
  uint64_t idx;
  double mn, mx;
  double l2;
};

constexpr int kStatThreads = 256;

__device__ __forceinline__ void stat_merge(StatPart& a, const StatPart& b) {
  if (b.maxe > a.maxe || (b.maxe == a.maxe && b.idx < a.idx)) { a.maxe = b.maxe; a.idx = b.idx; }
  a.mn = b.mn < a.mn ? b.mn : a.mn;
  a.mx = b.mx > a.mx ? b.mx : a.mx;
  a.l2 += b.l2;
}

template <class T>
__global__ void __launch_bounds__(kStatThreads)
stats_kernel(const T* __restrict__ ori, const T* __restrict__ dat, uint64_t n, StatPart* __restrict__ part) {
  __shared__ StatPart sh[kStatThreads];
  StatPart p;
  p.maxe = -1.0;
  p.idx = ~0ull;
  p.mn = (double)ori[0];
  p.mx = (double)ori[0];
  p.l2 = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const T o = __ldg(ori + i), d = __ldg(dat + i);
    const double err = fabs((double)(d - o));
    if (err > p.maxe) { p.maxe = err; p.idx = i; }  // per thread, indices increase
    const double od = (double)o;
    p.mn = od < p.mn ? od : p.mn;
    p.mx = od > p.mx ? od : p.mx;
    p.l2 = __fma_rn(err, err, p.l2);
  }
  sh[threadIdx.x] = p;
  __syncthreads();
  for (int s = kStatThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      StatPart a = sh[threadIdx.x];
      stat_merge(a, sh[threadIdx.x + s]);
      sh[threadIdx.x] = a;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void stats_final_kernel(StatPart* part, int nb) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  StatPart a = part[0];
  for (int b = 1; b < nb; ++b) stat_merge(a, part[b]);
  part[0] = a;
}

}  // namespace prism_b200
