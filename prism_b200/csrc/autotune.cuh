// Interpolation auto-tuning (InterpolationPredictor.cu:880-967 + host logic
// :2273-2355) and the per-field parameter setup.
//
// The reference samples 17^3 windows on a stride-128 grid placed around the
// field centre, evaluates 15 candidate interpolation variants per window on
// the original data (sum of |x - prediction|) and picks per level whether to
// use the multi-dimensional stages and/or the reverse sweep order.  The sample
// grid is computed with uint32 / int arithmetic whose wrap-around decides what
// 1-D and 2-D fields get; sample_grid() reproduces that arithmetic exactly and
// returns only the windows that actually touch the field.
//
// B200 mapping: one CTA per (sample window, variant group); per-thread partial
// sums, a fixed-order block reduction, then one CTA sums the windows in order
// and makes the decisions, so the result is deterministic (the reference's
// float atomics are not).
#pragma once
#include <vector>
#include "predict.cuh"

namespace prism_b200 {

struct SampleWindow { uint32_t gs[3]; };

// calc_start_size (:2277-2283) per axis + the launch-size check; returns the
// windows that lie (at least partly) inside the field.
inline std::vector<SampleWindow> sample_grid(uint32_t nx, uint32_t ny, uint32_t nz) {
  uint32_t dims[3] = {nx, ny, nz};
  uint32_t s_start[3], s_size[3];
  for (int d = 0; d < 3; ++d) {
    uint32_t dim = dims[d], mid = dim / 2;
    uint32_t k = (mid - 8u) / 128u;
    uint32_t t = (dim - 8u - 1u - mid) / 128u;
    s_start[d] = mid - k * 128u;
    s_size[d] = k + t + 1u;
  }
  std::vector<SampleWindow> out;
  int32_t block_num = (int32_t)(s_size[0] * s_size[1] * s_size[2]);
  if (block_num <= 0) return out;  // the reference launch is rejected
  std::vector<uint32_t> cand[3];
  for (int d = 0; d < 3; ++d) {
    for (uint64_t k = 0; k < 3; ++k) {
      uint64_t lo = k << 32;
      int64_t first = (int64_t)lo - (int64_t)s_start[d] > 0 ? ((int64_t)lo - (int64_t)s_start[d] + 127) / 128 : 0;
      for (int64_t i = first; i < (int64_t)s_size[d]; ++i) {
        uint64_t v = (uint64_t)s_start[d] + 128ull * (uint64_t)i;
        if (v >= lo + dims[d]) break;
        if (v >= lo) cand[d].push_back((uint32_t)i);
      }
    }
  }
  for (uint32_t iz : cand[2])
    for (uint32_t iy : cand[1])
      for (uint32_t ix : cand[0]) {
        uint64_t bix = ix + (uint64_t)s_size[0] * (iy + (uint64_t)s_size[1] * iz);
        if (bix >= (uint64_t)(uint32_t)block_num) continue;
        SampleWindow w;
        w.gs[0] = s_start[0] + ix * 128u;
        w.gs[1] = s_start[1] + iy * 128u;
        w.gs[2] = s_start[2] + iz * 128u;
        out.push_back(w);
      }
  return out;
}

constexpr int kAttThreads = 256;

template <class T>
__device__ T att_level(const TileCtx<T>& t, int level, bool md, bool rev, bool nat) {
  int u = 1 << level, N = 16 / (2 * u);
  T err = T(0);
  using F = Fp<T>;
  if (md) {
    for (int kind = 1; kind <= 3; ++kind) {
      int total = kind == 1 ? 3 * N * (N + 1) * (N + 1) : (kind == 2 ? 3 * N * N * (N + 1) : N * N * N);
      for (int i = threadIdx.x; i < total; i += blockDim.x) {
        int x, y, z;
        if (kind == 1) {
          int L = N * (N + 1) * (N + 1), Q = (N + 1) * (N + 1);
          int grp = i / L, m = i % L, a = m / Q, b = (m % Q) / (N + 1), c = (m % Q) % (N + 1);
          if (grp == 0) { x = 2 * u * a + u; y = 2 * u * b; z = 2 * u * c; }
          else if (grp == 1) { x = 2 * u * c; y = 2 * u * a + u; z = 2 * u * b; }
          else { x = 2 * u * b; y = 2 * u * c; z = 2 * u * a + u; }
        } else if (kind == 2) {
          int L = N * N * (N + 1), Q = N * N;
          int grp = i / L, m = i % L, a = m / Q, b = (m % Q) / N, c = (m % Q) % N;
          if (grp == 0) { x = 2 * u * a; y = 2 * u * b + u; z = 2 * u * c + u; }
          else if (grp == 1) { x = 2 * u * c + u; y = 2 * u * a; z = 2 * u * b + u; }
          else { x = 2 * u * b + u; y = 2 * u * c + u; z = 2 * u * a; }
        } else {
          int Q = N * N;
          x = 2 * u * (i / Q) + u; y = 2 * u * ((i % Q) / N) + u; z = 2 * u * ((i % Q) % N) + u;
        }
        if (!t.in_data(x, y, z)) continue;
        T pred = kind == 1 ? pred_line(t, (z % (2 * u)) ? 2 : ((y % (2 * u)) ? 1 : 0), x, y, z, u, true, nat)
                           : (kind == 2 ? pred_face(t, x, y, z, u, nat) : pred_cube(t, x, y, z, u, nat));
        err = F::add(err, F::abs(F::sub(t.at(x, y, z), pred)));
      }
    }
    return err;
  }
  // per-axis: {axis, nxs, xst, xo, nys, yst, yo, nzs, zst, zo}
  int st[3][10];
  if (rev) {
    int v[3][10] = {{0, N, 2, 1, N + 1, 2, 0, N + 1, 2, 0},
                    {1, 2 * N + 1, 1, 0, N, 2, 1, N + 1, 2, 0},
                    {2, 2 * N + 1, 1, 0, 2 * N + 1, 1, 0, N, 2, 1}};
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 10; ++b) st[a][b] = v[a][b];
  } else {
    int v[3][10] = {{2, N + 1, 2, 0, N + 1, 2, 0, N, 2, 1},
                    {1, N + 1, 2, 0, N, 2, 1, 2 * N + 1, 1, 0},
                    {0, N, 2, 1, 2 * N + 1, 1, 0, 2 * N + 1, 1, 0}};
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 10; ++b) st[a][b] = v[a][b];
  }
  for (int s = 0; s < 3; ++s) {
    int total = st[s][1] * st[s][4] * st[s][7];
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      int ii = i % st[s][1], jj = (i / st[s][1]) % st[s][4], kk = i / st[s][1] / st[s][4];
      int x = u * (ii * st[s][2] + st[s][3]), y = u * (jj * st[s][5] + st[s][6]), z = u * (kk * st[s][8] + st[s][9]);
      if (!t.in_data(x, y, z)) continue;
      T pred = pred_line(t, st[s][0], x, y, z, u, false, nat);
      err = F::add(err, F::abs(F::sub(t.at(x, y, z), pred)));
    }
  }
  return err;
}

template <class T>
__device__ T block_sum(T v, T* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = Fp<T>::add(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  T r = red[0];
  __syncthreads();
  return r;
}

// grid (windows, 6): blockIdx.y is the reference's variant group
// (pre_compute_att :111-141): 0 -> levels 3 and 2, 1-2 -> level 1
// (2 = natural cubic), 3-5 -> level 0.  partial[window][15].
template <class T>
__device__ __forceinline__ void autotune_window(T* win, T* red, const T* __restrict__ data, const Geometry& g,
                                                const SampleWindow w, int biy, T* out) {
  TileCtx<T> t;
  t.s = win;
  t.dim[0] = g.nx; t.dim[1] = g.ny; t.dim[2] = g.nz;
#pragma unroll
  for (int d = 0; d < 3; ++d) { t.gs[d] = w.gs[d]; t.notlast_[d] = w.gs[d] + 16u < t.dim[d]; }
  const uint64_t sy = g.nx, sz = (uint64_t)g.nx * g.ny;
  for (int i = threadIdx.x; i < kWinVol; i += blockDim.x) {
    int x = i % kWin, y = (i / kWin) % kWin, z = i / (kWin * kWin);
    T v = T(0);
    if (t.in_data(x, y, z)) v = data[(uint64_t)(t.gs[0] + x) + (uint64_t)(t.gs[1] + y) * sy + (uint64_t)(t.gs[2] + z) * sz];
    win[i] = v;
  }
  __syncthreads();
  if (biy == 0) {
    T e[6];
    e[0] = att_level(t, 3, false, false, false);
    e[1] = att_level(t, 3, false, true, false);
    e[2] = att_level(t, 3, true, true, false);
    e[3] = att_level(t, 2, false, false, false);
    e[4] = att_level(t, 2, false, true, false);
    e[5] = att_level(t, 2, true, true, false);
    for (int k = 0; k < 6; ++k) {
      T s = block_sum(e[k], red);
      if (threadIdx.x == 0) out[k] = s;
    }
  } else if (biy <= 2) {
    bool nat = biy == 2;
    T e0 = att_level(t, 1, false, false, nat), e1 = att_level(t, 1, false, true, nat);
    T e2 = att_level(t, 1, true, true, nat);
    T s0 = block_sum(e0, red), s1 = block_sum(e1, red), s2 = block_sum(e2, red);
    if (threadIdx.x == 0) { out[3 + biy * 3] = s0; out[4 + biy * 3] = s1; out[5 + biy * 3] = s2; }
  } else {
    T e = att_level(t, 0, biy == 5, biy % 3 != 0, false);
    T s = block_sum(e, red);
    if (threadIdx.x == 0) out[9 + biy] = s;
  }
}

template <class T>
__global__ void __launch_bounds__(kAttThreads)
autotune_kernel(const T* __restrict__ data, Geometry g, const SampleWindow* __restrict__ wins, T* __restrict__ partial) {
  __shared__ T win[kWinVol];
  __shared__ T red[kAttThreads];
  autotune_window<T>(win, red, data, g, wins[blockIdx.x], blockIdx.y, partial + (size_t)blockIdx.x * 15);
}

// Field parameters, computed on the device so nothing waits for the host:
// bound (ABS, or REL x range), calc_eb per level (:1825-1839) with the double
// alpha/beta and, when `partial` is given, the auto-tune decisions (:2306-2355)
// from the window sums.  Flags otherwise come from `flags_in` (a container).
template <class T>
__device__ __forceinline__ void compute_params(int mode, double bound, const double* __restrict__ range, double alpha,
                                               const T* __restrict__ partial, int nwin,
                                               const uint8_t* __restrict__ flags_in, int maxlevel,
                                               PredParams<T>* __restrict__ out, T* __restrict__ errors_out,
                                               double* __restrict__ eb_out, const T* __restrict__ sums = nullptr) {
  using F = Fp<T>;
  PredParams<T> p;
  double eb = mode == 1 ? __dmul_rn(bound, *range) : bound;
  T ebx2 = F::from_double(__dmul_rn(eb, 2.0)), ebr = F::from_double(__ddiv_rn(1.0, eb));
  const double beta = 4.0;
  int level = 3;
  for (int unit = 8; unit >= 1; unit >>= 1, --level) {
    T cx = ebx2, cr = ebr;
    for (int temp = 1; temp < unit; temp *= 2) {
      cr = F::from_double(__dmul_rn((double)cr, alpha));
      cx = F::from_double(__ddiv_rn((double)cx, alpha));
    }
    if ((double)cx < __ddiv_rn((double)ebx2, beta)) {
      cx = F::from_double(__ddiv_rn((double)ebx2, beta));
      cr = F::from_double(__dmul_rn((double)ebr, beta));
    }
    p.ebx2[level] = cx;
    p.ebr[level] = cr;
  }
  for (int l = 0; l < 4; ++l) p.natural[l] = 0;
  if (partial || sums) {
    T e[15];
    for (int k = 0; k < 15; ++k) {
      T s = T(0);
      if (sums) {
        s = sums[k];
      } else {
        for (int w = 0; w < nwin; ++w) s = F::add(s, partial[(size_t)w * 15 + k]);
      }
      e[k] = s;
      if (errors_out) errors_out[k] = s;
    }
    T best;
    int idx;
    if (e[0] > e[1]) { best = e[1]; p.reverse[3] = 1; } else { best = e[0]; p.reverse[3] = 0; }
    p.use_md[3] = e[2] < best;
    if (e[3] > e[4]) { best = e[4]; p.reverse[2] = 1; } else { best = e[3]; p.reverse[2] = 0; }
    p.use_md[2] = e[5] < best;
    best = e[6]; idx = 6;
    for (int i = 6; i < 12; ++i) if (e[i] < best) { best = e[i]; idx = i; }
    p.use_md[1] = idx == 8 || idx == 11;
    p.reverse[1] = idx % 3 != 0;
    best = e[12]; idx = 12;
    for (int i = 12; i < 15; ++i) if (e[i] < best) { best = e[i]; idx = i; }
    p.use_md[0] = idx == 14;
    p.reverse[0] = idx % 3 != 0;
  } else {
    for (int l = 0; l < 4; ++l) { p.use_md[l] = flags_in[l] != 0; p.reverse[l] = flags_in[4 + l] != 0; }
  }
  p.maxlevel = maxlevel;
  *out = p;
  if (eb_out) *eb_out = eb;
}

// One warp: lane k < 15 sums variant k's errors over the windows in window
// order (the same sums, in the same order, as a single thread would form),
// then lane 0 decides.
template <class T>
__global__ void params_kernel(int mode, double bound, const double* __restrict__ range, double alpha,
                              const T* __restrict__ partial, int nwin, const uint8_t* __restrict__ flags_in,
                              int maxlevel, PredParams<T>* __restrict__ out, T* __restrict__ errors_out,
                              double* __restrict__ eb_out) {
  __shared__ T sums[15];
  if (blockIdx.x != 0) return;
  const int k = threadIdx.x;
  if (partial && k < 15) {
    T s = T(0);
    for (int w = 0; w < nwin; ++w) s = Fp<T>::add(s, partial[(size_t)w * 15 + k]);
    sums[k] = s;
  }
  __syncthreads();
  if (k != 0) return;
  compute_params<T>(mode, bound, range, alpha, partial, nwin, flags_in, maxlevel, out, errors_out, eb_out,
                    partial ? sums : nullptr);
}

// Global min / max (compressor.cu:230-302): per-block partials, then one block.
constexpr int kExtThreads = 512;

// 16-byte vectors of values for the extrema scan
template <class T> struct Vec16;
template <> struct Vec16<double> {
  using type = double2;
  static __device__ __forceinline__ void fold(const double2& v, double& mn, double& mx) {
    mn = v.x < mn ? v.x : mn;
    mx = v.x > mx ? v.x : mx;
    mn = v.y < mn ? v.y : mn;
    mx = v.y > mx ? v.y : mx;
  }
};
template <> struct Vec16<float> {
  using type = float4;
  static __device__ __forceinline__ void fold(const float4& v, float& mn, float& mx) {
    mn = v.x < mn ? v.x : mn;
    mx = v.x > mx ? v.x : mx;
    mn = v.y < mn ? v.y : mn;
    mx = v.y > mx ? v.y : mx;
    mn = v.z < mn ? v.z : mn;
    mx = v.z > mx ? v.z : mx;
    mn = v.w < mn ? v.w : mn;
    mx = v.w > mx ? v.w : mx;
  }
};

// The folds start from in[0] and keep the running value unless the new one
// compares below (above) it, so a NaN is skipped unless it is in[0], and the
// result does not depend on the order in which values are folded.
template <class T>
__global__ void __launch_bounds__(kExtThreads)
extrema_kernel(const T* __restrict__ in, uint64_t n, T* __restrict__ part) {
  using V = typename Vec16<T>::type;
  constexpr uint64_t W = 16 / sizeof(T);
  __shared__ T smin[kExtThreads], smax[kExtThreads];
  T mn = in[0], mx = in[0];
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // values before the first 16-byte boundary, the 16-byte vectors (four
  // independent loads in flight), the values after the last whole vector
  uint64_t head = ((16 - (reinterpret_cast<uintptr_t>(in) & 15)) & 15) / sizeof(T);
  head = head < n ? head : n;
  const uint64_t nv = (n - head) / W, tail = head + nv * W;
  if (tid < head) {
    const T v = __ldg(in + tid);
    mn = v < mn ? v : mn;
    mx = v > mx ? v : mx;
  }
  const V* vin = reinterpret_cast<const V*>(in + head);
  uint64_t i = tid;
  for (; i + 3 * stride < nv; i += 4 * stride) {
    V v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = __ldg(vin + i + k * stride);
#pragma unroll
    for (int k = 0; k < 4; ++k) Vec16<T>::fold(v[k], mn, mx);
  }
  for (; i < nv; i += stride) Vec16<T>::fold(__ldg(vin + i), mn, mx);
  if (tail + tid < n) {
    const T v = __ldg(in + tail + tid);
    mn = v < mn ? v : mn;
    mx = v > mx ? v : mx;
  }
  smin[threadIdx.x] = mn;
  smax[threadIdx.x] = mx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      T a = smin[threadIdx.x + s], b = smax[threadIdx.x + s];
      if (a < smin[threadIdx.x]) smin[threadIdx.x] = a;
      if (b > smax[threadIdx.x]) smax[threadIdx.x] = b;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = smin[0]; part[2 * blockIdx.x + 1] = smax[0]; }
}

// one warp folds the per-block extrema (min/max are order independent)
template <class T>
__global__ void extrema_final_kernel(const T* __restrict__ part, int nblocks, double* __restrict__ range,
                                     double* __restrict__ minmax = nullptr) {
  const int lane = threadIdx.x;
  T mn = part[0], mx = part[1];
  for (int b = lane; b < nblocks; b += 32) {
    T a = part[2 * b], c = part[2 * b + 1];
    mn = a < mn ? a : mn;
    mx = c > mx ? c : mx;
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    T a = __shfl_xor_sync(0xffffffffu, mn, d), c = __shfl_xor_sync(0xffffffffu, mx, d);
    mn = a < mn ? a : mn;
    mx = c > mx ? c : mx;
  }
  if (lane == 0) {
    *range = __dsub_rn((double)mx, (double)mn);
    if (minmax) {
      minmax[0] = (double)mn;
      minmax[1] = (double)mx;
    }
  }
}

}  // namespace prism_b200
