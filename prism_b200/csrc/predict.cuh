// Multi-level cubic-spline predictor + error-bounded quantiser (compress) and
// the matching reconstruction (full and progressive), one 16^3 tile per CTA.
//
// Restates InterpolationPredictor.cu (interpolation :2137-2173,
// interpolation_reverse :2177-2207, interpolation_progressive_reverse
// :2209-2239): a tile works in a 17^3 shared-memory window (its own 16^3
// points plus the first plane of the next tile in x, y and z), sweeps levels
// 3..0 (unit 8, 4, 2, 1) and per level runs three stages: either
// line/face/cube ("md") or three axis sweeps in blue-yellow-hollow (z, y, x)
// order or its reverse.  Each stage predicts a set of independent points from
// already reconstructed ones, quantises the residual and reconstructs in
// place.  Codes go straight to their level-major slot (no linear scratch
// pass).  All arithmetic uses explicitly rounded intrinsics (fp.cuh) so the
// results equal the reference build bit for bit.
#pragma once
#include "fp.cuh"
#include "geometry.h"

namespace prism_b200 {

// Per-field predictor parameters, resident in device memory so a pipeline can
// compute them on the GPU (REL bound from the extrema kernel, flags from the
// auto-tuner) without a host round trip.
template <class T>
struct PredParams {
  T ebr[4];        // 1/eb scaled per level (calc_eb, :1825-1839)
  T ebx2[4];       // 2*eb scaled per level
  uint8_t use_md[4];
  uint8_t reverse[4];
  uint8_t natural[4];
  int32_t maxlevel;  // levels above are skipped (:1848-1849)
};

template <class T>
struct Expr {
  using F = Fp<T>;
  // nan_cubic_interp (:1811-1813): (-a + 9b + 9c - d) / 16
  static __device__ __forceinline__ T cubic_md(T a, T b, T c, T d) {
    T s = F::fma(T(9), b, -a);
    s = F::fma(T(9), c, s);
    s = F::sub(s, d);
    return F::mul(s, T(0.0625));
  }
  // nat_cubic_interp (:1815-1817): (-3a + 23b + 23c - 3d) / 40
  static __device__ __forceinline__ T cubic_nat(T a, T b, T c, T d) {
    T s = F::fma(T(-3), a, F::mul(T(23), b));
    s = F::fma(T(23), c, s);
    s = F::fma(T(-3), d, s);
    return F::div(s, T(40));
  }
  static __device__ __forceinline__ T cubic_lambda(T a, T b, T c, T d, bool nat) {
    return nat ? cubic_nat(a, b, c, d) : cubic_md(a, b, c, d);
  }
  // per-axis cubic (:1248-1251, :1325): (p1 a + p2 b + p3 c + p4 d) / p5
  static __device__ __forceinline__ T cubic_axis(T a, T b, T c, T d, bool nat) {
    T p1 = nat ? T(-3) : T(-1), p2 = nat ? T(23) : T(9), p5 = nat ? T(40) : T(16);
    T s = F::fma(p1, a, F::mul(p2, b));
    s = F::fma(p2, c, s);
    s = F::fma(p1, d, s);
    return F::div(s, p5);
  }
  // (-t0 + 6 t1 + 3 t2) / 8
  static __device__ __forceinline__ T quad_l(T t0, T t1, T t2) {
    T s = F::fma(T(6), t1, -t0);
    s = F::fma(T(3), t2, s);
    return F::mul(s, T(0.125));
  }
  // (3 t1 + 6 t2 - t3) / 8
  static __device__ __forceinline__ T quad_r(T t1, T t2, T t3) {
    T s = F::fma(T(3), t1, F::mul(T(6), t2));
    s = F::sub(s, t3);
    return F::mul(s, T(0.125));
  }
  // the same expression inside the md cube stage is contracted the other way
  // round: fma(6, t2, 3*t1) - t3 (measured against the reference build)
  static __device__ __forceinline__ T quad_r_cube(T t1, T t2, T t3) {
    T s = F::fma(T(6), t2, F::mul(T(3), t1));
    s = F::sub(s, t3);
    return F::mul(s, T(0.125));
  }
  static __device__ __forceinline__ T lin(T a, T b) { return F::mul(F::add(a, b), T(0.5)); }
  static __device__ __forceinline__ T half(T a) { return F::mul(a, T(0.5)); }
};

constexpr int kWin = 17;
constexpr int kWinVol = kWin * kWin * kWin;

template <class T>
struct TileCtx {
  T* s;  // shared window, s[(z*17 + y)*17 + x]
  uint32_t gs[3];      // global start of the window (uint32 arithmetic)
  bool notlast[3];     // the window does not reach the field's end
  uint32_t dim[3];
  __device__ __forceinline__ T& at(int x, int y, int z) const { return s[(z * kWin + y) * kWin + x]; }
  __device__ __forceinline__ T get(int axis, int x, int y, int z, int c) const {
    return axis == 0 ? at(c, y, z) : (axis == 1 ? at(x, c, z) : at(x, y, c));
  }
  __device__ __forceinline__ bool in_data(int x, int y, int z) const {
    return gs[0] + (uint32_t)x < dim[0] && gs[1] + (uint32_t)y < dim[1] && gs[2] + (uint32_t)z < dim[2];
  }
  // xyz_predicate (:1173-1185); the exclusive form is used by the last stage
  // of level 0
  __device__ __forceinline__ bool pred_ok(int x, int y, int z, bool inclusive) const {
    if (inclusive) return in_data(x, y, z);
    return x < 16 && y < 16 && z < 16 + !notlast[2] && in_data(x, y, z);
  }
  __device__ __forceinline__ bool owned(int x, int y, int z) const {
    return (x < 16 || !notlast[0]) && (y < 16 || !notlast[1]) && (z < 16 || !notlast[2]);
  }
};

__device__ __forceinline__ int nb_idx(int c, int u, int k) {  // id_x/id_y/id_z (:1426-1439)
  switch (k) {
    case 0: return c - 3 * u >= 0 ? c - 3 * u : 0;
    case 1: return c - u >= 0 ? c - u : 0;
    case 2: return c + u <= 16 ? c + u : 0;
    default: return c + 3 * u <= 16 ? c + 3 * u : 0;
  }
}

// 1-D prediction with the per-axis boundary cases (:1300-1326, :1506-1535)
template <class T>
__device__ __forceinline__ T pred_line(const TileCtx<T>& t, int axis, int x, int y, int z, int u,
                                       bool md, bool nat) {
  using E = Expr<T>;
  int ix = axis == 0 ? x : (axis == 1 ? y : z);
  uint32_t gx = t.gs[axis] + (uint32_t)ix, gs = t.dim[axis];
  bool c1 = t.notlast[axis];
  bool c2 = ix >= 3 * u, c3 = ix + 3 * u <= 16;
  bool c4 = gx + 3u * u < gs, c5 = gx + (uint32_t)u < gs;
  T t1 = t.get(axis, x, y, z, nb_idx(ix, u, 1));
  if ((c1 && !c2 && !c3) || (!c1 && !c2 && !(c3 && c4) && c5))
    return E::lin(t1, t.get(axis, x, y, z, nb_idx(ix, u, 2)));
  if ((c1 && !c2 && c3) || (!c1 && !c2 && c3 && c4))
    return E::quad_r(t1, t.get(axis, x, y, z, nb_idx(ix, u, 2)), t.get(axis, x, y, z, nb_idx(ix, u, 3)));
  if ((c1 && c2 && !c3) || (!c1 && c2 && !(c3 && c4) && c5))
    return E::quad_l(t.get(axis, x, y, z, nb_idx(ix, u, 0)), t1, t.get(axis, x, y, z, nb_idx(ix, u, 2)));
  if ((c1 && c2 && c3) || (!c1 && c2 && c3 && c4)) {
    T t0 = t.get(axis, x, y, z, nb_idx(ix, u, 0)), t2 = t.get(axis, x, y, z, nb_idx(ix, u, 2));
    T t3 = t.get(axis, x, y, z, nb_idx(ix, u, 3));
    return md ? E::cubic_lambda(t0, t1, t2, t3, nat) : E::cubic_axis(t0, t1, t2, t3, nat);
  }
  return t1;
}

// get_interp_order (:1538-1545): 4 cubic, 3 quad-left, 2 quad-right, 1 linear, 0 none
template <class T>
__device__ __forceinline__ int interp_order(const TileCtx<T>& t, int axis, int c, int u) {
  uint32_t gx = t.gs[axis] + (uint32_t)c, gs = t.dim[axis];
  bool notlast = t.notlast[axis];
  int b = c >= 3 * u ? 3 : 1;
  int f = (c + 3 * u <= 16 && (notlast || gx + 3u * u < gs)) ? 3 : ((notlast || gx + (uint32_t)u < gs) ? 1 : 0);
  return b == 3 ? (f == 3 ? 4 : (f == 1 ? 3 : 0)) : (f == 3 ? 2 : (f == 1 ? 1 : 0));
}

// FACE (:1546-1668)
template <class T>
__device__ __forceinline__ T pred_face(const TileCtx<T>& t, int x, int y, int z, int u, bool nat) {
  using E = Expr<T>;
  using F = Fp<T>;
  int a1, a2;
  T pred;
  if (x % (2 * u) == 0) { a1 = 2; a2 = 1; pred = t.at(x, nb_idx(y, u, 1), nb_idx(z, u, 1)); }
  else if (y % (2 * u) == 0) { a1 = 2; a2 = 0; pred = t.at(nb_idx(x, u, 1), y, nb_idx(z, u, 1)); }
  else { a1 = 1; a2 = 0; pred = t.at(nb_idx(x, u, 1), nb_idx(y, u, 1), z); }
  int c1 = a1 == 1 ? y : z, c2 = a2 == 0 ? x : y;
  T s1[4], s2[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    s1[k] = t.get(a1, x, y, z, nb_idx(c1, u, k));
    s2[k] = t.get(a2, x, y, z, nb_idx(c2, u, k));
  }
  int i1 = interp_order(t, a1, c1, u), i2 = interp_order(t, a2, c2, u);
  if (i1 == 4 && i2 == 4)
    return E::half(F::add(E::cubic_lambda(s1[0], s1[1], s1[2], s1[3], nat),
                          E::cubic_lambda(s2[0], s2[1], s2[2], s2[3], nat)));
  if (i1 != 4 && i2 == 4) return E::cubic_lambda(s2[0], s2[1], s2[2], s2[3], nat);
  if (i1 == 4 && i2 != 4) return E::cubic_lambda(s1[0], s1[1], s1[2], s1[3], nat);
  if (i1 == 3 && i2 == 3) return E::half(F::add(E::quad_l(s2[0], s2[1], s2[2]), E::quad_l(s1[0], s1[1], s1[2])));
  if (i1 == 3 && i2 == 2) return E::half(F::add(E::quad_r(s2[1], s2[2], s2[3]), E::quad_l(s1[0], s1[1], s1[2])));
  if (i1 == 3 && i2 < 2) return E::quad_l(s1[0], s1[1], s1[2]);
  if (i1 == 2 && i2 == 3) return E::half(F::add(E::quad_r(s1[1], s1[2], s1[3]), E::quad_l(s2[0], s2[1], s2[2])));
  if (i1 == 2 && i2 == 2) return E::half(F::add(E::quad_r(s1[1], s1[2], s1[3]), E::quad_r(s2[1], s2[2], s2[3])));
  if (i1 == 2 && i2 < 2) return E::quad_r(s1[1], s1[2], s1[3]);
  if (i1 <= 1 && i2 == 3) return E::quad_l(s2[0], s2[1], s2[2]);
  if (i1 <= 1 && i2 == 2) return E::quad_r(s2[1], s2[2], s2[3]);
  if (i1 == 1 && i2 == 1) return E::half(F::add(E::lin(s2[1], s2[2]), E::lin(s1[1], s1[2])));
  if (i1 == 1 && i2 < 1) return E::lin(s1[1], s1[2]);
  if (i1 == 0 && i2 == 1) return E::lin(s2[1], s2[2]);
  return F::sub(F::add(s1[1], s2[1]), pred);
}

// CUBE (:1671-1723)
template <class T>
__device__ __forceinline__ T pred_cube(const TileCtx<T>& t, int x, int y, int z, int u, bool nat) {
  using E = Expr<T>;
  using F = Fp<T>;
  int oz = interp_order(t, 2, z, u), oy = interp_order(t, 1, y, u), ox = interp_order(t, 0, x, u);
  T tx[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) tx[k] = t.at(nb_idx(x, u, k), y, z);
  auto cz = [&]() { return E::cubic_lambda(t.at(x, y, nb_idx(z, u, 0)), t.at(x, y, nb_idx(z, u, 1)),
                                           t.at(x, y, nb_idx(z, u, 2)), t.at(x, y, nb_idx(z, u, 3)), nat); };
  auto cy = [&]() { return E::cubic_lambda(t.at(x, nb_idx(y, u, 0), z), t.at(x, nb_idx(y, u, 1), z),
                                           t.at(x, nb_idx(y, u, 2), z), t.at(x, nb_idx(y, u, 3), z), nat); };
  auto cx = [&]() { return E::cubic_lambda(tx[0], tx[1], tx[2], tx[3], nat); };
  if (oz == 4 && oy == 4 && ox == 4) return F::div(F::add(F::add(cx(), cy()), cz()), T(3));
  if (oz == 4 && oy == 4) return E::half(F::add(cz(), cy()));
  if (oz == 4 && ox == 4) return E::half(F::add(cz(), cx()));
  if (oy == 4 && ox == 4) return E::half(F::add(cy(), cx()));
  if (oz == 4) return cz();
  if (oy == 4) return cy();
  if (ox == 4) return cx();
  if (ox == 3) return E::quad_l(tx[0], tx[1], tx[2]);
  if (ox == 2) return E::quad_r_cube(tx[1], tx[2], tx[3]);
  if (ox == 1) return E::lin(tx[1], tx[2]);
  return tx[1];
}

// Quantise one residual (:1330-1342) and reconstruct; returns the code.
template <class T>
__device__ __forceinline__ int32_t quantize(T orig, T pred, T ebr, T ebx2, T* rec) {
  using F = Fp<T>;
  T err = F::sub(orig, pred);
  T code = F::fma(F::abs(err), ebr, T(1));
  code = err < T(0) ? -code : code;
  int qi = F::to_int_rz(F::mul(code, T(0.5)));
  T qt = F::from_int(qi);
  *rec = F::fma(qt, ebx2, pred);
  return F::to_int_rz(qt);
}

template <class T, bool COMPRESS>
struct StageRunner {
  const TileCtx<T>& t;
  const Geometry& g;
  int32_t* qc;
  T ebr, ebx2;
  __device__ __forceinline__ void emit(int x, int y, int z, T pred) const {
    uint64_t gx = (uint64_t)t.gs[0] + x, gy = (uint64_t)t.gs[1] + y, gz = (uint64_t)t.gs[2] + z;
    if (COMPRESS) {
      T rec;
      int32_t code = quantize(t.at(x, y, z), pred, ebr, ebx2, &rec);
      t.at(x, y, z) = rec;
      if (t.owned(x, y, z)) qc[level_major_index(g, gx, gy, gz)] = code;
    } else {
      int32_t code = qc[level_major_index(g, gx, gy, gz)];
      t.at(x, y, z) = Fp<T>::fma(Fp<T>::from_int(code), ebx2, pred);
    }
  }
  // one per-axis sweep (interpolate_stage :1186-1386)
  __device__ void axis_stage(int axis, int u, int nxs, int xst, int xo, int nys, int yst, int yo,
                             int nzs, int zst, int zo, bool inclusive, bool nat) const {
    int total = nxs * nys * nzs;
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      int ii = i % nxs, jj = (i / nxs) % nys, kk = i / nxs / nys;
      int x = u * (ii * xst + xo), y = u * (jj * yst + yo), z = u * (kk * zst + zo);
      if (!t.pred_ok(x, y, z, inclusive)) continue;
      emit(x, y, z, pred_line(t, axis, x, y, z, u, false, nat));
    }
    __syncthreads();
  }
  // md stages (interpolate_stage_md :1388-1768) with the xyzmap_* point sets
  __device__ void md_stage(int kind, int u, bool inclusive, bool nat) const {
    int N = 16 / (2 * u);
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
      if (!t.pred_ok(x, y, z, inclusive)) continue;
      T pred;
      if (kind == 1) {
        int axis = (z % (2 * u)) ? 2 : ((y % (2 * u)) ? 1 : 0);
        pred = pred_line(t, axis, x, y, z, u, true, nat);
      } else if (kind == 2) {
        pred = pred_face(t, x, y, z, u, nat);
      } else {
        pred = pred_cube(t, x, y, z, u, nat);
      }
      emit(x, y, z, pred);
    }
    __syncthreads();
  }
};

// spline_layout_interpolate (:1771-2027)
template <class T, bool COMPRESS>
__device__ void run_levels(const TileCtx<T>& t, const Geometry& g, const PredParams<T>& p, int32_t* qc) {
  int level = 3;
  for (int u = 8; u >= 1; u >>= 1, --level) {
    if (level > p.maxlevel) continue;
    StageRunner<T, COMPRESS> r{t, g, qc, p.ebr[level], p.ebx2[level]};
    int N = 16 / (2 * u);
    bool last = level == 0;
    bool nat = p.natural[level];
    if (p.use_md[level]) {
      r.md_stage(1, u, true, nat);
      r.md_stage(2, u, true, nat);
      r.md_stage(3, u, !last, nat);
    } else if (p.reverse[level]) {
      r.axis_stage(0, u, N, 2, 1, N + 1, 2, 0, N + 1, 2, 0, true, nat);
      r.axis_stage(1, u, 2 * N + 1, 1, 0, N, 2, 1, N + 1, 2, 0, true, nat);
      r.axis_stage(2, u, 2 * N + 1, 1, 0, 2 * N + 1, 1, 0, N, 2, 1, !last, nat);
    } else {
      r.axis_stage(2, u, N + 1, 2, 0, N + 1, 2, 0, N, 2, 1, true, nat);
      r.axis_stage(1, u, N + 1, 2, 0, N, 2, 1, 2 * N + 1, 1, 0, true, nat);
      r.axis_stage(0, u, N, 2, 1, 2 * N + 1, 1, 0, 2 * N + 1, 1, 0, !last, nat);
    }
  }
}

constexpr int kPredThreads = 256;

// Compression: data -> anchors + level-major codes.
template <class T>
__global__ void __launch_bounds__(kPredThreads)
predict_compress_kernel(const T* __restrict__ data, Geometry g, const PredParams<T>* __restrict__ pp,
                        T* __restrict__ anchors, int32_t* __restrict__ qc) {
  __shared__ T win[kWinVol];
  __shared__ PredParams<T> p;
  uint32_t tile = blockIdx.x;
  TileCtx<T> t;
  t.s = win;
  uint32_t bi[3] = {tile % g.ax, (tile / g.ax) % g.ay, tile / g.ax / g.ay};
  uint32_t gd[3] = {g.ax, g.ay, g.az};
  t.dim[0] = g.nx; t.dim[1] = g.ny; t.dim[2] = g.nz;
#pragma unroll
  for (int d = 0; d < 3; ++d) { t.gs[d] = bi[d] * 16u; t.notlast[d] = bi[d] != gd[d] - 1; }
  if (threadIdx.x == 0) p = *pp;
  const uint64_t sy = g.nx, sz = (uint64_t)g.nx * g.ny;
  for (int i = threadIdx.x; i < kWinVol; i += blockDim.x) {
    int x = i % kWin, y = (i / kWin) % kWin, z = i / (kWin * kWin);
    T v = T(0);
    if (t.in_data(x, y, z))
      v = data[((uint64_t)t.gs[0] + x) + ((uint64_t)t.gs[1] + y) * sy + ((uint64_t)t.gs[2] + z) * sz];
    win[i] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) anchors[bi[0] + (uint64_t)bi[1] * g.ax + (uint64_t)bi[2] * g.ax * g.ay] = win[0];
  run_levels<T, true>(t, g, p, qc);
}

// Reconstruction: anchors + codes -> values; PROG adds the previous values
// (shmem2global_data_progressive :1123-1147).
template <class T, bool PROG>
__global__ void __launch_bounds__(kPredThreads)
reconstruct_kernel(const int32_t* __restrict__ qc, const T* __restrict__ anchors, Geometry g,
                   const PredParams<T>* __restrict__ pp, const T* old, T* out) {
  __shared__ T win[kWinVol];
  __shared__ PredParams<T> p;
  uint32_t tile = blockIdx.x;
  TileCtx<T> t;
  t.s = win;
  uint32_t bi[3] = {tile % g.ax, (tile / g.ax) % g.ay, tile / g.ax / g.ay};
  uint32_t gd[3] = {g.ax, g.ay, g.az};
  t.dim[0] = g.nx; t.dim[1] = g.ny; t.dim[2] = g.nz;
#pragma unroll
  for (int d = 0; d < 3; ++d) { t.gs[d] = bi[d] * 16u; t.notlast[d] = bi[d] != gd[d] - 1; }
  if (threadIdx.x == 0) p = *pp;
  for (int i = threadIdx.x; i < kWinVol; i += blockDim.x) win[i] = T(0);
  __syncthreads();
  if (threadIdx.x < 8) {  // x_reset_scratch_data (:1027-1067): anchors at the corners
    int x = (threadIdx.x & 1) * 16, y = ((threadIdx.x >> 1) & 1) * 16, z = (threadIdx.x >> 2) * 16;
    uint32_t ax = x / 16 + bi[0], ay = y / 16 + bi[1], az = z / 16 + bi[2];
    if (ax < g.ax && ay < g.ay && az < g.az) win[(z * kWin + y) * kWin + x] = anchors[ax + (uint64_t)ay * g.ax + (uint64_t)az * g.ax * g.ay];
  }
  __syncthreads();
  run_levels<T, false>(t, g, p, const_cast<int32_t*>(qc));
  const uint64_t sy = g.nx, sz = (uint64_t)g.nx * g.ny;
  int xs = 16 + !t.notlast[0], ys = 16 + !t.notlast[1], zs = 16 + !t.notlast[2];
  int total = xs * ys * zs;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    int x = i % xs, y = (i / xs) % ys, z = i / (xs * ys);
    if (!t.in_data(x, y, z)) continue;
    uint64_t gid = ((uint64_t)t.gs[0] + x) + ((uint64_t)t.gs[1] + y) * sy + ((uint64_t)t.gs[2] + z) * sz;
    T v = t.at(x, y, z);
    out[gid] = PROG ? Fp<T>::add(v, old[gid]) : v;
  }
}

}  // namespace prism_b200
