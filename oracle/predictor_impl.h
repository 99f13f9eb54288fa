/* Oracle predictor, instantiated for float and double by predictor.c --
 * TEST INFRASTRUCTURE ONLY.  Restates InterpolationPredictor.cu: one 16^3
 * tile at a time inside a 17^3 window, exactly the reference's stage order,
 * boundary cases and arithmetic (with the FP contraction chosen by or_policy).
 *
 * Expects: T, FN(x), FMA, FABS.
 */

/* ---- expression kernels with the reference's rounding (or_policy) ----
 * FN(ctx) selects per-context overrides: 0 none, 1 md line, 2 face, 3 cube */
static _Thread_local int FN(ctx) = 0;
static inline int FN(knob)(int base, int line, int face, int cube) {
  int v = FN(ctx) == 1 ? line : (FN(ctx) == 2 ? face : (FN(ctx) == 3 ? cube : -1));
  return v >= 0 ? v : base;
}
static inline T FN(cubic_md)(T a, T b, T c, T d, int natural) {
  /* nan_cubic_interp / nat_cubic_interp lambdas (:1811-1817, :738-744) */
  T s;
  if (!natural) {
    int k = FN(knob)(or_policy.cubic_md, or_policy.line_cubic, or_policy.face_cubic, or_policy.cube_cubic);
    if (k == 1) { s = FMA((T)9, b, -a); s = FMA((T)9, c, s); }
    else if (k == 2) { s = FMA((T)9, c, FMA((T)9, b, -a)); }
    else if (k == 3) { s = -a + (T)9 * b; s = FMA((T)9, c, s); }
    else if (k == 4) { s = FMA((T)9, b, -a); s = s + (T)9 * c; }
    else { s = -a + (T)9 * b; s = s + (T)9 * c; }
    s = s - d;
    return s / (T)16;
  }
  if (or_policy.cubic_md) {
    s = FMA((T)-3, a, (T)23 * b); s = FMA((T)23, c, s); s = FMA((T)-3, d, s);
  } else {
    s = (T)-3 * a + (T)23 * b; s = s + (T)23 * c; s = s - (T)3 * d;
  }
  return s / (T)40;
}

static inline T FN(cubic_axis)(T a, T b, T c, T d, int natural) {
  /* (p1*tmp0 + p2*tmp1 + p3*tmp2 + p4*tmp3) / p5 (:1248-1251, :1325) */
  T p1 = natural ? (T)-3 : (T)-1, p2 = natural ? (T)23 : (T)9;
  T p3 = p2, p4 = p1, p5 = natural ? (T)40 : (T)16;
  T s;
  switch (or_policy.cubic_axis) {
    case 1: s = FMA(p1, a, p2 * b); s = FMA(p3, c, s); s = FMA(p4, d, s); break;
    case 2: s = FMA(p2, b, p1 * a); s = FMA(p3, c, s); s = FMA(p4, d, s); break;
    default: s = p1 * a + p2 * b; s = s + p3 * c; s = s + p4 * d; break;
  }
  return s / p5;
}

static inline T FN(quad_l)(T t0, T t1, T t2) { /* (-t0 + 6 t1 + 3 t2) / 8 */
  T s;
  int k = FN(knob)(or_policy.quad_l, or_policy.line_quad_l, or_policy.face_quad_l, or_policy.cube_quad_l);
  if (k == 1) { s = FMA((T)6, t1, -t0); s = FMA((T)3, t2, s); }
  else if (k == 2) { s = -t0 + (T)6 * t1; s = FMA((T)3, t2, s); }
  else if (k == 3) { s = FMA((T)6, t1, -t0); s = s + (T)3 * t2; }
  else { s = -t0 + (T)6 * t1; s = s + (T)3 * t2; }
  return s / (T)8;
}

static inline T FN(quad_r)(T t1, T t2, T t3) { /* (3 t1 + 6 t2 - t3) / 8 */
  T s;
  switch (FN(knob)(or_policy.quad_r, or_policy.line_quad_r, or_policy.face_quad_r, or_policy.cube_quad_r)) {
    case 1: s = FMA((T)3, t1, (T)6 * t2); break;
    case 2: s = FMA((T)6, t2, (T)3 * t1); break;
    default: s = (T)3 * t1 + (T)6 * t2; break;
  }
  s = s - t3;
  return s / (T)8;
}

static inline T FN(recon)(T pred, T q, T ebx2) {
  return or_policy.recon ? FMA(q, ebx2, pred) : pred + q * ebx2;
}

/* CUDA's float->int conversion saturates and maps NaN to 0 (cvt.rzi.s32). */
static inline int32_t FN(to_i32)(T v) {
  if (v != v) return 0;
  if (v >= (T)2147483648.0) return INT32_MAX;
  if (v <= (T)-2147483648.0) return INT32_MIN;
  return (int32_t)v;
}

/* quantisation (:1330-1342): returns the stored code, updates *rec. */
static inline int32_t FN(quantize)(T orig, T pred, T eb_r, T ebx2, T* rec) {
  T err = orig - pred;
  T code = or_policy.quant ? FMA(FABS(err), eb_r, (T)1) : FABS(err) * eb_r + (T)1;
  code = err < 0 ? -code : code;
  int32_t qi = FN(to_i32)(code / (T)2); /* int(code / 2) + radius, radius = 0 */
  T qt = (T)qi;
  *rec = FN(recon)(pred, qt, ebx2);
  return FN(to_i32)(qt);
}

/* ---- tile context ---- */
typedef struct {
  T s[17][17][17]; /* [z][y][x] */
  const or_geom* g;
  uint32_t bi[3], gd[3]; /* block index / grid dim, [0]=x [1]=y [2]=z */
  int compress;
  const T* data;
  int32_t* ectrl_tmp;     /* compress: linear codes written here */
  const int32_t* qc;      /* decompress: level-major codes read from here */
  T eb_r, ebx2;           /* current level's bound (calc_eb) */
  const or_intp* p;
} FN(tile);

static inline T* FN(at)(FN(tile) * t, int x, int y, int z) { return &t->s[z][y][x]; }

static inline uint32_t FN(size_of)(const or_geom* g, int axis) {
  return axis == 0 ? g->nx : (axis == 1 ? g->ny : g->nz);
}

/* process one predicted point (compress or decompress workflow) */
static void FN(emit)(FN(tile) * t, int x, int y, int z, T pred) {
  const or_geom* g = t->g;
  uint64_t gx = (uint64_t)t->bi[0] * 16 + x, gy = (uint64_t)t->bi[1] * 16 + y,
           gz = (uint64_t)t->bi[2] * 16 + z;
  uint64_t gid = gx + gy * g->nx + gz * (uint64_t)g->nx * g->ny;
  if (t->compress) {
    T rec;
    int32_t code = FN(quantize)(t->s[z][y][x], pred, t->eb_r, t->ebx2, &rec);
    /* faces shared with the next tile are computed identically by both
     * tiles; only the owner stores, which keeps the OpenMP loop race-free */
    if ((x < 16 || t->bi[0] == t->gd[0] - 1) && (y < 16 || t->bi[1] == t->gd[1] - 1) &&
        (z < 16 || t->bi[2] == t->gd[2] - 1))
      t->ectrl_tmp[gid] = code;
    t->s[z][y][x] = rec;
  } else {
    int32_t code = t->qc[or_level_major_index(g, gx, gy, gz)];
    t->s[z][y][x] = FN(recon)(pred, (T)code, t->ebx2);
  }
}

static int FN(in_data)(FN(tile) * t, int x, int y, int z) {
  return (uint64_t)t->bi[0] * 16 + x < t->g->nx && (uint64_t)t->bi[1] * 16 + y < t->g->ny &&
         (uint64_t)t->bi[2] * 16 + z < t->g->nz;
}

/* xyz_predicate (:1173-1185) */
static int FN(pred_ok)(FN(tile) * t, int x, int y, int z, int inclusive) {
  if (inclusive) return x <= 16 && y <= 16 && z <= 16 && FN(in_data)(t, x, y, z);
  return x < 16 && y < 16 && z < 16 + (t->bi[2] == t->gd[2] - 1) && FN(in_data)(t, x, y, z);
}

static inline T FN(get)(FN(tile) * t, int axis, int x, int y, int z, int c) {
  if (axis == 0) return t->s[z][y][c];
  if (axis == 1) return t->s[z][c][x];
  return t->s[c][y][x];
}

/* 1-D prediction along `axis` with the per-axis boundary cases
 * (interpolate_stage :1300-1326; interpolate_stage_md LINE :1506-1535). */
static T FN(pred_line)(FN(tile) * t, int axis, int x, int y, int z, int u, int md, int natural) {
  int ix = axis == 0 ? x : (axis == 1 ? y : z);
  int id0 = ix - 3 * u >= 0 ? ix - 3 * u : 0;
  int id1 = ix - u >= 0 ? ix - u : 0;
  int id2 = ix + u < 17 ? ix + u : 0;
  int id3 = ix + 3 * u < 17 ? ix + 3 * u : 0;
  uint64_t gx = (uint64_t)t->bi[axis] * 16 + ix, gs = FN(size_of)(t->g, axis);
  int c1 = t->bi[axis] != t->gd[axis] - 1;
  int c2 = ix >= 3 * u, c3 = ix + 3 * u <= 16;
  int c4 = gx + 3 * u < gs, c5 = gx + u < gs;
  T t0 = FN(get)(t, axis, x, y, z, id0), t1 = FN(get)(t, axis, x, y, z, id1);
  T t2 = FN(get)(t, axis, x, y, z, id2), t3 = FN(get)(t, axis, x, y, z, id3);
  T pred = t1;
  if ((c1 && !c2 && !c3) || (!c1 && !c2 && !(c3 && c4) && c5)) pred = (t1 + t2) / (T)2;
  else if ((c1 && !c2 && c3) || (!c1 && !c2 && c3 && c4)) pred = FN(quad_r)(t1, t2, t3);
  else if ((c1 && c2 && !c3) || (!c1 && c2 && !(c3 && c4) && c5)) pred = FN(quad_l)(t0, t1, t2);
  else if ((c1 && c2 && c3) || (!c1 && c2 && c3 && c4))
    pred = md ? FN(cubic_md)(t0, t1, t2, t3, natural) : FN(cubic_axis)(t0, t1, t2, t3, natural);
  return pred;
}

/* get_interp_order (:1538-1545) */
static int FN(order)(FN(tile) * t, int axis, int c, int u) {
  uint64_t gx = (uint64_t)t->bi[axis] * 16 + c, gs = FN(size_of)(t->g, axis);
  int notlast = t->bi[axis] != t->gd[axis] - 1;
  int b = c >= 3 * u ? 3 : 1;
  int f = (c + 3 * u <= 16 && (notlast || gx + 3 * u < gs)) ? 3 : ((notlast || gx + u < gs) ? 1 : 0);
  return b == 3 ? (f == 3 ? 4 : (f == 1 ? 3 : 0)) : (f == 3 ? 2 : (f == 1 ? 1 : 0));
}

static inline int FN(idn)(int c, int u, int k) { /* id_z/id_y/id_x (:1426-1439) */
  switch (k) {
    case 0: return c - 3 * u >= 0 ? c - 3 * u : 0;
    case 1: return c - u >= 0 ? c - u : 0;
    case 2: return c + u <= 16 ? c + u : 0;
    default: return c + 3 * u <= 16 ? c + 3 * u : 0;
  }
}

/* FACE prediction (:1546-1668) */
static T FN(pred_face)(FN(tile) * t, int x, int y, int z, int u, int natural) {
  int a1, a2; /* dir1, dir2 axes */
  T pred;
  if (x % (2 * u) == 0) { a1 = 2; a2 = 1; pred = t->s[FN(idn)(z, u, 1)][FN(idn)(y, u, 1)][x]; }
  else if (y % (2 * u) == 0) { a1 = 2; a2 = 0; pred = t->s[FN(idn)(z, u, 1)][y][FN(idn)(x, u, 1)]; }
  else { a1 = 1; a2 = 0; pred = t->s[z][FN(idn)(y, u, 1)][FN(idn)(x, u, 1)]; }
  int c1 = a1 == 0 ? x : (a1 == 1 ? y : z), c2 = a2 == 0 ? x : (a2 == 1 ? y : z);
  T s1[4], s2[4];
  for (int k = 0; k < 4; ++k) {
    s1[k] = FN(get)(t, a1, x, y, z, FN(idn)(c1, u, k));
    s2[k] = FN(get)(t, a2, x, y, z, FN(idn)(c2, u, k));
  }
  int i1 = FN(order)(t, a1, c1, u), i2 = FN(order)(t, a2, c2, u);
  if (i1 == 4 && i2 == 4)
    pred = (FN(cubic_md)(s1[0], s1[1], s1[2], s1[3], natural) +
            FN(cubic_md)(s2[0], s2[1], s2[2], s2[3], natural)) / (T)2;
  else if (i1 != 4 && i2 == 4) pred = FN(cubic_md)(s2[0], s2[1], s2[2], s2[3], natural);
  else if (i1 == 4 && i2 != 4) pred = FN(cubic_md)(s1[0], s1[1], s1[2], s1[3], natural);
  else if (i1 == 3 && i2 == 3) { pred = FN(quad_l)(s2[0], s2[1], s2[2]); pred += FN(quad_l)(s1[0], s1[1], s1[2]); pred /= (T)2; }
  else if (i1 == 3 && i2 == 2) { pred = FN(quad_r)(s2[1], s2[2], s2[3]); pred += FN(quad_l)(s1[0], s1[1], s1[2]); pred /= (T)2; }
  else if (i1 == 3 && i2 < 2) pred = FN(quad_l)(s1[0], s1[1], s1[2]);
  else if (i1 == 2 && i2 == 3) { pred = FN(quad_r)(s1[1], s1[2], s1[3]); pred += FN(quad_l)(s2[0], s2[1], s2[2]); pred /= (T)2; }
  else if (i1 == 2 && i2 == 2) { pred = FN(quad_r)(s1[1], s1[2], s1[3]); pred += FN(quad_r)(s2[1], s2[2], s2[3]); pred /= (T)2; }
  else if (i1 == 2 && i2 < 2) pred = FN(quad_r)(s1[1], s1[2], s1[3]);
  else if (i1 <= 1 && i2 == 3) pred = FN(quad_l)(s2[0], s2[1], s2[2]);
  else if (i1 <= 1 && i2 == 2) pred = FN(quad_r)(s2[1], s2[2], s2[3]);
  else if (i1 == 1 && i2 == 1) { pred = (s2[1] + s2[2]) / (T)2; pred += (s1[1] + s1[2]) / (T)2; pred /= (T)2; }
  else if (i1 == 1 && i2 < 1) pred = (s1[1] + s1[2]) / (T)2;
  else if (i1 == 0 && i2 == 1) pred = (s2[1] + s2[2]) / (T)2;
  else pred = s1[1] + s2[1] - pred;
  return pred;
}

/* CUBE prediction (:1671-1723) */
static T FN(pred_cube)(FN(tile) * t, int x, int y, int z, int u, int natural) {
  int oz = FN(order)(t, 2, z, u), oy = FN(order)(t, 1, y, u), ox = FN(order)(t, 0, x, u);
  T tx[4], ty[4] = {0, 0, 0, 0}, tz[4] = {0, 0, 0, 0};
  for (int k = 0; k < 4; ++k) tx[k] = t->s[z][y][FN(idn)(x, u, k)];
  if (oz == 4) for (int k = 0; k < 4; ++k) tz[k] = t->s[FN(idn)(z, u, k)][y][x];
  if (oy == 4) for (int k = 0; k < 4; ++k) ty[k] = t->s[z][FN(idn)(y, u, k)][x];
  T px0 = tx[1];
  T pred = px0;
  if (oz == 4 && oy == 4 && ox == 4)
    pred = (FN(cubic_md)(tx[0], tx[1], tx[2], tx[3], natural) + FN(cubic_md)(ty[0], ty[1], ty[2], ty[3], natural) +
            FN(cubic_md)(tz[0], tz[1], tz[2], tz[3], natural)) / (T)3;
  else if (oz == 4 && oy == 4) pred = (FN(cubic_md)(tz[0], tz[1], tz[2], tz[3], natural) + FN(cubic_md)(ty[0], ty[1], ty[2], ty[3], natural)) / (T)2;
  else if (oz == 4 && ox == 4) pred = (FN(cubic_md)(tz[0], tz[1], tz[2], tz[3], natural) + FN(cubic_md)(tx[0], tx[1], tx[2], tx[3], natural)) / (T)2;
  else if (oy == 4 && ox == 4) pred = (FN(cubic_md)(ty[0], ty[1], ty[2], ty[3], natural) + FN(cubic_md)(tx[0], tx[1], tx[2], tx[3], natural)) / (T)2;
  else if (oz == 4) pred = FN(cubic_md)(tz[0], tz[1], tz[2], tz[3], natural);
  else if (oy == 4) pred = FN(cubic_md)(ty[0], ty[1], ty[2], ty[3], natural);
  else if (ox == 4) pred = FN(cubic_md)(tx[0], tx[1], tx[2], tx[3], natural);
  else if (ox == 3) pred = FN(quad_l)(tx[0], tx[1], tx[2]);
  else if (ox == 2) pred = FN(quad_r)(tx[1], tx[2], tx[3]);
  else if (ox == 1) pred = (tx[1] + tx[2]) / (T)2;
  return pred;
}

/* per-axis sweep stage (interpolate_stage :1186-1386): the point set is the
 * product of three index maps; `axis` is the sweep axis */
static void FN(stage_axis)(FN(tile) * t, int axis, int u, int nxs, int xstep, int xoff, int nys,
                           int ystep, int yoff, int nzs, int zstep, int zoff, int inclusive,
                           int natural) {
  for (int k = 0; k < nzs; ++k)
    for (int j = 0; j < nys; ++j)
      for (int i = 0; i < nxs; ++i) {
        int x = u * (i * xstep + xoff), y = u * (j * ystep + yoff), z = u * (k * zstep + zoff);
        if (!FN(pred_ok)(t, x, y, z, inclusive)) continue;
        FN(emit)(t, x, y, z, FN(pred_line)(t, axis, x, y, z, u, 0, natural));
      }
}

/* multi-dimensional stages (interpolate_stage_md :1388-1768) */
static void FN(stage_md)(FN(tile) * t, int kind /*1 line,2 face,3 cube*/, int u, int inclusive,
                         int natural) {
  for (int z = 0; z <= 16; z += u)
    for (int y = 0; y <= 16; y += u)
      for (int x = 0; x <= 16; x += u) {
        int ox = (x / u) & 1, oy = (y / u) & 1, oz = (z / u) & 1;
        if (ox + oy + oz != kind) continue;
        if (!FN(pred_ok)(t, x, y, z, inclusive)) continue;
        T pred;
        FN(ctx) = kind;
        if (kind == 1) {
          int axis = oz ? 2 : (oy ? 1 : 0);
          pred = FN(pred_line)(t, axis, x, y, z, u, 1, natural);
        } else if (kind == 2) {
          pred = FN(pred_face)(t, x, y, z, u, natural);
        } else {
          pred = FN(pred_cube)(t, x, y, z, u, natural);
        }
        FN(ctx) = 0;
        FN(emit)(t, x, y, z, pred);
      }
}

/* spline_layout_interpolate (:1771-2027) */
static void FN(layout)(FN(tile) * t, T eb_r, T ebx2, int maxlevel) {
  const or_intp* p = t->p;
  int level_id = 3;
  for (int unit = 8; unit >= 1; unit /= 2, level_id--) {
    if (level_id > maxlevel) continue;
    /* calc_eb (:1825-1839): FP values scaled by the double alpha/beta */
    T cur_ebx2 = ebx2, cur_eb_r = eb_r;
    for (int temp = 1; temp < unit; temp *= 2) {
      cur_eb_r = (T)((double)cur_eb_r * p->alpha);
      cur_ebx2 = (T)((double)cur_ebx2 / p->alpha);
    }
    if ((double)cur_ebx2 < (double)ebx2 / p->beta) {
      cur_ebx2 = (T)((double)ebx2 / p->beta);
      cur_eb_r = (T)((double)eb_r * p->beta);
    }
    t->eb_r = cur_eb_r;
    t->ebx2 = cur_ebx2;
    int N = 16 / (unit * 2);
    int last = level_id == 0; /* the last stage of level 0 is border-exclusive */
    int nat = p->use_natural[level_id];
    if (p->use_md[level_id]) {
      FN(stage_md)(t, 1, unit, 1, nat);
      FN(stage_md)(t, 2, unit, 1, nat);
      FN(stage_md)(t, 3, unit, !last, nat);
    } else if (p->reverse[level_id]) {
      /* hollow_reverse, yellow_reverse, blue_reverse (:1892-1913) */
      FN(stage_axis)(t, 0, unit, N, 2, 1, N + 1, 2, 0, N + 1, 2, 0, 1, nat);
      FN(stage_axis)(t, 1, unit, 2 * N + 1, 1, 0, N, 2, 1, N + 1, 2, 0, 1, nat);
      FN(stage_axis)(t, 2, unit, 2 * N + 1, 1, 0, 2 * N + 1, 1, 0, N, 2, 1, !last, nat);
    } else {
      /* blue, yellow, hollow (:1915-1936) */
      FN(stage_axis)(t, 2, unit, N + 1, 2, 0, N + 1, 2, 0, N, 2, 1, 1, nat);
      FN(stage_axis)(t, 1, unit, N + 1, 2, 0, N, 2, 1, 2 * N + 1, 1, 0, 1, nat);
      FN(stage_axis)(t, 0, unit, N, 2, 1, 2 * N + 1, 1, 0, 2 * N + 1, 1, 0, !last, nat);
    }
  }
}

static void FN(tile_init)(FN(tile) * t, const or_geom* g, uint32_t bx, uint32_t by, uint32_t bz) {
  memset(t->s, 0, sizeof(t->s));
  t->g = g;
  t->bi[0] = bx; t->bi[1] = by; t->bi[2] = bz;
  t->gd[0] = g->ax; t->gd[1] = g->ay; t->gd[2] = g->az;
}

/* interpolation kernel (:2137-2173) over all tiles */
void FN(or_predict)(const T* data, const or_geom* g, double eb, const or_intp* p, T* anchors,
                    int32_t* qc, int32_t* ectrl_tmp) {
  T ebx2 = (T)(eb * 2), eb_r = (T)(1 / eb);
  int64_t ntiles = (int64_t)g->ax * g->ay * g->az;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t tix = 0; tix < ntiles; ++tix) {
    FN(tile)* t = (FN(tile)*)malloc(sizeof(FN(tile)));
    uint32_t bx = (uint32_t)(tix % g->ax), by = (uint32_t)((tix / g->ax) % g->ay),
             bz = (uint32_t)(tix / g->ax / g->ay);
    FN(tile_init)(t, g, bx, by, bz);
    t->compress = 1; t->data = data; t->ectrl_tmp = ectrl_tmp; t->p = p;
    for (int z = 0; z < 17; ++z)
      for (int y = 0; y < 17; ++y)
        for (int x = 0; x < 17; ++x)
          if (FN(in_data)(t, x, y, z)) {
            uint64_t gid = (uint64_t)bx * 16 + x + ((uint64_t)by * 16 + y) * g->nx +
                           ((uint64_t)bz * 16 + z) * (uint64_t)g->nx * g->ny;
            t->s[z][y][x] = data[gid];
          }
    anchors[bx + (uint64_t)by * g->ax + (uint64_t)bz * g->ax * g->ay] = t->s[0][0][0];
    FN(layout)(t, eb_r, ebx2, 4);
    free(t);
  }
  /* shmem2global_data_with_compaction (:2028-2088): owned points -> qc */
#pragma omp parallel for schedule(static)
  for (int64_t gz = 0; gz < g->nz; ++gz)
    for (uint64_t gy = 0; gy < g->ny; ++gy)
      for (uint64_t gx = 0; gx < g->nx; ++gx) {
        uint64_t gid = gx + gy * g->nx + (uint64_t)gz * g->nx * g->ny;
        qc[or_level_major_index(g, gx, gy, (uint64_t)gz)] = ectrl_tmp[gid];
      }
}

/* interpolation_reverse / interpolation_progressive_reverse (:2177-2239) */
void FN(or_reconstruct)(const int32_t* qc, const T* anchors, const or_geom* g, double eb,
                        const or_intp* p, int maxlevel, const T* old, T* out) {
  T ebx2 = (T)(eb * 2), eb_r = (T)(1 / eb);
  int64_t ntiles = (int64_t)g->ax * g->ay * g->az;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t tix = 0; tix < ntiles; ++tix) {
    FN(tile)* t = (FN(tile)*)malloc(sizeof(FN(tile)));
    uint32_t bx = (uint32_t)(tix % g->ax), by = (uint32_t)((tix / g->ax) % g->ay),
             bz = (uint32_t)(tix / g->ax / g->ay);
    FN(tile_init)(t, g, bx, by, bz);
    t->compress = 0; t->qc = qc; t->p = p;
    /* x_reset_scratch_data (:1027-1067): zeros plus the anchors */
    for (int z = 0; z <= 16; z += 16)
      for (int y = 0; y <= 16; y += 16)
        for (int x = 0; x <= 16; x += 16) {
          uint64_t ax = x / 16 + bx, ay = y / 16 + by, az = z / 16 + bz;
          if (ax < g->ax && ay < g->ay && az < g->az)
            t->s[z][y][x] = anchors[ax + ay * g->ax + az * (uint64_t)g->ax * g->ay];
        }
    FN(layout)(t, eb_r, ebx2, maxlevel);
    /* shmem2global_data[_progressive] (:1097-1147): the tile's own points */
    int xs = 16 + (bx == g->ax - 1), ys = 16 + (by == g->ay - 1), zs = 16 + (bz == g->az - 1);
    for (int z = 0; z < zs; ++z)
      for (int y = 0; y < ys; ++y)
        for (int x = 0; x < xs; ++x) {
          uint64_t gx = (uint64_t)bx * 16 + x, gy = (uint64_t)by * 16 + y, gz = (uint64_t)bz * 16 + z;
          if (gx < g->nx && gy < g->ny && gz < g->nz) {
            uint64_t gid = gx + gy * g->nx + gz * (uint64_t)g->nx * g->ny;
            out[gid] = old ? t->s[z][y][x] + old[gid] : t->s[z][y][x];
          }
        }
    free(t);
  }
}

/* ======================= auto-tuning (:110-967) ======================= */

typedef struct {
  T s[17][17][17];
  uint32_t gs[3];     /* sample tile start (uint32 wrap-around) */
  uint32_t size[3];
} FN(att);

static int FN(att_in)(FN(att) * a, int x, int y, int z) {
  return (uint32_t)(a->gs[0] + x) < a->size[0] && (uint32_t)(a->gs[1] + y) < a->size[1] &&
         (uint32_t)(a->gs[2] + z) < a->size[2];
}

static inline T FN(att_get)(FN(att) * a, int axis, int x, int y, int z, int c) {
  if (axis == 0) return a->s[z][y][c];
  if (axis == 1) return a->s[z][c][x];
  return a->s[c][y][x];
}

/* interpolate_stage_att / LINE of interpolate_stage_md_att (:221-317, :554-651) */
static T FN(att_line)(FN(att) * a, int axis, int x, int y, int z, int u, int md, int natural) {
  int ix = axis == 0 ? x : (axis == 1 ? y : z);
  int id0 = ix - 3 * u >= 0 ? ix - 3 * u : 0, id1 = ix - u >= 0 ? ix - u : 0;
  int id2 = ix + u < 17 ? ix + u : 0, id3 = ix + 3 * u < 17 ? ix + 3 * u : 0;
  uint32_t gstart = a->gs[axis], gsz = a->size[axis];
  uint32_t gx = gstart + (uint32_t)ix;
  int c1 = gstart + 16u < gsz, c2 = ix >= 3 * u, c3 = ix + 3 * u <= 16;
  int c4 = gx + 3u * u < gsz, c5 = gx + (uint32_t)u < gsz;
  T t0 = FN(att_get)(a, axis, x, y, z, id0), t1 = FN(att_get)(a, axis, x, y, z, id1);
  T t2 = FN(att_get)(a, axis, x, y, z, id2), t3 = FN(att_get)(a, axis, x, y, z, id3);
  T pred = t1;
  if ((c1 && !c2 && !c3) || (!c1 && !c2 && !(c3 && c4) && c5)) pred = (t1 + t2) / (T)2;
  else if ((c1 && !c2 && c3) || (!c1 && !c2 && c3 && c4)) pred = FN(quad_r)(t1, t2, t3);
  else if ((c1 && c2 && !c3) || (!c1 && c2 && !(c3 && c4) && c5)) pred = FN(quad_l)(t0, t1, t2);
  else if ((c1 && c2 && c3) || (!c1 && c2 && c3 && c4))
    pred = md ? FN(cubic_md)(t0, t1, t2, t3, natural) : FN(cubic_axis)(t0, t1, t2, t3, natural);
  return pred;
}

static int FN(att_order)(FN(att) * a, int axis, int c, int u) { /* :318-325 */
  uint32_t gx = a->gs[axis] + (uint32_t)c, gsz = a->size[axis];
  int b = c >= 3 * u ? 3 : 1;
  int f = (c + 3 * u <= 16 && gx + 3u * u < gsz) ? 3 : ((gx + (uint32_t)u < gsz) ? 1 : 0);
  return b == 3 ? (f == 3 ? 4 : (f == 1 ? 3 : 0)) : (f == 3 ? 2 : (f == 1 ? 1 : 0));
}

static T FN(att_face)(FN(att) * a, int x, int y, int z, int u, int natural) { /* :326-442 */
  int a1, a2;
  T pred;
  if (x % (2 * u) == 0) { a1 = 2; a2 = 1; pred = a->s[FN(idn)(z, u, 1)][FN(idn)(y, u, 1)][x]; }
  else if (y % (2 * u) == 0) { a1 = 2; a2 = 0; pred = a->s[FN(idn)(z, u, 1)][y][FN(idn)(x, u, 1)]; }
  else { a1 = 1; a2 = 0; pred = a->s[z][FN(idn)(y, u, 1)][FN(idn)(x, u, 1)]; }
  int c1 = a1 == 0 ? x : (a1 == 1 ? y : z), c2 = a2 == 0 ? x : (a2 == 1 ? y : z);
  T s1[4], s2[4];
  for (int k = 0; k < 4; ++k) {
    s1[k] = FN(att_get)(a, a1, x, y, z, FN(idn)(c1, u, k));
    s2[k] = FN(att_get)(a, a2, x, y, z, FN(idn)(c2, u, k));
  }
  int i1 = FN(att_order)(a, a1, c1, u), i2 = FN(att_order)(a, a2, c2, u);
  if (i1 == 4 && i2 == 4)
    pred = (FN(cubic_md)(s1[0], s1[1], s1[2], s1[3], natural) + FN(cubic_md)(s2[0], s2[1], s2[2], s2[3], natural)) / (T)2;
  else if (i1 != 4 && i2 == 4) pred = FN(cubic_md)(s2[0], s2[1], s2[2], s2[3], natural);
  else if (i1 == 4 && i2 != 4) pred = FN(cubic_md)(s1[0], s1[1], s1[2], s1[3], natural);
  else if (i1 == 3 && i2 == 3) { pred = FN(quad_l)(s2[0], s2[1], s2[2]); pred += FN(quad_l)(s1[0], s1[1], s1[2]); pred /= (T)2; }
  else if (i1 == 3 && i2 == 2) { pred = FN(quad_r)(s2[1], s2[2], s2[3]); pred += FN(quad_l)(s1[0], s1[1], s1[2]); pred /= (T)2; }
  else if (i1 == 3 && i2 < 2) pred = FN(quad_l)(s1[0], s1[1], s1[2]);
  else if (i1 == 2 && i2 == 3) { pred = FN(quad_r)(s1[1], s1[2], s1[3]); pred += FN(quad_l)(s2[0], s2[1], s2[2]); pred /= (T)2; }
  else if (i1 == 2 && i2 == 2) { pred = FN(quad_r)(s1[1], s1[2], s1[3]); pred += FN(quad_r)(s2[1], s2[2], s2[3]); pred /= (T)2; }
  else if (i1 == 2 && i2 < 2) pred = FN(quad_r)(s1[1], s1[2], s1[3]);
  else if (i1 <= 1 && i2 == 3) pred = FN(quad_l)(s2[0], s2[1], s2[2]);
  else if (i1 <= 1 && i2 == 2) pred = FN(quad_r)(s2[1], s2[2], s2[3]);
  else if (i1 == 1 && i2 == 1) { pred = (s2[1] + s2[2]) / (T)2; pred += (s1[1] + s1[2]) / (T)2; pred /= (T)2; }
  else if (i1 == 1 && i2 < 1) pred = (s1[1] + s1[2]) / (T)2;
  else if (i1 == 0 && i2 == 1) pred = (s2[1] + s2[2]) / (T)2;
  else pred = s1[1] + s2[1] - pred;
  return pred;
}

static T FN(att_cube)(FN(att) * a, int x, int y, int z, int u, int natural) { /* :444-498 */
  int oz = FN(att_order)(a, 2, z, u), oy = FN(att_order)(a, 1, y, u), ox = FN(att_order)(a, 0, x, u);
  T tx[4], ty[4] = {0, 0, 0, 0}, tz[4] = {0, 0, 0, 0};
  for (int k = 0; k < 4; ++k) tx[k] = a->s[z][y][FN(idn)(x, u, k)];
  if (oz == 4) for (int k = 0; k < 4; ++k) tz[k] = a->s[FN(idn)(z, u, k)][y][x];
  if (oy == 4) for (int k = 0; k < 4; ++k) ty[k] = a->s[z][FN(idn)(y, u, k)][x];
  T pred = tx[1];
  if (oz == 4 && oy == 4 && ox == 4)
    pred = (FN(cubic_md)(tx[0], tx[1], tx[2], tx[3], natural) + FN(cubic_md)(ty[0], ty[1], ty[2], ty[3], natural) +
            FN(cubic_md)(tz[0], tz[1], tz[2], tz[3], natural)) / (T)3;
  else if (oz == 4 && oy == 4) pred = (FN(cubic_md)(tz[0], tz[1], tz[2], tz[3], natural) + FN(cubic_md)(ty[0], ty[1], ty[2], ty[3], natural)) / (T)2;
  else if (oz == 4 && ox == 4) pred = (FN(cubic_md)(tz[0], tz[1], tz[2], tz[3], natural) + FN(cubic_md)(tx[0], tx[1], tx[2], tx[3], natural)) / (T)2;
  else if (oy == 4 && ox == 4) pred = (FN(cubic_md)(ty[0], ty[1], ty[2], ty[3], natural) + FN(cubic_md)(tx[0], tx[1], tx[2], tx[3], natural)) / (T)2;
  else if (oz == 4) pred = FN(cubic_md)(tz[0], tz[1], tz[2], tz[3], natural);
  else if (oy == 4) pred = FN(cubic_md)(ty[0], ty[1], ty[2], ty[3], natural);
  else if (ox == 4) pred = FN(cubic_md)(tx[0], tx[1], tx[2], tx[3], natural);
  else if (ox == 3) pred = FN(quad_l)(tx[0], tx[1], tx[2]);
  else if (ox == 2) pred = FN(quad_r)(tx[1], tx[2], tx[3]);
  else if (ox == 1) pred = (tx[1] + tx[2]) / (T)2;
  return pred;
}

static int FN(att_ok)(FN(att) * a, int x, int y, int z) { /* xyz_predicate_att, inclusive */
  return x <= 16 && y <= 16 && z <= 16 && FN(att_in)(a, x, y, z);
}

/* one level of spline_layout_interpolate_att (:704-878): returns sum |x - pred| */
static T FN(att_level)(FN(att) * a, int level, int use_md, int reverse, int natural) {
  int u = 1 << level, N = 16 / (u * 2);
  T err = 0;
  if (use_md) {
    for (int kind = 1; kind <= 3; ++kind)
      for (int z = 0; z <= 16; z += u)
        for (int y = 0; y <= 16; y += u)
          for (int x = 0; x <= 16; x += u) {
            int ox = (x / u) & 1, oy = (y / u) & 1, oz = (z / u) & 1;
            if (ox + oy + oz != kind || !FN(att_ok)(a, x, y, z)) continue;
            T pred = kind == 1 ? FN(att_line)(a, oz ? 2 : (oy ? 1 : 0), x, y, z, u, 1, natural)
                               : (kind == 2 ? FN(att_face)(a, x, y, z, u, natural)
                                            : FN(att_cube)(a, x, y, z, u, natural));
            err += FABS(a->s[z][y][x] - pred);
          }
    return err;
  }
  /* per-axis sweeps; same point sets as the main path */
  int st[3][10];
  if (reverse) {
    int v[3][10] = {{0, N, 2, 1, N + 1, 2, 0, N + 1, 2, 0},
                    {1, 2 * N + 1, 1, 0, N, 2, 1, N + 1, 2, 0},
                    {2, 2 * N + 1, 1, 0, 2 * N + 1, 1, 0, N, 2, 1}};
    memcpy(st, v, sizeof(v));
  } else {
    int v[3][10] = {{2, N + 1, 2, 0, N + 1, 2, 0, N, 2, 1},
                    {1, N + 1, 2, 0, N, 2, 1, 2 * N + 1, 1, 0},
                    {0, N, 2, 1, 2 * N + 1, 1, 0, 2 * N + 1, 1, 0}};
    memcpy(st, v, sizeof(v));
  }
  for (int s = 0; s < 3; ++s) {
    int axis = st[s][0];
    for (int k = 0; k < st[s][7]; ++k)
      for (int j = 0; j < st[s][4]; ++j)
        for (int i = 0; i < st[s][1]; ++i) {
          int x = u * (i * st[s][2] + st[s][3]), y = u * (j * st[s][5] + st[s][6]),
              z = u * (k * st[s][8] + st[s][9]);
          if (!FN(att_ok)(a, x, y, z)) continue;
          T pred = FN(att_line)(a, axis, x, y, z, u, 0, natural);
          err += FABS(a->s[z][y][x] - pred);
        }
  }
  return err;
}

/* Per-axis candidate sample starts with uint32 wrap (:2277-2289): indices idx
 * in [0, size) whose start (s_start + 128*idx mod 2^32) lies inside [0, dim). */
static int FN(att_axis_candidates)(uint32_t dim, uint32_t s_start, uint32_t s_size,
                                   uint32_t* idx_out, int cap) {
  int cnt = 0;
  for (uint64_t k = 0; k < 3; ++k) {
    uint64_t lo = k << 32; /* need s_start + 128 idx in [lo, lo + dim) */
    int64_t first = ((int64_t)lo - (int64_t)s_start + 127) / 128;
    if ((int64_t)lo - (int64_t)s_start < 0) first = 0;
    for (int64_t i = first; i < (int64_t)s_size; ++i) {
      uint64_t v = (uint64_t)s_start + 128ull * (uint64_t)i;
      if (v >= lo + dim) break;
      if (v >= lo && cnt < cap) idx_out[cnt++] = (uint32_t)i;
    }
  }
  return cnt;
}

void FN(or_autotune)(const T* data, const or_geom* g, double eb, double rel_eb, const or_intp* in,
                     T errors[18]) {
  (void)eb; (void)rel_eb; (void)in;
  for (int i = 0; i < 18; ++i) errors[i] = 0;
  uint32_t dims[3] = {g->nx, g->ny, g->nz};
  uint32_t s_start[3], s_size[3];
  for (int d = 0; d < 3; ++d) { /* calc_start_size with unsigned arithmetic */
    uint32_t dim = dims[d], mid = dim / 2;
    uint32_t k = (mid - 8u) / 128u;
    uint32_t t = (dim - 8u - 1u - mid) / 128u;
    s_start[d] = mid - k * 128u;
    s_size[d] = k + t + 1u;
  }
  int32_t block_num = (int32_t)(s_size[0] * s_size[1] * s_size[2]);
  if (block_num <= 0) return; /* the launch is rejected; sums stay 0 */
  static const int CAP = 4096;
  uint32_t* cand[3];
  int nc[3];
  for (int d = 0; d < 3; ++d) {
    cand[d] = (uint32_t*)malloc(sizeof(uint32_t) * CAP);
    nc[d] = FN(att_axis_candidates)(dims[d], s_start[d], s_size[d], cand[d], CAP);
  }
  FN(att)* a = (FN(att)*)malloc(sizeof(FN(att)));
  for (int iz = 0; iz < nc[2]; ++iz)
    for (int iy = 0; iy < nc[1]; ++iy)
      for (int ix = 0; ix < nc[0]; ++ix) {
        uint64_t bix = cand[0][ix] + (uint64_t)s_size[0] * (cand[1][iy] + (uint64_t)s_size[1] * cand[2][iz]);
        if (bix >= (uint64_t)(uint32_t)block_num) continue;
        memset(a->s, 0, sizeof(a->s));
        a->size[0] = dims[0]; a->size[1] = dims[1]; a->size[2] = dims[2];
        a->gs[0] = s_start[0] + cand[0][ix] * 128u;
        a->gs[1] = s_start[1] + cand[1][iy] * 128u;
        a->gs[2] = s_start[2] + cand[2][iz] * 128u;
        for (int z = 0; z < 17; ++z)
          for (int y = 0; y < 17; ++y)
            for (int x = 0; x < 17; ++x)
              if (FN(att_in)(a, x, y, z)) {
                uint64_t gid = (uint64_t)(a->gs[0] + x) + (uint64_t)(a->gs[1] + y) * g->nx +
                               (uint64_t)(a->gs[2] + z) * (uint64_t)g->nx * g->ny;
                a->s[z][y][x] = data[gid];
              }
        /* BIY = 0: levels 3 and 2 (:900-935) */
        errors[0] += FN(att_level)(a, 3, 0, 0, 0);
        errors[1] += FN(att_level)(a, 3, 0, 1, 0);
        errors[2] += FN(att_level)(a, 3, 1, 1, 0);
        errors[3] += FN(att_level)(a, 2, 0, 0, 0);
        errors[4] += FN(att_level)(a, 2, 0, 1, 0);
        errors[5] += FN(att_level)(a, 2, 1, 1, 0);
        /* BIY = 1, 2: level 1, natural for BIY = 2 (:936-953) */
        for (int biy = 1; biy <= 2; ++biy) {
          int nat = biy == 2;
          errors[3 + biy * 3 + 0] += FN(att_level)(a, 1, 0, 0, nat);
          errors[3 + biy * 3 + 1] += FN(att_level)(a, 1, 0, 1, nat);
          errors[3 + biy * 3 + 2] += FN(att_level)(a, 1, 1, 1, nat);
        }
        /* BIY = 3..5: level 0 (:955-961, pre_compute_att :130-134) */
        for (int biy = 3; biy <= 5; ++biy)
          errors[9 + biy] += FN(att_level)(a, 0, biy == 5, biy % 3 != 0, 0);
      }
  free(a);
  for (int d = 0; d < 3; ++d) free(cand[d]);
}

void FN(or_decide)(const T errors[18], or_intp* p) { /* :2306-2355 */
  T best;
  int idx;
  if (errors[0] > errors[1]) { best = errors[1]; p->reverse[3] = 1; }
  else { best = errors[0]; p->reverse[3] = 0; }
  p->use_md[3] = errors[2] < best;
  if (errors[3] > errors[4]) { best = errors[4]; p->reverse[2] = 1; }
  else { best = errors[3]; p->reverse[2] = 0; }
  p->use_md[2] = errors[5] < best;
  best = errors[6]; idx = 6;
  for (int i = 6; i < 12; ++i) if (errors[i] < best) { best = errors[i]; idx = i; }
  p->use_md[1] = idx == 8 || idx == 11;
  p->reverse[1] = idx % 3 != 0;
  best = errors[12]; idx = 12;
  for (int i = 12; i < 15; ++i) if (errors[i] < best) { best = errors[i]; idx = i; }
  p->use_md[0] = idx == 14;
  p->reverse[0] = idx % 3 != 0;
}
