/* Oracle pipeline for one value type -- TEST INFRASTRUCTURE ONLY.
 * Restates Compressor::compress_pipeline / decompress_pipeline /
 * decompress_progressive_pipeline (src/compressor.cu:120-226) and the
 * container trailer (compress_merge :139-151, decompress_scatter :192-210).
 * Expects T, FN(x). */

/* code buffer: n codes plus the slack the reference reads/writes past its end */
static int32_t* FN(alloc_qc)(const or_geom* g) {
  size_t cnt = g->n + g->anchors + 2 * 16384 + 64;
  return (int32_t*)calloc(cnt, sizeof(int32_t));
}

static uint8_t* FN(alloc_planes)(const or_geom* g) {
  return (uint8_t*)calloc(g->aligned_size + (1u << 20), 1);
}

uint64_t FN(or_compress)(const T* data, uint32_t nx, uint32_t ny, uint32_t nz, int mode,
                         double bound, int bt, const or_intp* force, uint8_t* out, or_intp* used,
                         T errors[18]) {
  or_geom g;
  or_geometry(nx, ny, nz, (int)sizeof(T), &g);
  double range = 1.0, eb, rel_eb;
  if (mode == 1) { /* REL: StatBuffer::findMinMax (compressor.hpp:23-31) */
    T mn = data[0], mx = data[0];
    for (uint64_t i = 1; i < g.n; ++i) { mn = data[i] < mn ? data[i] : mn; mx = data[i] > mx ? data[i] : mx; }
    range = (double)mx - (double)mn;
    eb = bound * range;
    rel_eb = bound;
  } else {
    eb = bound;
    rel_eb = 0;
  }
  or_intp p;
  or_intp_default(&p);
  p.alpha = or_alpha(rel_eb);
  p.beta = 4.0;
  T err[18];
  FN(or_autotune)(data, &g, eb, rel_eb, &p, err);
  if (errors) memcpy(errors, err, sizeof(err));
  if (force) {
    memcpy(p.use_md, force->use_md, 4);
    memcpy(p.reverse, force->reverse, 4);
  } else {
    FN(or_decide)(err, &p);
  }
  if (used) *used = p;
  T* anchors = (T*)calloc(g.anchors, sizeof(T));
  int32_t* qc = FN(alloc_qc)(&g);
  uint8_t* planes = FN(alloc_planes)(&g);
  /* the predictor's linear scratch is the plane buffer (compressor.cu:328) */
  FN(or_predict)(data, &g, eb, &p, anchors, qc, (int32_t*)planes);
  or_bitshuffle(qc, &g, bt, planes);
  uint64_t csbp[128];
  uint64_t lossless = or_zbpc_encode(planes, &g, out, csbp);
  uint8_t* tr = out + lossless; /* compress_merge */
  memcpy(tr, p.use_md, 4);
  memcpy(tr + 4, p.reverse, 4);
  memcpy(tr + 8, &range, 8);
  memcpy(tr + 16, csbp, 1024);
  memcpy(tr + 1040, anchors, g.anchors * sizeof(T));
  free(anchors); free(qc); free(planes);
  return lossless + g.header_size;
}

static int FN(parse)(const uint8_t* cont, uint64_t size, const or_geom* g, or_intp* p,
                     double* range, uint64_t csbp[128], const uint8_t** anchors) {
  if (size < g->header_size + 8) return -10;
  const uint8_t* tr = cont + (size - g->header_size);
  or_intp_default(p);
  memcpy(p->use_md, tr, 4);
  memcpy(p->reverse, tr + 4, 4);
  memcpy(range, tr + 8, 8);
  memcpy(csbp, tr + 16, 1024);
  *anchors = tr + 1040;
  return 0;
}

int FN(or_decompress)(const uint8_t* cont, uint64_t size, uint32_t nx, uint32_t ny, uint32_t nz,
                      int mode, double bound, T* out) {
  or_geom g;
  or_geometry(nx, ny, nz, (int)sizeof(T), &g);
  or_intp p; double range; uint64_t csbp[128]; const uint8_t* ap;
  int rc = FN(parse)(cont, size, &g, &p, &range, csbp, &ap);
  if (rc) return rc;
  double eb = mode == 1 ? bound * range : bound;
  p.alpha = or_alpha(mode == 1 ? bound : 0);
  p.beta = 4.0;
  uint8_t* planes = FN(alloc_planes)(&g);
  rc = or_zbpc_decode(cont, &g, planes);
  if (rc) { free(planes); return rc; }
  int32_t* qc = FN(alloc_qc)(&g);
  or_inverse_bitshuffle(planes, &g, 1, qc);
  T* anchors = (T*)malloc(g.anchors * sizeof(T));
  memcpy(anchors, ap, g.anchors * sizeof(T));
  FN(or_reconstruct)(qc, anchors, &g, eb, &p, 4, NULL, out);
  free(anchors); free(qc); free(planes);
  return 0;
}

static int FN(progressive_step_impl)(const uint8_t* cont, uint64_t size, uint32_t nx, uint32_t ny,
                                     uint32_t nz, int mode, double bound, double target, double last,
                                     int begin[4], int end[4], int* maxlevel, const T* old, T* out,
                                     int exact) {
  or_geom g;
  or_geometry(nx, ny, nz, (int)sizeof(T), &g);
  or_intp p; double range; uint64_t csbp[128]; const uint8_t* ap;
  int rc = FN(parse)(cont, size, &g, &p, &range, csbp, &ap);
  if (rc) return rc;
  int first = last == 0;
  double eb = bound;
  if (mode == 1) { eb = bound * range; target *= range; }
  p.alpha = or_alpha(mode == 1 ? bound : 0);
  p.beta = 4.0;
  or_find_strategy(csbp, eb, target, begin, end, maxlevel);
  uint8_t* planes = FN(alloc_planes)(&g);
  int dec_begin[4];
  for (int i = 0; i < 4; ++i) dec_begin[i] = exact && begin[i] > 0 && begin[i] < end[i] ? begin[i] - 1 : begin[i];
  rc = or_zbpc_decode_progressive(cont, &g, dec_begin, end, planes);
  if (rc) { free(planes); return rc; }
  int32_t* qc = FN(alloc_qc)(&g);
  or_inverse_bitshuffle_progressive(planes, &g, begin, end, qc);
  T* anchors = (T*)calloc(g.anchors, sizeof(T));
  if (first) memcpy(anchors, ap, g.anchors * sizeof(T)); /* decompress_scatter<1> */
  FN(or_reconstruct)(qc, anchors, &g, eb, &p, *maxlevel, first ? NULL : old, out);
  free(anchors); free(qc); free(planes);
  return 0;
}

int FN(or_progressive_step)(const uint8_t* cont, uint64_t size, uint32_t nx, uint32_t ny,
                            uint32_t nz, int mode, double bound, double target, double last,
                            int begin[4], int end[4], int* maxlevel, const T* old, T* out) {
  return FN(progressive_step_impl)(cont, size, nx, ny, nz, mode, bound, target, last, begin, end, maxlevel, old,
                                   out, 0);
}

int FN(or_progressive_step_exact)(const uint8_t* cont, uint64_t size, uint32_t nx, uint32_t ny,
                                  uint32_t nz, int mode, double bound, double target, double last,
                                  int begin[4], int end[4], int* maxlevel, const T* old, T* out) {
  return FN(progressive_step_impl)(cont, size, nx, ny, nz, mode, bound, target, last, begin, end, maxlevel, old,
                                   out, 1);
}
