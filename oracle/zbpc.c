/* Oracle ZBPC lossless coder -- TEST INFRASTRUCTURE ONLY (see prism_oracle.h).
 * Restates RZE.hpp:10-167 for byte words (zero elimination + three levels of
 * repetition elimination on the bitmaps), the raw fallback of
 * zbpc.cu:222-243, the chunk walk of zbpc.cu:185-262 and the stream layout
 * (int64 size, uint16 chunk sizes, chunk payloads, pad to 8; zbpc.cu:179-181,
 * 255-260, 513-516). */
#include <stdlib.h>
#include <string.h>
#include "prism_oracle.h"

#define CS 16384

/* repetition elimination (d_repetition_elimination.hpp): keep byte i iff it
 * differs from byte i-1 (byte -1 == 0); bitmap bit i (LSB first) marks kept */
static int re_encode(const uint8_t* in, int n, uint8_t* out, uint8_t* bm) {
  int cnt = 0;
  memset(bm, 0, (size_t)(n + 7) / 8);
  for (int i = 0; i < n; ++i) {
    uint8_t prev = i == 0 ? 0 : in[i - 1];
    if (in[i] != prev) { bm[i / 8] |= (uint8_t)(1u << (i % 8)); out[cnt++] = in[i]; }
  }
  return cnt;
}

static int re_decode(const uint8_t* data, const uint8_t* bm, int n, uint8_t* out) {
  int j = 0;
  for (int i = 0; i < n; ++i) {
    if ((bm[i / 8] >> (i % 8)) & 1) out[i] = data[j++];
    else out[i] = i == 0 ? 0 : out[i - 1];
  }
  return j;
}

static int popcount_bytes(const uint8_t* b, int n) {
  int c = 0;
  for (int i = 0; i < n; ++i) c += __builtin_popcount(b[i]);
  return c;
}

int or_zbpc_encode_chunk(const uint8_t* in, int osize, uint8_t* out) {
  uint8_t bm0[2048], bm1[256], bm2[32], bm3[4];
  uint8_t* tmp = (uint8_t*)malloc(CS + 64);
  /* zero elimination (d_ZEencodebyteshort): nonzero bytes + bitmap */
  memset(bm0, 0, sizeof(bm0));
  int nz = 0;
  for (int i = 0; i < osize; ++i)
    if (in[i]) { bm0[i / 8] |= (uint8_t)(1u << (i % 8)); tmp[nz++] = in[i]; }
  int csize;
  if (nz == 0) {
    out[0] = (uint8_t)osize; out[1] = (uint8_t)(osize >> 8); /* RZE.hpp:79-84 */
    free(tmp);
    return 2;
  }
  uint8_t k1[2048], k2[256], k3[32];
  int c1 = re_encode(bm0, 2048, k1, bm1);
  int c2 = re_encode(bm1, 256, k2, bm2);
  int c3 = re_encode(bm2, 32, k3, bm3);
  csize = nz + c1 + c2 + c3 + 4 + 2;
  if (csize >= osize) { /* raw fallback (zbpc.cu:230) */
    memcpy(out, in, (size_t)osize);
    free(tmp);
    return osize;
  }
  int w = 0;
  memcpy(out + w, tmp, (size_t)nz); w += nz;
  memcpy(out + w, k1, (size_t)c1); w += c1;
  memcpy(out + w, k2, (size_t)c2); w += c2;
  memcpy(out + w, k3, (size_t)c3); w += c3;
  memcpy(out + w, bm3, 4); w += 4;
  out[w++] = (uint8_t)osize;
  out[w++] = (uint8_t)(osize >> 8);
  free(tmp);
  return csize;
}

int or_zbpc_decode_chunk(const uint8_t* in, int csize, int osize, uint8_t* out) {
  if (csize == osize) { memcpy(out, in, (size_t)osize); return 0; }
  if (csize < 2) return -1;
  int rpos = csize - 2;
  int orig = in[rpos] | (in[rpos + 1] << 8);
  if (orig != osize) return -2;
  if (rpos == 0) { memset(out, 0, (size_t)osize); return 0; }
  uint8_t bm0[2048], bm1[256], bm2[32], bm3[4];
  if (rpos < 4) return -3;
  rpos -= 4;
  memcpy(bm3, in + rpos, 4);
  int c3 = popcount_bytes(bm3, 4);
  if (rpos < c3) return -3;
  rpos -= c3;
  re_decode(in + rpos, bm3, 32, bm2);
  int c2 = popcount_bytes(bm2, 32);
  if (rpos < c2) return -3;
  rpos -= c2;
  re_decode(in + rpos, bm2, 256, bm1);
  int c1 = popcount_bytes(bm1, 256);
  if (rpos < c1) return -3;
  rpos -= c1;
  re_decode(in + rpos, bm1, 2048, bm0);
  int j = 0;
  for (int i = 0; i < osize; ++i) {
    if ((bm0[i / 8] >> (i % 8)) & 1) {
      if (j >= rpos) return -4;
      out[i] = in[j++];
    } else {
      out[i] = 0;
    }
  }
  return 0;
}

/* chunk -> (host level, plane, offset) walk of zbpc.cu:191-206 */
static void chunk_locate(const or_geom* g, int64_t id, int* l_out, int64_t* bp_id,
                         int64_t* bp_off, int64_t* base, int* osize) {
  int64_t real = id;
  int l = 3;
  while (real >= g->chunks_level[l]) real -= g->chunks_level[l--];
  int64_t cpp = g->chunks_level[l] >> 5;
  *bp_id = real / cpp;
  *bp_off = real % cpp;
  int64_t b = 0;
  for (int i = 3; i > l; --i) b += g->hastride[i] << 5;
  b += *bp_id * g->hastride[l] + *bp_off * CS;
  *base = b;
  int64_t rem = g->hastride[l] - *bp_off * CS;
  *osize = (int)(rem < CS ? rem : CS);
  *l_out = l;
}

uint64_t or_zbpc_encode(const uint8_t* planes, const or_geom* g, uint8_t* out,
                        uint64_t comp_size_bp[128]) {
  int64_t chunks = g->chunks;
  uint16_t* sizes = (uint16_t*)(out + 8);
  uint8_t* data = out + 8 + 2 * chunks;
  uint64_t off = 0;
  for (int64_t id = 0; id < chunks; ++id) {
    int l; int64_t bp_id, bp_off, base; int osize;
    chunk_locate(g, id, &l, &bp_id, &bp_off, &base, &osize);
    int cs = or_zbpc_encode_chunk(planes + base, osize, data + off);
    sizes[id] = (uint16_t)cs;
    off += (uint64_t)cs;
    if (bp_off == (g->chunks_level[l] >> 5) - 1) comp_size_bp[(3 - l) * 32 + bp_id] = off;
  }
  int64_t hdr = (int64_t)g->aligned_size;
  memcpy(out, &hdr, 8);
  uint64_t total = 8 + 2 * (uint64_t)chunks + off;
  uint64_t pad = (8 - total % 8) % 8;
  memset(out + total, 0, pad);
  return total + pad;
}

static int decode_impl(const uint8_t* stream, const or_geom* g, const int* begin, const int* end,
                       uint8_t* planes) {
  int64_t chunks = g->chunks;
  const uint16_t* sizes = (const uint16_t*)(stream + 8);
  const uint8_t* data = stream + 8 + 2 * chunks;
  uint64_t off = 0;
  for (int64_t id = 0; id < chunks; ++id) {
    int l; int64_t bp_id, bp_off, base; int osize;
    chunk_locate(g, id, &l, &bp_id, &bp_off, &base, &osize);
    int cs = sizes[id];
    if (begin) { /* zbpc.cu:420-423 */
      int64_t cpp = g->chunks_level[l] >> 5;
      int64_t real = bp_id * cpp + bp_off;
      if (real < begin[3 - l] * cpp || real >= end[3 - l] * cpp) { off += (uint64_t)cs; continue; }
    }
    int rc = or_zbpc_decode_chunk(data + off, cs, osize, planes + base);
    if (rc) return rc;
    off += (uint64_t)cs;
  }
  return 0;
}

int or_zbpc_decode(const uint8_t* stream, const or_geom* g, uint8_t* planes) {
  return decode_impl(stream, g, NULL, NULL, planes);
}

int or_zbpc_decode_progressive(const uint8_t* stream, const or_geom* g, const int begin[4],
                               const int end[4], uint8_t* planes) {
  return decode_impl(stream, g, begin, end, planes);
}
