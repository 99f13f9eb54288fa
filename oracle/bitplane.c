/* Oracle bit-plane shuffle -- TEST INFRASTRUCTURE ONLY (see prism_oracle.h).
 * Lane-by-lane emulation of bitplane.cu: the 8-lane warp-shuffle/byte_perm
 * transpose, the per-block position bookkeeping (including the last block's
 * element count, bitplane.cu:200-260) and the device plane placement
 * (bitplane.cu:142-154).  Blocks are applied in launch order, so writes of
 * the last block land last. */
#include <string.h>
#include "prism_oracle.h"

#define CS 16384
#define TPB 512

/* __byte_perm(x, y, s): byte i of the result = byte ((s >> 4i) & 7) of {y:x} */
static uint32_t byte_perm(uint32_t x, uint32_t y, uint32_t s) {
  uint64_t v = ((uint64_t)y << 32) | x;
  uint32_t r = 0;
  for (int i = 0; i < 4; ++i) {
    uint32_t sel = (s >> (4 * i)) & 7;
    r |= (uint32_t)((v >> (8 * sel)) & 0xFF) << (8 * i);
  }
  return r;
}

/* byte-level exchange: bitplane.cu:112-124 (forward) == :328-340 (inverse) */
static void byte_steps(uint32_t a[8]) {
  uint32_t q[8];
  for (int l = 0; l < 8; ++l) q[l] = a[l ^ 4];
  for (int l = 0; l < 8; ++l)
    a[l] = (l & 4) == 0 ? byte_perm(a[l], q[l], (3 << 12) | (2 << 8) | (7 << 4) | 6)
                        : byte_perm(a[l], q[l], (5 << 12) | (4 << 8) | (1 << 4) | 0);
  for (int l = 0; l < 8; ++l) q[l] = a[l ^ 2];
  for (int l = 0; l < 8; ++l)
    a[l] = (l & 2) == 0 ? byte_perm(a[l], q[l], (3 << 12) | (7 << 8) | (1 << 4) | 5)
                        : byte_perm(a[l], q[l], (6 << 12) | (2 << 8) | (4 << 4) | 0);
  for (int l = 0; l < 8; ++l) q[l] = a[l ^ 1];
  const uint32_t mask = 0x0F0F0F0F;
  for (int l = 0; l < 8; ++l)
    a[l] = (l & 1) == 0 ? (a[l] & ~mask) | ((q[l] >> 4) & mask)
                        : ((q[l] << 4) & ~mask) | (a[l] & mask);
}

static uint32_t bit_steps_fwd(uint32_t a) { /* :126-131 */
  uint32_t q;
  q = (a ^ (a >> 3)) & 0x0A0A0A0AU; a = a ^ q ^ (q << 3);
  q = (a ^ (a >> 6)) & 0x00CC00CCU; a = a ^ q ^ (q << 6);
  q = (a ^ (a >> 12)) & 0x0000F0F0U; a = a ^ q ^ (q << 12);
  return a;
}

static uint32_t bit_steps_inv(uint32_t a) { /* :321-326 */
  uint32_t q;
  q = (a ^ (a >> 12)) & 0x0000F0F0U; a = a ^ q ^ (q << 12);
  q = (a ^ (a >> 6)) & 0x00CC00CCU; a = a ^ q ^ (q << 6);
  q = (a ^ (a >> 3)) & 0x0A0A0A0AU; a = a ^ q ^ (q << 3);
  return a;
}

void or_shuffle_network(const uint32_t in[8], uint32_t out[8]) {
  uint32_t a[8];
  memcpy(a, in, sizeof(a));
  byte_steps(a);
  for (int l = 0; l < 8; ++l) out[l] = bit_steps_fwd(a[l]);
}

static void inverse_network(uint32_t a[8]) {
  for (int l = 0; l < 8; ++l) a[l] = bit_steps_inv(a[l]);
  byte_steps(a);
}

static uint32_t to_planes_word(int32_t code, int bt) { /* :102-111 */
  uint32_t a = (uint32_t)code;
  if (bt == 0) return (a + 0xaaaaaaaau) ^ 0xaaaaaaaau; /* NB */
  uint32_t sign = (uint32_t)(((int32_t)a) >> 31);
  return (a & 0x7FFFFFFF) ^ sign; /* SM */
}

static int32_t from_planes_word(uint32_t a, int bt) { /* :387-392 */
  if (bt == 0) return (int32_t)((a ^ 0xaaaaaaaau) - 0xaaaaaaaau);
  uint32_t sign = (uint32_t)(((int32_t)a) >> 31);
  return (int32_t)((a & 0x7FFFFFFF) ^ sign);
}

/* byte offset of plane 4*(idx&7) for code index c (:143-149) */
static int64_t place(const or_geom* g, int64_t c, int* level_out) {
  int level = 0;
  while (c < g->dprefix[level]) ++level;
  int64_t idx = c - g->dprefix[level];
  *level_out = level;
  return (idx >> 3) + g->dstride[level] * ((idx & 7) << 2) + g->daprefix[level];
}

static void write_word(uint8_t* planes, const or_geom* g, int64_t c, uint32_t a) {
  int level;
  int64_t s = place(g, c, &level);
  int64_t st = g->dstride[level];
  planes[s] = (uint8_t)(a >> 24);
  planes[s + st] = (uint8_t)(a >> 8);
  planes[s + 2 * st] = (uint8_t)(a >> 16);
  planes[s + 3 * st] = (uint8_t)a;
}

/* The 8-lane network with some lanes inactive: an inactive lane keeps 0 in
 * its register and the active lanes read that 0 from it.  The reference's
 * last block runs the network under __activemask() (bitplane.cu:220-240);
 * what an inactive source lane returns is undefined in CUDA, zero is the value
 * its register holds.  Inactive lanes output 0. */
static void network_partial(const uint32_t in[8], const int act[8], uint32_t out[8]) {
  uint32_t a[8], q[8];
  for (int l = 0; l < 8; ++l) a[l] = act[l] ? in[l] : 0;
  for (int l = 0; l < 8; ++l) q[l] = act[l ^ 4] ? a[l ^ 4] : 0;
  for (int l = 0; l < 8; ++l)
    if (act[l]) a[l] = (l & 4) == 0 ? byte_perm(a[l], q[l], (3 << 12) | (2 << 8) | (7 << 4) | 6)
                                    : byte_perm(a[l], q[l], (5 << 12) | (4 << 8) | (1 << 4) | 0);
  for (int l = 0; l < 8; ++l) q[l] = act[l ^ 2] ? a[l ^ 2] : 0;
  for (int l = 0; l < 8; ++l)
    if (act[l]) a[l] = (l & 2) == 0 ? byte_perm(a[l], q[l], (3 << 12) | (7 << 8) | (1 << 4) | 5)
                                    : byte_perm(a[l], q[l], (6 << 12) | (2 << 8) | (4 << 4) | 0);
  for (int l = 0; l < 8; ++l) q[l] = act[l ^ 1] ? a[l ^ 1] : 0;
  const uint32_t mask = 0x0F0F0F0F;
  for (int l = 0; l < 8; ++l)
    if (act[l]) a[l] = (l & 1) == 0 ? (a[l] & ~mask) | ((q[l] >> 4) & mask)
                                    : ((q[l] << 4) & ~mask) | (a[l] & mask);
  for (int l = 0; l < 8; ++l) out[l] = act[l] ? bit_steps_fwd(a[l]) : 0;
}

/* Per-thread element count of the last shuffle block: `align` is a local
 * that d_comput updates in thread 0 only (bitplane.cu:32-57, 90-91), so
 * res = align + tail for thread 0 and res = tail for every other thread. */
static int64_t last_res(const or_geom* g, int t) {
  int64_t tail = (int64_t)(g->n % CS);
  if (tail == 0) tail = CS;
  return tail + (t == 0 ? g->align_dev : 0);
}

/* Order of the last block's writes relative to the others where they overlap
 * (its zero bytes can spill into the first bytes of the next level-0 plane,
 * which another block writes): 1 = last block lands last, 0 = first,
 * -1 = decide like a B200 schedules the reference launch.  With more blocks
 * than fit at once (148 SMs x 4 CTAs of 512 threads) the last block starts
 * after the first wave has finished.  Otherwise all blocks run together and
 * the order follows the loop iteration in which each side writes those bytes. */
int or_shuffle_last_block_last = -1;

static int last_block_lands_last(const or_geom* g) {
  if (or_shuffle_last_block_last >= 0) return or_shuffle_last_block_last;
  if (g->sh_grid > 148 * 4) return 1;
  int64_t tail = (int64_t)(g->n % CS);
  if (tail == 0) tail = CS;
  int64_t it_last = (tail + 511) / 512 - 1;         /* zero-tail iteration */
  int64_t it_first = (g->dprefix[0] % CS) / TPB;    /* level-0 start writes */
  return it_first <= it_last;
}

static void last_block_fwd(const int32_t* in, const or_geom* g, int bt, uint8_t* planes);

void or_bitshuffle(const int32_t* qc, const or_geom* g, int bt, uint8_t* planes) {
  const int32_t* in = qc + g->anchors;
  int lbl = last_block_lands_last(g);
  if (!lbl) last_block_fwd(in, g, bt, planes);
  for (int64_t b = 0; b + 1 < g->sh_grid; ++b) {
    int64_t start = b * CS;
    for (int64_t base = 0; base < CS; base += 8) {
      uint32_t w[8], o[8];
      for (int l = 0; l < 8; ++l) w[l] = to_planes_word(in[start + base + l], bt);
      or_shuffle_network(w, o);
      for (int l = 0; l < 8; ++l) write_word(planes, g, start + base + l, o[l]);
    }
  }
  if (lbl) last_block_fwd(in, g, bt, planes);
}

/* last block (bitplane.cu:200-260), thread by thread */
static void last_block_fwd(const int32_t* in, const or_geom* g, int bt, uint8_t* planes) {
  int64_t start = (g->sh_grid - 1) * CS;
  int64_t res[TPB], ares[TPB], maxa = 0;
  for (int t = 0; t < TPB; ++t) {
    res[t] = last_res(g, t);
    ares[t] = (res[t] + 511) / 512 * 512;
    if (ares[t] > maxa) maxa = ares[t];
  }
  static uint32_t shm[TPB];
  memset(shm, 0, sizeof(shm));
  for (int64_t base = 0; base < maxa; base += TPB) {
    for (int grp = 0; grp < TPB / 8; ++grp) {
      uint32_t w[8], o[8];
      int act[8], part[8];
      for (int l = 0; l < 8; ++l) {
        int t = grp * 8 + l;
        part[l] = base < ares[t];
        act[l] = part[l] && base + t < res[t];
        w[l] = act[l] ? to_planes_word(in[start + base + t], bt) : 0;
      }
      network_partial(w, act, o);
      for (int l = 0; l < 8; ++l)
        if (part[l]) shm[grp * 8 + l] = o[l];
    }
    for (int t = 0; t < TPB; ++t) {
      if (base >= ares[t]) continue;
      int write_pos = ((t & 63) << 3) + (t >> 6);
      if (write_pos < res[t]) write_word(planes, g, start + base + write_pos, shm[write_pos]);
    }
  }
}

static uint32_t gather_word(const uint8_t* planes, const or_geom* g, int64_t c, const int* begin,
                            const int* end) {
  int level;
  int64_t s = place(g, c, &level);
  int64_t st = g->dstride[level];
  int lane = (int)(((c - g->dprefix[level]) & 7) << 2);
  uint32_t v = 0;
  int lo = 0, hi = 32;
  if (begin) { lo = begin[3 - level]; hi = end[3 - level]; }
  if (lo < hi) {
    if (lane >= lo && lane < hi) v |= (uint32_t)planes[s] << 24;
    if (lane + 1 >= lo && lane + 1 < hi) v |= (uint32_t)planes[s + st] << 8;
    if (lane + 2 >= lo && lane + 2 < hi) v |= (uint32_t)planes[s + 2 * st] << 16;
    if (lane + 3 >= lo && lane + 3 < hi) v |= (uint32_t)planes[s + 3 * st];
  }
  return v;
}

/* Inverse network with lanes that left the loop: they are modelled as
 * supplying 0 to the xor-shuffles (bitplane.cu:403-448 shuffles with a full
 * mask after some lanes exited -- undefined in CUDA). */
static void inverse_network_partial(uint32_t a[8], const int act[8]) {
  for (int l = 0; l < 8; ++l) a[l] = act[l] ? bit_steps_inv(a[l]) : 0;
  uint32_t q[8];
  for (int l = 0; l < 8; ++l) q[l] = act[l ^ 4] ? a[l ^ 4] : 0;
  for (int l = 0; l < 8; ++l)
    if (act[l]) a[l] = (l & 4) == 0 ? byte_perm(a[l], q[l], (3 << 12) | (2 << 8) | (7 << 4) | 6)
                                    : byte_perm(a[l], q[l], (5 << 12) | (4 << 8) | (1 << 4) | 0);
  for (int l = 0; l < 8; ++l) q[l] = act[l ^ 2] ? a[l ^ 2] : 0;
  for (int l = 0; l < 8; ++l)
    if (act[l]) a[l] = (l & 2) == 0 ? byte_perm(a[l], q[l], (3 << 12) | (7 << 8) | (1 << 4) | 5)
                                    : byte_perm(a[l], q[l], (6 << 12) | (2 << 8) | (4 << 4) | 0);
  for (int l = 0; l < 8; ++l) q[l] = act[l ^ 1] ? a[l ^ 1] : 0;
  const uint32_t mask = 0x0F0F0F0F;
  for (int l = 0; l < 8; ++l)
    if (act[l]) a[l] = (l & 1) == 0 ? (a[l] & ~mask) | ((q[l] >> 4) & mask)
                                    : ((q[l] << 4) & ~mask) | (a[l] & mask);
}

/* shared by the full and the plane-masked inverse */
static void inverse_impl(const uint8_t* planes, const or_geom* g, int bt, const int* begin,
                         const int* end, int32_t* qc) {
  int32_t* out = qc + g->anchors;
  for (int64_t b = 0; b + 1 < g->sh_grid; ++b) {
    int64_t start = b * CS;
    for (int64_t base = 0; base < CS; base += 8) {
      uint32_t a[8];
      for (int l = 0; l < 8; ++l) a[l] = gather_word(planes, g, start + base + l, begin, end);
      inverse_network(a);
      for (int l = 0; l < 8; ++l) out[start + base + l] = from_planes_word(a[l], bt);
    }
  }
  /* last block: thread t handles positions t, t+512, ... below its res */
  int64_t start = (g->sh_grid - 1) * CS;
  int64_t res[TPB], maxr = 0;
  for (int t = 0; t < TPB; ++t) { res[t] = last_res(g, t); if (res[t] > maxr) maxr = res[t]; }
  for (int64_t base = 0; base < maxr; base += TPB) {
    for (int grp = 0; grp < TPB / 8; ++grp) {
      uint32_t a[8];
      int act[8], any = 0;
      for (int l = 0; l < 8; ++l) {
        int t = grp * 8 + l;
        act[l] = base + t < res[t];
        any |= act[l];
        a[l] = act[l] ? gather_word(planes, g, start + base + t, begin, end) : 0;
      }
      if (!any) continue;
      inverse_network_partial(a, act);
      for (int l = 0; l < 8; ++l)
        if (act[l]) out[start + base + grp * 8 + l] = from_planes_word(a[l], bt);
    }
  }
}

void or_inverse_bitshuffle(const uint8_t* planes, const or_geom* g, int bt, int32_t* qc) {
  inverse_impl(planes, g, bt, NULL, NULL, qc);
}

void or_inverse_bitshuffle_progressive(const uint8_t* planes, const or_geom* g,
                                       const int begin[4], const int end[4], int32_t* qc) {
  inverse_impl(planes, g, 0, begin, end, qc);
}
