/* CPU oracle for the PRISM compression hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's algorithm (BingluCS/PRISM), stage
 * by stage, used by tests/ (as the checker), __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py.  Product code never links or calls it.
 * Every function cites the reference file:line it restates.
 *
 * Parity status: pinned against stage dumps of the reference build run on a
 * B200 (tests/golden/, produced by tests/golden/make_golden.py).
 */
#ifndef PRISM_ORACLE_H
#define PRISM_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- geometry (io.hpp:104-132, io.cu:117-127,
 *                   bitplane.cu:10-53, InterpolationPredictor.cu:969-995) */
typedef struct {
  uint32_t nx, ny, nz;
  uint64_t n;
  uint32_t ax, ay, az;            /* anchor grid (stride 16)               */
  uint64_t anchors;
  uint64_t leaps[5][2];           /* pre_compute grid_leaps                */
  uint64_t lm_prefix[5];          /* pre_compute prefix_nums (level-major) */
  int64_t dprefix[5];             /* d_comput prefix_nums (code space)     */
  int64_t align_dev;
  int64_t dstride[4];             /* device plane stride (bytes) / level   */
  int64_t daprefix[4];            /* byte offset of each level's planes    */
  int64_t hprefix[5];             /* h_comput prefix_nums                  */
  int64_t align_host;
  int64_t hstride[4];             /* host strides (bytes)                  */
  int64_t hastride[4];            /* host aligned strides (x8)             */
  uint64_t aligned_size;          /* plane buffer bytes = sum 32*hastride  */
  uint64_t aligned_len;           /* n + align_host                        */
  int64_t sh_grid;                /* bitShuffle grid                        */
  int64_t sh_res;                 /* codes in its last block                */
  int64_t chunks_level[4];        /* zbpc chunks per host level (x32)       */
  int64_t chunks;
  uint64_t header_size;           /* trailer bytes (needs dtype size)       */
} or_geom;

void or_geometry(uint32_t nx, uint32_t ny, uint32_t nz, int tsize, or_geom* g);
uint64_t or_level_major_index(const or_geom* g, uint64_t gx, uint64_t gy, uint64_t gz);

/* ---------------- interpolation parameters (parameters.hpp:8-24) */
typedef struct {
  double alpha, beta;
  uint8_t use_md[4];
  uint8_t use_natural[4];
  uint8_t reverse[4];
} or_intp;

void or_intp_default(or_intp* p);
double or_alpha(double rel_eb); /* InterpolationPredictor.cu:2248-2271 */

/* FP contraction policy of the reference build.  Each knob
 * selects how one expression of the reference is rounded.  0 = every
 * operation rounded separately; other values = a specific fused pattern. */
typedef struct {
  int quant;      /* fabs(err)*eb_r + 1           (:1335, :1731)            */
  int recon;      /* pred + q*ebx2                (:1342, :1349, :1738,:1746)*/
  int cubic_md;   /* (-a+9b+9c-d)/16              (:1811-1813)              */
  int cubic_axis; /* (p1 a + p2 b + p3 c + p4 d)/p5 (:1325)                  */
  int quad_l;     /* (-t0 + 6 t1 + 3 t2)/8        (:1322, :1528, ...)       */
  int quad_r;     /* (3 t1 + 6 t2 - t3)/8         (:1319, :1531, ...)       */
  int att;        /* same knobs applied inside the auto-tune kernel         */
  /* per-context overrides (-1 = use the base knob): md LINE, FACE, CUBE */
  int line_cubic, line_quad_l, line_quad_r;
  int face_cubic, face_quad_l, face_quad_r;
  int cube_cubic, cube_quad_l, cube_quad_r;
} or_fp_policy;

extern or_fp_policy or_policy;          /* process-wide, default = pinned */
void or_set_policy(const or_fp_policy* p);
void or_get_policy(or_fp_policy* p);

/* ---------------- predictor (InterpolationPredictor.cu) */
/* Auto-tune error sums (:880-967) over the sample grid (:2273-2299),
 * including the uint32/int wrap-around of the sample-grid arithmetic.
 * errors[18] receives the sums (T precision, deterministic order). */
void or_autotune_f32(const float* data, const or_geom* g, double eb, double rel_eb,
                     const or_intp* in, float errors[18]);
void or_autotune_f64(const double* data, const or_geom* g, double eb, double rel_eb,
                     const or_intp* in, double errors[18]);
/* Host decisions from the sums (:2306-2355). */
void or_decide_f32(const float errors[18], or_intp* p);
void or_decide_f64(const double errors[18], or_intp* p);

/* Compression kernel (:2137-2173): fills anchors, level-major codes qc
 * (n + slack entries, zero-initialised by the caller) and the linear scratch
 * ectrl_tmp (int32[n], zero-initialised by the caller). */
void or_predict_f32(const float* data, const or_geom* g, double eb, const or_intp* p,
                    float* anchors, int32_t* qc, int32_t* ectrl_tmp);
void or_predict_f64(const double* data, const or_geom* g, double eb, const or_intp* p,
                    double* anchors, int32_t* qc, int32_t* ectrl_tmp);
/* Reconstruction (:2177-2207) and progressive reconstruction (:2209-2239).
 * old == NULL selects the full reconstruction. */
void or_reconstruct_f32(const int32_t* qc, const float* anchors, const or_geom* g, double eb,
                        const or_intp* p, int maxlevel, const float* old, float* out);
void or_reconstruct_f64(const int32_t* qc, const double* anchors, const or_geom* g, double eb,
                        const or_intp* p, int maxlevel, const double* old, double* out);

/* ---------------- bit-plane shuffle (bitplane.cu) */
/* bt: 0 = NB (negabinary), 1 = SM (sign-magnitude) -- traits.hpp:108-112 */
/* Forward (bitplane.cu:61-253, launcher :604-622): reads qc+anchors, writes
 * `planes` (aligned_size bytes, pre-filled by the caller with the predictor's
 * scratch bytes, exactly as the reference reuses that buffer). */
void or_bitshuffle(const int32_t* qc, const or_geom* g, int bt, uint8_t* planes);
extern int or_shuffle_last_block_last;
/* Inverse (:262-430) -> qc+anchors codes. */
void or_inverse_bitshuffle(const uint8_t* planes, const or_geom* g, int bt, int32_t* qc);
/* Progressive inverse, NB only (:433-601). */
void or_inverse_bitshuffle_progressive(const uint8_t* planes, const or_geom* g,
                                       const int begin[4], const int end[4], int32_t* qc);
/* Lane-exact emulation of the 8-lane shuffle network (:112-131) for one group
 * of 8 transformed codes -> 8 words (test hook). */
void or_shuffle_network(const uint32_t in[8], uint32_t out[8]);

/* ---------------- ZBPC lossless coder (zbpc.cu, RZE.hpp, d_*_elimination.hpp) */
/* Encode one chunk (RZE.hpp:10-86 + zbpc.cu:222-243 raw fallback).
 * Returns csize; out must hold >= osize bytes. */
int or_zbpc_encode_chunk(const uint8_t* in, int osize, uint8_t* out);
/* Decode one chunk (RZE.hpp:88-167); csize == osize means raw. */
int or_zbpc_decode_chunk(const uint8_t* in, int csize, int osize, uint8_t* out);
/* Whole stream (zbpc.cu:155-263, 476-520).  Writes the lossless stream (padded
 * to x8) into out, returns its size; fills comp_size_bp[128]. */
uint64_t or_zbpc_encode(const uint8_t* planes, const or_geom* g, uint8_t* out,
                        uint64_t comp_size_bp[128]);
/* Full decode (zbpc.cu:265-365): planes must be zero-initialised. */
int or_zbpc_decode(const uint8_t* stream, const or_geom* g, uint8_t* planes);
/* Progressive decode (zbpc.cu:368-473). */
int or_zbpc_decode_progressive(const uint8_t* stream, const or_geom* g, const int begin[4],
                               const int end[4], uint8_t* planes);

/* ---------------- strategy search (dataloader.cu:13-208) */
/* Updates begin/end/maxlevel exactly as findStrategy_h does (maxlevel is
 * reset to 4 first). */
void or_find_strategy(const uint64_t comp_size_bp[128], double eb, double target_error,
                      int begin[4], int end[4], int* maxlevel);
void or_strategy_costs(uint64_t cost[4][33]);

/* ---------------- whole pipeline (compressor.cu, prism.cu) */
/* Compress: returns container size; out must hold n*tsize + 64 KiB + trailer.
 * mode: 0 ABS, 1 REL. bt: 0 NB (progressive), 1 SM.
 * force != NULL skips the auto-tune and uses its use_md/reverse flags. */
uint64_t or_compress_f32(const float* data, uint32_t nx, uint32_t ny, uint32_t nz, int mode,
                         double bound, int bt, const or_intp* force, uint8_t* out,
                         or_intp* used, float errors[18]);
uint64_t or_compress_f64(const double* data, uint32_t nx, uint32_t ny, uint32_t nz, int mode,
                         double bound, int bt, const or_intp* force, uint8_t* out,
                         or_intp* used, double errors[18]);
int or_decompress_f32(const uint8_t* cont, uint64_t size, uint32_t nx, uint32_t ny, uint32_t nz,
                      int mode, double bound, float* out);
int or_decompress_f64(const uint8_t* cont, uint64_t size, uint32_t nx, uint32_t ny, uint32_t nz,
                      int mode, double bound, double* out);
/* One progressive step (compressor.cu:166-190): first = (last_error == 0).
 * begin/end/maxlevel are the persistent strategy state (start at 0/0/4). */
int or_progressive_step_f32(const uint8_t* cont, uint64_t size, uint32_t nx, uint32_t ny,
                            uint32_t nz, int mode, double bound, double target, double last,
                            int begin[4], int end[4], int* maxlevel, const float* old, float* out);
int or_progressive_step_f64(const uint8_t* cont, uint64_t size, uint32_t nx, uint32_t ny,
                            uint32_t nz, int mode, double bound, double target, double last,
                            int begin[4], int end[4], int* maxlevel, const double* old, double* out);
/* The same step in this library's exact refinement (prism_progressive_exact;
 * not a reference behaviour): a later step also decodes the chunks of plane
 * begin - 1 of every level that gains planes, and the inverse shuffle keeps
 * planes [begin, end) of what was decoded. */
int or_progressive_step_exact_f32(const uint8_t* cont, uint64_t size, uint32_t nx, uint32_t ny,
                                  uint32_t nz, int mode, double bound, double target, double last,
                                  int begin[4], int end[4], int* maxlevel, const float* old, float* out);
int or_progressive_step_exact_f64(const uint8_t* cont, uint64_t size, uint32_t nx, uint32_t ny,
                                  uint32_t nz, int mode, double bound, double target, double last,
                                  int begin[4], int end[4], int* maxlevel, const double* old, double* out);

#ifdef __cplusplus
}
#endif
#endif
