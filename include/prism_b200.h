/*
 * prism_b200 -- C ABI of the B200-native PRISM compression hot path.
 *
 * Drop-in boundary for PRISM's pipeline entry points.  Every call works on
 * device pointers on a caller-supplied CUDA stream, returns a status code and
 * never exits the process (the reference exits on CUDA errors, err.hpp:3-11).
 * Containers are byte-compatible with the reference in both directions.
 *
 * Reference interfaces replaced (paths inside BingluCS/PRISM):
 *   prism_compress              Compressor<T,i4>::init + compress_pipeline
 *                               (include/compressor.hpp:44-52,
 *                                src/compressor.cu:77-151) with REL range from
 *                               StatBuffer::findMinMax (compressor.hpp:23-31)
 *   prism_decompress            Compressor<T,i4>::decompress_pipeline
 *                               (compressor.hpp:54-57, compressor.cu:153-164)
 *   prism_progressive_open/step Compressor<T,i4>::decompress_progressive_pipeline
 *                               (compressor.hpp:59-61, compressor.cu:166-190) with
 *                               the begin/end/maxlevel state of prism_context
 *                               (include/utils/parameters.hpp:54-55,
 *                                src/loader/dataloader.cu:11)
 *   stage entry points          spline_construct / spline_reconstruct /
 *                               spline_progressive_reconstruct
 *                               (include/predictor/InterpolationPredictor.hpp:12-21),
 *                               convert_to_bitplane / inverse_convert_to_bitplane[_progressive]
 *                               (include/predictor/bitplane.hpp:15-22),
 *                               lossless_encode / lossless_decode[_progressive]
 *                               (include/encoder/zbpc.hpp:11-15),
 *                               findStrategy_h (include/loader/dataloader.hpp:8),
 *                               extrema_scan (include/compressor.hpp:10)
 *
 * dtype_size: 4 = float (PRISM -f), 8 = double (-d).
 * mode: 0 = ABS (-A), 1 = REL (-R).
 * progressive: 0 = sign-magnitude planes (default CLI), 1 = negabinary (-prog).
 * Dimensions: nx fastest (-3 nx ny nz; -2 nx ny; -1 nx).
 */
#ifndef PRISM_B200_H
#define PRISM_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum prism_status {
  PRISM_OK = 0,
  PRISM_ERR_ARG = -1,        /* bad argument (dims, dtype, bound, capacity) */
  PRISM_ERR_CUDA = -2,       /* CUDA runtime error */
  PRISM_ERR_CORRUPT = -3,    /* container does not parse / decode */
  PRISM_ERR_TIMEOUT = -4,    /* a device-side wait hit its iteration limit */
  PRISM_ERR_NOMEM = -5,      /* device workspace allocation failed */
  PRISM_ERR_LIMIT = -6       /* input larger than a fixed-size entry point accepts */
};

typedef struct prism_handle prism_handle;
typedef struct prism_prog prism_prog;

/* Handle owning the device workspace (grown on demand, reused across calls).
 * The calls on one handle share that workspace: enqueue them on one stream,
 * or order the streams they use (one handle per concurrent stream, as the
 * server's workers do). */
int prism_create(prism_handle** out);
void prism_destroy(prism_handle* h);
/* Human-readable description of the last failure on this handle. */
const char* prism_last_error(const prism_handle* h);

/* Stage timing: with profiling on, every pipeline call records CUDA events
 * around its stages on the caller's stream (no extra synchronisation) and
 * accumulates device milliseconds per stage.  prism_stage_times copies up to n
 * accumulators (order: extrema, autotune, predict, shuffle, encode, trailer,
 * strategy, decode, inverse shuffle, reconstruct), returns the stage count and
 * clears them when reset != 0.  No counterpart in the reference, which times
 * its stages with blocking GPUTimer pairs (include/utils/timer.hpp:21-30).
 * prism_profile_stages times only the stages whose bit (1 << index, order
 * above) is set in mask: each timing event drains the stream, so timing
 * every stage costs a few microseconds per launch. */
int prism_profile(prism_handle* h, int enable);
int prism_profile_stages(prism_handle* h, uint32_t mask);
int prism_stage_times(prism_handle* h, double* ms, int* counts, int n, int reset);
/* Number of kernels this handle has launched. */
uint64_t prism_launch_count(const prism_handle* h);

/* Upper bound of the container size (all chunks stored raw). */
uint64_t prism_max_container_size(uint32_t nx, uint32_t ny, uint32_t nz, int dtype_size);
/* Size of the plane buffer (host aligned_size, io.cu:117-127) and the trailer. */
uint64_t prism_plane_buffer_size(uint32_t nx, uint32_t ny, uint32_t nz);
uint64_t prism_trailer_size(uint32_t nx, uint32_t ny, uint32_t nz, int dtype_size);

/* Compress d_in (n values) into the container at d_out.  *out_size receives
 * the container size.  flags_out (host, may be NULL) receives use_md[4] then
 * reverse[4] as chosen by the auto-tuner. */
int prism_compress(prism_handle* h, const void* d_in, int dtype_size, uint32_t nx, uint32_t ny,
                   uint32_t nz, int mode, double bound, int progressive, void* d_out,
                   uint64_t out_capacity, uint64_t* out_size, uint8_t flags_out[8], void* stream);

/* Same, with host buffers: host->device copy of the input, compression, and
 * device->host copy of the container all inside the call. */
int prism_compress_host(prism_handle* h, const void* h_in, int dtype_size, uint32_t nx, uint32_t ny,
                        uint32_t nz, int mode, double bound, int progressive, void* h_out,
                        uint64_t out_capacity, uint64_t* out_size, void* stream);

/* Full decompression of a non-progressive (sign-magnitude) container. */
int prism_decompress(prism_handle* h, const void* d_container, uint64_t size, int dtype_size,
                     uint32_t nx, uint32_t ny, uint32_t nz, int mode, double bound, void* d_out,
                     void* stream);
int prism_decompress_host(prism_handle* h, const void* h_container, uint64_t size, int dtype_size,
                          uint32_t nx, uint32_t ny, uint32_t nz, int mode, double bound, void* h_out,
                          void* stream);

/* Progressive retrieval of a negabinary (-prog) container that stays resident
 * on the device (the caller keeps d_container alive).  Each step picks the
 * planes the target error needs, decodes only their chunks and refines the
 * values in d_values in place (the first step overwrites them).  A step is
 * enqueued on `stream` and returns without waiting (the plane state stays in
 * device memory); prism_progressive_state waits for the last step and
 * returns PRISM_ERR_CORRUPT if any step met a corrupt chunk.  From an
 * object's second step on, the handle holds a second code buffer
 * (prism_code_buffer_len entries) so that a step's decode and inverse shuffle
 * can run beside the previous step's reconstruction. */
int prism_progressive_open(prism_handle* h, const void* d_container, uint64_t size, int dtype_size,
                           uint32_t nx, uint32_t ny, uint32_t nz, int mode, double bound,
                           prism_prog** out);
int prism_progressive_step(prism_prog* p, double target_error, void* d_values, void* stream);
/* The same step out of place, as decompress_progressive_pipeline(config,
 * output_old, output_new, ...) (include/compressor.hpp:80-81,
 * src/prism.cu:112-138): reads the previous step's values from d_prev
 * (ignored by the first step; may equal d_out) and writes the refined values
 * to d_out.  Alternating two buffers lets the caller copy one step's result
 * to the host while the next step runs. */
int prism_progressive_step_into(prism_prog* p, double target_error, const void* d_prev, void* d_out,
                                void* stream);
/* Start an object from a state whose planes [0, end[l]) of every level are
 * already reconstructed (values the caller holds, e.g. a cached earlier
 * retrieval of the same container): the next step refines them, as the
 * reference's later steps refine output_old into output_new
 * (src/prism.cu:126-138, compressor.cu:166-190).  Only before the first step;
 * the next step needs d_prev (prism_progressive_step_into). */
int prism_progressive_resume(prism_prog* p, const int end[4], void* stream);
/* Exact refinement (no counterpart in the reference; off by default, which is
 * the reference's behaviour).  The container's chunks are cut at the host
 * plane stride, which can exceed the device stride the planes are laid out
 * with (by 8 bytes per plane when a plane's size is a multiple of 8 bytes,
 * plus 256 bytes per earlier level), so the first bytes of device plane b can
 * lie in the chunks of plane b - 1.  A reference step that loads planes
 * [b, e) decodes the chunks of planes b..e-1 only, and the step that loaded
 * plane b - 1 masked plane b out: a chained retrieval never sees those bytes,
 * its values differ from the one-step retrieval to the same planes and can
 * miss the requested bound (on a 64x48x40 double field the chain 1e-2 ->
 * 1e-4 ends 0.45% of the range away from the data).  With
 * exact mode on, a step also decodes the chunks of plane b - 1 of every level
 * that gains planes and keeps planes [b, e) of them, so after every step the
 * values hold complete device planes [0, e) and equal the one-step retrieval
 * up to the rounding of the sum (when the object starts from values that
 * hold complete planes: a first step, an exact step, or a resume from
 * either).  Set before the step it should apply to. */
int prism_progressive_exact(prism_prog* p, int enable);
/* begin/end/maxlevel after the last step; loaded = payload bytes of the
 * planes selected so far (calculate_accumulate_size, analyze.hpp:118-159). */
int prism_progressive_state(const prism_prog* p, int begin[4], int end[4], int* maxlevel,
                            uint64_t* loaded);
void prism_progressive_close(prism_prog* p);

/* ---- stage entry points (device buffers; for tests and custom pipelines) */
/* Global range max-min in double (extrema_scan). */
int prism_extrema(prism_handle* h, const void* d_in, int dtype_size, uint64_t n, double* range_out,
                  void* stream);
/* Minimum and maximum of n values (host minmax_out[0], [1], converted to
 * double): the two results of extrema_scan (include/compressor.hpp:10-31),
 * which StatBuffer::findMinMax turns into the REL range. */
int prism_extrema_minmax(prism_handle* h, const void* d_in, int dtype_size, uint64_t n, double minmax_out[2],
                         void* stream);
/* Auto-tune error sums (15 values, host) and the decisions (use_md[4], reverse[4]). */
int prism_autotune(prism_handle* h, const void* d_in, int dtype_size, uint32_t nx, uint32_t ny,
                   uint32_t nz, double* errors_out, uint8_t flags_out[8], void* stream);
/* Predictor + quantiser with given flags (use_md[4], reverse[4]); eb is the
 * absolute bound, rel_eb selects the level schedule (0 for ABS).  Writes the
 * level-major codes (prism_code_buffer_len entries) and the anchors. */
uint64_t prism_code_buffer_len(uint32_t nx, uint32_t ny, uint32_t nz);
int prism_predict(prism_handle* h, const void* d_in, int dtype_size, uint32_t nx, uint32_t ny,
                  uint32_t nz, double eb, double rel_eb, const uint8_t flags[8], int32_t* d_codes,
                  void* d_anchors, void* stream);
/* Reconstruction from codes + anchors; d_old != NULL adds the previous values
 * (progressive delta); maxlevel = 4 for a full reconstruction. */
int prism_reconstruct(prism_handle* h, const int32_t* d_codes, const void* d_anchors, int dtype_size,
                      uint32_t nx, uint32_t ny, uint32_t nz, double eb, double rel_eb,
                      const uint8_t flags[8], int maxlevel, const void* d_old, void* d_out, void* stream);
/* Codes -> planes (prism_plane_buffer_size bytes), including the bytes the
 * reference leaves holding the predictor's scratch. */
int prism_bitshuffle(prism_handle* h, const int32_t* d_codes, uint32_t nx, uint32_t ny, uint32_t nz,
                     int progressive, uint8_t* d_planes, void* stream);
/* Planes -> codes; begin/end (host, may be NULL) restrict each level to the
 * planes [begin[3-l], end[3-l]) like the progressive inverse. */
int prism_inverse_bitshuffle(prism_handle* h, const uint8_t* d_planes, uint32_t nx, uint32_t ny,
                             uint32_t nz, int progressive, const int begin[4], const int end[4],
                             int32_t* d_codes, void* stream);
/* Planes -> lossless stream (8-byte header, size table, payloads, pad to 8);
 * comp_size_bp (host, may be NULL) receives the 128 cumulative plane sizes. */
int prism_lossless_encode(prism_handle* h, const uint8_t* d_planes, uint32_t nx, uint32_t ny,
                          uint32_t nz, uint8_t* d_stream, uint64_t capacity, uint64_t* size_out,
                          uint64_t comp_size_bp[128], void* stream);
/* Self-test of the failure detection in the encoder's look-back (no
 * counterpart in the reference, whose decoupled look-back in zbpc_encode,
 * src/encoder/zbpc.cu:113-153, spins without a limit).  Runs the kernels of
 * prism_lossless_encode with the chunk tickets starting at 1, so chunk 0 never
 * publishes its size and every wait that reaches it gives up after
 * `spin_limit` polls (about 64 ns apart).  Returns PRISM_ERR_TIMEOUT when the
 * bounded wait works; the stream bytes it leaves are meaningless.  The handle
 * stays usable.  Needs a field of at least two chunks. */
int prism_lossless_wait_selftest(prism_handle* h, const uint8_t* d_planes, uint32_t nx, uint32_t ny,
                                 uint32_t nz, uint8_t* d_stream, uint64_t capacity, long long spin_limit,
                                 void* stream);
/* Number of level-0 codes whose bits the reference's last bit-plane shuffle
 * block does not carry for these dimensions (src/predictor/bitplane.cu:180-181,
 * 200-260): on some shapes the block stops short of the end of the code space
 * (trailing codes decode as 0), and on many small shapes its zero words past
 * the end of the last level-0 plane land on the first bytes of the next
 * planes (leading level-0 codes lose their low bits).  The container bytes
 * stay identical to the reference's, so the points of these codes are
 * reconstructed from a wrong code and may miss the bound.  0 for shapes
 * without the effect.  Geometry only; no device work. */
uint64_t prism_lost_codes(uint32_t nx, uint32_t ny, uint32_t nz);
/* Lossless stream -> planes.  With begin/end (host, both or neither), only
 * the chunks of planes [begin[3-l], end[3-l]) of each level are decoded; of
 * the other planes, the bytes that the inverse shuffle of the selected planes
 * reads (their device placement reaches into neighbouring host planes) are
 * written as zeros and the rest of the buffer is left as it is. */
int prism_lossless_decode(prism_handle* h, const uint8_t* d_stream, uint32_t nx, uint32_t ny,
                          uint32_t nz, const int begin[4], const int end[4], uint8_t* d_planes,
                          void* stream);
/* Lossless encode that allocates nothing.  No counterpart in the reference.
 *
 * Same result as prism_lossless_encode (bit-identical stream, size and plane
 * sizes) without a handle: its scratch (look-back status words, chunk ticket,
 * error flag, plane sizes; about 130 KiB) is a fixed device array inside the
 * library, so neither this call nor anything it calls allocates device or host
 * memory.  Meant for callers that cannot allocate at this point, e.g. a process
 * whose device memory is fully reserved by another allocator, or a
 * latency-critical loop in which cudaMalloc/cudaFree would synchronise the
 * device and stall the work on other streams.
 *
 * Limit: at most 16384 lossless chunks, i.e. a plane buffer
 * (prism_plane_buffer_size) of at most 256 MiB, about 64 million values;
 * larger fields return PRISM_ERR_LIMIT before any device work.
 * Zero state: the call itself resets, on `stream`, every scratch word the
 * kernels expect to start at zero; the caller zeroes nothing.
 * Overlap: there is one scratch per device for the whole process, so two calls
 * whose device work may overlap (different streams, different host threads)
 * race on it and produce wrong output; order them on one stream or with
 * events.  The call waits for its stream before it returns.
 * Setup: the first call on each device (with that device current) looks up
 * the scratch address and sets the encode kernel's shared-memory limit; make
 * that first call before any stream capture begins.
 * Other errors: PRISM_ERR_ARG for bad arguments or capacity, PRISM_ERR_CUDA,
 * PRISM_ERR_TIMEOUT as for prism_lossless_encode. */
int prism_lossless_encode_static(const uint8_t* d_planes, uint32_t nx, uint32_t ny, uint32_t nz,
                                 uint8_t* d_stream, uint64_t capacity, uint64_t* size_out,
                                 uint64_t comp_size_bp[128], void* stream);
/* Strategy step: updates begin/end/maxlevel (host arrays) from the cumulative
 * plane sizes (host), the absolute bound and the absolute target error. */
int prism_find_strategy(prism_handle* h, const uint64_t comp_size_bp[128], double eb,
                        double target_error, int begin[4], int end[4], int* maxlevel, void* stream);
/* Many strategy steps at once (no counterpart in the reference, which runs
 * findStrategy_h, dataloader.cu:179-334, one target at a time): search i
 * reads comp_size_bp[128 i .. 128 i + 127], the absolute bound eb[i] and
 * target target_error[i], and updates begin[4 i ..], end[4 i ..] and
 * maxlevel[i] (host arrays) exactly as prism_find_strategy would.  One scan
 * launch and one reduction launch for all n (1 <= n <= 65535) searches, then
 * a wait for `stream`. */
int prism_find_strategy_batch(prism_handle* h, int n, const uint64_t* comp_size_bp, const double* eb,
                              const double* target_error, int* begin, int* end, int* maxlevel, void* stream);

/* Error statistics of a reconstruction against the original (both device
 * arrays of n values): out = {max |error|, max |error| / range, PSNR, NRMSE,
 * min, max (of the original), sum of squared errors}; *max_err_index = first
 * index with the max error.  Replaces statistic (include/utils/analyze.hpp:
 * 5-73), which loops over host copies. */
int prism_statistics(prism_handle* h, const void* d_original, const void* d_data, int dtype_size, uint64_t n,
                     double out[7], uint64_t* max_err_index, void* stream);

/* ---- container files ----------------------------------------------------
 * Save a device-resident container to `path`: device-to-host copies through
 * two pinned staging buffers overlap the file writes.  Waits for `stream`. */
int prism_file_save(const char* path, const void* d_container, uint64_t size, void* stream);

typedef struct prism_file prism_file;
/* Open a -prog container file for progressive retrieval.  Reads only the
 * stream header, the chunk size table and the trailer; later steps read only
 * the chunks of the planes they add.  Replaces the reference's whole-file
 * reload per target (src/prism.cu:131-135). */
int prism_file_open(prism_handle* h, const char* path, int dtype_size, uint32_t nx, uint32_t ny, uint32_t nz,
                    int mode, double bound, prism_file** out);
/* One progressive step from the file: values equal prism_progressive_step on
 * the whole container. */
int prism_file_step(prism_file* f, double target_error, void* d_values, void* stream);
/* File size, bytes read from it so far, planes loaded per level. */
int prism_file_info(const prism_file* f, uint64_t* file_bytes, uint64_t* bytes_read, int end[4]);
void prism_file_close(prism_file* f);

/* ---- batched compression ----------------------------------------------
 * Many fields of uneven shapes compressed by one launch per pipeline stage;
 * no counterpart in the reference, whose pipeline handles one field per call
 * (Compressor<T,i4>::compress_pipeline, src/compressor.cu:120-151).  Every
 * field's container is byte-identical to prism_compress of that field. */
typedef struct prism_field_desc {
  const void* d_in;       /* device input, nx*ny*nz values, x fastest */
  void* d_out;            /* device container buffer */
  uint64_t out_capacity;  /* >= prism_max_container_size of the field */
  uint32_t nx, ny, nz;
  int dtype_size;         /* 4 or 8 */
  int mode;               /* 0 ABS, 1 REL */
  double bound;
  int progressive;        /* 0 sign-magnitude planes, 1 negabinary */
} prism_field_desc;

typedef struct prism_batch prism_batch;

/* Plan a batch for these fields and buffers: one device workspace for all
 * fields, work tables per stage, a schedule tuned on the batch itself (CTAs
 * per SM of the persistent predictor and encoder, timed on the first runs),
 * and, when use_graph != 0, the whole pipeline captured in a CUDA graph.
 * Runs the pipeline a few times while tuning, on the current device. */
int prism_batch_create(const prism_field_desc* fields, int n, int use_graph, prism_batch** out);
/* Compress the current contents of the batch's input buffers into its output
 * buffers; sizes_out[i] receives field i's container size and flags_out
 * (may be NULL) its use_md[4], reverse[4].  Waits for `stream`. */
int prism_batch_compress(prism_batch* b, void* stream, uint64_t* sizes_out, uint8_t* flags_out);
/* The tuned schedule: predictor CTAs per SM for float and double fields (0 =
 * one CTA per tile instead of persistent CTAs), encoder CTAs per SM, the
 * tuned stage times (ms) and kernels per run. */
int prism_batch_schedule(const prism_batch* b, int pred_ctas_per_sm[2], int* enc_ctas_per_sm, double tuned_ms[2],
                         uint64_t* launches_per_run);
const char* prism_batch_last_error(const prism_batch* b);
void prism_batch_destroy(prism_batch* b);

/* ---- progressive-retrieval server -----------------------------------------
 * No counterpart in the reference, whose CLI reloads and re-decodes the whole
 * container for each -errors target (src/prism.cu:131-190).  The server keeps
 * -prog containers and reconstructions resident on the current device and
 * answers "field f at error bound t" requests from `slots` worker threads
 * (one stream and workspace each) under an HBM budget.  A request's values are
 * the progressive retrieval of f to the planes that t selects: either one step
 * from no planes (prism_progressive_open + one prism_progressive_step) or,
 * when a reconstruction of f with a subset of those planes is resident, a
 * refinement step from it (prism_progressive_resume +
 * prism_progressive_step_into, src/prism.cu:126-138, in exact mode:
 * prism_progressive_exact).  The two carry the same planes and differ only by
 * floating-point rounding of the refinement sum: at most 64 units in the last
 * place of the field's largest magnitude
 * (prism_server_set_refine(s, 0) makes every result the one-step retrieval,
 * bit for bit).
 * Reconstructions are cached per selected plane set and reused as they are. */
typedef struct prism_server prism_server;
typedef struct prism_server_stats {
  uint64_t completed, cache_hits, shared, evictions, failed;
  uint64_t bytes_out, bytes_resident, bytes_reserved, bytes_peak;
  double p50_ms, p99_ms, mean_ms, max_ms, elapsed_s;  /* submit -> completion */
  double queue_p50_ms, queue_p99_ms;                  /* submit -> a slot takes it */
  double service_p50_ms, service_p99_ms;              /* slot start -> completion */
  uint64_t refined;                                   /* misses refined from a coarser entry */
  uint64_t plan_calls;  /* batched plane searches run: each searches the plane selections of the request a
                         * worker takes and of up to 31 other queued requests (prism_find_strategy_batch) */
} prism_server_stats;

/* hbm_budget: bytes of device memory the server may hold (containers,
 * cached reconstructions, per-slot workspaces). */
int prism_server_create(uint64_t hbm_budget, int slots, prism_server** out);
/* Copy a -prog container (host, or device when on_device != 0) into the
 * server; *field_id names it in requests.  PRISM_ERR_NOMEM beyond the budget. */
int prism_server_add_field(prism_server* s, const void* container, uint64_t size, int on_device, int dtype_size,
                           uint32_t nx, uint32_t ny, uint32_t nz, int mode, double bound, int* field_id);
/* Queue a retrieval of field_id at target_error (the same kind of bound as
 * the field's mode) into `out` (nx*ny*nz values; device memory when
 * out_on_device != 0, else host memory).  Returns at once. */
int prism_server_submit(prism_server* s, int field_id, double target_error, void* out, int out_on_device,
                        uint64_t* request_id);
/* Wait for a request; latency = submit to completion.  end/maxlevel receive
 * the plane selection; from_cache = 1 when a resident reconstruction served
 * it, 2 when it was refined from a resident coarser one, 0 when computed from
 * no planes.  Returns the request's status. */
int prism_server_wait(prism_server* s, uint64_t request_id, double* latency_ms, int end[4], int* maxlevel,
                      int* from_cache);
/* Non-blocking: *done = 1 once the request has completed (then wait). */
int prism_server_poll(prism_server* s, uint64_t request_id, int* done);
/* Refinement of misses from coarser resident entries: on (default) or off
 * (every miss from no planes). */
int prism_server_set_refine(prism_server* s, int enable);
/* Latency percentiles and counters of the completed requests. */
int prism_server_stats_get(prism_server* s, prism_server_stats* out, int reset);
void prism_server_destroy(prism_server* s);

#ifdef __cplusplus
}
#endif
#endif
