// Host side of the batched compression (prism_batch_* in prism_b200.h).
// Included at the end of prism_b200.cu, whose helpers it uses.
//
// A batch is planned once for a fixed set of fields and buffers: the planner
// lays out one device workspace for all fields, builds the per-stage work
// tables, tunes the persistent kernels' CTAs per SM on the batch itself, and
// captures the whole pipeline in a CUDA graph.  Each prism_batch_compress is
// then one graph launch plus one small device-to-host copy of the results.
#include "batch.cuh"

struct prism_batch {
  std::string err;
  int n = 0;
  std::vector<prism_field_desc> desc;
  std::vector<Geometry> geo;
  unsigned char* dev = nullptr;  // one allocation for all device state
  BatchField* d_fields = nullptr;
  BatchState* d_states = nullptr;
  unsigned long long* d_status = nullptr;
  size_t status_bytes = 0;
  unsigned long long* d_counters = nullptr;  // predict f32 x2, f64 x2, encode
  BatchResult* d_results = nullptr;
  BatchResult* h_results = nullptr;  // pinned
  struct Group {
    int tsize = 0;
    int n = 0;
    int* d_idx = nullptr;
    uint64_t* d_ext_prefix = nullptr;
    uint64_t ext_items = 0;
    void* d_ext_part = nullptr;
    uint64_t* d_win_prefix = nullptr;
    uint64_t nwin = 0;
    BatchWindow* d_wins = nullptr;
    void* d_partial = nullptr;
    uint64_t* d_tile_prefix[2] = {nullptr, nullptr};
    uint64_t tiles[2] = {0, 0};
    uint64_t* d_tr_prefix = nullptr;
    uint64_t tr_items = 0;
  } grp[2];  // [0] float, [1] double
  uint64_t* d_shuf_prefix = nullptr;
  uint64_t shuf_items = 0;
  uint64_t* d_chunk_prefix = nullptr;
  uint64_t chunk_items = 0;
  BatchRange* d_ranges = nullptr;
  int nranges = 0;
  BatchLastCta* d_pre = nullptr;
  int npre = 0;
  BatchLastCta* d_post = nullptr;
  int npost = 0;
  BatchZero* d_zero = nullptr;
  int nzero = 0;
  int sm_count = 148;
  int pred_ctas[2] = {0, 0};  // CTAs per SM of the persistent predictor, per dtype
  int enc_ctas = 0;           // CTAs per SM of the persistent encoder
  int pred_max[2] = {0, 0}, enc_max = 0;
  double tuned_ms[2] = {0, 0};  // predictor and encoder stage time of the chosen schedule
  bool use_graph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t launches_per_run = 0;
};

namespace {

int bfail(prism_batch* b, int code, const std::string& what, cudaError_t e = cudaSuccess) {
  if (b) {
    b->err = what;
    if (e != cudaSuccess) b->err += std::string(": ") + cudaGetErrorString(e);
  }
  return code;
}

#define BCK(call)                                                      \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess) return bfail(b, PRISM_ERR_CUDA, #call, e_); \
  } while (0)

// bump allocator over the batch's single device allocation
struct Carve {
  size_t off = 0;
  template <class U>
  size_t take(size_t count, size_t align = 256) {
    off = (off + align - 1) / align * align;
    size_t at = off;
    off += count * sizeof(U) + 64;
    return at;
  }
};

template <class T>
int enqueue_group_front(prism_batch* b, const prism_batch::Group& gr, cudaStream_t st, uint64_t& launches) {
  if (gr.n == 0) return PRISM_OK;
  if (gr.ext_items) {
    int blocks = (int)std::min<uint64_t>(gr.ext_items, (uint64_t)b->sm_count * 4);
    batch_extrema_kernel<T><<<blocks, kExtThreads, 0, st>>>(b->d_fields, gr.d_idx, gr.d_ext_prefix, gr.n,
                                                            gr.ext_items, reinterpret_cast<T*>(gr.d_ext_part));
    ++launches;
  }
  batch_extrema_final_kernel<T><<<gr.n, 32, 0, st>>>(b->d_fields, gr.d_idx, gr.d_ext_prefix, gr.n,
                                                     reinterpret_cast<const T*>(gr.d_ext_part));
  ++launches;
  if (gr.nwin) {
    batch_autotune_kernel<T><<<dim3((unsigned)gr.nwin, 6), kAttThreads, 0, st>>>(
        b->d_fields, gr.d_wins, reinterpret_cast<T*>(gr.d_partial));
    ++launches;
  }
  batch_params_kernel<T><<<(gr.n + 63) / 64, 64, 0, st>>>(b->d_fields, gr.d_idx, gr.d_win_prefix, gr.n,
                                                           reinterpret_cast<const T*>(gr.d_partial));
  ++launches;
  BCK(cudaGetLastError());
  return PRISM_OK;
}

template <class T>
int enqueue_group_predict(prism_batch* b, const prism_batch::Group& gr, int g, int ctas, cudaStream_t st,
                          uint64_t& launches) {
  const int smem = compress_smem_bytes<T>();
  // ctas > 0: persistent CTAs (ctas per SM) on the tile counter; 0: one CTA
  // per tile
  for (int part = 0; part < 2; ++part) {
    if (!gr.tiles[part]) continue;
    unsigned grid = ctas > 0 ? (unsigned)std::min<uint64_t>(gr.tiles[part], (uint64_t)b->sm_count * ctas)
                             : (unsigned)gr.tiles[part];
    unsigned long long* counter = b->d_counters + 2 * g + part;
    const uint64_t* pre = gr.d_tile_prefix[part];
    if (ctas == 0 && part == 0)
      batch_predict_kernel<T, 0><<<grid, kPredThreads, smem, st>>>(b->d_fields, gr.d_idx, pre, gr.n, gr.tiles[0]);
    else if (ctas == 0)
      batch_predict_kernel<T, 1><<<grid, kPredThreads, smem, st>>>(b->d_fields, gr.d_idx, pre, gr.n, gr.tiles[1]);
    else if (part == 0)
      batch_predict_persistent_kernel<T, 0><<<grid, kPredThreads, smem, st>>>(b->d_fields, gr.d_idx, pre, gr.n,
                                                                              gr.tiles[0], counter);
    else
      batch_predict_persistent_kernel<T, 1><<<grid, kPredThreads, smem, st>>>(b->d_fields, gr.d_idx, pre, gr.n,
                                                                              gr.tiles[1], counter);
    ++launches;
  }
  BCK(cudaGetLastError());
  return PRISM_OK;
}

template <class T>
int enqueue_group_back(prism_batch* b, const prism_batch::Group& gr, cudaStream_t st, uint64_t& launches) {
  if (gr.n == 0) return PRISM_OK;
  int blocks = (int)std::min<uint64_t>(gr.tr_items, 4096);
  batch_trailer_kernel<T><<<blocks, 256, 0, st>>>(b->d_fields, gr.d_idx, gr.d_tr_prefix, gr.n, gr.tr_items);
  batch_collect_kernel<T><<<(gr.n + 63) / 64, 64, 0, st>>>(b->d_fields, gr.d_idx, gr.n, b->d_results);
  launches += 2;
  BCK(cudaGetLastError());
  return PRISM_OK;
}

int enqueue_encode(prism_batch* b, int ctas, cudaStream_t st, uint64_t& launches) {
  unsigned grid = (unsigned)std::min<uint64_t>(b->chunk_items, (uint64_t)b->sm_count * ctas);
  batch_encode_kernel<<<grid, kZThreads, sizeof(EncodeShared), st>>>(b->d_fields, b->d_chunk_prefix, b->n,
                                                                     b->chunk_items, b->d_counters + 4,
                                                                     (long long)1 << 22);
  ++launches;
  BCK(cudaGetLastError());
  return PRISM_OK;
}

// The whole pipeline on stream st (what the graph holds).
int enqueue_all(prism_batch* b, cudaStream_t st, uint64_t& launches) {
  launches = 0;
  BCK(cudaMemsetAsync(b->d_states, 0, sizeof(BatchState) * b->n, st));
  BCK(cudaMemsetAsync(b->d_status, 0, b->status_bytes, st));
  BCK(cudaMemsetAsync(b->d_counters, 0, 8 * sizeof(unsigned long long), st));
  int rc;
  if ((rc = enqueue_group_front<float>(b, b->grp[0], st, launches))) return rc;
  if ((rc = enqueue_group_front<double>(b, b->grp[1], st, launches))) return rc;
  if (b->nzero) {
    batch_zero_kernel<<<std::min(b->nzero, 4096), 256, 0, st>>>(b->d_zero, b->nzero);
    ++launches;
  }
  if ((rc = enqueue_group_predict<float>(b, b->grp[0], 0, b->pred_ctas[0], st, launches))) return rc;
  if ((rc = enqueue_group_predict<double>(b, b->grp[1], 1, b->pred_ctas[1], st, launches))) return rc;
  if (b->nranges) {
    batch_leftover_kernel<<<std::min(b->nranges, 4096), 256, 0, st>>>(b->d_fields, b->d_ranges, b->nranges);
    ++launches;
  }
  if (b->npre) {
    batch_last_block_kernel<<<b->npre, 512, 0, st>>>(b->d_fields, b->d_pre);
    ++launches;
  }
  if (b->shuf_items) {
    batch_shuffle_kernel<<<(unsigned)((b->shuf_items + kShufWarps - 1) / kShufWarps), kShufWarps * 32, 0, st>>>(
        b->d_fields, b->d_shuf_prefix, b->n, b->shuf_items);
    ++launches;
  }
  if (b->npost) {
    batch_last_block_kernel<<<b->npost, 512, 0, st>>>(b->d_fields, b->d_post);
    ++launches;
  }
  if ((rc = enqueue_encode(b, b->enc_ctas, st, launches))) return rc;
  batch_finish_kernel<<<b->n, 32, 0, st>>>(b->d_fields, b->n);
  ++launches;
  if ((rc = enqueue_group_back<float>(b, b->grp[0], st, launches))) return rc;
  if ((rc = enqueue_group_back<double>(b, b->grp[1], st, launches))) return rc;
  BCK(cudaMemcpyAsync(b->h_results, b->d_results, sizeof(BatchResult) * b->n, cudaMemcpyDeviceToHost, st));
  BCK(cudaGetLastError());
  return PRISM_OK;
}

// Time `fn` (which enqueues on st) over two runs; the faster one counts.
template <class Fn>
int time_stage(prism_batch* b, cudaStream_t st, Fn fn, double* ms) {
  cudaEvent_t e0, e1;
  BCK(cudaEventCreate(&e0));
  BCK(cudaEventCreate(&e1));
  double best = 1e30;
  int rc = PRISM_OK;
  for (int r = 0; r < 2 && rc == PRISM_OK; ++r) {
    cudaEventRecord(e0, st);
    rc = fn();
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) rc = bfail(b, PRISM_ERR_CUDA, "schedule timing");
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    best = std::min(best, (double)t);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = best;
  return rc;
}

// Schedule tuner: for the predictor (per dtype) one CTA per tile or
// persistent CTAs with 1..max per SM, for the encoder 1..max persistent CTAs
// per SM; every feasible value is timed on the batch and the fastest kept.
int tune_schedule(prism_batch* b, cudaStream_t st) {
  uint64_t launches = 0;
  int rc = enqueue_all(b, st, launches);  // warm-up; leaves params and planes in place
  if (rc) return rc;
  BCK(cudaStreamSynchronize(st));
  for (int g = 0; g < 2; ++g) {
    if (!b->grp[g].n) continue;
    double best = 1e30;
    int pick = b->pred_max[g];
    for (int c = 0; c <= b->pred_max[g]; ++c) {  // 0: one CTA per tile
      double ms = 0;
      rc = time_stage(b, st, [&]() -> int {
        cudaMemsetAsync(b->d_counters + 2 * g, 0, 2 * sizeof(unsigned long long), st);
        uint64_t l = 0;
        return g == 0 ? enqueue_group_predict<float>(b, b->grp[0], 0, c, st, l)
                      : enqueue_group_predict<double>(b, b->grp[1], 1, c, st, l);
      }, &ms);
      if (rc) return rc;
      if (ms < best) { best = ms; pick = c; }
    }
    b->pred_ctas[g] = pick;
    b->tuned_ms[0] += best;
  }
  double best = 1e30;
  int pick = b->enc_max;
  for (int c = 1; c <= b->enc_max; ++c) {
    double ms = 0;
    rc = time_stage(b, st, [&]() -> int {
      cudaMemsetAsync(b->d_status, 0, b->status_bytes, st);
      cudaMemsetAsync(b->d_counters + 4, 0, sizeof(unsigned long long), st);
      uint64_t l = 0;
      return enqueue_encode(b, c, st, l);
    }, &ms);
    if (rc) return rc;
    if (ms < best) { best = ms; pick = c; }
  }
  b->enc_ctas = pick;
  b->tuned_ms[1] = best;
  return PRISM_OK;
}

template <auto Kernel>
int max_ctas(prism_batch* b, int threads, int smem, int* out) {
  BCK(cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int nb = 0;
  BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, Kernel, threads, smem));
  *out = std::max(nb, 1);
  return PRISM_OK;
}

int batch_plan(prism_batch* b) {
  const int n = b->n;
  int dev = 0;
  BCK(cudaGetDevice(&dev));
  BCK(cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, dev));
  // ---- host tables ----
  std::vector<BatchField> fields(n);
  std::vector<uint64_t> shuf_prefix(n + 1, 0), chunk_prefix(n + 1, 0);
  std::vector<BatchRange> ranges;
  std::vector<BatchLastCta> pre, post;
  std::vector<std::pair<size_t, uint64_t>> zero_rel;  // (field qc offset in ints, len) resolved later
  struct GroupHost {
    std::vector<int> idx;
    std::vector<uint64_t> ext{0}, win{0}, tile0{0}, tile1{0}, tr{0};
    std::vector<BatchWindow> wins;
  } gh[2];
  Carve cv;
  std::vector<size_t> off_qc(n), off_planes(n), off_anchors(n), off_status(n);
  size_t status_total = 0;
  for (int i = 0; i < n; ++i) {
    const prism_field_desc& d = b->desc[i];
    const Geometry& g = b->geo[i];
    BatchField& f = fields[i];
    memset(&f, 0, sizeof(f));
    f.g = g;
    f.plan = make_shuf_plan(g, (g.sh_grid - 1) * (int64_t)kChunk);
    f.in = d.d_in;
    f.out = reinterpret_cast<uint8_t*>(d.d_out);
    f.mode = d.mode;
    f.nb = d.progressive ? 1 : 0;
    f.tsize = d.dtype_size;
    f.bound = d.bound;
    f.alpha = alpha_of(d.mode == 1 ? d.bound : 0.0);
    off_qc[i] = cv.take<int32_t>(qc_len(g));
    off_planes[i] = cv.take<uint8_t>(g.aligned_size + 64);
    off_anchors[i] = cv.take<double>(g.anchors);
    off_status[i] = status_total;
    status_total += (size_t)g.chunks;
    // work items
    shuf_prefix[i + 1] = shuf_prefix[i] + (uint64_t)f.plan.items;
    chunk_prefix[i + 1] = chunk_prefix[i] + (uint64_t)g.chunks;
    ByteRange rng[160];
    int nr = fill_ranges(g, f.plan, rng, 160);
    for (int r = 0; r < nr; ++r) ranges.push_back(BatchRange{rng[r].start, rng[r].len, i, 0});
    const bool last_last = last_block_lands_last(g);
    const int grid = shuffle_last_block_grid(g);
    for (int c = 0; c < grid; ++c) (last_last ? post : pre).push_back(BatchLastCta{i, c, grid, 0});
    uint64_t c3 = g.grid[2] - g.grid[3], c2 = g.grid[1] - g.grid[2], c1 = g.grid[0] - g.grid[1];
    uint64_t c0 = g.n - g.grid[0];
    uint64_t segs[4][2] = {{g.anchors + c3, g.lm_prefix[2]},
                           {g.lm_prefix[2] + c2, g.lm_prefix[1]},
                           {g.lm_prefix[1] + c1, g.lm_prefix[0]},
                           {g.lm_prefix[0] + c0, qc_len(g)}};
    for (auto& sg : segs)
      if (sg[1] > sg[0]) zero_rel.push_back({off_qc[i] / sizeof(int32_t) + sg[0], sg[1] - sg[0]});
    GroupHost& G = gh[d.dtype_size == 8 ? 1 : 0];
    const int e = (int)G.idx.size();
    G.idx.push_back(i);
    G.ext.push_back(G.ext.back() + (d.mode == 1 ? (g.n + kBatchExtSeg - 1) / kBatchExtSeg : 0));
    std::vector<SampleWindow> w = sample_grid(g.nx, g.ny, g.nz);
    for (const SampleWindow& sw : w) G.wins.push_back(BatchWindow{sw, i, 0});
    G.win.push_back(G.win.back() + w.size());
    G.tile0.push_back(G.tile0.back() + tiles_in_part(g, 0));
    G.tile1.push_back(G.tile1.back() + tiles_in_part(g, 1));
    const uint64_t tr_bytes = 1040 + g.anchors * (uint64_t)d.dtype_size;
    G.tr.push_back(G.tr.back() + (tr_bytes + kBatchTrailerSeg - 1) / kBatchTrailerSeg);
    (void)e;
  }
  // ---- device layout ----
  size_t o_fields = cv.take<BatchField>(n), o_states = cv.take<BatchState>(n);
  size_t o_status = cv.take<unsigned long long>(std::max<size_t>(status_total, 1));
  size_t o_counters = cv.take<unsigned long long>(8), o_results = cv.take<BatchResult>(n);
  size_t o_shuf = cv.take<uint64_t>(n + 1), o_chunk = cv.take<uint64_t>(n + 1);
  size_t o_ranges = cv.take<BatchRange>(std::max<size_t>(ranges.size(), 1));
  size_t o_pre = cv.take<BatchLastCta>(std::max<size_t>(pre.size(), 1));
  size_t o_post = cv.take<BatchLastCta>(std::max<size_t>(post.size(), 1));
  size_t o_zero = cv.take<BatchZero>(std::max<size_t>(zero_rel.size(), 1));
  struct GroupOff { size_t idx, ext, extpart, win, wins, partial, t0, t1, tr; } go[2];
  for (int k = 0; k < 2; ++k) {
    GroupHost& G = gh[k];
    const int gn = (int)G.idx.size();
    const size_t ts = k ? 8 : 4;
    go[k].idx = cv.take<int>(std::max(gn, 1));
    go[k].ext = cv.take<uint64_t>(gn + 1);
    go[k].extpart = cv.take<unsigned char>(2 * ts * std::max<uint64_t>(G.ext.back(), 1));
    go[k].win = cv.take<uint64_t>(gn + 1);
    go[k].wins = cv.take<BatchWindow>(std::max<size_t>(G.wins.size(), 1));
    go[k].partial = cv.take<unsigned char>(15 * ts * std::max<size_t>(G.wins.size(), 1));
    go[k].t0 = cv.take<uint64_t>(gn + 1);
    go[k].t1 = cv.take<uint64_t>(gn + 1);
    go[k].tr = cv.take<uint64_t>(gn + 1);
  }
  cudaError_t e = cudaMalloc((void**)&b->dev, cv.off);
  if (e != cudaSuccess) return bfail(b, PRISM_ERR_NOMEM, "batch workspace", e);
  e = cudaMallocHost((void**)&b->h_results, sizeof(BatchResult) * n);
  if (e != cudaSuccess) return bfail(b, PRISM_ERR_NOMEM, "batch results", e);
  unsigned char* base = b->dev;
  for (int i = 0; i < n; ++i) {
    fields[i].qc = reinterpret_cast<int32_t*>(base + off_qc[i]);
    fields[i].planes = base + off_planes[i];
    fields[i].anchors = base + off_anchors[i];
    fields[i].status = reinterpret_cast<unsigned long long*>(base + o_status) + off_status[i];
    fields[i].st = reinterpret_cast<BatchState*>(base + o_states) + i;
  }
  std::vector<BatchZero> zeros;
  for (auto& z : zero_rel) zeros.push_back(BatchZero{reinterpret_cast<int32_t*>(base) + z.first, z.second});
  b->d_fields = reinterpret_cast<BatchField*>(base + o_fields);
  b->d_states = reinterpret_cast<BatchState*>(base + o_states);
  b->d_status = reinterpret_cast<unsigned long long*>(base + o_status);
  b->status_bytes = std::max<size_t>(status_total, 1) * sizeof(unsigned long long);
  b->d_counters = reinterpret_cast<unsigned long long*>(base + o_counters);
  b->d_results = reinterpret_cast<BatchResult*>(base + o_results);
  b->d_shuf_prefix = reinterpret_cast<uint64_t*>(base + o_shuf);
  b->d_chunk_prefix = reinterpret_cast<uint64_t*>(base + o_chunk);
  b->d_ranges = reinterpret_cast<BatchRange*>(base + o_ranges);
  b->d_pre = reinterpret_cast<BatchLastCta*>(base + o_pre);
  b->d_post = reinterpret_cast<BatchLastCta*>(base + o_post);
  b->d_zero = reinterpret_cast<BatchZero*>(base + o_zero);
  b->shuf_items = shuf_prefix[n];
  b->chunk_items = chunk_prefix[n];
  b->nranges = (int)ranges.size();
  b->npre = (int)pre.size();
  b->npost = (int)post.size();
  b->nzero = (int)zeros.size();
  auto up = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
    return bytes ? cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
  };
  BCK(up(b->d_fields, fields.data(), sizeof(BatchField) * n));
  BCK(up(b->d_shuf_prefix, shuf_prefix.data(), sizeof(uint64_t) * (n + 1)));
  BCK(up(b->d_chunk_prefix, chunk_prefix.data(), sizeof(uint64_t) * (n + 1)));
  BCK(up(b->d_ranges, ranges.data(), sizeof(BatchRange) * ranges.size()));
  BCK(up(b->d_pre, pre.data(), sizeof(BatchLastCta) * pre.size()));
  BCK(up(b->d_post, post.data(), sizeof(BatchLastCta) * post.size()));
  BCK(up(b->d_zero, zeros.data(), sizeof(BatchZero) * zeros.size()));
  for (int k = 0; k < 2; ++k) {
    GroupHost& G = gh[k];
    prism_batch::Group& gr = b->grp[k];
    gr.tsize = k ? 8 : 4;
    gr.n = (int)G.idx.size();
    gr.d_idx = reinterpret_cast<int*>(base + go[k].idx);
    gr.d_ext_prefix = reinterpret_cast<uint64_t*>(base + go[k].ext);
    gr.ext_items = G.ext.back();
    gr.d_ext_part = base + go[k].extpart;
    gr.d_win_prefix = reinterpret_cast<uint64_t*>(base + go[k].win);
    gr.nwin = G.wins.size();
    gr.d_wins = reinterpret_cast<BatchWindow*>(base + go[k].wins);
    gr.d_partial = base + go[k].partial;
    gr.d_tile_prefix[0] = reinterpret_cast<uint64_t*>(base + go[k].t0);
    gr.d_tile_prefix[1] = reinterpret_cast<uint64_t*>(base + go[k].t1);
    gr.tiles[0] = G.tile0.back();
    gr.tiles[1] = G.tile1.back();
    gr.d_tr_prefix = reinterpret_cast<uint64_t*>(base + go[k].tr);
    gr.tr_items = G.tr.back();
    if (!gr.n) continue;
    BCK(up(gr.d_idx, G.idx.data(), sizeof(int) * gr.n));
    BCK(up(gr.d_ext_prefix, G.ext.data(), sizeof(uint64_t) * (gr.n + 1)));
    BCK(up(gr.d_win_prefix, G.win.data(), sizeof(uint64_t) * (gr.n + 1)));
    BCK(up(gr.d_wins, G.wins.data(), sizeof(BatchWindow) * G.wins.size()));
    BCK(up(gr.d_tile_prefix[0], G.tile0.data(), sizeof(uint64_t) * (gr.n + 1)));
    BCK(up(gr.d_tile_prefix[1], G.tile1.data(), sizeof(uint64_t) * (gr.n + 1)));
    BCK(up(gr.d_tr_prefix, G.tr.data(), sizeof(uint64_t) * (gr.n + 1)));
  }
  // ---- occupancy limits of the persistent kernels ----
  int rc;
  int dummy = 0;
  if ((rc = max_ctas<batch_predict_kernel<float, 0>>(b, kPredThreads, compress_smem_bytes<float>(), &dummy))) return rc;
  if ((rc = max_ctas<batch_predict_kernel<float, 1>>(b, kPredThreads, compress_smem_bytes<float>(), &dummy))) return rc;
  if ((rc = max_ctas<batch_predict_kernel<double, 0>>(b, kPredThreads, compress_smem_bytes<double>(), &dummy)))
    return rc;
  if ((rc = max_ctas<batch_predict_kernel<double, 1>>(b, kPredThreads, compress_smem_bytes<double>(), &dummy)))
    return rc;
  if ((rc = max_ctas<batch_predict_persistent_kernel<float, 0>>(b, kPredThreads, compress_smem_bytes<float>(),
                                                                &b->pred_max[0])))
    return rc;
  if ((rc = max_ctas<batch_predict_persistent_kernel<float, 1>>(b, kPredThreads, compress_smem_bytes<float>(),
                                                                &dummy)))
    return rc;
  b->pred_max[0] = std::min(b->pred_max[0], dummy);
  if ((rc = max_ctas<batch_predict_persistent_kernel<double, 0>>(b, kPredThreads, compress_smem_bytes<double>(),
                                                                 &b->pred_max[1])))
    return rc;
  if ((rc = max_ctas<batch_predict_persistent_kernel<double, 1>>(b, kPredThreads, compress_smem_bytes<double>(),
                                                                 &dummy)))
    return rc;
  b->pred_max[1] = std::min(b->pred_max[1], dummy);
  if ((rc = max_ctas<batch_encode_kernel>(b, kZThreads, (int)sizeof(EncodeShared), &b->enc_max))) return rc;
  b->pred_ctas[0] = b->pred_max[0];
  b->pred_ctas[1] = b->pred_max[1];
  b->enc_ctas = b->enc_max;
  return PRISM_OK;
}

}  // namespace

int prism_batch_create(const prism_field_desc* fields, int n, int use_graph, prism_batch** out) {
  if (!fields || n <= 0 || !out) return PRISM_ERR_ARG;
  *out = nullptr;
  prism_batch* b = new (std::nothrow) prism_batch();
  if (!b) return PRISM_ERR_NOMEM;
  b->n = n;
  b->use_graph = use_graph != 0;
  b->desc.assign(fields, fields + n);
  b->geo.resize(n);
  for (int i = 0; i < n; ++i) {
    const prism_field_desc& d = fields[i];
    if (!d.d_in || !d.d_out || (d.dtype_size != 4 && d.dtype_size != 8) || !dims_ok(d.nx, d.ny, d.nz) ||
        !(d.bound > 0) || (d.mode != 0 && d.mode != 1)) {
      delete b;
      return PRISM_ERR_ARG;
    }
    make_geometry(d.nx, d.ny, d.nz, d.dtype_size, &b->geo[i]);
    const Geometry& g = b->geo[i];
    if (d.out_capacity < 8 + 2 * (uint64_t)g.chunks + g.aligned_size + 8 + g.header_size) {
      delete b;
      return PRISM_ERR_ARG;
    }
  }
  int rc = batch_plan(b);
  cudaStream_t st = nullptr;
  if (!rc && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) rc = PRISM_ERR_CUDA;
  if (!rc) rc = tune_schedule(b, st);
  if (!rc && b->use_graph) {
    uint64_t launches = 0;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = PRISM_ERR_CUDA;
    if (!rc) {
      rc = enqueue_all(b, st, launches);
      cudaGraph_t graph = nullptr;
      cudaError_t e = cudaStreamEndCapture(st, &graph);
      if (!rc && e != cudaSuccess) rc = PRISM_ERR_CUDA;
      b->graph = graph;
      if (!rc && cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) rc = PRISM_ERR_CUDA;
      b->launches_per_run = launches;
    }
  }
  if (st) cudaStreamDestroy(st);
  if (rc) {
    prism_batch_destroy(b);
    return rc;
  }
  *out = b;
  return PRISM_OK;
}

int prism_batch_compress(prism_batch* b, void* stream, uint64_t* sizes_out, uint8_t* flags_out) {
  if (!b || !sizes_out) return PRISM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (b->exec) {
    BCK(cudaGraphLaunch(b->exec, st));
  } else {
    uint64_t launches = 0;
    int rc = enqueue_all(b, st, launches);
    if (rc) return rc;
    b->launches_per_run = launches;
  }
  BCK(cudaStreamSynchronize(st));
  for (int i = 0; i < b->n; ++i) {
    const BatchResult& r = b->h_results[i];
    if (r.error_flag == 1) return bfail(b, PRISM_ERR_TIMEOUT, "look-back wait exceeded its limit");
    sizes_out[i] = r.padded_size + b->geo[i].header_size;
    if (flags_out) memcpy(flags_out + 8 * i, r.flags, 8);
  }
  return PRISM_OK;
}

int prism_batch_schedule(const prism_batch* b, int pred_ctas_per_sm[2], int* enc_ctas_per_sm, double tuned_ms[2],
                         uint64_t* launches_per_run) {
  if (!b) return PRISM_ERR_ARG;
  if (pred_ctas_per_sm) { pred_ctas_per_sm[0] = b->pred_ctas[0]; pred_ctas_per_sm[1] = b->pred_ctas[1]; }
  if (enc_ctas_per_sm) *enc_ctas_per_sm = b->enc_ctas;
  if (tuned_ms) { tuned_ms[0] = b->tuned_ms[0]; tuned_ms[1] = b->tuned_ms[1]; }
  if (launches_per_run) *launches_per_run = b->launches_per_run;
  return PRISM_OK;
}

const char* prism_batch_last_error(const prism_batch* b) { return b ? b->err.c_str() : "null batch"; }

void prism_batch_destroy(prism_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->dev) cudaFree(b->dev);
  if (b->h_results) cudaFreeHost(b->h_results);
  delete b;
}
