// Host side of the progressive-retrieval server (prism_server_* in
// prism_b200.h).  Included at the end of prism_b200.cu.
//
// The server keeps compressed fields and their partial reconstructions
// resident on the device and serves requests "field f at error bound t".
// A request's result is the reference's progressive retrieval of f to the
// plane selection that t calls for (the strategy from no planes): either in
// one step from no planes (strategy, decode of the selected planes, inverse
// shuffle, reconstruction), or -- when a reconstruction of f with a coarser
// selection is resident -- as a refinement step from that entry
// (src/prism.cu:126-138: output_old -> output_new, only the planes the entry
// lacks are decoded and their delta added) in exact mode
// (prism_progressive_exact: the reference's own refinement step misses the
// head of the first new plane and can end far from the one-step result).
// Both carry the same planes; they differ only by the floating-point
// rounding of the refinement sum.  Reconstructions are cached per (field,
// selected planes): a request whose selection is cached or being computed is
// served from that entry.
//
// Continuous batching: `slots` worker threads, each with its own stream and
// workspace, pull requests from one queue; a request is admitted when a slot
// is free and its reconstruction fits the HBM budget (least recently used
// idle entries are evicted first), so requests that arrive while others run
// start as soon as a slot and memory free up, and their kernels overlap on
// the device.  Requests that need the same entry at the same time share one
// computation.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <list>
#include <memory>
#include <thread>
#include <unordered_map>

namespace {

using SrvClock = std::chrono::steady_clock;

struct SrvField {
  uint8_t* d_cont = nullptr;
  uint64_t size = 0;
  int tsize = 4;
  uint32_t nx = 1, ny = 1, nz = 1;
  int mode = 1;
  double bound = 0, range = 1;
  uint64_t csbp[128];
  uint64_t value_bytes = 0;
  uint64_t workspace = 0;  // per-slot handle workspace this field needs
};

struct SrvEntry {
  int field = -1;
  int end[4] = {0, 0, 0, 0};
  int maxlevel = 0;
  void* d_values = nullptr;
  uint64_t bytes = 0;
  int pins = 0;
  bool ready = false;
  bool failed = false;
  uint64_t last_use = 0;
};

struct SrvRequest {
  uint64_t id = 0;
  int field = -1;
  double target = 0;
  void* out = nullptr;
  bool out_on_device = true;
  int status = 0;
  bool done = false;
  bool hit = false;
  bool refined = false;
  SrvClock::time_point t_submit, t_start, t_done;
  int end[4] = {0, 0, 0, 0};
  int maxlevel = 0;
  // plane selection: 0 not searched, 1 being searched (in another worker's
  // batch), 2 done (plan_* hold the result)
  int plan = 0;
  int plan_rc = 0;
  int plan_end[4] = {0, 0, 0, 0};
  int plan_maxlevel = 4;
};

// requests whose plane selections one worker searches in one batch
constexpr int kPlanBatch = 32;

// Handle workspace one slot needs for a field (what prism_progressive_step
// allocates: codes, planes, chunk tables, anchors, small state).
uint64_t srv_workspace_bytes(uint32_t nx, uint32_t ny, uint32_t nz, int tsize) {
  Geometry g;
  make_geometry(nx, ny, nz, tsize, &g);
  uint64_t b = qc_len(g) * 4 + g.aligned_size + 64 + (uint64_t)g.chunks * 24 + g.anchors * 16 + 65536;
  return b + b / 8;
}

}  // namespace

struct prism_server {
  std::mutex m;
  std::condition_variable cv_work, cv_done;
  std::deque<SrvRequest*> queue;
  std::unordered_map<uint64_t, SrvRequest*> reqs;
  std::vector<SrvField> fields;
  std::list<SrvEntry> cache;
  uint64_t budget = 0, used = 0, peak = 0, reserved = 0;
  uint64_t next_id = 1, clock = 0;
  int nslots = 1;
  std::vector<std::thread> workers;
  std::vector<cudaStream_t> streams;
  std::vector<prism_handle*> handles;
  std::vector<std::unique_ptr<std::mutex>> slot_mu;  // held while a slot's handle is in use
  bool stop = false;
  bool warmed = false;
  bool refine = true;  // misses refine the finest resident coarser entry of the field
  int device = 0;
  // statistics
  std::vector<double> lat_ms, queue_ms, service_ms;
  uint64_t completed = 0, hits = 0, shared = 0, evictions = 0, failed = 0, bytes_out = 0, refined = 0;
  uint64_t plan_calls = 0;  // batched plane searches run (each for up to kPlanBatch requests)
  SrvClock::time_point t0;
  std::string err;
};

namespace {

// Make room for `bytes` in the budget by evicting idle entries (LRU).  Caller
// holds the lock.
bool srv_reserve(prism_server* s, uint64_t bytes, cudaStream_t st) {
  while (s->used + s->reserved + bytes > s->budget) {
    auto victim = s->cache.end();
    for (auto it = s->cache.begin(); it != s->cache.end(); ++it)
      if (it->ready && it->pins == 0 && (victim == s->cache.end() || it->last_use < victim->last_use)) victim = it;
    if (victim == s->cache.end()) return false;
    cudaFreeAsync(victim->d_values, st);
    s->used -= victim->bytes;
    s->cache.erase(victim);
    ++s->evictions;
  }
  s->used += bytes;
  s->peak = std::max(s->peak, s->used + s->reserved);
  return true;
}

// The worker of one slot.
void srv_worker(prism_server* s, int slot) {
  cudaSetDevice(s->device);
  cudaStream_t st = s->streams[slot];
  prism_handle* h = s->handles[slot];
  std::unique_lock<std::mutex> lk(s->m);
  while (true) {
    s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
    if (s->stop) return;
    SrvRequest* r = s->queue.front();
    s->queue.pop_front();
    r->t_start = SrvClock::now();
    const SrvField f = s->fields[r->field];  // a copy: add_field may grow the vector
    // Plane selection of the one-step retrieval (the strategy of
    // prism_progressive_step from no planes, in absolute terms).  A request
    // not yet searched is searched together with up to kPlanBatch - 1 other
    // queued requests in one prism_find_strategy_batch call; a request that
    // another worker's batch is searching is waited for.
    std::vector<SrvRequest*> batch;
    std::vector<uint64_t> b_cs;
    std::vector<double> b_eb, b_te;
    if (r->plan == 0) {
      auto add = [&](SrvRequest* q) {
        const SrvField& fq = s->fields[q->field];
        q->plan = 1;
        batch.push_back(q);
        b_cs.insert(b_cs.end(), fq.csbp, fq.csbp + 128);
        b_eb.push_back(fq.mode == 1 ? fq.bound * fq.range : fq.bound);
        b_te.push_back(fq.mode == 1 ? q->target * fq.range : q->target);
      };
      add(r);
      for (SrvRequest* q : s->queue) {
        if ((int)batch.size() >= kPlanBatch) break;
        if (q->plan == 0) add(q);
      }
    } else {
      s->cv_done.wait(lk, [&] { return r->plan == 2; });
    }
    lk.unlock();
    std::unique_lock<std::mutex> slot_lk(*s->slot_mu[slot]);
    if (!batch.empty()) {
      const int nb = (int)batch.size();
      std::vector<int> bb(4 * nb, 0), be(4 * nb, 0), bm(nb, 4);
      const int brc = prism_find_strategy_batch(h, nb, b_cs.data(), b_eb.data(), b_te.data(), bb.data(), be.data(),
                                                bm.data(), st);
      lk.lock();
      ++s->plan_calls;
      for (int i = 0; i < nb; ++i) {
        SrvRequest* q = batch[i];
        q->plan_rc = brc;
        std::copy(be.begin() + 4 * i, be.begin() + 4 * i + 4, q->plan_end);
        q->plan_maxlevel = bm[i];
        q->plan = 2;
      }
      s->cv_done.notify_all();
      lk.unlock();
    }
    int end[4], maxlevel = r->plan_maxlevel;
    std::copy(r->plan_end, r->plan_end + 4, end);
    int rc = r->plan_rc;
    lk.lock();
    SrvEntry* e = nullptr;
    if (!rc) {
      for (auto& c : s->cache)
        if (c.field == r->field && !c.failed && std::equal(c.end, c.end + 4, end)) {
          e = &c;
          break;
        }
      if (e) {
        ++e->pins;
        if (e->ready) ++s->hits;
        else ++s->shared;
        r->hit = true;
        s->cv_done.wait(lk, [&] { return e->ready; });
        if (e->failed) rc = PRISM_ERR_CUDA;
      } else {
        // admission: wait until the entry fits, evicting idle entries; give
        // up only when nothing is in use that could still be released
        bool got = false;
        s->cv_done.wait(lk, [&] {
          if (s->stop) return true;
          if (srv_reserve(s, f.value_bytes, st)) {
            got = true;
            return true;
          }
          bool busy = false;
          for (auto& c : s->cache) busy |= c.pins > 0;
          return !busy;
        });
        if (!got) {
          rc = PRISM_ERR_NOMEM;
        } else {
          // refinement base: the finest resident entry of the field whose
          // planes are a subset of this selection (pinned while in use)
          SrvEntry* base = nullptr;
          int best = -1;
          if (s->refine)
            for (auto& c : s->cache) {
              if (c.field != r->field || !c.ready || c.failed || std::equal(c.end, c.end + 4, end)) continue;
              bool sub = true;
              int sum = 0;
              for (int l = 0; l < 4; ++l) {
                sub &= c.end[l] <= end[l];
                sum += c.end[l];
              }
              if (sub && sum > best) {
                best = sum;
                base = &c;
              }
            }
          if (base) {
            ++base->pins;
            ++s->refined;
            r->refined = true;
          }
          s->cache.emplace_back();
          e = &s->cache.back();
          e->field = r->field;
          std::copy(end, end + 4, e->end);
          e->maxlevel = maxlevel;
          e->bytes = f.value_bytes;
          e->pins = 1;
          const void* base_values = base ? base->d_values : nullptr;
          int base_end[4] = {0, 0, 0, 0};
          if (base) std::copy(base->end, base->end + 4, base_end);
          lk.unlock();
          void* p = nullptr;
          rc = cudaMallocAsync(&p, f.value_bytes, st) == cudaSuccess ? PRISM_OK : PRISM_ERR_NOMEM;
          prism_prog* pg = nullptr;
          if (!rc) rc = prism_progressive_open(h, f.d_cont, f.size, f.tsize, f.nx, f.ny, f.nz, f.mode, f.bound, &pg);
          if (!rc && base) rc = prism_progressive_exact(pg, 1);
          if (!rc && base) rc = prism_progressive_resume(pg, base_end, st);
          if (!rc) rc = base ? prism_progressive_step_into(pg, r->target, base_values, p, st)
                             : prism_progressive_step(pg, r->target, p, st);
          if (!rc) rc = prism_progressive_state(pg, nullptr, nullptr, nullptr, nullptr);  // waits, reports errors
          if (pg) prism_progressive_close(pg);
          lk.lock();
          if (base) --base->pins;
          e->d_values = p;
          e->ready = true;
          e->failed = rc != 0;
          s->cv_done.notify_all();
        }
      }
    }
    if (!rc && e) {
      e->last_use = ++s->clock;
      lk.unlock();
      cudaError_t ce = cudaMemcpyAsync(r->out, e->d_values, f.value_bytes,
                                       r->out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
      lk.lock();
      if (ce != cudaSuccess) rc = PRISM_ERR_CUDA;
    }
    if (e) {
      --e->pins;
      if (e->failed && e->pins == 0) {
        for (auto it = s->cache.begin(); it != s->cache.end(); ++it)
          if (&*it == e) {
            if (it->d_values) cudaFreeAsync(it->d_values, st);
            s->used -= it->bytes;
            s->cache.erase(it);
            break;
          }
      }
    }
    slot_lk.unlock();
    r->status = rc;
    std::copy(end, end + 4, r->end);
    r->maxlevel = maxlevel;
    r->t_done = SrvClock::now();
    r->done = true;
    if (rc) ++s->failed;
    else {
      ++s->completed;
      s->bytes_out += f.value_bytes;
      s->lat_ms.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
      s->queue_ms.push_back(std::chrono::duration<double, std::milli>(r->t_start - r->t_submit).count());
      s->service_ms.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_start).count());
    }
    s->cv_done.notify_all();
  }
}

}  // namespace

int prism_server_create(uint64_t hbm_budget, int slots, prism_server** out) {
  if (!out || slots < 1 || slots > 64 || hbm_budget == 0) return PRISM_ERR_ARG;
  *out = nullptr;
  prism_server* s = new (std::nothrow) prism_server();
  if (!s) return PRISM_ERR_NOMEM;
  s->budget = hbm_budget;
  s->nslots = slots;
  s->t0 = SrvClock::now();
  if (cudaGetDevice(&s->device) != cudaSuccess) {
    delete s;
    return PRISM_ERR_CUDA;
  }
  for (int i = 0; i < slots; ++i) {
    cudaStream_t st = nullptr;
    prism_handle* h = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess || prism_create(&h) != PRISM_OK) {
      if (st) cudaStreamDestroy(st);
      prism_server_destroy(s);
      return PRISM_ERR_CUDA;
    }
    s->streams.push_back(st);
    s->handles.push_back(h);
    s->slot_mu.emplace_back(new std::mutex());
  }
  // keep freed reconstruction memory in the stream-ordered pool instead of
  // returning it to the driver at every synchronisation (this process's
  // default pool only)
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  for (int i = 0; i < slots; ++i) s->workers.emplace_back(srv_worker, s, i);
  *out = s;
  return PRISM_OK;
}

int prism_server_add_field(prism_server* s, const void* container, uint64_t size, int on_device, int dtype_size,
                           uint32_t nx, uint32_t ny, uint32_t nz, int mode, double bound, int* field_id) {
  if (!s || !container || !field_id || (dtype_size != 4 && dtype_size != 8) || !dims_ok(nx, ny, nz) ||
      !(bound > 0) || (mode != 0 && mode != 1))
    return PRISM_ERR_ARG;
  Geometry g;
  make_geometry(nx, ny, nz, dtype_size, &g);
  if (size < g.header_size + 8 + 2 * (uint64_t)g.chunks) return PRISM_ERR_CORRUPT;
  SrvField f;
  f.size = size;
  f.tsize = dtype_size;
  f.nx = nx; f.ny = ny; f.nz = nz;
  f.mode = mode;
  f.bound = bound;
  f.value_bytes = g.n * (uint64_t)dtype_size;
  f.workspace = srv_workspace_bytes(nx, ny, nz, dtype_size);
  // trailer: range and cumulative plane sizes, needed for the plane selection
  std::vector<uint8_t> tr(1040);
  const uint8_t* src_tr = (const uint8_t*)container + (size - g.header_size);
  if (on_device) {
    if (cudaMemcpy(tr.data(), src_tr, 1040, cudaMemcpyDeviceToHost) != cudaSuccess) return PRISM_ERR_CUDA;
  } else {
    memcpy(tr.data(), src_tr, 1040);
  }
  memcpy(&f.range, tr.data() + 8, 8);
  memcpy(f.csbp, tr.data() + 16, 1024);
  std::unique_lock<std::mutex> lk(s->m);
  uint64_t ws = f.workspace * s->nslots;
  uint64_t new_reserved = std::max(s->reserved, ws);
  if (s->used + new_reserved + size > s->budget) return PRISM_ERR_NOMEM;
  s->reserved = new_reserved;
  s->used += size;
  s->peak = std::max(s->peak, s->used + s->reserved);
  lk.unlock();
  if (cudaMalloc(&f.d_cont, size) != cudaSuccess ||
      cudaMemcpy(f.d_cont, container, size, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    if (f.d_cont) cudaFree(f.d_cont);
    lk.lock();
    s->used -= size;
    return PRISM_ERR_CUDA;
  }
  // size every slot's workspace for this field now, so that no request grows
  // it (a cudaFree of the old workspace would stall the whole device); a
  // slot's mutex keeps its worker off the handle meanwhile
  for (size_t i = 0; i < s->handles.size(); ++i) {
    std::lock_guard<std::mutex> slk(*s->slot_mu[i]);
    prism_handle* h = s->handles[i];
    if (ensure_common(h, g) != PRISM_OK || h->zero_anchors.ensure(g.anchors * 8 + 64) != cudaSuccess) {
      lk.lock();
      s->used -= size;
      cudaFree(f.d_cont);
      return PRISM_ERR_NOMEM;
    }
  }
  lk.lock();
  s->fields.push_back(f);
  *field_id = (int)s->fields.size() - 1;
  return PRISM_OK;
}

int prism_server_submit(prism_server* s, int field_id, double target_error, void* out, int out_on_device,
                        uint64_t* request_id) {
  if (!s || !out || !request_id || !(target_error > 0)) return PRISM_ERR_ARG;
  SrvRequest* r = new (std::nothrow) SrvRequest();
  if (!r) return PRISM_ERR_NOMEM;
  std::lock_guard<std::mutex> lk(s->m);
  if (field_id < 0 || field_id >= (int)s->fields.size()) {
    delete r;
    return PRISM_ERR_ARG;
  }
  if (!s->warmed) {
    // Map the reconstruction part of the budget into the stream-ordered pool
    // once, so that cache misses sub-allocate instead of growing the pool
    // (a fresh mapping of a GB-sized entry costs tens of milliseconds).
    s->warmed = true;
    const uint64_t room = s->budget > s->used + s->reserved ? s->budget - s->used - s->reserved : 0;
    void* p = nullptr;
    if (room > 0 && cudaMallocAsync(&p, room, s->streams[0]) == cudaSuccess) cudaFreeAsync(p, s->streams[0]);
    cudaStreamSynchronize(s->streams[0]);
    cudaGetLastError();  // a refused warm-up only costs speed
  }
  r->id = s->next_id++;
  r->field = field_id;
  r->target = target_error;
  r->out = out;
  r->out_on_device = out_on_device != 0;
  r->t_submit = SrvClock::now();
  s->reqs[r->id] = r;
  s->queue.push_back(r);
  s->cv_work.notify_one();
  *request_id = r->id;
  return PRISM_OK;
}

int prism_server_wait(prism_server* s, uint64_t request_id, double* latency_ms, int end[4], int* maxlevel,
                      int* from_cache) {
  if (!s) return PRISM_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) return PRISM_ERR_ARG;
  SrvRequest* r = it->second;
  s->cv_done.wait(lk, [&] { return r->done; });
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  if (end) std::copy(r->end, r->end + 4, end);
  if (maxlevel) *maxlevel = r->maxlevel;
  if (from_cache) *from_cache = r->hit ? 1 : (r->refined ? 2 : 0);
  int rc = r->status;
  s->reqs.erase(it);
  delete r;
  return rc;
}

int prism_server_poll(prism_server* s, uint64_t request_id, int* done) {
  if (!s || !done) return PRISM_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->m);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) return PRISM_ERR_ARG;
  *done = it->second->done ? 1 : 0;
  return PRISM_OK;
}

int prism_server_stats_get(prism_server* s, prism_server_stats* out, int reset) {
  if (!s || !out) return PRISM_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->m);
  memset(out, 0, sizeof(*out));
  out->completed = s->completed;
  out->cache_hits = s->hits;
  out->shared = s->shared;
  out->evictions = s->evictions;
  out->failed = s->failed;
  out->bytes_out = s->bytes_out;
  out->bytes_resident = s->used;
  out->bytes_reserved = s->reserved;
  out->bytes_peak = s->peak;
  out->elapsed_s = std::chrono::duration<double>(SrvClock::now() - s->t0).count();
  out->refined = s->refined;
  out->plan_calls = s->plan_calls;
  auto pct = [](std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    return v[std::min(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5))];
  };
  if (!s->lat_ms.empty()) {
    out->p50_ms = pct(s->lat_ms, 0.50);
    out->p99_ms = pct(s->lat_ms, 0.99);
    double sum = 0;
    for (double x : s->lat_ms) sum += x;
    out->mean_ms = sum / s->lat_ms.size();
    out->max_ms = pct(s->lat_ms, 1.0);
    out->queue_p50_ms = pct(s->queue_ms, 0.50);
    out->queue_p99_ms = pct(s->queue_ms, 0.99);
    out->service_p50_ms = pct(s->service_ms, 0.50);
    out->service_p99_ms = pct(s->service_ms, 0.99);
  }
  if (reset) {
    s->lat_ms.clear();
    s->queue_ms.clear();
    s->service_ms.clear();
    s->completed = s->hits = s->shared = s->evictions = s->failed = s->bytes_out = s->refined = s->plan_calls = 0;
    s->t0 = SrvClock::now();
  }
  return PRISM_OK;
}

int prism_server_set_refine(prism_server* s, int enable) {
  if (!s) return PRISM_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->m);
  s->refine = enable != 0;
  return PRISM_OK;
}

void prism_server_destroy(prism_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->stop = true;
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  for (auto& t : s->workers) t.join();
  for (size_t i = 0; i < s->streams.size(); ++i) cudaStreamSynchronize(s->streams[i]);
  for (auto& c : s->cache)
    if (c.d_values) cudaFree(c.d_values);
  for (auto& f : s->fields)
    if (f.d_cont) cudaFree(f.d_cont);
  for (prism_handle* h : s->handles) prism_destroy(h);
  for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
  for (auto& kv : s->reqs) delete kv.second;
  delete s;
}
