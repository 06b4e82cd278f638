// server.cu -- resident columns under a memory budget and continuously batched requests.
//
// The reference has no serving layer: every LeCoGPU<T> method is a blocking host round trip
// (api/G-LeCo.cuh:615-678 random access, :1878-1928 fixed random access).  Here compressed
// columns stay resident in HBM and a worker thread turns a stream of lookup and range-decode
// requests into shared launches:
//  - a request is scheduled once its arrival time (not_before_ns) has passed;
//  - every request waiting when a launch slot is free goes into that slot: all lookup requests
//    into one lookup launch (any columns, any element types), range requests as pieces of at most
//    max_range_values values into one persistent decode launch over a device work list
//    (batch_decode_kernel), so a 16M-value range cannot hold back small requests;
//  - up to `slots` launches are on the GPU at once, each on its own stream; requests that arrive
//    meanwhile wait for the next free slot (continuous batching);
//  - a request completes when the last launch carrying a piece of it has completed.
// Admission keeps the device bytes of resident columns under the budget, evicting idle columns
// least recently used first.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <queue>
#include <thread>
#include <vector>

#include "glc_internal.h"

using namespace glc;

namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Device bytes a column holds: the reference SoA arrays (start, end, model type, 4 parameters,
// bits, bit offset, error bound), the partition descriptors, the tile table, the padded
// bitstream and the optional pre-unpacked residuals.
uint64_t column_device_bytes(const glc_column* c) {
  const uint64_t P = (uint64_t)c->P;
  if (c->blob_view)  // an attached blob: the blob (or its bitstream) it holds and its derived tables
    return c->owned_bytes + P * sizeof(PartDesc) + sizeof(TileInfo) * (uint64_t)(c->ntiles + 1) +
           (c->d_plain ? 8ull * (uint64_t)c->n + 16 : 0);
  uint64_t b = P * (4 + 4 + 4 + 32 + 4 + 8 + 8) + P * sizeof(PartDesc) + sizeof(TileInfo) * (uint64_t)(c->ntiles + 1);
  if (c->d_words) b += 4ull * (uint64_t)c->nwords_alloc;
  if (c->d_plain) b += 8ull * (uint64_t)c->n + 16;
  return b;
}

constexpr int kMaxSlots = 16;
constexpr int kMaxColsPerLaunch = 256;

struct SrvColumn {
  glc_column* col = nullptr;  // null once freed
  uint64_t bytes = 0;
  int64_t pins = 0;           // submitted requests not yet completed
  uint64_t last_use = 0;
  bool evicting = false;
  RAColumn ra{};
  BatchColumn bc{};
};

struct Req {
  glc_request r;
  int64_t arrival = 0;
  int64_t next = 0;      // RANGE: first position not yet scheduled
  int32_t pieces = 0;    // pieces in launches that have not completed
  int32_t launches = 0;
  int32_t status = GLC_OK;
  int32_t esize = 0;
  bool in_place = false;  // RANGE: out - first * esize is 16-byte aligned
  RAColumn ra{};
  BatchColumn bc{};
  bool scheduled() const { return r.kind == GLC_REQ_LOOKUP ? launches > 0 : next == r.first + r.count; }
};

struct Copy {
  void* dst;
  const void* src;
  size_t bytes;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;     // everything of the launch has completed
  cudaEvent_t lk_done = nullptr;  // its lookup kernel has completed (lookups finish early)
  uint8_t* h_meta = nullptr;      // pinned staging of the launch's tables
  uint8_t* d_meta = nullptr;
  uint8_t* d_stage = nullptr;     // range pieces whose output is not 16-byte aligned
  int* h_err = nullptr;           // mapped host word: the launch's device error code
  int* d_err = nullptr;           // its device address
  bool busy = false;
  bool lookups_pending = false;   // lreqs not yet reported
  std::vector<Req*> lreqs;        // lookup requests of the launch
  std::vector<Req*> rreqs;        // one entry per range piece
};

}  // namespace

struct glc_server {
  glc_ctx* ctx = nullptr;
  glc_server_config cfg{};
  cudaMemPool_t pool = nullptr;  // arrays of the columns admitted from blobs
  int64_t max_work = 0;
  size_t meta_cap = 0, stage_cap = 0;

  std::mutex mu;                  // everything below up to `worker`
  std::condition_variable wake;   // worker: new requests or stop
  std::condition_variable idle;   // drain: completed == submitted
  std::vector<SrvColumn> cols;    // id = index
  std::vector<Req*> incoming;
  std::deque<glc_completion> done;
  std::vector<glc_column*> to_free;  // evicted columns whose requests have all completed
  uint64_t resident_bytes = 0;
  int32_t resident_columns = 0;
  uint64_t tick = 0;
  glc_server_stats st{};
  bool stop = false;
  std::atomic<int> n_incoming{0};
  std::atomic<int> in_flight{0};

  std::thread worker;
  Slot slots[kMaxSlots];
  // worker-only state
  std::vector<RAColumn> w_ra;
  std::vector<BatchColumn> w_bc;
  std::vector<RARequest> w_req;
  std::vector<BatchWork> w_work;  // range pieces of the launch being built
  std::vector<int64_t> w_tb;       // tiles before each piece
  std::vector<Copy> w_copy;
  std::vector<int32_t> w_dtype;
  std::vector<int32_t> w_colmap;    // column id -> local index + 1 (valid when w_epoch matches)
  std::vector<uint64_t> w_epoch;
  uint64_t launch_no = 0;
};

namespace {

glc_status sfail(glc_ctx* ctx, glc_status s, const char* msg) {
  if (ctx) ctx->err = msg;
  return s;
}

glc_status scuda(glc_ctx* ctx, cudaError_t e, const char* where) {
  if (ctx) ctx->err = std::string(where) + ": " + cudaGetErrorString(e);
  return GLC_ERR_CUDA;
}

size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

// Completes a request whose last piece has finished (caller holds mu).
void complete_locked(glc_server* S, Req* r, int64_t t) {
  glc_completion c;
  c.tag = r->r.tag;
  c.status = r->status;
  c.launches = r->launches;
  c.arrival_ns = r->arrival;
  c.done_ns = t;
  S->done.push_back(c);
  SrvColumn& col = S->cols[r->r.column];
  if (--col.pins == 0 && col.evicting && col.col) {
    S->to_free.push_back(col.col);
    col.col = nullptr;
  }
  S->st.completed++;
  if (r->r.kind == GLC_REQ_LOOKUP) S->st.lookups += r->r.count;
  else S->st.range_values += r->r.count;
  delete r;
}

// Reports the pieces in v as finished with `status` (launch errors override GLC_OK).
void finish_pieces(glc_server* S, std::vector<Req*>& v, int32_t status) {
  if (v.empty()) return;
  const int64_t t = now_ns();
  bool all_done;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    for (Req* r : v) {
      if (status != GLC_OK) r->status = status;
      if (--r->pieces == 0 && r->scheduled()) complete_locked(S, r, t);
    }
    all_done = S->st.completed == S->st.submitted;
  }
  v.clear();
  if (all_done) S->idle.notify_all();
}

void finish_slot(glc_server* S, Slot& sl, cudaError_t q) {
  const int dev_err = (q == cudaSuccess) ? *sl.h_err : 0;
  const int32_t status = q != cudaSuccess ? GLC_ERR_CUDA : (dev_err ? GLC_ERR_TIMEOUT : GLC_OK);
  finish_pieces(S, sl.lreqs, q != cudaSuccess ? GLC_ERR_CUDA : GLC_OK);
  finish_pieces(S, sl.rreqs, status);
  sl.lookups_pending = false;
  sl.busy = false;
  S->in_flight.fetch_sub(1);
}

int local_col(glc_server* S, const Req* r) {
  const int32_t id = r->r.column;
  if ((size_t)id >= S->w_colmap.size()) {
    S->w_colmap.resize((size_t)id + 64, 0);
    S->w_epoch.resize((size_t)id + 64, 0);
  }
  if (S->w_epoch[id] == S->launch_no) return S->w_colmap[id] - 1;
  if ((int)S->w_ra.size() >= kMaxColsPerLaunch) return -1;
  S->w_epoch[id] = S->launch_no;
  S->w_colmap[id] = (int32_t)S->w_ra.size() + 1;
  S->w_ra.push_back(r->ra);
  S->w_bc.push_back(r->bc);
  return (int)S->w_ra.size() - 1;
}

// Packs waiting requests into slot sl and launches it.
void launch_slot(glc_server* S, Slot& sl, std::deque<Req*>& ready_l, std::deque<Req*>& ready_r) {
  S->launch_no++;
  S->w_ra.clear();
  S->w_bc.clear();
  S->w_req.clear();
  S->w_work.clear();
  S->w_copy.clear();
  const glc_server_config& cfg = S->cfg;

  int64_t nl = 0;
  while (!ready_l.empty() && (int64_t)S->w_req.size() < cfg.max_requests) {
    Req* r = ready_l.front();
    if (nl > 0 && nl + r->r.count > cfg.max_lookups) break;
    const int li = local_col(S, r);
    if (li < 0) break;
    RARequest q;
    q.base = nl;
    q.col = li;
    q.pad = 0;
    q.pos = r->r.positions;
    q.out = (uint8_t*)r->r.out;
    S->w_req.push_back(q);
    nl += r->r.count;
    r->pieces++;
    r->launches++;
    sl.lreqs.push_back(r);
    ready_l.pop_front();
  }

  int64_t budget = cfg.max_range_values;
  int max_bits = 0;
  size_t stage_off = 0;
  int npieces = 0;
  while (!ready_r.empty() && budget > 0 && npieces < cfg.max_requests) {
    Req* r = ready_r.front();
    const int li = local_col(S, r);
    if (li < 0) break;
    const int64_t end = r->r.first + r->r.count;
    const int64_t lo = r->next, hi = std::min(end, lo + budget);
    const int64_t es = r->esize;
    uintptr_t base;
    if (r->in_place) {
      base = (uintptr_t)r->r.out - (uintptr_t)(r->r.first * es);
    } else {  // stage so that stage + off - lo * es is 16-byte aligned, then copy out
      const size_t want = (size_t)(lo * es) & 15;
      stage_off += (want - (stage_off & 15)) & 15;
      base = (uintptr_t)sl.d_stage + stage_off - (uintptr_t)(lo * es);
      S->w_copy.push_back(Copy{(uint8_t*)r->r.out + (lo - r->r.first) * es, sl.d_stage + stage_off,
                               (size_t)((hi - lo) * es)});
      stage_off += (size_t)((hi - lo) * es);
    }
    S->w_work.push_back(BatchWork{li, (int32_t)(lo / kDecodeTile), lo, hi, (void*)base});  // one per piece
    max_bits = std::max(max_bits, (int)r->bc.max_bits);
    budget -= hi - lo;
    r->next = hi;
    r->pieces++;
    r->launches++;
    sl.rreqs.push_back(r);
    npieces++;
    if (hi == end) ready_r.pop_front();
  }

  // Range pieces grouped by element type (the decode runs one type per CTA); their tiles become
  // the decode's work items on the device (expand_pieces_kernel), group order kept.
  int64_t group_begin[5] = {0, 0, 0, 0, 0};
  npieces = (int)S->w_work.size();  // pieces after the loop (equal to its count)
  S->w_tb.assign((size_t)npieces + 1, 0);
  if (npieces > 0) {
    S->w_dtype.resize(S->w_bc.size());
    for (size_t i = 0; i < S->w_bc.size(); i++) S->w_dtype[i] = S->w_bc[i].dtype;
    group_work_by_type(S->w_work, S->w_dtype, group_begin);
    for (int p = 0; p < npieces; p++) {
      const BatchWork& w = S->w_work[p];
      S->w_tb[p + 1] = S->w_tb[p] + (w.hi + kDecodeTile - 1) / kDecodeTile - w.lo / kDecodeTile;
    }
    for (int d = 0; d < 5; d++) group_begin[d] = S->w_tb[group_begin[d]];  // in tiles
  }
  const int64_t ntiles = S->w_tb[npieces];

  // One host-to-device copy of all tables: [4 decode work counters u64][lookup columns]
  // [decode columns][lookup requests][range pieces][piece tile bases]; the per-tile work items
  // follow on the device only.
  const size_t o_ra = 32;
  const size_t o_bc = align16(o_ra + sizeof(RAColumn) * S->w_ra.size());
  const size_t o_req = align16(o_bc + sizeof(BatchColumn) * S->w_bc.size());
  const size_t o_piece = align16(o_req + sizeof(RARequest) * S->w_req.size());
  const size_t o_tb = align16(o_piece + sizeof(BatchWork) * (size_t)npieces);
  const size_t o_work = align16(o_tb + sizeof(int64_t) * ((size_t)npieces + 1));
  const size_t total = o_work;
  std::memset(sl.h_meta, 0, 32);
  std::memcpy(sl.h_meta + o_ra, S->w_ra.data(), sizeof(RAColumn) * S->w_ra.size());
  std::memcpy(sl.h_meta + o_bc, S->w_bc.data(), sizeof(BatchColumn) * S->w_bc.size());
  std::memcpy(sl.h_meta + o_req, S->w_req.data(), sizeof(RARequest) * S->w_req.size());
  std::memcpy(sl.h_meta + o_piece, S->w_work.data(), sizeof(BatchWork) * (size_t)npieces);
  std::memcpy(sl.h_meta + o_tb, S->w_tb.data(), sizeof(int64_t) * ((size_t)npieces + 1));
  *sl.h_err = 0;

  cudaError_t e = cudaMemcpyAsync(sl.d_meta, sl.h_meta, total, cudaMemcpyHostToDevice, sl.stream);
  if (e == cudaSuccess && nl > 0)
    e = launch_multi_lookup((const RAColumn*)(sl.d_meta + o_ra), (const RARequest*)(sl.d_meta + o_req),
                            (int)S->w_req.size(), nl, S->ctx->num_sms, sl.stream);
  sl.lookups_pending = false;
  if (e == cudaSuccess && nl > 0 && npieces > 0) {  // lookups need not wait for the decode
    e = cudaEventRecord(sl.lk_done, sl.stream);
    sl.lookups_pending = e == cudaSuccess;
  }
  if (e == cudaSuccess && npieces > 0)
    e = launch_expand_pieces((const BatchWork*)(sl.d_meta + o_piece), (const int64_t*)(sl.d_meta + o_tb), npieces,
                             ntiles, (BatchWork*)(sl.d_meta + o_work), S->ctx->num_sms, sl.stream);
  if (e == cudaSuccess && npieces > 0) {
    BatchDecodeArgs a;
    a.cols = (const BatchColumn*)(sl.d_meta + o_bc);
    a.work = (const BatchWork*)(sl.d_meta + o_work);
    a.nwork = ntiles;
    for (int d = 0; d < 5; d++) a.group_begin[d] = group_begin[d];
    a.counter = (unsigned long long*)sl.d_meta;
    a.err = sl.d_err;
    a.stage_bytes = batch_stage_bytes(max_bits);
    e = launch_batch_decode_zeroed(a, S->ctx->num_sms, sl.stream);
  }
  for (size_t i = 0; e == cudaSuccess && i < S->w_copy.size(); i++)
    e = cudaMemcpyAsync(S->w_copy[i].dst, S->w_copy[i].src, S->w_copy[i].bytes, cudaMemcpyDeviceToDevice, sl.stream);
  if (e != cudaSuccess) {
    for (Req* r : sl.lreqs) r->status = GLC_ERR_CUDA;
    for (Req* r : sl.rreqs) r->status = GLC_ERR_CUDA;
  }
  sl.busy = true;
  S->in_flight.fetch_add(1);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->st.launches++;
  }
  if (cudaEventRecord(sl.done, sl.stream) != cudaSuccess) finish_slot(S, sl, cudaErrorUnknown);
}

void worker_main(glc_server* S) {
  cudaSetDevice(S->ctx->device);
  // Requests not yet arrived: a FIFO for the usual case of submissions in arrival order, and a
  // heap for the ones that arrive earlier than a request already queued.
  auto later = [](const Req* a, const Req* b) { return a->arrival > b->arrival; };
  std::priority_queue<Req*, std::vector<Req*>, decltype(later)> future_heap(later);
  std::deque<Req*> future_fifo;
  std::deque<Req*> ready_l, ready_r;
  std::vector<Req*> fresh;
  const int nslots = S->cfg.slots;
  auto next_arrival = [&]() -> int64_t {
    int64_t t = INT64_MAX;
    if (!future_fifo.empty()) t = future_fifo.front()->arrival;
    if (!future_heap.empty() && future_heap.top()->arrival < t) t = future_heap.top()->arrival;
    return t;
  };
  for (;;) {
    bool any_busy = false;
    for (int i = 0; i < nslots; i++) {
      Slot& sl = S->slots[i];
      if (!sl.busy) continue;
      if (sl.lookups_pending && cudaEventQuery(sl.lk_done) == cudaSuccess) {
        finish_pieces(S, sl.lreqs, GLC_OK);
        sl.lookups_pending = false;
      }
      const cudaError_t q = cudaEventQuery(sl.done);
      if (q == cudaErrorNotReady) {
        any_busy = true;
        continue;
      }
      finish_slot(S, sl, q);
    }
    if (S->n_incoming.load(std::memory_order_acquire) > 0) {
      {
        std::lock_guard<std::mutex> lk(S->mu);
        fresh.swap(S->incoming);
        S->n_incoming.store(0, std::memory_order_relaxed);
      }
      for (Req* r : fresh) {
        if (future_fifo.empty() || r->arrival >= future_fifo.back()->arrival) future_fifo.push_back(r);
        else future_heap.push(r);
      }
      fresh.clear();
    }
    const int64_t t = now_ns();
    for (;;) {  // move every arrived request to its ready queue, in arrival order
      Req* r = nullptr;
      const bool f = !future_fifo.empty() && future_fifo.front()->arrival <= t;
      const bool h = !future_heap.empty() && future_heap.top()->arrival <= t;
      if (f && (!h || future_fifo.front()->arrival <= future_heap.top()->arrival)) {
        r = future_fifo.front();
        future_fifo.pop_front();
      } else if (h) {
        r = future_heap.top();
        future_heap.pop();
      } else {
        break;
      }
      (r->r.kind == GLC_REQ_LOOKUP ? ready_l : ready_r).push_back(r);
    }
    if (!ready_l.empty() || !ready_r.empty()) {
      Slot* free_slot = nullptr;
      for (int i = 0; i < nslots && !free_slot; i++)
        if (!S->slots[i].busy) free_slot = &S->slots[i];
      if (free_slot) {
        launch_slot(S, *free_slot, ready_l, ready_r);
        continue;
      }
    }
    if (any_busy || !ready_l.empty() || !ready_r.empty()) {
      std::this_thread::yield();
      continue;
    }
    // Nothing on the GPU and nothing ready: wait for a submission, the next arrival or stop.
    const int64_t na = next_arrival();
    if (na != INT64_MAX && na - t < 200000) {
      std::this_thread::yield();  // arrival within 200 us: keep polling for punctual scheduling
      continue;
    }
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->stop && S->incoming.empty() && na == INT64_MAX) break;
    if (!S->incoming.empty()) continue;
    if (na == INT64_MAX) {
      S->wake.wait(lk, [&] { return S->stop || !S->incoming.empty(); });
    } else {
      const auto until = std::chrono::steady_clock::time_point(std::chrono::nanoseconds(na - 100000));
      S->wake.wait_until(lk, until, [&] { return S->stop || !S->incoming.empty(); });
    }
  }
}

// Frees evicted columns whose requests have completed (outside the lock: cudaFree synchronises).
void free_pending(glc_server* S) {
  std::vector<glc_column*> v;
  std::vector<uint64_t> bytes;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    v.swap(S->to_free);
  }
  uint64_t freed = 0;
  for (glc_column* c : v) {
    freed += column_device_bytes(c);
    glc_column_free(c);
  }
  if (!v.empty()) {
    std::lock_guard<std::mutex> lk(S->mu);
    S->resident_bytes -= freed;
    S->resident_columns -= (int32_t)v.size();
  }
}

void fill_views(SrvColumn& sc) {
  const glc_column* c = sc.col;
  sc.ra.desc = c->d_desc;
  sc.ra.starts = c->d_start;
  sc.ra.words = c->d_words;
  sc.ra.P = c->P;
  sc.ra.n = c->n;
  sc.ra.fixed_len = c->fixed_len;
  sc.ra.dtype = (int32_t)c->dtype;
  sc.bc.desc = c->d_desc;
  sc.bc.starts = c->d_start;
  sc.bc.tiles = c->d_tiles;
  sc.bc.words = c->d_words;
  sc.bc.n = c->n;
  sc.bc.dtype = (int32_t)c->dtype;
  sc.bc.max_bits = c->max_bits;
}

void destroy_slots(glc_server* S) {
  for (int i = 0; i < kMaxSlots; i++) {
    Slot& sl = S->slots[i];
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.lk_done) cudaEventDestroy(sl.lk_done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    if (sl.h_meta) cudaFreeHost(sl.h_meta);
    if (sl.h_err) cudaFreeHost(sl.h_err);
    if (sl.d_meta) cudaFree(sl.d_meta);
    if (sl.d_stage) cudaFree(sl.d_stage);
    sl = Slot();
  }
}

}  // namespace

extern "C" {

int64_t glc_server_now_ns(void) { return now_ns(); }

glc_status glc_server_create(glc_ctx* ctx, const glc_server_config* config, glc_server** out) {
  if (!ctx || !config || !out) return sfail(ctx, GLC_ERR_INVALID_ARG, "server: null argument");
  *out = nullptr;
  glc_server_config c = *config;
  if (c.budget_bytes == 0) return sfail(ctx, GLC_ERR_INVALID_ARG, "server: budget_bytes must be > 0");
  if (c.slots == 0) c.slots = 4;
  if (c.max_requests == 0) c.max_requests = 4096;
  if (c.max_lookups == 0) c.max_lookups = 1ll << 22;
  if (c.max_range_values == 0) c.max_range_values = 1ll << 24;
  if (c.slots < 1 || c.slots > kMaxSlots || c.max_requests < 1 || c.max_requests > (1 << 20) || c.max_lookups < 1 ||
      c.max_range_values < 1 || c.max_range_values > (1ll << 30) || (c.flags & ~GLC_SERVER_RESERVE) != 0)
    return sfail(ctx, GLC_ERR_INVALID_ARG, "server: configuration out of range");
  glc_server* S = new (std::nothrow) glc_server();
  if (!S) return GLC_ERR_OOM;
  S->ctx = ctx;
  S->cfg = c;
  // Work items: every full tile of the launch's range values plus two partial tiles per piece.
  S->max_work = c.max_range_values / kDecodeTile + 2ll * c.max_requests + 2;
  S->meta_cap = align16(32 + (sizeof(RAColumn) + sizeof(BatchColumn)) * kMaxColsPerLaunch + 64 +
                        sizeof(RARequest) * (size_t)c.max_requests + sizeof(BatchWork) * (size_t)c.max_requests +
                        sizeof(int64_t) * ((size_t)c.max_requests + 1) + 48 + sizeof(BatchWork) * (size_t)S->max_work);
  S->stage_cap = (size_t)c.max_range_values * 8 + 16 * (size_t)c.max_requests + 256;
  glc::DeviceScope device_scope(ctx->device);
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < c.slots && e == cudaSuccess; i++) {
    Slot& sl = S->slots[i];
    if ((e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking)) != cudaSuccess) break;
    if ((e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming)) != cudaSuccess) break;
    if ((e = cudaEventCreateWithFlags(&sl.lk_done, cudaEventDisableTiming)) != cudaSuccess) break;
    if ((e = cudaHostAlloc((void**)&sl.h_meta, S->meta_cap, cudaHostAllocDefault)) != cudaSuccess) break;
    // the decode kernel stores its error code straight into this mapped host word
    if ((e = cudaHostAlloc((void**)&sl.h_err, 64, cudaHostAllocMapped)) != cudaSuccess) break;
    if ((e = cudaHostGetDevicePointer((void**)&sl.d_err, sl.h_err, 0)) != cudaSuccess) break;
    if ((e = cudaMalloc((void**)&sl.d_meta, S->meta_cap)) != cudaSuccess) break;
    e = cudaMalloc((void**)&sl.d_stage, S->stage_cap);
  }
  if (e == cudaSuccess) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctx->device;
    uint64_t keep = ~0ull;
    e = cudaMemPoolCreate(&S->pool, &props);
    if (e == cudaSuccess) e = cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e == cudaSuccess && (c.flags & GLC_SERVER_RESERVE)) {  // grow the pool once; freed memory stays
      void* p = nullptr;
      e = cudaMallocFromPoolAsync(&p, c.budget_bytes, S->pool, ctx->own_stream);
      if (e == cudaSuccess) e = cudaFreeAsync(p, ctx->own_stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->own_stream);
    }
  }
  if (e != cudaSuccess) {
    destroy_slots(S);
    if (S->pool) cudaMemPoolDestroy(S->pool);
    delete S;
    return scuda(ctx, e, "server: slot resources");
  }
  S->worker = std::thread(worker_main, S);
  *out = S;
  return GLC_OK;
}

glc_status glc_server_drain(glc_server* S, int64_t timeout_ms) {
  if (!S) return GLC_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto pred = [&] { return S->st.completed == S->st.submitted; };
  if (timeout_ms < 0) {
    S->idle.wait(lk, pred);
    return GLC_OK;
  }
  if (!S->idle.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred))
    return sfail(S->ctx, GLC_ERR_TIMEOUT, "server: requests still outstanding");
  return GLC_OK;
}

glc_status glc_server_destroy(glc_server* S) {
  if (!S) return GLC_ERR_INVALID_ARG;
  glc_server_drain(S, -1);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->wake.notify_all();
  if (S->worker.joinable()) S->worker.join();
  glc::DeviceScope device_scope(S->ctx->device);
  for (int i = 0; i < kMaxSlots; i++)
    if (S->slots[i].stream) cudaStreamSynchronize(S->slots[i].stream);
  free_pending(S);
  for (SrvColumn& c : S->cols)
    if (c.col) glc_column_free(c.col);
  cudaStreamSynchronize(S->ctx->own_stream);  // pooled arrays are released on the context's stream
  destroy_slots(S);
  cudaMemPoolDestroy(S->pool);
  delete S;
  return GLC_OK;
}

glc_status glc_server_admit(glc_server* S, glc_column* col, int32_t* id) {
  if (!S || !col || !id) return sfail(S ? S->ctx : nullptr, GLC_ERR_INVALID_ARG, "server admit: null argument");
  if (col->view) return sfail(S->ctx, GLC_ERR_INVALID_ARG, "server admit: column is owned by a batch");
  if (col->ctx && col->ctx->device != S->ctx->device)
    return sfail(S->ctx, GLC_ERR_INVALID_ARG, "server admit: column is on another device");
  if (!col->d_words || col->n <= 0)
    return sfail(S->ctx, GLC_ERR_UNSUPPORTED, "server admit: column has no packed bitstream or no values");
  free_pending(S);
  const uint64_t need = column_device_bytes(col);
  std::vector<glc_column*> victims;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (need > S->cfg.budget_bytes) {
      S->st.admissions_refused++;
      return sfail(S->ctx, GLC_ERR_BUDGET, "server admit: column larger than the budget");
    }
    if (S->resident_bytes + need > S->cfg.budget_bytes) {
      std::vector<int32_t> idle;
      for (size_t i = 0; i < S->cols.size(); i++) {
        const SrvColumn& c = S->cols[i];
        if (c.col && !c.evicting && c.pins == 0) idle.push_back((int32_t)i);
      }
      std::sort(idle.begin(), idle.end(),
                [&](int32_t a, int32_t b) { return S->cols[a].last_use < S->cols[b].last_use; });
      uint64_t avail = S->cfg.budget_bytes - std::min(S->cfg.budget_bytes, S->resident_bytes);
      size_t k = 0;
      while (avail < need && k < idle.size()) avail += S->cols[idle[k++]].bytes;
      if (avail < need) {
        S->st.admissions_refused++;
        return sfail(S->ctx, GLC_ERR_BUDGET, "server admit: budget exceeded and idle columns cannot make room");
      }
      for (size_t j = 0; j < k; j++) {
        SrvColumn& c = S->cols[idle[j]];
        victims.push_back(c.col);
        c.col = nullptr;
        c.evicting = true;
        S->resident_bytes -= c.bytes;
        S->resident_columns--;
        S->st.evictions++;
      }
    }
    SrvColumn sc;
    sc.col = col;
    sc.bytes = need;
    sc.last_use = ++S->tick;
    fill_views(sc);
    *id = (int32_t)S->cols.size();
    S->cols.push_back(sc);
    S->resident_bytes += need;
    S->resident_columns++;
  }
  for (glc_column* v : victims) glc_column_free(v);  // idle: no launch references them
  return GLC_OK;
}

glc_status glc_server_admit_blob(glc_server* S, glc_dtype dtype, const void* blob, uint64_t size, int flags,
                                 int32_t* id, glc_stream stream) {
  if (!S || !id) return GLC_ERR_INVALID_ARG;
  glc_column* col = nullptr;
  // the blob itself stays resident (copied once into the server's pool) and is read in place
  glc_status st = attach_column(S->ctx, dtype, blob, size, flags, 0, &col, stream, S->pool, true);
  if (st != GLC_OK) return st;
  st = glc_server_admit(S, col, id);
  if (st != GLC_OK) glc_column_free(col);
  return st;
}

glc_status glc_server_evict(glc_server* S, int32_t id) {
  if (!S) return GLC_ERR_INVALID_ARG;
  glc_column* now = nullptr;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (id < 0 || (size_t)id >= S->cols.size() || !S->cols[id].col || S->cols[id].evicting)
      return sfail(S->ctx, GLC_ERR_INVALID_ARG, "server evict: unknown or evicted column");
    SrvColumn& c = S->cols[id];
    c.evicting = true;
    S->st.evictions++;
    if (c.pins == 0) {
      now = c.col;
      c.col = nullptr;
      S->resident_bytes -= c.bytes;
      S->resident_columns--;
    }
    // otherwise the last completion moves it to to_free; its bytes count until then
  }
  if (now) glc_column_free(now);
  free_pending(S);
  return GLC_OK;
}

glc_status glc_server_submit(glc_server* S, const glc_request* reqs, int32_t count) {
  if (!S || count < 0 || (count > 0 && !reqs)) return GLC_ERR_INVALID_ARG;
  if (count == 0) return GLC_OK;
  const int64_t t = now_ns();
  std::vector<Req*> made;
  made.reserve((size_t)count);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    for (int32_t i = 0; i < count; i++) {
      const glc_request& q = reqs[i];
      const bool col_ok = q.column >= 0 && (size_t)q.column < S->cols.size() && S->cols[q.column].col &&
                          !S->cols[q.column].evicting;
      bool ok = col_ok && q.count >= 1 && q.out && (q.kind == GLC_REQ_LOOKUP || q.kind == GLC_REQ_RANGE);
      const uintptr_t es = col_ok ? (uintptr_t)dtype_size(S->cols[q.column].col->dtype) : 1;
      if (ok) ok = ((uintptr_t)q.out % es) == 0;
      if (ok && q.kind == GLC_REQ_LOOKUP) ok = q.positions != nullptr && ((uintptr_t)q.positions & 3) == 0;
      if (ok && q.kind == GLC_REQ_RANGE)
        ok = q.first >= 0 && q.first <= S->cols[q.column].col->n && q.count <= S->cols[q.column].col->n - q.first;
      if (!ok) return sfail(S->ctx, GLC_ERR_INVALID_ARG, "server submit: invalid request (nothing queued)");
    }
    for (int32_t i = 0; i < count; i++) {
      const glc_request& q = reqs[i];
      SrvColumn& c = S->cols[q.column];
      Req* r = new Req();
      r->r = q;
      r->arrival = q.not_before_ns > t ? q.not_before_ns : t;
      r->next = q.first;
      r->esize = dtype_size(c.col->dtype);
      r->in_place = q.kind == GLC_REQ_RANGE && (((uintptr_t)q.out - (uintptr_t)(q.first * r->esize)) & 15) == 0;
      r->ra = c.ra;
      r->bc = c.bc;
      c.pins++;
      c.last_use = ++S->tick;
      S->incoming.push_back(r);
    }
    S->st.submitted += count;
    S->n_incoming.store((int)S->incoming.size(), std::memory_order_release);
  }
  S->wake.notify_one();
  return GLC_OK;
}

glc_status glc_server_poll(glc_server* S, glc_completion* out, int32_t max, int32_t* got) {
  if (!S || !got || max < 0 || (max > 0 && !out)) return GLC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  int32_t k = 0;
  while (k < max && !S->done.empty()) {
    out[k++] = S->done.front();
    S->done.pop_front();
  }
  *got = k;
  return GLC_OK;
}

glc_status glc_server_get_stats(glc_server* S, glc_server_stats* stats) {
  if (!S || !stats) return GLC_ERR_INVALID_ARG;
  free_pending(S);
  std::lock_guard<std::mutex> lk(S->mu);
  *stats = S->st;
  stats->resident_bytes = S->resident_bytes;
  stats->resident_columns = S->resident_columns;
  stats->in_flight = S->in_flight.load();
  return GLC_OK;
}

glc_status glc_server_columns(glc_server* S, int32_t* ids, int32_t max, int32_t* got) {
  if (!S || !got || max < 0 || (max > 0 && !ids)) return GLC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  int32_t k = 0;
  for (size_t i = 0; i < S->cols.size() && k < max; i++)
    if (S->cols[i].col && !S->cols[i].evicting) ids[k++] = (int32_t)i;
  *got = k;
  return GLC_OK;
}

}  // extern "C"
