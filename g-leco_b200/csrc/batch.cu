// batch.cu -- many columns per launch: batched compress and batched decode (device work list).
//
// No counterpart in the reference, which compresses and decodes one column per API call
// (api/G-LeCo.cuh:349, :680).  Thousands of columns of uneven length and mixed int32 / int64 /
// uint64 / uint32 are handled by a fixed number of launches instead of a launch chain per column:
//
// compress (fixed-length partitions; the length is picked per column by compressed size):
//   1. per candidate length (1024, 2048, 4096): one launch fits every partition of every column
//      and adds each column's residual bits; the smallest compressed size picks the length
//      (skipped when the caller fixes the length);
//   2. one launch writes all partitions, one launch fits them all (a CTA per partition: exact
//      128-bit sums, line, max |delta|, width), one scan over all widths gives the bit offsets;
//   3. one launch packs every column's words (a CTA per 8 KB output tile of any column), one
//      builds all descriptors, one all decode-tile tables.
//   Each column's arrays are slices of batch-wide allocations; a column compressed here is
//   identical, byte for byte, to glc_compress of the same values with the same length.
// decode: one persistent launch (decode.cu batch_decode_kernel) over a work list with one item
//   per (column, 4096-value tile); optionally captured once in a CUDA graph and replayed.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>
#include "glc_internal.h"
#include "glc_scan.cuh"

using namespace glc;

struct glc_batch {
  glc_ctx* ctx = nullptr;
  std::vector<glc_column*> cols;  // views into `storage` when the batch compressed them
  bool owns_columns = false;
  glc_column* col_block = nullptr;  // the owned columns, when allocated as one array
  std::vector<void*> storage;     // device allocations owned by the batch
  BatchColumn* d_cols = nullptr;
  int max_bits = 0;
  // decode work list for the last set of outputs
  std::vector<void*> outs;
  BatchWork* d_work = nullptr;
  int64_t nwork = 0;
  unsigned long long* d_counter = nullptr;
  int64_t group_begin[5] = {0, 0, 0, 0, 0};  // work items grouped by element type
  cudaStream_t alloc_stream = nullptr;        // stream of the pool allocations in `storage`
  int* d_err = nullptr;
  cudaGraphExec_t graph = nullptr;
  // batches compressed by the one-pass kernel (lengths 1024 / 2048 / 4096): what
  // glc_batch_recompress needs -- the columns' element types, sizes and lengths, and after its
  // first call word arrays of the widest size, the launch tables and scratch of each element type
  bool one_pass = false;
  std::vector<glc_dtype> dtypes;
  std::vector<int64_t> ns;
  std::vector<int32_t> lens;
  struct ReGroup {
    glc_dtype dt;
    std::vector<int> cols;  // batch columns of this type with values
    CfColumn* d_tab = nullptr;
    int32_t* d_owner = nullptr;
    int64_t nitems = 0;
    void* scratch = nullptr;
  };
  std::vector<ReGroup> re;
  std::vector<const void*> re_values;      // the values the launch tables point at
  unsigned long long* re_stats = nullptr;  // 2 per column (total bits, widest field), then a status
  cudaGraphExec_t re_graph = nullptr;
  bool re_stale = false;                   // the host-side column sizes await glc_batch_sync
};

namespace {

constexpr int kFitCTA = 256;
constexpr int kMaxBatchPartLen = 8192;
const int kCandidates[3] = {1024, 2048, 4096};

glc_status bfail(glc_ctx* ctx, glc_status st, const char* msg) {
  if (ctx) ctx->err = msg;
  return st;
}

glc_status bcuda(glc_ctx* ctx, cudaError_t e, const char* where) {
  if (ctx) ctx->err = std::string(where) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? GLC_ERR_OOM : GLC_ERR_CUDA;
}

#define BCK(call, where)                                  \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return bcuda(ctx, e_, where);  \
  } while (0)

// Per batch column, on the device.
struct FitCol {
  const void* values;
  int64_t n;
  int64_t part_base;  // first global partition of the column
  int32_t len;        // partition length
  int32_t dtype;
};

__device__ __forceinline__ int col_of(const int64_t* __restrict__ base, int ncols, int64_t x) {
  int lo = 0, hi = ncols - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (base[mid] <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <typename T>
__device__ void fit_one(const T* __restrict__ v, int64_t len, int& type, double& t0, double& t1, long long& err,
                        int& bits) {
  __shared__ i128 s_a[kFitCTA / 32], s_b[kFitCTA / 32];
  __shared__ long long s_m[kFitCTA / 32];
  __shared__ int s_o[kFitCTA / 32];
  __shared__ double s_t0, s_t1;
  __shared__ int s_over;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  HalfSums<T> hs;  // exact 64-bit partials (len <= 8192: at most 32 values per thread)
  int ovf = 0;
  for (int64_t i = threadIdx.x; i < len; i += kFitCTA) {
    const T x = __ldg(v + i);
    ovf |= overflows_double<T>(x) ? 1 : 0;
    hs.add(x, (int)i);
  }
  i128 sy = hs.sy(), sxy = hs.sxy();
  sy = warp_sum_i128(sy);
  sxy = warp_sum_i128(sxy);
  ovf = __any_sync(FULL_MASK, ovf);
  if (lane == 0) { s_a[warp] = sy; s_b[warp] = sxy; s_o[warp] = ovf; }
  __syncthreads();
  if (threadIdx.x == 0) {
    i128 a = 0, b = 0;
    int o = 0;
    for (int w = 0; w < kFitCTA / 32; w++) { a += s_a[w]; b += s_b[w]; o |= s_o[w]; }
    double x0 = 0.0, x1 = 0.0;
    if (!o) solve_line(len, a, b, x0, x1);
    s_t0 = x0;
    s_t1 = x1;
    s_over = o;
  }
  __syncthreads();
  const double a0 = s_t0, a1 = s_t1;
  const bool over = s_over != 0;
  long long m = 0;
  bool exact = !over;
  if (!over && len > 0 && line_fp64_safe<T>(a0, a1, 0, len - 1)) {  // exact in FP64 (glc_device.cuh)
    double md = 0.0, id = (double)threadIdx.x;
    bool ok = true;
    for (int64_t i = threadIdx.x; i < len; i += kFitCTA, id += (double)kFitCTA) {
      const T y = __ldg(v + i);
      ok &= value_fp64_safe<T>(y);
      md = fmax(md, abs_resid_fp64((double)(long long)y, __fma_rn(a1, id, a0)));
    }
    if (ok) { m = (long long)md; exact = false; }
  }
  if (exact)
    for (int64_t i = threadIdx.x; i < len; i += kFitCTA) {
      const long long d = abs_ref(calc_delta<T>(__ldg(v + i), predict<T>(a0, a1, i)));
      m = d > m ? d : m;
    }
  m = warp_max_ll(m);
  if (lane == 0) s_m[warp] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < kFitCTA / 32; w++) t = s_m[w] > t ? s_m[w] : t;
    type = over ? MODEL_DIRECT_COPY : MODEL_LINEAR;
    t0 = a0;
    t1 = a1;
    err = over ? 0 : t;
    bits = over ? (int)sizeof(T) * 8 : bits_for(t);
  }
}

// One CTA per global partition.  size_only: add the column's residual bits into col_bits[c];
// otherwise write the partition's SoA entries and its width.
__global__ void __launch_bounds__(kFitCTA)
batch_fit_kernel(const FitCol* __restrict__ cols, const int64_t* __restrict__ part_base, int ncols, int size_only,
                 unsigned long long* __restrict__ col_bits, int32_t* __restrict__ starts, int32_t* __restrict__ ends,
                 int32_t* __restrict__ types, double* __restrict__ params, int32_t* __restrict__ bits,
                 int64_t* __restrict__ errs, int64_t* __restrict__ widths) {
  const int64_t p = blockIdx.x;
  const int c = col_of(part_base, ncols, p);
  const FitCol fc = cols[c];
  const int64_t k = p - fc.part_base;
  const int64_t s = k * fc.len;
  const int64_t len = (s + fc.len < fc.n ? s + fc.len : fc.n) - s;
  int type = 0, b = 0;
  double t0 = 0.0, t1 = 0.0;
  long long err = 0;
  switch (fc.dtype) {
    case GLC_I32: fit_one<int32_t>((const int32_t*)fc.values + s, len, type, t0, t1, err, b); break;
    case GLC_I64: fit_one<int64_t>((const int64_t*)fc.values + s, len, type, t0, t1, err, b); break;
    case GLC_U64: fit_one<uint64_t>((const uint64_t*)fc.values + s, len, type, t0, t1, err, b); break;
    default: fit_one<uint32_t>((const uint32_t*)fc.values + s, len, type, t0, t1, err, b); break;
  }
  if (threadIdx.x != 0) return;
  if (size_only) {
    atomicAdd(col_bits + c, (unsigned long long)(len * b));
    return;
  }
  starts[p] = (int32_t)s;
  ends[p] = (int32_t)(s + len);
  types[p] = type;
  params[4 * p] = t0;
  params[4 * p + 1] = t1;
  params[4 * p + 2] = 0.0;
  params[4 * p + 3] = 0.0;
  bits[p] = b;
  errs[p] = err;
  widths[p] = len * b;
}

// Global exclusive bit prefix -> column-local offsets; col_stats[c] = {total bits, max bits}.
__global__ void batch_local_offsets_kernel(const int64_t* __restrict__ gofs, const int64_t* __restrict__ part_base,
                                           const int32_t* __restrict__ bits, int ncols, int64_t P,
                                           const int64_t* __restrict__ grand, int64_t* __restrict__ offs,
                                           int64_t* __restrict__ col_stats) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const int c = col_of(part_base, ncols, p);
  const int64_t base = gofs[part_base[c]];
  offs[p] = gofs[p] - base;
  atomicMax((unsigned long long*)(col_stats + 2 * c + 1), (unsigned long long)bits[p]);
  if (p == part_base[c]) {
    // the next column's first partition, or the grand total when every later column is empty
    const int64_t nb = (c + 1 < ncols) ? part_base[c + 1] : P;
    const int64_t next = nb < P ? gofs[nb] : *grand;
    col_stats[2 * c] = next - base;
  }
}

struct TileCol {
  const int32_t* starts;
  const int32_t* bits;
  const int64_t* offs;
  glc::TileInfo* tiles;
  int64_t P, n, ntiles, total_bits;
};

__device__ __forceinline__ int64_t owner_in(const int32_t* __restrict__ starts, int64_t P, int64_t e) {
  int64_t lo = 0, hi = P - 1;
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if ((int64_t)starts[mid] <= e) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// One thread per tile-table entry of any column (ntiles + 1 entries per column).
__global__ void batch_tiles_kernel(const TileCol* __restrict__ cols, const int64_t* __restrict__ entry_base, int ncols,
                                   int64_t total) {
  const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= total) return;
  const int c = col_of(entry_base, ncols, x);
  const TileCol tc = cols[c];
  const int64_t t = x - entry_base[c];
  glc::TileInfo ti;
  if (t == tc.ntiles) {
    ti.bit_lo = tc.total_bits;
    ti.p_first = (int32_t)(tc.P - 1);
    ti.p_last = (int32_t)(tc.P - 1);
  } else {
    const int64_t e0 = t * kDecodeTile;
    const int64_t e1 = e0 + kDecodeTile < tc.n ? e0 + kDecodeTile : tc.n;
    const int64_t pf = owner_in(tc.starts, tc.P, e0);
    ti.bit_lo = tc.offs[pf] + (e0 - tc.starts[pf]) * (int64_t)tc.bits[pf];
    ti.p_first = (int32_t)pf;
    ti.p_last = (int32_t)owner_in(tc.starts, tc.P, e1 - 1);
  }
  tc.tiles[t] = ti;
}

__global__ void batch_desc_kernel(const int32_t* __restrict__ starts, const int32_t* __restrict__ types,
                                  const double* __restrict__ params, const int32_t* __restrict__ bits,
                                  const int64_t* __restrict__ offs, int64_t P, PartDesc* __restrict__ desc) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  PartDesc d;
  d.theta0 = params[4 * p];
  d.theta1 = params[4 * p + 1];
  d.bit_off = offs[p];
  d.start = starts[p];
  d.bits_type = (bits[p] & 0xff) | (types[p] << 8);
  desc[p] = d;
}

// The batch's arrays come from the context's stream-ordered pool (no device-wide synchronisation
// per allocation); they are returned to it when the batch is freed.
template <typename V> cudaError_t dalloc(glc_batch* b, V** p, size_t count) {
  void* q = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&q, count * sizeof(V) + 16, b->ctx->pool, b->alloc_stream);
  if (e == cudaSuccess) b->storage.push_back(q);
  *p = (V*)q;
  return e;
}

void free_batch(glc_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->re_graph) cudaGraphExecDestroy(b->re_graph);
  if (b->col_block) delete[] b->col_block;  // views: their arrays are in storage
  else if (b->owns_columns)
    for (glc_column* c : b->cols) delete c;
  for (void* q : b->storage) cudaFreeAsync(q, b->ctx->own_stream);
  if (!b->storage.empty()) cudaStreamSynchronize(b->ctx->own_stream);
  if (b->d_cols) cudaFree(b->d_cols);
  if (b->d_work) cudaFree(b->d_work);
  if (b->d_counter) cudaFree(b->d_counter);
  delete b;
}

glc_status finish_batch(glc_ctx* ctx, glc_batch* b, cudaStream_t s) {
  std::vector<BatchColumn> h(b->cols.size());
  b->max_bits = 0;
  for (size_t i = 0; i < b->cols.size(); i++) {
    const glc_column* c = b->cols[i];
    h[i] = BatchColumn{c->d_desc, c->d_start, c->d_tiles, c->d_words, c->n, (int32_t)c->dtype, c->max_bits};
    b->max_bits = std::max(b->max_bits, c->max_bits);
  }
  BCK(cudaMalloc(&b->d_cols, sizeof(BatchColumn) * std::max<size_t>(1, h.size())), "batch: column table");
  BCK(cudaMemcpyAsync(b->d_cols, h.data(), sizeof(BatchColumn) * h.size(), cudaMemcpyHostToDevice, s), "batch: column table");
  void* q = nullptr;
  BCK(cudaMalloc(&q, 64), "batch: counters");
  BCK(cudaMemsetAsync(q, 0, 64, s), "batch: counters");
  b->d_counter = (unsigned long long*)q;  // 4 counters, one per element type
  b->d_err = (int*)((char*)q + 32);
  BCK(cudaStreamSynchronize(s), "batch: sync");
  return GLC_OK;
}

glc_status build_work(glc_ctx* ctx, glc_batch* b, void* const* outs, cudaStream_t s) {
  const size_t nc = b->cols.size();
  bool same = b->d_work && b->outs.size() == nc;
  for (size_t i = 0; same && i < nc; i++) same = b->outs[i] == outs[i];
  if (same) return GLC_OK;
  std::vector<BatchWork> w;
  for (size_t i = 0; i < nc; i++) {
    const glc_column* c = b->cols[i];
    if (c->n == 0) continue;
    if (!outs[i]) return bfail(ctx, GLC_ERR_INVALID_ARG, "null output for a column of the batch");
    if (((uintptr_t)outs[i] & 15) != 0) return bfail(ctx, GLC_ERR_INVALID_ARG, "batch outputs must be 16-byte aligned");
    if (!c->d_words) return bfail(ctx, GLC_ERR_UNSUPPORTED, "a column of the batch has no packed bitstream");
    for (int64_t t = 0; t < c->ntiles; t++) w.push_back(BatchWork{(int32_t)i, (int32_t)t, 0, c->n, outs[i]});
  }
  std::vector<int32_t> col_dtype(nc);
  for (size_t i = 0; i < nc; i++) col_dtype[i] = (int32_t)b->cols[i]->dtype;
  group_work_by_type(w, col_dtype, b->group_begin);
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  if (b->d_work) {
    cudaStreamSynchronize(s);
    cudaFree(b->d_work);
    b->d_work = nullptr;
  }
  b->nwork = (int64_t)w.size();
  if (!w.empty()) {
    BCK(cudaMalloc(&b->d_work, sizeof(BatchWork) * w.size()), "batch: work list");
    BCK(cudaMemcpyAsync(b->d_work, w.data(), sizeof(BatchWork) * w.size(), cudaMemcpyHostToDevice, s), "batch: work list");
    BCK(cudaStreamSynchronize(s), "batch: work list");
  }
  b->outs.assign(outs, outs + nc);
  return GLC_OK;
}

// One-pass batched compress (compress_fixed.cu): every column's partition length divides the
// 4096-value tile, and its exact bit count is known from the choice pass (the same exact-sum fit,
// so the same widths), so every array is allocated at its exact size before one launch per element
// type fits, offsets, packs and tabulates all of that type's columns.  The values are read twice
// in all: once by the choice, once by this launch.
// The length choice's pass over one element type, which also packed every tile at length 4096:
// its column table and work list (the choice's item numbering), the tiles' slots and bits
// (scratch), their descriptors and max errors, and each column's widest field at 4096.
struct PrePacked {
  glc_dtype dt;
  int64_t nitems = 0;
  std::vector<int> cols;          // the batch's column index of each entry of the table
  std::vector<int64_t> item_base; // per entry
  int32_t* d_owner = nullptr;
  void* scratch = nullptr;        // from the context's pool, returned after the place
  PartDesc* tdesc = nullptr;
  long long* terr = nullptr;
};

// What the one-pass batched compress sets up before the lengths are known (so that it overlaps the
// length choice on the device): the columns, their partition arrays sized for the shortest
// candidate length (a column's arrays are a prefix of its region), the decode tables, the status
// words, and each column's launch-table entry without its length-dependent fields.
struct OnePassPrep {
  std::vector<CfColumn> hc;
  unsigned long long* stats = nullptr;  // 2 per column, then the status word
};

glc_status prepare_one_pass(glc_ctx* ctx, glc_batch* b, const glc_dtype* dtypes, const void* const* values,
                            const int64_t* ns, int nc, int32_t shortest_len, cudaStream_t s, OnePassPrep* prep) {
  std::vector<int64_t> pb(nc + 1, 0), eb(nc + 1, 0);
  glc_column* block = new (std::nothrow) glc_column[nc > 0 ? nc : 1];
  if (!block) return GLC_ERR_OOM;
  b->col_block = block;
  for (int i = 0; i < nc; i++) {
    glc_column* c = block + i;
    b->cols.push_back(c);
    c->ctx = ctx;
    c->view = true;
    c->dtype = dtypes[i];
    c->n = ns[i];
    c->ntiles = (c->n + kDecodeTile - 1) / kDecodeTile;
    pb[i + 1] = pb[i] + (c->n > 0 ? (c->n + shortest_len - 1) / shortest_len : 0);
    eb[i + 1] = eb[i] + (c->n ? c->ntiles + 1 : 0);
  }
  const int64_t P = pb[nc];
  int32_t *starts, *ends, *types, *bits;
  double* params;
  int64_t *offs, *errs;
  PartDesc* desc;
  TileInfo* tiles;
  unsigned long long* stats;
  cudaError_t e;
  if ((e = dalloc(b, &starts, P)) || (e = dalloc(b, &ends, P)) || (e = dalloc(b, &types, P)) ||
      (e = dalloc(b, &bits, P)) || (e = dalloc(b, &params, 4 * P)) || (e = dalloc(b, &offs, P)) ||
      (e = dalloc(b, &errs, P)) || (e = dalloc(b, &desc, P)) || (e = dalloc(b, &tiles, eb[nc])) ||
      (e = dalloc(b, &stats, 2 * (size_t)nc + 1)))
    return bcuda(ctx, e, "batch compress: allocation");
  BCK(cudaMemsetAsync(stats, 0, sizeof(unsigned long long) * (2 * (size_t)nc + 1), s), "batch compress: stats");
  prep->stats = stats;
  prep->hc.assign(nc, CfColumn{});
  for (int i = 0; i < nc; i++) {
    glc_column* c = block + i;
    const int64_t p0 = pb[i];
    c->d_start = starts + p0;
    c->d_end = ends + p0;
    c->d_types = types + p0;
    c->d_params = params + 4 * p0;
    c->d_bits = bits + p0;
    c->d_offs = offs + p0;
    c->d_err = errs + p0;
    c->d_desc = desc + p0;
    c->d_tiles = tiles + eb[i];
    CfColumn& f = prep->hc[i];
    f.values = values[i];
    f.n = c->n;
    f.ntiles = c->ntiles;
    f.starts = c->d_start;
    f.ends = c->d_end;
    f.types = c->d_types;
    f.params = c->d_params;
    f.bits = c->d_bits;
    f.offs = c->d_offs;
    f.err = c->d_err;
    f.desc = c->d_desc;
    f.tiles = c->d_tiles;
    f.stats = stats + 2 * i;
  }
  return GLC_OK;
}

glc_status compress_one_pass(glc_ctx* ctx, glc_batch* b, const glc_dtype* dtypes, const void* const* values,
                             const int64_t* ns, int nc, const std::vector<int32_t>& len,
                             const std::vector<unsigned long long>& hbits, cudaStream_t s, int64_t* total_size,
                             std::vector<PrePacked>* pre, unsigned long long* pre_stats, OnePassPrep& prep) {
  (void)values;
  std::vector<int64_t> wb(nc + 1, 0);
  for (int i = 0; i < nc; i++) {  // the length-dependent fields
    glc_column* c = b->cols[i];
    c->fixed_len = len[i];
    c->P = c->n > 0 ? (c->n + len[i] - 1) / len[i] : 0;
    const int k = len[i] == 1024 ? 0 : (len[i] == 2048 ? 1 : 2);
    c->total_bits = c->n > 0 ? (int64_t)hbits[3 * (size_t)i + k] : 0;
    c->nwords = (c->total_bits + 31) / 32;
    c->nwords_alloc = ((c->nwords + 3) & ~3ll) + 8;
    c->reported_size = c->n ? 64 * c->P + 120 + (c->total_bits + 7) / 8 : 0;  // api/G-LeCo.cuh:589-603
    wb[i + 1] = wb[i] + c->nwords_alloc;
  }
  uint32_t* words;
  cudaError_t e;
  if ((e = dalloc(b, &words, wb[nc])) != cudaSuccess) return bcuda(ctx, e, "batch compress: allocation");
  unsigned long long* stats = prep.stats;
  std::vector<CfColumn>& hc = prep.hc;
  std::vector<glc_column*> cols(b->cols.begin(), b->cols.end());
  for (int i = 0; i < nc; i++) {
    glc_column* c = cols[i];
    c->d_words = words + wb[i];
    CfColumn& f = hc[i];
    f.L = len[i];
    f.parts_per_tile = kDecodeTile / len[i];
    f.P = c->P;
    f.nwords_alloc = c->nwords_alloc;
    f.words_cap = c->nwords_alloc;
    f.words = c->d_words;
  }
  // a column the length choice already packed (it keeps length 4096) is only placed
  std::vector<char> prepacked(nc, 0);
  if (pre)
    for (const PrePacked& pp : *pre)
      for (int i : pp.cols) prepacked[i] = len[i] == 4096;
  // one launch per element type over the tiles of that type's other columns, in column order; the
  // host tables stay alive until the stream is synchronised
  std::vector<std::vector<CfColumn>> keep_g;
  std::vector<std::vector<int64_t>> keep_ib;
  if (pre) {
    for (PrePacked& pp : *pre) {
      keep_g.emplace_back();
      std::vector<CfColumn>& tab = keep_g.back();
      bool any = false;
      for (size_t k = 0; k < pp.cols.size(); k++) {
        CfColumn f{};
        const int i = pp.cols[k];
        if (prepacked[i]) {
          f = hc[i];
          any = true;
        }
        f.n = ns[i];
        f.ntiles = (ns[i] + kDecodeTile - 1) / kDecodeTile;
        f.item_base = pp.item_base[k];  // words stay null for a column placed elsewhere: skipped
        tab.push_back(f);
      }
      cudaError_t ee = cudaSuccess;
      if (any) {
        CfColumn* d_tab;
        if ((e = dalloc(b, &d_tab, tab.size())) != cudaSuccess) return bcuda(ctx, e, "batch compress: allocation");
        ee = cudaMemcpyAsync(d_tab, tab.data(), sizeof(CfColumn) * tab.size(), cudaMemcpyHostToDevice, s);
        if (ee == cudaSuccess)
          ee = launch_place_prepacked(pp.dt, d_tab, pp.d_owner, pp.nitems, pp.scratch, pp.tdesc, pp.terr,
                                      stats + 2 * (size_t)nc, ctx->num_sms, s);
      }
      cudaFreeAsync(pp.scratch, s);
      pp.scratch = nullptr;
      BCK(ee, "batch compress: place of the columns packed by the length choice");
    }
  }
  for (glc_dtype dt : {GLC_I32, GLC_I64, GLC_U64, GLC_U32}) {
    keep_g.emplace_back();
    keep_ib.emplace_back(1, 0);
    std::vector<CfColumn>& g = keep_g.back();
    std::vector<int64_t>& ib = keep_ib.back();
    for (int i = 0; i < nc; i++) {
      if (dtypes[i] != dt || ns[i] == 0 || prepacked[i]) continue;
      CfColumn f = hc[i];
      f.item_base = ib.back();
      g.push_back(f);
      ib.push_back(ib.back() + f.ntiles);
    }
    if (g.empty()) continue;
    const int64_t nitems = ib.back();
    CfColumn* d_g;
    int64_t* d_ib;
    int32_t* d_owner;
    uint8_t* scratch;
    if ((e = dalloc(b, &d_g, g.size())) || (e = dalloc(b, &d_ib, ib.size())) || (e = dalloc(b, &d_owner, nitems)))
      return bcuda(ctx, e, "batch compress: allocation");
    // the tiles' slots are scratch: from the context's pool, returned after the launch
    BCK(cudaMallocFromPoolAsync((void**)&scratch, fixed_compress_scratch_bytes(dt, nitems), ctx->pool, s),
        "batch compress: scratch");
    BCK(cudaMemcpyAsync(d_g, g.data(), sizeof(CfColumn) * g.size(), cudaMemcpyHostToDevice, s), "batch compress: columns");
    BCK(cudaMemcpyAsync(d_ib, ib.data(), sizeof(int64_t) * ib.size(), cudaMemcpyHostToDevice, s), "batch compress: columns");
    BCK(launch_pack_item_owner(d_ib, (int)g.size(), d_owner, s), "batch compress: work list");
    e = launch_fixed_compress_batch(dt, d_g, d_owner, nitems, scratch, stats + 2 * (size_t)nc, ctx->num_sms, s);
    cudaFreeAsync(scratch, s);
    BCK(e, "batch compress: one-pass compress");
  }
  std::vector<unsigned long long> hs(2 * (size_t)nc + 1), hp(pre_stats ? 2 * (size_t)nc : 0);
  BCK(cudaMemcpyAsync(hs.data(), stats, sizeof(unsigned long long) * hs.size(), cudaMemcpyDeviceToHost, s),
      "batch compress: stats");
  if (pre_stats)
    BCK(cudaMemcpyAsync(hp.data(), pre_stats, sizeof(unsigned long long) * hp.size(), cudaMemcpyDeviceToHost, s),
        "batch compress: stats");
  BCK(cudaStreamSynchronize(s), "batch compress: sync");
  for (int i = 0; i < nc && pre_stats; i++)
    if (prepacked[i]) hs[2 * (size_t)i + 1] = hp[2 * (size_t)i + 1];  // widest field at 4096
  if (hs[2 * (size_t)nc] == DEVERR_TIMEOUT) return bfail(ctx, GLC_ERR_TIMEOUT, "batch compress: a device-side wait gave up");
  if (hs[2 * (size_t)nc] != DEVERR_NONE) return bfail(ctx, GLC_ERR_CUDA, "batch compress: words beyond their array");
  int64_t total = 0;
  for (int i = 0; i < nc; i++) {
    glc_column* c = cols[i];
    if (c->n > 0 && (int64_t)hs[2 * (size_t)i] != c->total_bits)
      return bfail(ctx, GLC_ERR_CUDA, "batch compress: the pass and the length choice disagree on a column's bits");
    c->max_bits = (int32_t)hs[2 * (size_t)i + 1];
    total += c->reported_size;
  }
  if (total_size) *total_size = total;
  b->one_pass = true;
  b->dtypes.assign(dtypes, dtypes + nc);
  b->ns.assign(ns, ns + nc);
  b->lens = len;
  return GLC_OK;
}

// Word arrays of the widest size for every column, launch tables and scratch per element type
// (glc_batch_recompress's first call).
glc_status recompress_setup(glc_ctx* ctx, glc_batch* b, cudaStream_t s) {
  const int nc = (int)b->cols.size();
  std::vector<int64_t> cap(nc), wb(nc + 1, 0);
  for (int i = 0; i < nc; i++) {
    cap[i] = b->ns[i] > 0 ? ((fixed_compress_worst_words(b->dtypes[i], b->ns[i]) + 3) & ~3ll) : 4;
    wb[i + 1] = wb[i] + cap[i];
  }
  uint32_t* words;
  cudaError_t e;
  if ((e = dalloc(b, &words, wb[nc])) || (e = dalloc(b, &b->re_stats, 2 * (size_t)nc + 1)))
    return bcuda(ctx, e, "batch recompress: allocation");
  for (int i = 0; i < nc; i++) {
    glc_column* c = b->cols[i];
    c->d_words = words + wb[i];
    c->nwords_alloc = cap[i];
  }
  for (glc_dtype dt : {GLC_I32, GLC_I64, GLC_U64, GLC_U32}) {
    glc_batch::ReGroup g;
    g.dt = dt;
    for (int i = 0; i < nc; i++)
      if (b->dtypes[i] == dt && b->ns[i] > 0) {
        g.cols.push_back(i);
        g.nitems += b->cols[i]->ntiles;
      }
    if (g.cols.empty()) continue;
    if ((e = dalloc(b, &g.d_tab, g.cols.size())) || (e = dalloc(b, &g.d_owner, g.nitems)) ||
        (e = dalloc(b, (uint8_t**)&g.scratch, fixed_compress_scratch_bytes(dt, g.nitems))))
      return bcuda(ctx, e, "batch recompress: allocation");
    b->re.push_back(g);
  }
  // the decode reads the new word arrays
  std::vector<BatchColumn> h(nc);
  for (int i = 0; i < nc; i++) {
    const glc_column* c = b->cols[i];
    h[i] = BatchColumn{c->d_desc, c->d_start, c->d_tiles, c->d_words, c->n, (int32_t)c->dtype, c->max_bits};
  }
  BCK(cudaMemcpyAsync(b->d_cols, h.data(), sizeof(BatchColumn) * nc, cudaMemcpyHostToDevice, s), "batch recompress");
  BCK(cudaStreamSynchronize(s), "batch recompress");
  return GLC_OK;
}

// The launch tables of every element type for these values (columns' arrays, widest word arrays).
glc_status recompress_tables(glc_ctx* ctx, glc_batch* b, const void* const* values, cudaStream_t s) {
  for (glc_batch::ReGroup& g : b->re) {
    std::vector<CfColumn> tab;
    std::vector<int64_t> ib(1, 0);
    for (int i : g.cols) {
      const glc_column* c = b->cols[i];
      CfColumn f{};
      f.values = values[i];
      f.n = c->n;
      f.L = b->lens[i];
      f.parts_per_tile = kDecodeTile / f.L;
      f.P = c->P;
      f.ntiles = c->ntiles;
      f.item_base = ib.back();
      f.nwords_alloc = c->nwords_alloc;
      f.words_cap = c->nwords_alloc;
      f.starts = c->d_start;
      f.ends = c->d_end;
      f.types = c->d_types;
      f.params = c->d_params;
      f.bits = c->d_bits;
      f.offs = c->d_offs;
      f.err = c->d_err;
      f.desc = c->d_desc;
      f.tiles = c->d_tiles;
      f.words = c->d_words;
      f.stats = b->re_stats + 2 * (size_t)i;
      tab.push_back(f);
      ib.push_back(ib.back() + f.ntiles);
    }
    int64_t* d_ib;
    cudaError_t e;
    if ((e = dalloc(b, &d_ib, ib.size()))) return bcuda(ctx, e, "batch recompress: allocation");
    BCK(cudaMemcpyAsync(g.d_tab, tab.data(), sizeof(CfColumn) * tab.size(), cudaMemcpyHostToDevice, s),
        "batch recompress: tables");
    BCK(cudaMemcpyAsync(d_ib, ib.data(), sizeof(int64_t) * ib.size(), cudaMemcpyHostToDevice, s),
        "batch recompress: tables");
    BCK(launch_pack_item_owner(d_ib, (int)tab.size(), g.d_owner, s), "batch recompress: work list");
    BCK(cudaStreamSynchronize(s), "batch recompress: tables");
  }
  b->re_values.assign(values, values + b->cols.size());
  return GLC_OK;
}

// The launches of one recompress (stream-ordered, nothing read back; capturable).
cudaError_t recompress_launches(glc_ctx* ctx, glc_batch* b, cudaStream_t s) {
  const size_t nc = b->cols.size();
  cudaError_t e = cudaMemsetAsync(b->re_stats, 0, sizeof(unsigned long long) * (2 * nc + 1), s);
  for (const glc_batch::ReGroup& g : b->re) {
    if (e != cudaSuccess) break;
    e = launch_fixed_compress_batch(g.dt, g.d_tab, g.d_owner, g.nitems, g.scratch, b->re_stats + 2 * nc, ctx->num_sms,
                                    s);
  }
  return e;
}

}  // namespace

extern "C" {

glc_status glc_batch_create(glc_ctx* ctx, glc_column* const* cols, int32_t ncols, glc_batch** out) {
  if (!ctx || !out || ncols < 0 || (ncols > 0 && !cols)) return bfail(ctx, GLC_ERR_INVALID_ARG, "bad batch arguments");
  *out = nullptr;
  glc_batch* b = new (std::nothrow) glc_batch();
  if (!b) return GLC_ERR_OOM;
  b->ctx = ctx;
  for (int i = 0; i < ncols; i++) {
    if (!cols[i]) { delete b; return bfail(ctx, GLC_ERR_INVALID_ARG, "null column in batch"); }
    b->cols.push_back(cols[i]);
  }
  glc::DeviceScope device_scope(ctx->device);
  glc_status st = finish_batch(ctx, b, ctx->own_stream);
  if (st != GLC_OK) { free_batch(b); return st; }
  *out = b;
  return GLC_OK;
}

glc_status glc_batch_compress(glc_ctx* ctx, const glc_dtype* dtypes, const void* const* values, const int64_t* ns,
                              int32_t ncols, int32_t fixed_partition_len, glc_batch** out,
                              int64_t* compressed_size_bytes, glc_stream stream) {
  if (!ctx || !out || ncols <= 0 || !dtypes || !values || !ns) return bfail(ctx, GLC_ERR_INVALID_ARG, "bad batch arguments");
  if (fixed_partition_len < 0 || fixed_partition_len > kMaxBatchPartLen)
    return bfail(ctx, GLC_ERR_INVALID_ARG, "batch partition length must be in [1, 8192] (0 = chosen per column)");
  *out = nullptr;
  for (int i = 0; i < ncols; i++) {
    if (dtypes[i] < GLC_I32 || dtypes[i] > GLC_U32 || ns[i] < 0 || ns[i] > 0x7fffffffll || (ns[i] > 0 && !values[i]))
      return bfail(ctx, GLC_ERR_INVALID_ARG, "bad column in batch");
  }
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->own_stream;
  glc_batch* b = new (std::nothrow) glc_batch();
  if (!b) return GLC_ERR_OOM;
  b->ctx = ctx;
  b->owns_columns = true;
  b->alloc_stream = s;
  auto bail = [&](glc_status st) { cudaStreamSynchronize(s); free_batch(b); return st; };
  const int nc = ncols;

  // ---- partition length per column ----
  std::vector<int32_t> len(nc, fixed_partition_len > 0 ? fixed_partition_len : kCandidates[2]);
  std::vector<int64_t> pb(nc + 1, 0);
  FitCol* d_fc = nullptr;
  int64_t* d_pb = nullptr;
  unsigned long long* d_colbits = nullptr;
  cudaError_t e;
  auto upload_layout = [&](const std::vector<int32_t>& L) -> cudaError_t {
    std::vector<FitCol> fc(nc);
    pb[0] = 0;
    for (int i = 0; i < nc; i++) {
      const int64_t P = ns[i] > 0 ? (ns[i] + L[i] - 1) / L[i] : 0;
      pb[i + 1] = pb[i] + P;
      fc[i] = FitCol{values[i], ns[i], pb[i], L[i], (int32_t)dtypes[i]};
    }
    cudaError_t ee = cudaMemcpyAsync(d_fc, fc.data(), sizeof(FitCol) * nc, cudaMemcpyHostToDevice, s);
    if (ee == cudaSuccess) ee = cudaMemcpyAsync(d_pb, pb.data(), sizeof(int64_t) * (nc + 1), cudaMemcpyHostToDevice, s);
    if (ee == cudaSuccess) ee = cudaStreamSynchronize(s);  // host vectors are reused next
    return ee;
  };
  if ((e = dalloc(b, &d_fc, nc)) != cudaSuccess || (e = dalloc(b, &d_pb, nc + 1)) != cudaSuccess ||
      (e = dalloc(b, &d_colbits, 3 * (size_t)nc + 1)) != cudaSuccess)
    return bail(bcuda(ctx, e, "batch compress: allocation"));
  // lengths 1024 / 2048 / 4096: the choice pass measures the exact bits of all three, and the
  // one-pass kernel compresses every column at its chosen length
  const bool one_pass = fixed_partition_len == 0 || fixed_partition_len == 1024 || fixed_partition_len == 2048 ||
                        fixed_partition_len == 4096;
  std::vector<unsigned long long> hbits(3 * (size_t)nc);
  std::vector<PrePacked> pre;
  if (one_pass) {  // one read of every column measures all three candidate lengths
    if ((e = cudaMemsetAsync(d_colbits, 0, sizeof(unsigned long long) * (3 * (size_t)nc + 1), s)) != cudaSuccess)
      return bail(bcuda(ctx, e, "batch compress: sizes"));
    // one launch per element type, which also packs every tile at length 4096 (kept by most
    // columns); the host tables stay alive until the stream is synchronised
    std::vector<std::vector<CfColumn>> keep_g;
    std::vector<std::vector<int64_t>> keep_ib;
    const bool pack = fixed_partition_len == 0 || fixed_partition_len == 4096;
    unsigned long long* pre_stats = nullptr;  // per column: [1] widest field at 4096
    if (pack) {
      if ((e = dalloc(b, &pre_stats, 2 * (size_t)nc)) != cudaSuccess ||
          (e = cudaMemsetAsync(pre_stats, 0, sizeof(unsigned long long) * 2 * (size_t)nc, s)) != cudaSuccess)
        return bail(bcuda(ctx, e, "batch compress: allocation"));
    }
    auto release_pre = [&]() {
      for (PrePacked& pp : pre)
        if (pp.scratch) cudaFreeAsync(pp.scratch, s);
      pre.clear();
    };
    for (glc_dtype dt : {GLC_I32, GLC_I64, GLC_U64, GLC_U32}) {
      keep_g.emplace_back();
      keep_ib.emplace_back(1, 0);
      std::vector<CfColumn>& g = keep_g.back();
      std::vector<int64_t>& ib = keep_ib.back();
      PrePacked pp;
      pp.dt = dt;
      for (int i = 0; i < nc; i++) {
        if (dtypes[i] != dt || ns[i] == 0) continue;
        CfColumn f{};
        f.values = values[i];
        f.n = ns[i];
        f.ntiles = (ns[i] + kDecodeTile - 1) / kDecodeTile;
        f.item_base = ib.back();
        f.choice_bits = d_colbits + 3 * (size_t)i;
        f.stats = pack ? pre_stats + 2 * (size_t)i : nullptr;
        pp.cols.push_back(i);
        pp.item_base.push_back(ib.back());
        g.push_back(f);
        ib.push_back(ib.back() + f.ntiles);
      }
      if (g.empty()) continue;
      CfColumn* d_g;
      int64_t* d_ib;
      int32_t* d_owner;
      if ((e = dalloc(b, &d_g, g.size())) || (e = dalloc(b, &d_ib, ib.size())) || (e = dalloc(b, &d_owner, ib.back())))
        return release_pre(), bail(bcuda(ctx, e, "batch compress: allocation"));
      pp.nitems = ib.back();
      pp.d_owner = d_owner;
      if (pack) {
        if ((e = dalloc(b, &pp.tdesc, pp.nitems)) || (e = dalloc(b, &pp.terr, pp.nitems)) ||
            (e = cudaMallocFromPoolAsync(&pp.scratch, fixed_compress_scratch_bytes(dt, pp.nitems), ctx->pool, s)))
          return release_pre(), bail(bcuda(ctx, e, "batch compress: allocation"));
      }
      void* scratch = pp.scratch;
      PartDesc* tdesc = pp.tdesc;
      long long* terr = pp.terr;
      if (pack) pre.push_back(std::move(pp));
      if ((e = cudaMemcpyAsync(d_g, g.data(), sizeof(CfColumn) * g.size(), cudaMemcpyHostToDevice, s)) ||
          (e = cudaMemcpyAsync(d_ib, ib.data(), sizeof(int64_t) * ib.size(), cudaMemcpyHostToDevice, s)) ||
          (e = launch_pack_item_owner(d_ib, (int)g.size(), d_owner, s)) ||
          (e = launch_choose_lengths(dt, d_g, d_owner, ib.back(), d_colbits + 3 * (size_t)nc, ctx->num_sms, s,
                                     scratch, tdesc, terr)))
        return release_pre(), bail(bcuda(ctx, e, "batch compress: length choice"));
    }
    // everything that does not depend on the lengths, while the choice runs on the device
    OnePassPrep prep;
    {
      const glc_status ps = prepare_one_pass(ctx, b, dtypes, values, ns, nc,
                                             fixed_partition_len ? fixed_partition_len : kCandidates[0], s, &prep);
      if (ps != GLC_OK) return release_pre(), bail(ps);
    }
    unsigned long long choice_status = 0;
    if ((e = cudaMemcpyAsync(hbits.data(), d_colbits, sizeof(unsigned long long) * 3 * nc, cudaMemcpyDeviceToHost,
                             s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&choice_status, d_colbits + 3 * (size_t)nc, sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return release_pre(), bail(bcuda(ctx, e, "batch compress: sizes"));
    if (choice_status != DEVERR_NONE)
      return release_pre(), bail(bfail(ctx, GLC_ERR_TIMEOUT, "batch compress: a device-side wait gave up"));
    // the smallest compressed size; within 0.1 % of it, the length the tuner found to decode
    // fastest for the element type and the column's mean field width (when the table holds one)
    for (int i = 0; i < nc && fixed_partition_len == 0; i++) {
      int64_t size[3], best = INT64_MAX;
      for (int k = 0; k < 3; k++) {
        const int64_t cand = kCandidates[k];
        const int64_t P = ns[i] > 0 ? (ns[i] + cand - 1) / cand : 0;
        size[k] = 64 * P + 120 + (int64_t)(hbits[3 * i + k] + 7) / 8;  // api/G-LeCo.cuh:589-603
        if (size[k] < best) { best = size[k]; len[i] = (int32_t)cand; }
      }
      const int mean_bits = ns[i] > 0 ? (int)((hbits[3 * i + 2] + ns[i] - 1) / ns[i]) : 0;
      const int tuned = tune_entry(ctx, dtypes[i], mean_bits, 0).partition_len;
      for (int k = 0; k < 3; k++)
        if (kCandidates[k] == tuned && size[k] * 1000 <= best * 1001) len[i] = tuned;
    }
    int64_t total = 0;
    glc_status st = compress_one_pass(ctx, b, dtypes, values, ns, nc, len, hbits, s, &total, pack ? &pre : nullptr,
                                      pre_stats, prep);
    release_pre();  // what the place did not return (an error on the way)
    if (st == GLC_OK) st = finish_batch(ctx, b, s);
    if (st != GLC_OK) return bail(st);
    if (compressed_size_bytes) *compressed_size_bytes = total;
    *out = b;
    return GLC_OK;
  }
  if ((e = upload_layout(len)) != cudaSuccess) return bail(bcuda(ctx, e, "batch compress: layout"));
  const int64_t P = pb[nc];

  // ---- batch-wide arrays ----
  int32_t *starts, *ends, *types, *bits;
  double* params;
  int64_t *offs, *errs, *widths, *gofs, *scan_tmp, *grand, *col_stats;
  PartDesc* desc;
  if ((e = dalloc(b, &starts, P)) || (e = dalloc(b, &ends, P)) || (e = dalloc(b, &types, P)) ||
      (e = dalloc(b, &bits, P)) || (e = dalloc(b, &params, 4 * P)) || (e = dalloc(b, &offs, P)) ||
      (e = dalloc(b, &errs, P)) || (e = dalloc(b, &widths, P)) || (e = dalloc(b, &gofs, P)) ||
      (e = dalloc(b, &scan_tmp, scan_num_tiles(P) + 1)) || (e = dalloc(b, &grand, 1)) ||
      (e = dalloc(b, &col_stats, 2 * nc)) || (e = dalloc(b, &desc, P)))
    return bail(bcuda(ctx, e, "batch compress: allocation"));
  if (P > 0)
    batch_fit_kernel<<<(unsigned)P, kFitCTA, 0, s>>>(d_fc, d_pb, nc, 0, nullptr, starts, ends, types, params, bits, errs,
                                                     widths);
  if ((e = exclusive_scan<int64_t>(widths, gofs, P, grand, scan_tmp, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(col_stats, 0, sizeof(int64_t) * 2 * nc, s)) != cudaSuccess)
    return bail(bcuda(ctx, e, "batch compress: offsets"));
  if (P > 0)
    batch_local_offsets_kernel<<<(unsigned)((P + 255) / 256), 256, 0, s>>>(gofs, d_pb, bits, nc, P, grand, offs,
                                                                            col_stats);
  std::vector<int64_t> hstats(2 * nc);
  if ((e = cudaMemcpyAsync(hstats.data(), col_stats, sizeof(int64_t) * 2 * nc, cudaMemcpyDeviceToHost, s)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return bail(bcuda(ctx, e, "batch compress: column sizes"));

  // ---- column views, words, tables and packing ----
  std::vector<int64_t> word_base(nc + 1, 0), entry_base(nc + 1, 0);
  std::vector<glc_column*> cols(nc, nullptr);
  for (int i = 0; i < nc; i++) {
    glc_column* c = new (std::nothrow) glc_column();
    if (!c) return bail(GLC_ERR_OOM);
    cols[i] = c;
    b->cols.push_back(c);
    c->ctx = ctx;
    c->view = true;
    c->dtype = dtypes[i];
    c->n = ns[i];
    c->P = pb[i + 1] - pb[i];
    c->total_bits = hstats[2 * i];
    c->max_bits = (int32_t)hstats[2 * i + 1];
    c->fixed_len = len[i];
    c->nwords = (c->total_bits + 31) / 32;
    c->nwords_alloc = ((c->nwords + 3) & ~3ll) + 8;
    c->ntiles = (c->n + kDecodeTile - 1) / kDecodeTile;
    c->reported_size = c->n ? 64 * c->P + 120 + (c->total_bits + 7) / 8 : 0;
    word_base[i + 1] = word_base[i] + c->nwords_alloc;
    entry_base[i + 1] = entry_base[i] + (c->n ? c->ntiles + 1 : 0);
  }
  uint32_t* words;
  TileInfo* tiles;
  TileCol* d_tc;
  int64_t* d_eb;
  if ((e = dalloc(b, &words, word_base[nc])) || (e = dalloc(b, &tiles, entry_base[nc])) || (e = dalloc(b, &d_tc, nc)) ||
      (e = dalloc(b, &d_eb, nc + 1)))
    return bail(bcuda(ctx, e, "batch compress: allocation"));
  std::vector<TileCol> htc(nc);
  for (int i = 0; i < nc; i++) {
    glc_column* c = cols[i];
    const int64_t p0 = pb[i];
    c->d_start = starts + p0;
    c->d_end = ends + p0;
    c->d_types = types + p0;
    c->d_params = params + 4 * p0;
    c->d_bits = bits + p0;
    c->d_offs = offs + p0;
    c->d_err = errs + p0;
    c->d_desc = desc + p0;
    c->d_words = words + word_base[i];
    c->d_tiles = tiles + entry_base[i];
    htc[i] = TileCol{c->d_start, c->d_bits, c->d_offs, c->d_tiles, c->P, c->n, c->ntiles, c->total_bits};
  }
  // Work items of the value-tile pack, grouped by element type: one launch per type, each with its
  // own columns, item bases (first tile of each column) and item -> column table.
  struct PackGroup {
    glc_dtype dt;
    int64_t c0, ncols, ib0, own0, nitems;
  };
  std::vector<PackTileCol> hptc;
  std::vector<int64_t> hib;
  std::vector<PackGroup> groups;
  int64_t total_items = 0;
  for (glc_dtype dt : {GLC_I32, GLC_I64, GLC_U64, GLC_U32}) {
    PackGroup g{dt, (int64_t)hptc.size(), 0, (int64_t)hib.size(), total_items, 0};
    hib.push_back(0);
    for (int i = 0; i < nc; i++) {
      glc_column* c = cols[i];
      if (dtypes[i] != dt || c->n == 0) continue;
      hptc.push_back(PackTileCol{values[i], c->d_desc, c->d_tiles, c->n, c->ntiles, c->d_words});
      g.nitems += c->ntiles;
      hib.push_back(g.nitems);
    }
    g.ncols = (int64_t)hptc.size() - g.c0;
    total_items += g.nitems;
    groups.push_back(g);
  }
  PackTileCol* d_ptc;
  int64_t* d_ib;
  int32_t* d_owner;
  if ((e = dalloc(b, &d_ptc, hptc.size() + 1)) || (e = dalloc(b, &d_ib, hib.size())) ||
      (e = dalloc(b, &d_owner, total_items + 1)))
    return bail(bcuda(ctx, e, "batch compress: allocation"));
  if ((e = cudaMemcpyAsync(d_tc, htc.data(), sizeof(TileCol) * nc, cudaMemcpyHostToDevice, s)) ||
      (e = cudaMemcpyAsync(d_eb, entry_base.data(), sizeof(int64_t) * (nc + 1), cudaMemcpyHostToDevice, s)) ||
      (e = cudaMemcpyAsync(d_ptc, hptc.data(), sizeof(PackTileCol) * hptc.size(), cudaMemcpyHostToDevice, s)) ||
      (e = cudaMemcpyAsync(d_ib, hib.data(), sizeof(int64_t) * hib.size(), cudaMemcpyHostToDevice, s)) ||
      (e = cudaMemsetAsync(words, 0, sizeof(uint32_t) * word_base[nc], s)))
    return bail(bcuda(ctx, e, "batch compress: tables"));
  // descriptor and tile tables first: the packer reads them
  if (P > 0) batch_desc_kernel<<<(unsigned)((P + 255) / 256), 256, 0, s>>>(starts, types, params, bits, offs, P, desc);
  if (entry_base[nc] > 0)
    batch_tiles_kernel<<<(unsigned)((entry_base[nc] + 255) / 256), 256, 0, s>>>(d_tc, d_eb, nc, entry_base[nc]);
  for (const PackGroup& g : groups) {
    if (g.nitems == 0) continue;
    if ((e = launch_pack_item_owner(d_ib + g.ib0, (int)g.ncols, d_owner + g.own0, s)) != cudaSuccess ||
        (e = launch_batch_pack_tiles(g.dt, d_ptc + g.c0, d_owner + g.own0, d_ib + g.ib0, g.nitems,
                                     ctx->d_flags + kFlagError, ctx->num_sms, s)) != cudaSuccess)
      return bail(bcuda(ctx, e, "batch compress: pack"));
  }
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return bail(bcuda(ctx, e, "batch compress"));
  int64_t total = 0;
  for (glc_column* c : cols) total += c->reported_size;
  if (compressed_size_bytes) *compressed_size_bytes = total;
  glc_status st = finish_batch(ctx, b, s);
  if (st != GLC_OK) return bail(st);
  *out = b;
  return GLC_OK;
}

glc_status glc_batch_column(const glc_batch* b, int32_t i, glc_column** col) {
  if (!b || !col || i < 0 || i >= (int32_t)b->cols.size()) return GLC_ERR_INVALID_ARG;
  *col = b->cols[i];
  return GLC_OK;
}

glc_status glc_batch_decompress(glc_ctx* ctx, glc_batch* b, void* const* outs, int use_graph, glc_stream stream) {
  if (!ctx || !b || (!outs && !b->cols.empty())) return bfail(ctx, GLC_ERR_INVALID_ARG, "bad batch arguments");
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->own_stream;
  glc_status st = build_work(ctx, b, outs, s);
  if (st != GLC_OK) return st;
  if (b->nwork == 0) return GLC_OK;
  BatchDecodeArgs a;
  a.cols = b->d_cols;
  a.work = b->d_work;
  a.nwork = b->nwork;
  for (int d = 0; d < 5; d++) a.group_begin[d] = b->group_begin[d];
  a.counter = b->d_counter;
  a.err = b->d_err;
  a.stage_bytes = batch_stage_bytes(b->max_bits);
  if (!use_graph) {
    BCK(launch_batch_decode(a, ctx->num_sms, s), "batch decode");
    return GLC_OK;
  }
  if (!b->graph) {  // capture the counter reset and the launch once; replay afterwards
    cudaGraph_t g = nullptr;
    BCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "batch decode: capture");
    cudaError_t e = launch_batch_decode(a, ctx->num_sms, s);
    cudaError_t e2 = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); return bcuda(ctx, e, "batch decode: capture"); }
    if (e2 != cudaSuccess) return bcuda(ctx, e2, "batch decode: capture");
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { b->graph = nullptr; return bcuda(ctx, e, "batch decode: instantiate"); }
  }
  BCK(cudaGraphLaunch(b->graph, s), "batch decode: graph launch");
  return GLC_OK;
}

glc_status glc_batch_recompress(glc_ctx* ctx, glc_batch* b, const void* const* values, int use_graph,
                                glc_stream stream) {
  if (!ctx || !b || !values) return bfail(ctx, GLC_ERR_INVALID_ARG, "bad batch arguments");
  if (!b->one_pass)
    return bfail(ctx, GLC_ERR_UNSUPPORTED, "recompress needs a batch compressed at lengths 1024 / 2048 / 4096");
  for (size_t i = 0; i < b->cols.size(); i++)
    if (b->ns[i] > 0 && (!values[i] || ((uintptr_t)values[i] % dtype_size(b->dtypes[i])) != 0))
      return bfail(ctx, GLC_ERR_INVALID_ARG, "null or misaligned values for a column of the batch");
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->own_stream;
  glc_status st;
  if (b->re.empty() && !b->cols.empty()) {
    if ((st = recompress_setup(ctx, b, s)) != GLC_OK) return st;
  }
  bool same = b->re_values.size() == b->cols.size();
  for (size_t i = 0; same && i < b->cols.size(); i++) same = b->re_values[i] == values[i];
  if (!same) {
    if (b->re_graph) {
      cudaGraphExecDestroy(b->re_graph);
      b->re_graph = nullptr;
    }
    if ((st = recompress_tables(ctx, b, values, s)) != GLC_OK) return st;
  }
  // until glc_batch_sync, the decode stages the widest tiles the element types allow
  int widest = 0;
  for (glc_dtype dt : b->dtypes) widest = std::max(widest, dtype_size(dt) == 8 ? 64 : 33);
  if (b->max_bits != widest && b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->max_bits = widest;
  b->re_stale = true;
  if (!use_graph) {
    BCK(recompress_launches(ctx, b, s), "batch recompress");
    return GLC_OK;
  }
  if (!b->re_graph) {
    cudaGraph_t g = nullptr;
    BCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "batch recompress: capture");
    cudaError_t e = recompress_launches(ctx, b, s);
    cudaError_t e2 = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); return bcuda(ctx, e, "batch recompress: capture"); }
    if (e2 != cudaSuccess) return bcuda(ctx, e2, "batch recompress: capture");
    e = cudaGraphInstantiate(&b->re_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { b->re_graph = nullptr; return bcuda(ctx, e, "batch recompress: instantiate"); }
  }
  BCK(cudaGraphLaunch(b->re_graph, s), "batch recompress: graph launch");
  return GLC_OK;
}

glc_status glc_batch_sync(glc_ctx* ctx, glc_batch* b, glc_stream stream, int64_t* compressed_size_bytes) {
  if (!ctx || !b) return bfail(ctx, GLC_ERR_INVALID_ARG, "bad batch arguments");
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->own_stream;
  const size_t nc = b->cols.size();
  int64_t total = 0;
  if (b->re_stale) {
    std::vector<unsigned long long> hs(2 * nc + 1);
    BCK(cudaMemcpyAsync(hs.data(), b->re_stats, sizeof(unsigned long long) * hs.size(), cudaMemcpyDeviceToHost, s),
        "batch sync");
    BCK(cudaStreamSynchronize(s), "batch sync");
    if (hs[2 * nc] == DEVERR_TIMEOUT) return bfail(ctx, GLC_ERR_TIMEOUT, "batch recompress: a device-side wait gave up");
    if (hs[2 * nc] != DEVERR_NONE) return bfail(ctx, GLC_ERR_CUDA, "batch recompress: words beyond their array");
    std::vector<BatchColumn> h(nc);
    int mb = 0;
    for (size_t i = 0; i < nc; i++) {
      glc_column* c = b->cols[i];
      if (c->n > 0) {
        c->total_bits = (int64_t)hs[2 * i];
        c->max_bits = (int32_t)hs[2 * i + 1];
        c->nwords = (c->total_bits + 31) / 32;
        c->reported_size = 64 * c->P + 120 + (c->total_bits + 7) / 8;  // api/G-LeCo.cuh:589-603
      }
      mb = std::max(mb, c->max_bits);
      h[i] = BatchColumn{c->d_desc, c->d_start, c->d_tiles, c->d_words, c->n, (int32_t)c->dtype, c->max_bits};
    }
    BCK(cudaMemcpyAsync(b->d_cols, h.data(), sizeof(BatchColumn) * nc, cudaMemcpyHostToDevice, s), "batch sync");
    BCK(cudaStreamSynchronize(s), "batch sync");
    if (mb != b->max_bits && b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    b->max_bits = mb;
    b->re_stale = false;
  } else {
    BCK(cudaStreamSynchronize(s), "batch sync");
  }
  for (glc_column* c : b->cols) total += c->reported_size;
  if (compressed_size_bytes) *compressed_size_bytes = total;
  return GLC_OK;
}

glc_status glc_batch_free(glc_batch* b) {
  if (!b) return GLC_ERR_INVALID_ARG;
  glc::DeviceScope device_scope(b->ctx->device);
  cudaDeviceSynchronize();
  free_batch(b);
  return GLC_OK;
}

}  // extern "C"
