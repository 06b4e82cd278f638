// api.cu -- the C ABI (include/glc.h): contexts, columns, compress / decode / random access,
// pre-unpack and the version-5 blob.  Orchestration only; the kernels live in the other .cu
// files.  Nothing here exits the process or falls back to host computation: every failure is a
// glc_status with a message (the reference calls exit() on any CUDA error,
// core/CudaUtils.cuh:5-13).
#include <cstdio>
#include <cstring>
#include <new>
#include "glc_internal.h"

using namespace glc;

namespace {

struct BlobHeader {  // core/InternalTypes.cuh:39-63 (120 bytes, 4 trailing pad bytes)
  uint32_t magic, version, total_values, num_partitions;
  uint64_t start_off, end_off, types_off, params_off, bits_off, offsets_off, errb_off, delta_off;
  uint64_t params_size, delta_size;
  uint32_t type_size, checksum;
  uint32_t reserved[3];
  uint32_t pad;
};
static_assert(sizeof(BlobHeader) == 120, "blob header layout");
constexpr uint32_t kMagic = 0x4F43454C;

uint64_t align8(uint64_t x) { return (x + 7) & ~7ull; }

// api/G-LeCo.cuh:87-100: rotate-add (the build without SSE4.2) or byte-wise CRC32C from 0.
uint32_t header_checksum(const uint8_t* p, size_t n, int crc32c) {
  uint32_t c = 0;
  if (!crc32c) {
    for (size_t i = 0; i < n; i++) { c += p[i]; c = (c << 1) | (c >> 31); }
    return c;
  }
  for (size_t i = 0; i < n; i++) {
    c ^= p[i];
    for (int k = 0; k < 8; k++) c = (c >> 1) ^ (0x82F63B78u & (0u - (c & 1u)));
  }
  return c;
}

void fill_layout(BlobHeader& h, int64_t P, int64_t total_bits, int type_size, int64_t n) {
  std::memset(&h, 0, sizeof h);
  h.magic = kMagic;
  h.version = 5;
  h.total_values = (uint32_t)n;
  h.num_partitions = (uint32_t)P;
  uint64_t off = sizeof(BlobHeader);
  off = align8(off); h.start_off = off; off += 4 * (uint64_t)P;
  off = align8(off); h.end_off = off; off += 4 * (uint64_t)P;
  off = align8(off); h.types_off = off; off += 4 * (uint64_t)P;
  off = align8(off); h.params_off = off; h.params_size = 32 * (uint64_t)P; off += 32 * (uint64_t)P;
  off = align8(off); h.bits_off = off; off += 4 * (uint64_t)P;
  off = align8(off); h.offsets_off = off; off += 8 * (uint64_t)P;
  off = align8(off); h.errb_off = off; off += 8 * (uint64_t)P;
  off = align8(off); h.delta_off = off;
  h.delta_size = (uint64_t)(total_bits + 7) / 8;
  h.type_size = (uint32_t)type_size;
}

uint64_t blob_total(const BlobHeader& h) { return align8(h.delta_off + h.delta_size); }

glc_status fail(glc_ctx* ctx, glc_status st, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return st;
}

glc_status cuda_fail(glc_ctx* ctx, cudaError_t e, const char* where) {
  if (e == cudaErrorMemoryAllocation) return fail(ctx, GLC_ERR_OOM, std::string(where) + ": out of device memory");
  return fail(ctx, GLC_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call, where)                                  \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
  } while (0)

cudaStream_t pick(glc_ctx* ctx, glc_stream s) { return s ? (cudaStream_t)s : ctx->own_stream; }

bool valid_dtype(int d) { return d >= GLC_I32 && d <= GLC_U32; }

// Column arrays come from cudaMalloc, or from a stream-ordered pool when c->pool is set (the
// columns a server deserializes: their allocation and release never synchronise the device).
template <typename P> cudaError_t col_alloc(glc_column* c, P** p, size_t bytes, cudaStream_t s) {
  if (c->pool) return cudaMallocFromPoolAsync((void**)p, bytes, c->pool, s);
  return cudaMalloc((void**)p, bytes);
}

void col_release(glc_column* c, void* p) {
  if (!p) return;
  if (c->pool) cudaFreeAsync(p, c->ctx->own_stream);
  else cudaFree(p);
}

void free_column_arrays(glc_column* c) {
  if (c->blob_view) {  // the SoA arrays and the bitstream lie in the blob (owned or borrowed)
    void* ptrs[] = {c->d_plain, c->d_desc, c->d_tiles, c->owned};
    for (void* p : ptrs) col_release(c, p);
    c->owned = nullptr;
  } else {
    void* ptrs[] = {c->d_start, c->d_end, c->d_types, c->d_params, c->d_bits, c->d_offs, c->d_err,
                    c->d_words, c->d_plain, c->d_desc, c->d_tiles};
    for (void* p : ptrs) col_release(c, p);
  }
  c->d_start = c->d_end = c->d_types = c->d_bits = nullptr;
  c->d_params = nullptr;
  c->d_offs = c->d_err = c->d_plain = nullptr;
  c->d_words = nullptr;
  c->d_desc = nullptr;
  c->d_tiles = nullptr;
}

// Metadata arrays for P partitions and the decode tile table.
cudaError_t alloc_meta(glc_column* c, cudaStream_t s) {
  const int64_t P = c->P > 0 ? c->P : 1;
  cudaError_t e;
  if ((e = col_alloc(c, &c->d_start, 4 * P, s)) != cudaSuccess) return e;
  if ((e = col_alloc(c, &c->d_end, 4 * P, s)) != cudaSuccess) return e;
  if ((e = col_alloc(c, &c->d_types, 4 * P, s)) != cudaSuccess) return e;
  if ((e = col_alloc(c, &c->d_params, 32 * P, s)) != cudaSuccess) return e;
  if ((e = col_alloc(c, &c->d_bits, 4 * P, s)) != cudaSuccess) return e;
  if ((e = col_alloc(c, &c->d_offs, 8 * P, s)) != cudaSuccess) return e;
  if ((e = col_alloc(c, &c->d_err, 8 * P, s)) != cudaSuccess) return e;
  if ((e = col_alloc(c, &c->d_desc, sizeof(PartDesc) * P, s)) != cudaSuccess) return e;
  c->ntiles = (c->n + kDecodeTile - 1) / kDecodeTile;
  if ((e = col_alloc(c, &c->d_tiles, sizeof(TileInfo) * (c->ntiles + 1), s)) != cudaSuccess) return e;
  return cudaSuccess;
}

void set_word_counts(glc_column* c) {
  c->nwords = (c->total_bits + 31) / 32;
  c->nwords_alloc = ((c->nwords + 3) & ~3ll) + 8;  // decoders read up to 3 words past a field
}

// A private pool that keeps freed memory (release threshold = max), so per-call temporaries
// (host-output staging, scratch) cost no fresh device allocation after the first call.
cudaError_t create_pool(glc_ctx* ctx) {
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = ctx->device;
  cudaError_t e = cudaMemPoolCreate(&ctx->pool, &props);
  if (e != cudaSuccess) return e;
  uint64_t keep = ~0ull;
  return cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
}

int64_t reported_size(int64_t P, int64_t total_bits) {  // api/G-LeCo.cuh:589-603
  return 64 * P + 120 + (total_bits + 7) / 8;
}

}  // namespace

extern "C" {

const char* glc_status_string(glc_status s) {
  switch (s) {
    case GLC_OK: return "ok";
    case GLC_ERR_INVALID_ARG: return "invalid argument";
    case GLC_ERR_BAD_BLOB: return "bad blob";
    case GLC_ERR_OOM: return "out of memory";
    case GLC_ERR_CUDA: return "CUDA error";
    case GLC_ERR_TIMEOUT: return "device wait timed out";
    case GLC_ERR_BUDGET: return "memory budget exceeded";
    case GLC_ERR_UNSUPPORTED: return "unsupported for this column";
  }
  return "unknown status";
}

const char* glc_last_error(const glc_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

glc_status glc_create(glc_ctx** out, int device) {
  if (!out) return GLC_ERR_INVALID_ARG;
  *out = nullptr;
  glc_ctx* ctx = new (std::nothrow) glc_ctx();
  if (!ctx) return GLC_ERR_OOM;
  cudaError_t e;
  if (device < 0) {
    if ((e = cudaGetDevice(&device)) != cudaSuccess) { delete ctx; return GLC_ERR_CUDA; }
  }
  glc::DeviceScope device_scope(device);
  if (!device_scope.ok()) { delete ctx; return GLC_ERR_CUDA; }
  ctx->device = device;
  if ((e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = create_pool(ctx)) != cudaSuccess ||
      (e = cudaMalloc(&ctx->d_flags, sizeof(int) * kFlagWords)) != cudaSuccess ||
      (e = cudaMemset(ctx->d_flags, 0, sizeof(int) * kFlagWords)) != cudaSuccess ||
      (e = cudaMalloc(&ctx->d_stats, sizeof(int64_t) * 16)) != cudaSuccess ||
      (e = cudaMallocHost(&ctx->h_stats, sizeof(int64_t) * 16)) != cudaSuccess) {
    glc_destroy(ctx);
    return e == cudaErrorMemoryAllocation ? GLC_ERR_OOM : GLC_ERR_CUDA;
  }
  tune_defaults(ctx);
  const char* expire = getenv("GLC_TEST_EXPIRE_FIRST_WAIT");  // test hook: see glc_ctx::expire_next_wait
  if (expire && expire[0] == '1') ctx->expire_next_wait.store(1);
  const char* cache = getenv("GLC_TUNE_CACHE");  // results of an earlier glc_autotune, if they fit
  if (cache && *cache) tune_load(ctx, cache);
  *out = ctx;
  return GLC_OK;
}

glc_status glc_destroy(glc_ctx* ctx) {
  if (!ctx) return GLC_ERR_INVALID_ARG;
  glc::DeviceScope device_scope(ctx->device);
  if (ctx->own_stream) cudaStreamSynchronize(ctx->own_stream);
  if (ctx->d_flags) cudaFree(ctx->d_flags);
  if (ctx->d_stats) cudaFree(ctx->d_stats);
  if (ctx->h_stats) cudaFreeHost(ctx->h_stats);
  stager_free(ctx);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  for (cudaStream_t a : ctx->aux_stream)
    if (a) cudaStreamDestroy(a);
  if (ctx->pool) {
    cudaDeviceSynchronize();
    cudaMemPoolDestroy(ctx->pool);
  }
  delete ctx;
  return GLC_OK;
}

glc_status glc_sync(glc_ctx* ctx, glc_stream stream) {
  if (!ctx) return GLC_ERR_INVALID_ARG;
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = pick(ctx, stream);
  CK(cudaStreamSynchronize(s), "sync");
  int code = 0;
  CK(cudaMemcpy(&code, ctx->d_flags + kFlagError, sizeof(int), cudaMemcpyDeviceToHost), "sync: read error flag");
  if (code != DEVERR_NONE) {
    cudaMemset(ctx->d_flags + kFlagError, 0, sizeof(int));
    return fail(ctx, code == DEVERR_TIMEOUT ? GLC_ERR_TIMEOUT : GLC_ERR_CUDA, "a device-side wait gave up");
  }
  return GLC_OK;
}

glc_status glc_column_free(glc_column* col) {
  if (!col) return GLC_ERR_INVALID_ARG;
  if (col->view) return fail(col->ctx, GLC_ERR_INVALID_ARG, "a column of a batch is freed with its batch");
  glc::DeviceScope device_scope(col->ctx ? col->ctx->device : -1);
  if (col->sync_free) cudaDeviceSynchronize();  // work on any stream may still read the arrays
  free_column_arrays(col);
  delete col;
  return GLC_OK;
}

glc_status glc_column_get_info(const glc_column* c, glc_column_info* info) {
  if (!c || !info) return GLC_ERR_INVALID_ARG;
  info->dtype = c->dtype;
  info->total_values = c->n;
  info->num_partitions = c->P;
  info->total_bits = c->total_bits;
  info->compressed_size_bytes = c->reported_size;
  info->fixed_partition_len = c->fixed_len;
  info->has_packed = (c->d_words != nullptr) ? 1 : 0;
  info->has_preunpacked = (c->d_plain != nullptr) ? 1 : 0;
  info->d_start_indices = c->d_start;
  info->d_end_indices = c->d_end;
  info->d_model_types = c->d_types;
  info->d_model_params = c->d_params;
  info->d_delta_bits = c->d_bits;
  info->d_delta_array_bit_offsets = c->d_offs;
  info->d_error_bounds = c->d_err;
  info->delta_array = words_begin(c);
  info->d_plain_deltas = c->d_plain;
  info->max_delta_bits = c->max_bits;
  return GLC_OK;
}

// ---------------------------------------------------------------------------------------
// compress
// ---------------------------------------------------------------------------------------
static glc_status compress_impl(glc_ctx* ctx, glc_dtype dtype, const void* dev_values, int64_t n,
                                glc_partitioning mode, int32_t fixed_len, glc_column* c, cudaStream_t s) {
  c->ctx = ctx;
  c->dtype = dtype;
  c->n = n;
  // The column's arrays come from the context's pool (no cudaMalloc per array per call); freeing
  // the column synchronises the device first, so a free behaves as cudaFree does.
  c->pool = ctx->pool;
  c->sync_free = true;
  int32_t* tmp_s = nullptr;
  int32_t* tmp_e = nullptr;
  long long* part_err = nullptr;  // variable partitions: each partition's max |delta|, measured by the partitioner
  struct StreamFree {  // returned to the pool after the stream's work so far, on every exit
    void** p;
    cudaStream_t s;
    ~StreamFree() {
      if (*p) cudaFreeAsync(*p, s);
    }
  } part_err_free{reinterpret_cast<void**>(&part_err), s};
  if (mode == GLC_PART_FIXED) {
    c->P = (n + fixed_len - 1) / fixed_len;
    c->fixed_len = fixed_len;
  } else if (mode == GLC_PART_VARIABLE_V6) {
    int64_t P = 0;
    cudaError_t e = launch_partition_v6(ctx, dtype, dev_values, n, kV6Base, &tmp_s, &tmp_e, &P, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "GPU partitioner (V6)");
    c->P = P;
    c->fixed_len = 0;
  } else {
    std::string perr;
    int64_t P = 0;
    cudaError_t e = launch_partition_variable(ctx, dtype, dev_values, n, &tmp_s, &tmp_e, &P, s, &perr, &part_err);
    if (e != cudaSuccess) return perr.empty() ? cuda_fail(ctx, e, "variable partitioner") : fail(ctx, GLC_ERR_CUDA, perr);
    c->P = P;
    c->fixed_len = 0;
  }
  CK(alloc_meta(c, s), "compress: metadata allocation");
  if (mode == GLC_PART_FIXED && fixed_compress_supported(n, fixed_len)) {
    // one read of the values: fit, widths and words of every tile (into scratch slots), a scan of
    // the tiles' bits; then, with the total known, the words placed into an exact-size array
    void* scratch = nullptr;
    CK(pool_alloc(ctx, &scratch, fixed_compress_scratch_bytes(dtype, c->ntiles), s), "compress: scratch");
    unsigned long long* st = (unsigned long long*)ctx->d_stats;
    cudaError_t e = launch_fixed_compress(dtype, dev_values, c, fixed_len, scratch, st, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->h_stats, ctx->d_stats, 3 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && ctx->h_stats[2] != DEVERR_NONE) {
      cudaFreeAsync(scratch, s);
      return fail(ctx, GLC_ERR_TIMEOUT, "compress: a device-side wait gave up");
    }
    if (e == cudaSuccess) {
      c->total_bits = ctx->h_stats[0];
      c->max_bits = (int32_t)ctx->h_stats[1];
      set_word_counts(c);
      e = col_alloc(c, &c->d_words, 4 * c->nwords_alloc, s);
    }
    if (e == cudaSuccess) e = launch_fixed_place(dtype, c, fixed_len, scratch, st, s);
    cudaFreeAsync(scratch, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "compress: one-pass fixed compression");
    c->reported_size = reported_size(c->P, c->total_bits);
    return GLC_OK;
  }
  if (mode == GLC_PART_FIXED) {
    CK(launch_fixed_partitions(c->d_start, c->d_end, n, fixed_len, c->P, s), "compress: fixed partitions");
  } else {
    CK(cudaMemcpyAsync(c->d_start, tmp_s, 4 * c->P, cudaMemcpyDeviceToDevice, s), "compress: partition copy");
    CK(cudaMemcpyAsync(c->d_end, tmp_e, 4 * c->P, cudaMemcpyDeviceToDevice, s), "compress: partition copy");
    cudaFreeAsync(tmp_s, s);
    cudaFreeAsync(tmp_e, s);
  }
  const size_t sb = fit_scratch_bytes(nullptr, n, c->P);
  void* scratch = nullptr;
  CK(pool_alloc(ctx, &scratch, sb, s), "compress: scratch allocation");
  cudaError_t e = launch_fit(dtype, dev_values, c, scratch, sb, ctx->d_stats, s, part_err);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->h_stats, ctx->d_stats, 4 * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(scratch, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "compress: fit");
  if (ctx->h_stats[2] != DEVERR_NONE) return fail(ctx, GLC_ERR_TIMEOUT, "compress: a device-side wait of the fit gave up");
  c->total_bits = ctx->h_stats[0];
  c->max_bits = (int32_t)ctx->h_stats[1];
  set_word_counts(c);
  CK(col_alloc(c, &c->d_words, 4 * c->nwords_alloc, s), "compress: word allocation");
  const int64_t parts_per_tile = ctx->h_stats[3];
  CK(launch_desc_and_tiles(c, s), "compress: tables");
  CK(launch_pack(dtype, dev_values, c, parts_per_tile, ctx->d_flags + kFlagError, s), "compress: pack");
  c->reported_size = reported_size(c->P, c->total_bits);
  return GLC_OK;
}

glc_status glc_compress(glc_ctx* ctx, glc_dtype dtype, const void* values, int64_t n, int flags,
                        glc_partitioning mode, int32_t fixed_partition_len, glc_column** out,
                        int64_t* compressed_size_bytes, glc_stream stream) {
  if (!ctx || !out) return fail(ctx, GLC_ERR_INVALID_ARG, "null context or output");
  *out = nullptr;
  if (!valid_dtype(dtype)) return fail(ctx, GLC_ERR_INVALID_ARG, "unknown dtype");
  if (n < 0 || n > 0x7fffffffll) return fail(ctx, GLC_ERR_INVALID_ARG, "n must be in [0, 2^31)");
  if (n > 0 && !values) return fail(ctx, GLC_ERR_INVALID_ARG, "null values");
  if (mode != GLC_PART_FIXED && mode != GLC_PART_VARIABLE && mode != GLC_PART_VARIABLE_V6)
    return fail(ctx, GLC_ERR_INVALID_ARG, "unknown partitioning");
  if (mode == GLC_PART_FIXED && fixed_partition_len <= 0)
    return fail(ctx, GLC_ERR_INVALID_ARG, "fixed partition length must be positive");
  if (!(flags & GLC_HOST_IN) && ((uintptr_t)values % dtype_size(dtype)) != 0)
    return fail(ctx, GLC_ERR_INVALID_ARG, "device values must be aligned to the element size");
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = pick(ctx, stream);
  glc_column* c = new (std::nothrow) glc_column();
  if (!c) return fail(ctx, GLC_ERR_OOM, "host allocation");
  c->ctx = ctx;
  c->dtype = dtype;
  if (n == 0) {  // api/G-LeCo.cuh:355-371: an empty object, size 0
    c->n = 0;
    c->P = 0;
    set_word_counts(c);
    if (compressed_size_bytes) *compressed_size_bytes = 0;
    c->reported_size = 0;
    *out = c;
    return GLC_OK;
  }
  const void* dev_values = values;
  void* staged = nullptr;
  if (flags & GLC_HOST_IN) {
    const size_t bytes = (size_t)n * dtype_size(dtype);
    cudaError_t e = pool_alloc(ctx, &staged, bytes, s);
    if (e == cudaSuccess) e = host_upload(ctx, staged, values, bytes, s);
    if (e != cudaSuccess) {
      if (staged) cudaFreeAsync(staged, s);
      delete c;
      return cuda_fail(ctx, e, "compress: input upload");
    }
    dev_values = staged;
  }
  glc_status st;
  {
    std::lock_guard<std::mutex> lk(ctx->stats_mu);  // the fit's totals come back through h_stats
    st = compress_impl(ctx, dtype, dev_values, n, mode, fixed_partition_len, c, s);
  }
  if (staged) cudaFreeAsync(staged, s);
  if (st != GLC_OK) {
    cudaStreamSynchronize(s);
    free_column_arrays(c);
    delete c;
    return st;
  }
  if (compressed_size_bytes) *compressed_size_bytes = c->reported_size;
  *out = c;
  return GLC_OK;
}

// Partition boundaries only: the split/merge partitioner (v6_base == 0) or the reference's GPU
// partitioner with that base size.
static glc_status partition_only(glc_ctx* ctx, glc_dtype dtype, const void* values, int64_t n, int flags,
                                 int32_t v6_base, int32_t* starts, int32_t* ends, int64_t cap,
                                 int64_t* num_partitions, glc_stream stream) {
  if (!ctx || !num_partitions) return fail(ctx, GLC_ERR_INVALID_ARG, "null argument");
  if (!valid_dtype(dtype) || n < 0 || n > 0x7fffffffll) return fail(ctx, GLC_ERR_INVALID_ARG, "bad dtype or n");
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = pick(ctx, stream);
  *num_partitions = 0;
  if (n == 0) return GLC_OK;
  if (n > 0 && !values) return fail(ctx, GLC_ERR_INVALID_ARG, "null values");
  const void* dev_values = values;
  void* staged = nullptr;
  if (flags & GLC_HOST_IN) {
    const size_t bytes = (size_t)n * dtype_size(dtype);
    CK(pool_alloc(ctx, &staged, bytes, s), "partition: upload");
    CK(host_upload(ctx, staged, values, bytes, s), "partition: upload");
    dev_values = staged;
  }
  int32_t* ds = nullptr;
  int32_t* de = nullptr;
  int64_t P = 0;
  std::string perr;
  std::unique_lock<std::mutex> stats_lock(ctx->stats_mu);  // partition counts come back through h_stats
  cudaError_t e = v6_base > 0 ? launch_partition_v6(ctx, dtype, dev_values, n, v6_base, &ds, &de, &P, s)
                              : launch_partition_variable(ctx, dtype, dev_values, n, &ds, &de, &P, s, &perr);
  if (staged) cudaFreeAsync(staged, s);
  if (e != cudaSuccess) return perr.empty() ? cuda_fail(ctx, e, "partition") : fail(ctx, GLC_ERR_CUDA, perr);
  *num_partitions = P;
  glc_status st = GLC_OK;
  if (P > cap || !starts || !ends) {
    st = fail(ctx, GLC_ERR_INVALID_ARG, "partition output capacity too small");
  } else {
    const cudaMemcpyKind k = (flags & GLC_HOST_OUT) ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    e = cudaMemcpyAsync(starts, ds, 4 * P, k, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ends, de, 4 * P, k, s);
    if (e != cudaSuccess) st = cuda_fail(ctx, e, "partition: copy out");
  }
  cudaFreeAsync(ds, s);
  cudaFreeAsync(de, s);
  if (flags & GLC_HOST_OUT) CK(cudaStreamSynchronize(s), "partition: sync");
  return st;
}

glc_status glc_partition_variable(glc_ctx* ctx, glc_dtype dtype, const void* values, int64_t n, int flags,
                                  int32_t* starts, int32_t* ends, int64_t cap, int64_t* num_partitions,
                                  glc_stream stream) {
  return partition_only(ctx, dtype, values, n, flags, 0, starts, ends, cap, num_partitions, stream);
}

glc_status glc_partition_v6(glc_ctx* ctx, glc_dtype dtype, const void* values, int64_t n, int flags,
                            int32_t base_size, int32_t* starts, int32_t* ends, int64_t cap, int64_t* num_partitions,
                            glc_stream stream) {
  if (ctx && (base_size < 2 || base_size > (1 << 26) || (base_size & 1)))
    return fail(ctx, GLC_ERR_INVALID_ARG, "base size must be even and in [2, 2^26]");
  return partition_only(ctx, dtype, values, n, flags, base_size, starts, ends, cap, num_partitions, stream);
}

// ---------------------------------------------------------------------------------------
// decode / random access
// ---------------------------------------------------------------------------------------
static glc_status resolve_source(glc_ctx* ctx, const glc_column* c, glc_source src, int* plain) {
  if (src == GLC_SRC_AUTO) src = c->d_plain ? GLC_SRC_PREUNPACKED : GLC_SRC_PACKED;
  if (src == GLC_SRC_PREUNPACKED) {
    if (!c->d_plain) return fail(ctx, GLC_ERR_UNSUPPORTED, "column has no pre-unpacked residuals");
    *plain = 1;
  } else if (src == GLC_SRC_PACKED) {
    if (!c->d_words && c->n > 0) return fail(ctx, GLC_ERR_UNSUPPORTED, "column has no packed bitstream");
    *plain = 0;
  } else {
    return fail(ctx, GLC_ERR_INVALID_ARG, "unknown source");
  }
  return GLC_OK;
}

glc_status glc_decompress_range(glc_ctx* ctx, const glc_column* col, glc_source source, int64_t first, int64_t count,
                                void* out, int flags, glc_stream stream) {
  if (!ctx || !col) return fail(ctx, GLC_ERR_INVALID_ARG, "null argument");
  if (first < 0 || count < 0 || first > col->n || count > col->n - first)  // no signed overflow for any count
    return fail(ctx, GLC_ERR_INVALID_ARG, "range outside the column");
  if (count == 0) return GLC_OK;
  if (!out) return fail(ctx, GLC_ERR_INVALID_ARG, "null output");
  int plain = 0;
  glc_status st = resolve_source(ctx, col, source, &plain);
  if (st != GLC_OK) return st;
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = pick(ctx, stream);
  const size_t es = dtype_size(col->dtype);
  // The kernel writes value e at base + e with 16-byte stores, so base must be 16-byte aligned.
  // Host outputs and misaligned device outputs go through an aligned temporary.
  const size_t shift = (size_t)(first * (int64_t)es) & 15;
  const bool staged = (flags & GLC_HOST_OUT) || (((uintptr_t)out - shift) & 15) != 0;
  void* tmp = nullptr;
  char* dev_out = (char*)out;
  if (staged) {
    CK(pool_alloc(ctx, &tmp, count * es + 16, s), "decode: output allocation");
    dev_out = (char*)tmp + shift;
  }
  char* base = dev_out - first * (int64_t)es;
  cudaError_t e = launch_decode(ctx, col, plain, 0, first, first + count, base, s);
  if (e == cudaSuccess && staged)
    e = (flags & GLC_HOST_OUT) ? host_download(ctx, out, dev_out, count * es, s)
                               : cudaMemcpyAsync(out, dev_out, count * es, cudaMemcpyDeviceToDevice, s);
  if (tmp) cudaFreeAsync(tmp, s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "decode");
  if (flags & GLC_HOST_OUT) return glc_sync(ctx, stream);
  return GLC_OK;
}

glc_status glc_decompress_full(glc_ctx* ctx, const glc_column* col, glc_source source, void* out, int flags,
                               glc_stream stream) {
  if (!col) return fail(ctx, GLC_ERR_INVALID_ARG, "null column");
  return glc_decompress_range(ctx, col, source, 0, col->n, out, flags, stream);
}

glc_status glc_random_access(glc_ctx* ctx, const glc_column* col, glc_source source, const int32_t* positions,
                             int64_t count, void* out, int flags, int32_t fixed_partition_len, glc_stream stream) {
  if (!ctx || !col) return fail(ctx, GLC_ERR_INVALID_ARG, "null argument");
  if (count < 0) return fail(ctx, GLC_ERR_INVALID_ARG, "negative count");
  if (count == 0) return GLC_OK;
  if (!positions || !out) return fail(ctx, GLC_ERR_INVALID_ARG, "null positions or output");
  if (fixed_partition_len < 0) return fail(ctx, GLC_ERR_INVALID_ARG, "negative partition length");
  // a layout of fixed length L: every partition but the last has L values.  A single partition of
  // at most L values is one (the reference's TILE_SIZE layout of a short column).
  const bool single = col->P == 1 && col->n <= fixed_partition_len;
  if (fixed_partition_len > 0 && col->fixed_len != fixed_partition_len && !single)
    return fail(ctx, GLC_ERR_INVALID_ARG, "column is not partitioned with that fixed length");
  int plain = 0;
  glc_status st = resolve_source(ctx, col, source, &plain);
  if (st != GLC_OK) return st;
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = pick(ctx, stream);
  const size_t es = dtype_size(col->dtype);
  const int32_t* dpos = positions;
  void* dout = out;
  void* tpos = nullptr;
  if (flags & GLC_HOST_IN) {
    CK(pool_alloc(ctx, &tpos, 4 * count, s), "random access: positions");
    CK(host_upload(ctx, tpos, positions, 4 * count, s), "random access: positions");
    dpos = (const int32_t*)tpos;
  }
  if (flags & GLC_HOST_OUT) CK(pool_alloc(ctx, &dout, es * count, s), "random access: output");
  const int32_t fl = fixed_partition_len > 0 && !single ? fixed_partition_len : col->fixed_len;
  cudaError_t e = launch_random_access(ctx, col, plain, dpos, count, dout, fl, s);
  if (e == cudaSuccess && (flags & GLC_HOST_OUT)) e = host_download(ctx, out, dout, es * count, s);
  if (tpos) cudaFreeAsync(tpos, s);
  if (flags & GLC_HOST_OUT) cudaFreeAsync(dout, s);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "random access");
  if (flags & (GLC_HOST_OUT | GLC_HOST_IN)) CK(cudaStreamSynchronize(s), "random access: sync");
  return GLC_OK;
}

glc_status glc_preunpack(glc_ctx* ctx, glc_column* col, int drop_packed, glc_stream stream) {
  if (!ctx || !col) return fail(ctx, GLC_ERR_INVALID_ARG, "null argument");
  if (col->view && drop_packed) return fail(ctx, GLC_ERR_INVALID_ARG, "a batch column keeps its bitstream");
  if (col->blob_view && drop_packed) return fail(ctx, GLC_ERR_INVALID_ARG, "an attached blob keeps its bitstream");
  if (col->n == 0) return GLC_OK;
  if (!col->d_plain) {
    if (!col->d_words) return fail(ctx, GLC_ERR_UNSUPPORTED, "column has no packed bitstream");
    glc::DeviceScope device_scope(ctx->device);
    cudaStream_t s = pick(ctx, stream);
    CK(col_alloc(col, &col->d_plain, 8 * col->n + 16, s), "pre-unpack: allocation");  // +16: 16-byte TMA granules
    CK(cudaMemsetAsync((char*)col->d_plain + 8 * col->n, 0, 16, s), "pre-unpack: padding");
    CK(launch_decode(ctx, col, 0, 1, 0, col->n, col->d_plain, s), "pre-unpack");
    CK(cudaStreamSynchronize(s), "pre-unpack: sync");
  }
  if (drop_packed && col->d_words) {  // api/G-LeCo.cuh:2283-2287
    if (col->sync_free) cudaDeviceSynchronize();  // work on any stream may still read the bitstream
    col_release(col, col->d_words);
    col->d_words = nullptr;
  }
  return GLC_OK;
}

// ---------------------------------------------------------------------------------------
// blob version 5
// ---------------------------------------------------------------------------------------
glc_status glc_blob_size(const glc_column* c, uint64_t* size) {
  if (!c || !size) return GLC_ERR_INVALID_ARG;
  BlobHeader h;
  fill_layout(h, c->P, c->total_bits, dtype_size(c->dtype), c->n);
  *size = blob_total(h);
  return GLC_OK;
}

glc_status glc_serialize(glc_ctx* ctx, const glc_column* c, void* blob, uint64_t cap, int flags, int crc32c,
                         uint64_t* written, glc_stream stream) {
  if (!ctx || !c || !blob) return fail(ctx, GLC_ERR_INVALID_ARG, "null argument");
  if (!c->d_words && c->d_plain) {  // api/G-LeCo.cuh:2005-2011
    return fail(ctx, GLC_ERR_UNSUPPORTED, "a column whose bitstream was dropped cannot be serialized");
  }
  BlobHeader h;
  fill_layout(h, c->P, c->total_bits, dtype_size(c->dtype), c->n);
  const uint64_t total = blob_total(h);
  if (written) *written = total;
  if (cap < total) return fail(ctx, GLC_ERR_INVALID_ARG, "blob capacity too small");
  BlobHeader t = h;
  t.checksum = 0;
  h.checksum = header_checksum((const uint8_t*)&t, sizeof t, crc32c);
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = pick(ctx, stream);
  const bool host = (flags & GLC_HOST_OUT) != 0;
  uint8_t* b = (uint8_t*)blob;
  const cudaMemcpyKind k = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  const uint64_t P = c->P;
  struct Piece { uint64_t off; const void* src; uint64_t bytes; } pieces[8] = {
      {h.start_off, c->d_start, 4 * P}, {h.end_off, c->d_end, 4 * P},     {h.types_off, c->d_types, 4 * P},
      {h.params_off, c->d_params, 32 * P}, {h.bits_off, c->d_bits, 4 * P}, {h.offsets_off, c->d_offs, 8 * P},
      {h.errb_off, c->d_err, 8 * P},     {h.delta_off, words_begin(c), h.delta_size}};
  // zero the gaps (alignment padding and the tail), then the header, then the arrays
  uint64_t cursor = sizeof(BlobHeader);
  for (const Piece& pc : pieces) {
    if (pc.off > cursor) {
      if (host) std::memset(b + cursor, 0, pc.off - cursor);
      else CK(cudaMemsetAsync(b + cursor, 0, pc.off - cursor, s), "serialize: padding");
    }
    cursor = pc.off + pc.bytes;
  }
  if (total > cursor) {
    if (host) std::memset(b + cursor, 0, total - cursor);
    else CK(cudaMemsetAsync(b + cursor, 0, total - cursor, s), "serialize: padding");
  }
  if (host) std::memcpy(b, &h, sizeof h);
  else CK(cudaMemcpyAsync(b, &h, sizeof h, cudaMemcpyHostToDevice, s), "serialize: header");
  for (const Piece& pc : pieces)
    if (pc.bytes)
      CK(host ? host_download(ctx, b + pc.off, pc.src, pc.bytes, s) : cudaMemcpyAsync(b + pc.off, pc.src, pc.bytes, k, s),
         "serialize: arrays");
  CK(cudaStreamSynchronize(s), "serialize: sync");  // the header lives on this stack frame
  return GLC_OK;
}

glc_status glc_deserialize(glc_ctx* ctx, glc_dtype dtype, const void* blob, uint64_t size, int flags, int crc32c,
                           int pre_unpack, glc_column** out, glc_stream stream) {
  return glc::deserialize_column(ctx, dtype, blob, size, flags, crc32c, pre_unpack, out, stream, nullptr, false);
}

}  // extern "C"

namespace {

// Reads and checks a blob's header (api/G-LeCo.cuh:1029-1049: magic, version, element size,
// checksum, size), plus bounds checks on every array and on the partition count.
glc_status read_blob_header(glc_ctx* ctx, glc_dtype dtype, const void* blob, uint64_t size, bool host, int crc32c,
                            BlobHeader* out) {
  BlobHeader& h = *out;
  if (host) std::memcpy(&h, blob, sizeof h);
  else CK(cudaMemcpy(&h, blob, sizeof h, cudaMemcpyDeviceToHost), "blob: header");
  if (h.magic != kMagic || (h.version != 4 && h.version != 5)) return fail(ctx, GLC_ERR_BAD_BLOB, "bad magic or version");
  if ((int)h.type_size != dtype_size(dtype)) return fail(ctx, GLC_ERR_BAD_BLOB, "blob element size differs from dtype");
  BlobHeader t = h;
  t.checksum = 0;
  if (header_checksum((const uint8_t*)&t, sizeof t, crc32c) != h.checksum)
    return fail(ctx, GLC_ERR_BAD_BLOB, "header checksum mismatch");
  uint64_t expected = h.delta_off + h.delta_size;
  if (h.version == 5) expected = align8(expected);
  if (h.delta_off > size || h.delta_size > size || expected > size) return fail(ctx, GLC_ERR_BAD_BLOB, "blob is short");
  const uint64_t P = h.num_partitions;
  const uint64_t offs[7] = {h.start_off, h.end_off, h.types_off, h.params_off, h.bits_off, h.offsets_off, h.errb_off};
  const uint64_t lens[7] = {4 * P, 4 * P, 4 * P, 32 * P, 4 * P, 8 * P, 8 * P};
  for (int k = 0; k < 7; k++)
    if (offs[k] > size || lens[k] > size - offs[k]) return fail(ctx, GLC_ERR_BAD_BLOB, "array outside the blob");
  if ((P == 0) != (h.total_values == 0)) return fail(ctx, GLC_ERR_BAD_BLOB, "partition count and length disagree");
  return GLC_OK;
}

}  // namespace

glc_status glc::deserialize_column(glc_ctx* ctx, glc_dtype dtype, const void* blob, uint64_t size, int flags,
                                   int crc32c, int pre_unpack, glc_column** out, glc_stream stream,
                                   cudaMemPool_t pool, bool defer_words) {
  if (!ctx || !out) return fail(ctx, GLC_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> stats_lock(ctx->stats_mu);  // the checks come back through h_stats
  *out = nullptr;
  if (!valid_dtype(dtype)) return fail(ctx, GLC_ERR_INVALID_ARG, "unknown dtype");
  if (!blob || size < sizeof(BlobHeader)) return fail(ctx, GLC_ERR_BAD_BLOB, "blob shorter than its header");
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = pick(ctx, stream);
  const bool host = (flags & GLC_HOST_IN) != 0;
  BlobHeader h;
  glc_status hst = read_blob_header(ctx, dtype, blob, size, host, crc32c, &h);
  if (hst != GLC_OK) return hst;
  const uint64_t P = h.num_partitions;
  const uint64_t offs[7] = {h.start_off, h.end_off, h.types_off, h.params_off, h.bits_off, h.offsets_off, h.errb_off};
  const uint64_t lens[7] = {4 * P, 4 * P, 4 * P, 32 * P, 4 * P, 8 * P, 8 * P};

  glc_column* c = new (std::nothrow) glc_column();
  if (!c) return fail(ctx, GLC_ERR_OOM, "host allocation");
  c->ctx = ctx;
  c->pool = pool;
  c->dtype = dtype;
  c->n = h.total_values;
  c->P = (int64_t)P;
  c->total_bits = (int64_t)h.delta_size * 8;  // bound; refined below
  auto bail = [&](glc_status st) { cudaStreamSynchronize(s); free_column_arrays(c); delete c; return st; };
  if (c->n == 0) {
    set_word_counts(c);
    c->reported_size = 0;
    *out = c;
    return GLC_OK;
  }
  cudaError_t e = alloc_meta(c, s);
  if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "deserialize: allocation"));
  set_word_counts(c);
  if ((e = col_alloc(c, &c->d_words, 4 * c->nwords_alloc, s)) != cudaSuccess)
    return bail(cuda_fail(ctx, e, "deserialize: allocation"));
  const cudaMemcpyKind k = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  const uint8_t* b = (const uint8_t*)blob;
  void* dst[7] = {c->d_start, c->d_end, c->d_types, c->d_params, c->d_bits, c->d_offs, c->d_err};
  auto copy_in = [&](void* d, const void* src, size_t len) {
    return host ? host_upload(ctx, d, src, len, s) : cudaMemcpyAsync(d, src, len, k, s);
  };
  for (int j = 0; j < 7; j++)
    if (lens[j] && (e = copy_in(dst[j], b + offs[j], lens[j])) != cudaSuccess)
      return bail(cuda_fail(ctx, e, "deserialize: arrays"));
  if ((e = cudaMemsetAsync(c->d_words, 0, 4 * c->nwords_alloc, s)) != cudaSuccess ||
      (h.delta_size && !defer_words && (e = copy_in(c->d_words, b + h.delta_off, h.delta_size)) != cudaSuccess))
    return bail(cuda_fail(ctx, e, "deserialize: bitstream"));
  // structure check, fixed-length detection and max width
  int* d_chk = (int*)(ctx->d_stats + 4);
  if ((e = cudaMemsetAsync(ctx->d_stats, 0, 8 * sizeof(int64_t), s)) != cudaSuccess ||
      (e = launch_validate(c, d_chk, s)) != cudaSuccess || (e = launch_max_bits(c, ctx->d_stats + 1, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(ctx->h_stats, ctx->d_stats, 8 * sizeof(int64_t), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return bail(cuda_fail(ctx, e, "deserialize: validation"));
  const int* chk = (const int*)(ctx->h_stats + 4);
  if (chk[0]) return bail(fail(ctx, GLC_ERR_BAD_BLOB, "partition arrays are inconsistent"));
  c->max_bits = (int32_t)ctx->h_stats[1];
  c->fixed_len = 0;
  if (!chk[1]) {
    int32_t s0 = 0, e0 = 0;
    if (host) {
      std::memcpy(&s0, b + h.start_off, 4);
      std::memcpy(&e0, b + h.end_off, 4);
    } else {
      cudaMemcpy(&s0, c->d_start, 4, cudaMemcpyDeviceToHost);
      cudaMemcpy(&e0, c->d_end, 4, cudaMemcpyDeviceToHost);
    }
    c->fixed_len = e0 - s0;
  }
  // total bits: the end of the last partition's range (api/G-LeCo.cuh:2016-2044)
  {
    int32_t ls = 0, le = 0, lb = 0;
    int64_t lo = 0;
    const uint64_t L = P - 1;
    if (host) {
      std::memcpy(&ls, b + h.start_off + 4 * L, 4);
      std::memcpy(&le, b + h.end_off + 4 * L, 4);
      std::memcpy(&lb, b + h.bits_off + 4 * L, 4);
      std::memcpy(&lo, b + h.offsets_off + 8 * L, 8);
    } else {
      cudaMemcpy(&ls, c->d_start + L, 4, cudaMemcpyDeviceToHost);
      cudaMemcpy(&le, c->d_end + L, 4, cudaMemcpyDeviceToHost);
      cudaMemcpy(&lb, c->d_bits + L, 4, cudaMemcpyDeviceToHost);
      cudaMemcpy(&lo, c->d_offs + L, 8, cudaMemcpyDeviceToHost);
    }
    c->total_bits = lo + (int64_t)(le - ls) * lb;
  }
  if ((e = launch_desc_and_tiles(c, s)) != cudaSuccess) return bail(cuda_fail(ctx, e, "deserialize: tables"));
  c->reported_size = reported_size(c->P, c->total_bits);
  if (pre_unpack) {
    glc_status st = glc_preunpack(ctx, c, 1, stream);
    if (st != GLC_OK) return bail(st);
  }
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return bail(cuda_fail(ctx, e, "deserialize: sync"));
  *out = c;
  return GLC_OK;
}

// ---------------------------------------------------------------------------------------
// a column attached to a blob: the blob's arrays read where they lie
// ---------------------------------------------------------------------------------------
namespace {

// End of the device allocation holding p (the driver's cuMemGetAddressRange, fetched through the
// runtime so the library links no driver stub); 0 when it cannot be told.
uintptr_t allocation_end(const void* p) {
  typedef int (*AddrRange)(unsigned long long*, size_t*, unsigned long long);
  static AddrRange fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return (AddrRange)f;
  }();
  if (!fn) return 0;
  unsigned long long base = 0;
  size_t bytes = 0;
  if (fn(&base, &bytes, (unsigned long long)(uintptr_t)p) != 0) return 0;
  return (uintptr_t)(base + bytes);
}

constexpr uint64_t kAttachSlack = 64;  // readable bytes the decoders may touch past the bitstream

}  // namespace

glc_status glc::attach_column(glc_ctx* ctx, glc_dtype dtype, const void* blob, uint64_t size, int flags, int crc32c,
                              glc_column** out, glc_stream stream, cudaMemPool_t pool, bool own_copy) {
  if (!ctx || !out) return fail(ctx, GLC_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> stats_lock(ctx->stats_mu);  // the checks come back through h_stats
  *out = nullptr;
  if (!valid_dtype(dtype)) return fail(ctx, GLC_ERR_INVALID_ARG, "unknown dtype");
  if (!blob || size < sizeof(BlobHeader)) return fail(ctx, GLC_ERR_BAD_BLOB, "blob shorter than its header");
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = pick(ctx, stream);
  const bool host = (flags & GLC_HOST_IN) != 0;
  if (!host && ((uintptr_t)blob & 7) != 0) return fail(ctx, GLC_ERR_INVALID_ARG, "device blob must be 8-byte aligned");
  BlobHeader h;
  glc_status hst = read_blob_header(ctx, dtype, blob, size, host, crc32c, &h);
  if (hst != GLC_OK) return hst;
  glc_column* c = new (std::nothrow) glc_column();
  if (!c) return fail(ctx, GLC_ERR_OOM, "host allocation");
  c->ctx = ctx;
  c->pool = pool;
  c->sync_free = pool == nullptr || pool == ctx->pool;  // as the reference's cudaFree in cleanup()
  c->dtype = dtype;
  c->blob_view = true;
  c->n = h.total_values;
  c->P = (int64_t)h.num_partitions;
  auto bail = [&](glc_status st) { cudaStreamSynchronize(s); free_column_arrays(c); delete c; return st; };
  cudaError_t e;
  // where the blob lies on the device: borrowed in place, or a copy placed so that its bitstream
  // starts on a 16-byte boundary, with zeroed slack after it for the decoders' read-ahead
  const uint8_t* b = (const uint8_t*)blob;
  if (host || own_copy) {
    const uint64_t lead = (16 - (h.delta_off & 15)) & 15;
    c->owned_bytes = lead + size + kAttachSlack;
    if ((e = col_alloc(c, (uint8_t**)&c->owned, c->owned_bytes, s)) != cudaSuccess)
      return bail(cuda_fail(ctx, e, "attach: allocation"));
    uint8_t* d = (uint8_t*)c->owned + lead;
    e = host ? host_upload(ctx, d, blob, size, s) : cudaMemcpyAsync(d, blob, size, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d + size, 0, kAttachSlack, s);
    if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "attach: copy of the blob"));
    b = d;
  }
  c->d_start = (int32_t*)(b + h.start_off);
  c->d_end = (int32_t*)(b + h.end_off);
  c->d_types = (int32_t*)(b + h.types_off);
  c->d_params = (double*)(b + h.params_off);
  c->d_bits = (int32_t*)(b + h.bits_off);
  c->d_offs = (int64_t*)(b + h.offsets_off);
  c->d_err = (int64_t*)(b + h.errb_off);
  if (c->n == 0) {
    c->d_words = nullptr;
    set_word_counts(c);
    c->reported_size = 0;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return bail(cuda_fail(ctx, e, "attach: sync"));
    *out = c;
    return GLC_OK;
  }
  // total bits: the end of the last partition's range (api/G-LeCo.cuh:2016-2044)
  {
    struct { int32_t ls, le, lb, pad; int64_t lo; } last;
    const uint64_t L = h.num_partitions - 1;
    e = cudaMemcpyAsync(&last.ls, b + h.start_off + 4 * L, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last.le, b + h.end_off + 4 * L, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last.lb, b + h.bits_off + 4 * L, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last.lo, b + h.offsets_off + 8 * L, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "attach: last partition"));
    c->total_bits = last.lo + (int64_t)(last.le - last.ls) * last.lb;
  }
  set_word_counts(c);
  if ((uint64_t)((c->total_bits + 7) / 8) > h.delta_size && c->total_bits >= 0)
    return bail(fail(ctx, GLC_ERR_BAD_BLOB, "partition arrays are inconsistent"));
  // the kernels read the bitstream from a 16-byte aligned base in aligned 16-byte pieces, and up
  // to a few words past its last field
  const uintptr_t first = (uintptr_t)(b + h.delta_off);
  const uintptr_t base = first & ~(uintptr_t)15;
  const int shift = (int)((first - base) / 4);
  const uint64_t need = (uint64_t)((((c->total_bits + 32 * shift) >> 5) + 8) & ~3ll) * 4;  // bytes from base
  const bool in_place = host || own_copy || (allocation_end(b) >= base + need);
  if (in_place) {
    c->d_words = (uint32_t*)base;
    c->word_shift = shift;
  } else {  // a borrowed blob without room after its bitstream: its bitstream alone is copied
    c->owned_bytes = 4 * (uint64_t)c->nwords_alloc;
    if ((e = col_alloc(c, (uint32_t**)&c->owned, c->owned_bytes, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->owned, 0, c->owned_bytes, s)) != cudaSuccess ||
        (h.delta_size && (e = cudaMemcpyAsync(c->owned, b + h.delta_off, h.delta_size, cudaMemcpyDeviceToDevice, s)) !=
                             cudaSuccess))
      return bail(cuda_fail(ctx, e, "attach: bitstream copy"));
    c->d_words = (uint32_t*)c->owned;
    c->word_shift = 0;
  }
  const int64_t P = c->P;
  c->ntiles = (c->n + kDecodeTile - 1) / kDecodeTile;
  if ((e = col_alloc(c, &c->d_desc, sizeof(PartDesc) * P, s)) != cudaSuccess ||
      (e = col_alloc(c, &c->d_tiles, sizeof(TileInfo) * (c->ntiles + 1), s)) != cudaSuccess)
    return bail(cuda_fail(ctx, e, "attach: tables"));
  // structure check, fixed-length detection and max width (as deserialize)
  int* d_chk = (int*)(ctx->d_stats + 4);
  if ((e = cudaMemsetAsync(ctx->d_stats, 0, 8 * sizeof(int64_t), s)) != cudaSuccess ||
      (e = launch_validate(c, d_chk, s)) != cudaSuccess || (e = launch_max_bits(c, ctx->d_stats + 1, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(ctx->h_stats, ctx->d_stats, 8 * sizeof(int64_t), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return bail(cuda_fail(ctx, e, "attach: validation"));
  const int* chk = (const int*)(ctx->h_stats + 4);
  if (chk[0]) return bail(fail(ctx, GLC_ERR_BAD_BLOB, "partition arrays are inconsistent"));
  c->max_bits = (int32_t)ctx->h_stats[1];
  c->fixed_len = 0;
  if (!chk[1]) {
    int32_t se[2] = {0, 0};
    if ((e = cudaMemcpy(&se[0], c->d_start, 4, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(&se[1], c->d_end, 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
      return bail(cuda_fail(ctx, e, "attach: layout"));
    c->fixed_len = se[1] - se[0];
  }
  if ((e = launch_desc_and_tiles(c, s)) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return bail(cuda_fail(ctx, e, "attach: tables"));
  c->reported_size = reported_size(c->P, c->total_bits);
  *out = c;
  return GLC_OK;
}

extern "C" glc_status glc_attach_blob(glc_ctx* ctx, glc_dtype dtype, const void* blob, uint64_t size, int flags,
                                      int crc32c, glc_column** out, glc_stream stream) {
  return glc::attach_column(ctx, dtype, blob, size, flags, crc32c, out, stream, ctx ? ctx->pool : nullptr, false);
}

// ---------------------------------------------------------------------------------------
// streaming decode of a host blob into host memory
// ---------------------------------------------------------------------------------------
namespace {

template <typename V> V load_at(const uint8_t* p, int64_t i) {  // the blob may sit at any address
  V v;
  std::memcpy(&v, p + i * (int64_t)sizeof(V), sizeof(V));
  return v;
}

// Bit position of value e in a blob's column: offset of its partition + (e - start) * bits.
int64_t blob_bit_of(const uint8_t* starts, const uint8_t* bits, const uint8_t* offs, int64_t P, int64_t e) {
  int64_t lo = 0, hi = P - 1;
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if (load_at<int32_t>(starts, mid) <= e) lo = mid; else hi = mid - 1;
  }
  return load_at<int64_t>(offs, lo) + (e - load_at<int32_t>(starts, lo)) * (int64_t)load_at<int32_t>(bits, lo);
}

}  // namespace

extern "C" glc_status glc_decode_blob_to_host(glc_ctx* ctx, glc_dtype dtype, const void* blob, uint64_t size,
                                              int crc32c, void* out, glc_column** col_out, glc_stream stream) {
  if (!ctx || !blob || (!out && !col_out)) return fail(ctx, GLC_ERR_INVALID_ARG, "null argument");
  if (col_out) *col_out = nullptr;
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t up = pick(ctx, stream);
  // metadata, checks and lookup tables; the bitstream follows in chunks below
  glc_column* c = nullptr;
  glc_status st = deserialize_column(ctx, dtype, blob, size, GLC_HOST_IN, crc32c, 0, &c, stream,
                                     col_out ? nullptr : ctx->pool, true);
  if (st != GLC_OK) return st;
  BlobHeader h;
  std::memcpy(&h, blob, sizeof h);
  const uint8_t* b = (const uint8_t*)blob;
  auto finish = [&](glc_status r) {
    cudaStreamSynchronize(up);
    if (ctx->aux_stream[0]) cudaStreamSynchronize(ctx->aux_stream[0]);
    if (ctx->aux_stream[1]) cudaStreamSynchronize(ctx->aux_stream[1]);
    if (r == GLC_OK && col_out) *col_out = c;
    else glc_column_free(c);
    return r;
  };
  if (c->n == 0) return finish(GLC_OK);
  for (int i = 0; i < 2; i++)
    if (!ctx->aux_stream[i] && cudaStreamCreateWithFlags(&ctx->aux_stream[i], cudaStreamNonBlocking) != cudaSuccess)
      return finish(fail(ctx, GLC_ERR_CUDA, "streaming decode: stream"));
  cudaStream_t dec = ctx->aux_stream[1], down = ctx->aux_stream[0];
  const int64_t es = dtype_size(dtype);
  // chunks of whole decode tiles, about 64 MB of values each, through a ring of 3 staging slots
  const int64_t chunk = std::max<int64_t>(1, (64ll << 20) / (kDecodeTile * es)) * kDecodeTile;
  const int64_t nchunks = (c->n + chunk - 1) / chunk;
  constexpr int kSlots = 3;
  const size_t slot_bytes = (size_t)(chunk * es);
  uint8_t* ring = nullptr;
  std::vector<cudaEvent_t> ev_up(nchunks), ev_dec(nchunks), ev_down(nchunks);
  for (auto* v : {&ev_up, &ev_dec, &ev_down})
    for (auto& x : *v) x = nullptr;
  cudaError_t e = pool_alloc(ctx, &ring, slot_bytes * kSlots, up);
  const uint8_t* hs = b + h.start_off;
  const uint8_t* hb = b + h.bits_off;
  const uint8_t* ho = b + h.offsets_off;
  uint64_t uploaded = 0;  // bytes of the bitstream already queued
  for (int64_t k = 0; k < nchunks && e == cudaSuccess; k++) {
    const int64_t lo = k * chunk, hi = std::min(c->n, lo + chunk);
    // words the decode of [lo, hi) reads: through the last value's field plus the read-ahead
    const int64_t bit_hi = hi >= c->n ? c->total_bits : blob_bit_of(hs, hb, ho, c->P, hi);
    const uint64_t need = std::min<uint64_t>(h.delta_size, (uint64_t)((((bit_hi + 31) >> 5) + 8) * 4));
    for (auto* v : {&ev_up, &ev_dec, &ev_down})
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&(*v)[k], cudaEventDisableTiming);
    if (e == cudaSuccess && need > uploaded) {
      e = cudaMemcpyAsync((uint8_t*)c->d_words + uploaded, b + h.delta_off + uploaded, need - uploaded,
                          cudaMemcpyHostToDevice, up);
      uploaded = need;
    }
    if (e == cudaSuccess) e = cudaEventRecord(ev_up[k], up);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(dec, ev_up[k], 0);
    if (e == cudaSuccess && k >= kSlots) e = cudaStreamWaitEvent(dec, ev_down[k - kSlots], 0);  // slot free
    uint8_t* slot = ring + (size_t)(k % kSlots) * slot_bytes;
    if (e == cudaSuccess) e = launch_decode(ctx, c, 0, 0, lo, hi, slot - lo * es, dec);
    if (e == cudaSuccess) e = cudaEventRecord(ev_dec[k], dec);
    if (e == cudaSuccess && out) {
      e = cudaStreamWaitEvent(down, ev_dec[k], 0);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync((uint8_t*)out + lo * es, slot, (size_t)((hi - lo) * es), cudaMemcpyDeviceToHost, down);
    }
    if (e == cudaSuccess) e = cudaEventRecord(ev_down[k], down);
  }
  if (e == cudaSuccess && uploaded < h.delta_size)  // the rest of the bitstream (kept for later calls)
    e = cudaMemcpyAsync((uint8_t*)c->d_words + uploaded, b + h.delta_off + uploaded, h.delta_size - uploaded,
                        cudaMemcpyHostToDevice, up);
  if (e == cudaSuccess && nchunks > 0) e = cudaStreamWaitEvent(up, ev_down[nchunks - 1], 0);
  if (ring) cudaFreeAsync(ring, up);  // after the last download
  cudaStreamSynchronize(up);
  cudaStreamSynchronize(dec);
  cudaStreamSynchronize(down);
  for (auto* v : {&ev_up, &ev_dec, &ev_down})
    for (auto& x : *v)
      if (x) cudaEventDestroy(x);
  if (e != cudaSuccess) return finish(cuda_fail(ctx, e, "streaming decode"));
  return finish(glc_sync(ctx, stream));
}
