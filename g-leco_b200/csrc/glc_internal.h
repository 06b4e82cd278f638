// glc_internal.h -- host-side structures and kernel launchers of libglc (not part of the ABI).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <atomic>
#include <mutex>
#include <vector>
#include <string>
#include "glc.h"
#include "glc_device.cuh"

namespace glc {

// Decode work unit: a fixed run of output values.  4096 values are 16-32 KB of output, the
// unit each persistent CTA claims from the work counter.
constexpr int kDecodeTile = 4096;
constexpr int kDecodeThreads = 256;
constexpr int kDescCache = 128;  // partitions per tile kept in shared memory

// Per decode tile: bit position of its first value and the partitions it spans.  The table
// has ntiles + 1 entries; the last one holds total_bits.
struct TileInfo {
  int64_t bit_lo;
  int32_t p_first;
  int32_t p_last;
};

// Device scratch owned by a context (grow-only).
struct Scratch {
  void* ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace glc

namespace glc {
// Work counters of concurrent decode launches rotate through this many slots.
constexpr int kCounterSlots = 64;
constexpr int kFlagError = kCounterSlots;      // device error code (DEVERR_*)
constexpr int kFlagWords = kCounterSlots + 8;
}  // namespace glc

namespace glc {
struct HostStager;  // hostxfer.cu: pinned chunks and copy threads for pageable host transfers
// Launch choices per (element type, widest-field bucket, residual source), filled with measured
// defaults and replaced by glc_autotune.
constexpr int kTuneBuckets = 6;  // widest field <= 8, 16, 24, 32, 48, 64 bits
struct TuneEntry {
  int32_t decode_stages;  // TMA ring depth of the decode kernel (2, 3, 4)
  int32_t decode_unroll;  // unroll depth of its full-tile loop (1, 2, 4)
  int32_t ra_shape;       // random-access launch shape (0..4)
  int32_t measured;       // 1 when set by a measurement
  int32_t decode_cap_words;  // largest tile staged in shared memory, in words (0 = built-in)
  int32_t decode_warps;      // consumer warps per CTA of the packed decode: 4 or 8 (0 = 8)
  float decode_gbs;       // decoded GB/s of the chosen decode shape (when measured)
  float ra_glookups;      // G lookups/s of the chosen random-access shape (when measured)
  int32_t partition_len;  // fixed length (1024, 2048, 4096) whose column decoded fastest (0 = not measured)
  int32_t reserved;
};
inline int tune_bucket(int bits) {
  return bits <= 8 ? 0 : bits <= 16 ? 1 : bits <= 24 ? 2 : bits <= 32 ? 3 : bits <= 48 ? 4 : 5;
}
}  // namespace glc

struct glc_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t aux_stream[2] = {nullptr, nullptr};  // streaming decode: download, upload (lazy)
  cudaMemPool_t pool = nullptr;  // private stream-ordered pool; keeps freed memory for reuse
  int* d_flags = nullptr;      // [0, 64) decode work counters, [64] device error code
  int64_t* d_stats = nullptr;  // small readback area (total bits, max bits, ...)
  int64_t* h_stats = nullptr;  // pinned mirror of d_stats
  std::atomic<unsigned> next_slot{0};
  // test hook (GLC_TEST_EXPIRE_FIRST_WAIT=1 at glc_create): the next decode launch's consumers give
  // up their first wait at once, so that launch reports GLC_ERR_TIMEOUT on a healthy copy
  std::atomic<int> expire_next_wait{0};
  std::string err;
  glc::TuneEntry tune[4][glc::kTuneBuckets][2];  // [dtype][bucket][pre-unpacked source]
  std::mutex stats_mu;                     // held by calls that read results back through h_stats
  std::mutex stage_mu;                     // creates `stager` once
  glc::HostStager* stager = nullptr;       // created by the first large pageable transfer
};

struct glc_column {
  glc_ctx* ctx = nullptr;
  cudaMemPool_t pool = nullptr;  // arrays from this stream-ordered pool (else cudaMalloc)
  bool sync_free = false;    // glc_column_free synchronises the device first (as cudaFree would)
  bool view = false;         // arrays are slices of a batch's storage (freed with the batch)
  glc_dtype dtype = GLC_I32;
  int64_t n = 0;
  int64_t P = 0;
  int64_t total_bits = 0;
  int64_t nwords = 0;        // ceil(total_bits / 32)
  int64_t nwords_alloc = 0;  // nwords rounded up to 4 plus zeroed padding for over-reads
  int32_t max_bits = 0;
  int32_t fixed_len = 0;
  int64_t reported_size = 0;
  // reference SoA (CompressedData<T>)
  int32_t* d_start = nullptr;
  int32_t* d_end = nullptr;
  int32_t* d_types = nullptr;
  double* d_params = nullptr;
  int32_t* d_bits = nullptr;
  int64_t* d_offs = nullptr;
  int64_t* d_err = nullptr;
  uint32_t* d_words = nullptr;
  int64_t* d_plain = nullptr;
  // derived lookup tables
  glc::PartDesc* d_desc = nullptr;
  glc::TileInfo* d_tiles = nullptr;
  int64_t ntiles = 0;
  // A column attached to a blob (glc_attach_blob) reads the blob's arrays where they lie: the SoA
  // pointers point into the blob and are not freed with the column.  d_words is then the 16-byte
  // aligned address at or below the blob's bitstream, which starts word_shift words above it; the
  // descriptors and the tile table carry bit positions relative to d_words.  `owned` is device
  // memory the column holds (a copy of the blob, or of its bitstream), freed with it.
  bool blob_view = false;
  int32_t word_shift = 0;
  void* owned = nullptr;
  uint64_t owned_bytes = 0;
};

namespace glc {

inline int dtype_size(glc_dtype d) { return (d == GLC_I64 || d == GLC_U64) ? 8 : 4; }

// The first word of a column's bitstream (d_words is a kernel base below it for attached blobs).
inline const uint32_t* words_begin(const glc_column* c) { return c->d_words ? c->d_words + c->word_shift : nullptr; }

inline const TuneEntry& tune_entry(const glc_ctx* ctx, glc_dtype d, int bits, int plain) {
  return ctx->tune[(int)d & 3][tune_bucket(bits)][plain ? 1 : 0];
}
// hostxfer.cu: host <-> device copies in stream order; pageable buffers of 4 MB and more go
// through the context's pinned chunks (a download returns once `dst` holds the data)
cudaError_t host_upload(glc_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t s);
cudaError_t host_download(glc_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t s);
void stager_free(glc_ctx* ctx);
void tune_defaults(glc_ctx* ctx);                  // tune.cu
bool tune_load(glc_ctx* ctx, const char* path);   // tune.cu: true when the file fits this device

// One bit per device: a per-device launch step (a kernel attribute, which belongs to the
// device's copy of the kernel) has been done.  Safe for concurrent host threads.
struct PerDeviceFlag {
  std::atomic<unsigned long long> bits{0};
  bool test(int dev) const { return dev >= 0 && dev < 64 && ((bits.load(std::memory_order_acquire) >> dev) & 1ull); }
  void set(int dev) {
    if (dev >= 0 && dev < 64) bits.fetch_or(1ull << dev, std::memory_order_release);
  }
};
inline int current_device() {
  int d = 0;
  return cudaGetDevice(&d) == cudaSuccess ? d : -1;
}

// Makes `dev` the calling thread's current device for the scope and gives the caller's device
// back at its end, so that no entry point leaves the thread's device switched.  dev < 0: no change.
class DeviceScope {
 public:
  explicit DeviceScope(int dev) {
    if (dev < 0) return;
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) cur = -1;
    if (cur == dev) return;
    ok_ = cudaSetDevice(dev) == cudaSuccess;
    if (ok_ && cur >= 0) prev_ = cur;
  }
  ~DeviceScope() {
    if (prev_ >= 0) cudaSetDevice(prev_);
  }
  bool ok() const { return ok_; }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;

 private:
  int prev_ = -1;
  bool ok_ = true;
};

// Stream-ordered temporary allocation from the context's pool.
template <typename P> inline cudaError_t pool_alloc(glc_ctx* ctx, P** p, size_t bytes, cudaStream_t s) {
  return cudaMallocFromPoolAsync((void**)p, bytes, ctx->pool, s);
}

// ---- kernel launchers (defined in the .cu files) -------------------------------------
// fit.cu
cudaError_t launch_fixed_partitions(int32_t* starts, int32_t* ends, int64_t n, int32_t len, int64_t P, cudaStream_t s);
size_t fit_scratch_bytes(const int32_t* unused, int64_t n, int64_t P);
// Fits every partition of c (starts/ends set); d_stats[0] = total bits, d_stats[1] = max bits.
// known_err: each partition's max |delta| against its exact least-squares line when already
// measured (the variable partitioner's), so partitions longer than one chunk need no second pass.
cudaError_t launch_fit(glc_dtype dt, const void* values, glc_column* c, void* scratch, size_t scratch_bytes,
                       int64_t* d_stats, cudaStream_t s, const long long* known_err = nullptr);
cudaError_t launch_desc_and_tiles(glc_column* c, cudaStream_t s);
// compress_fixed.cu: one-pass compression of fixed partitions of L values, L a divisor of 4096 and >= 256
// One column of a launch (its arrays are the column's own, or its slices of a batch's arrays).
struct CfColumn {
  const void* values;
  int64_t n;
  int32_t L;
  int32_t parts_per_tile;  // 4096 / L
  int64_t P, ntiles;
  int64_t item_base;       // work item of the column's tile 0
  int64_t nwords_alloc;    // > 0: the edge pass also zeroes the words [total words, nwords_alloc)
  int64_t words_cap;       // words the column's word array holds: nothing is written past it
  int32_t* starts;
  int32_t* ends;
  int32_t* types;
  double* params;
  int32_t* bits;
  int64_t* offs;
  int64_t* err;
  PartDesc* desc;
  TileInfo* tiles;
  uint32_t* words;             // the column's words (interior words of each tile)
  unsigned long long* stats;   // [0] total bits (written by the last tile), [1] widest field
  unsigned long long* choice_bits;  // length choice: the column's bits at lengths 1024, 2048, 4096
};

bool fixed_compress_supported(int64_t n, int32_t L);
int64_t fixed_compress_slot_words(glc_dtype dt);
int64_t fixed_compress_worst_words(glc_dtype dt, int64_t n);  // the widest fields of the type, + padding
size_t fixed_compress_scratch_bytes(glc_dtype dt, int64_t nitems);  // nitems = 4096-value tiles of the launch
cudaError_t launch_fixed_compress(glc_dtype dt, const void* values, glc_column* c, int32_t L, void* scratch,
                                  unsigned long long* stats, cudaStream_t s);
cudaError_t launch_fixed_place(glc_dtype dt, glc_column* c, int32_t L, void* scratch, unsigned long long* stats,
                               cudaStream_t s);
cudaError_t launch_fixed_compress_batch(glc_dtype dt, const CfColumn* cols, const int32_t* owner, int64_t nitems,
                                        void* scratch, unsigned long long* status, int num_sms, cudaStream_t s);
// The exact bits of every column of one element type at partition lengths 1024, 2048 and 4096
// (added into each column's choice_bits, zeroed by the caller), in one read of the values.
// With scratch (fixed_compress_scratch_bytes(dt, nitems)) the same pass also compresses every tile
// at length 4096: its words into its slot, its descriptor and max error into tdesc / terr (nitems
// each); launch_place_prepacked then places the columns that keep length 4096.
cudaError_t launch_choose_lengths(glc_dtype dt, const CfColumn* cols, const int32_t* owner, int64_t nitems,
                                  unsigned long long* status, int num_sms, cudaStream_t s, void* scratch = nullptr,
                                  PartDesc* tdesc = nullptr, long long* terr = nullptr);
cudaError_t launch_place_prepacked(glc_dtype dt, const CfColumn* cols, const int32_t* owner, int64_t nitems,
                                   void* scratch, PartDesc* tdesc, long long* terr, unsigned long long* status,
                                   int num_sms, cudaStream_t s);
cudaError_t launch_validate(const glc_column* c, int* d_bad, cudaStream_t s);
cudaError_t launch_max_bits(const glc_column* c, int64_t* d_out, cudaStream_t s);
// pack.cu: one column's arrays for the packer
struct PackArgs {
  const int32_t* starts;
  const int32_t* ends;
  const int32_t* types;
  const double* params;
  const int32_t* bits;
  const int64_t* offs;
  int64_t P;
  uint32_t* words;
  int64_t nwords_alloc;
};
// pack.cu: one column of a value-tile pack (its decode tile table and descriptors built)
struct PackTileCol {
  const void* v;
  const PartDesc* desc;
  const TileInfo* tiles;
  int64_t n, ntiles;
  uint32_t* words;
};
constexpr int kPackTilePartsMax = 40;  // partitions a 4096-value tile may span in the value-tile pack
cudaError_t launch_batch_pack_tiles(glc_dtype dt, const PackTileCol* cols, const int32_t* owner,
                                    const int64_t* item_base, int64_t nitems, int* status, int num_sms, cudaStream_t s);
cudaError_t launch_pack_item_owner(const int64_t* item_base, int ncols, int32_t* owner, cudaStream_t s);
// pack.cu: packs c's values; the column's descriptor and tile tables must be built.
// parts_per_tile bounds the partitions a 4096-value tile spans (the fit's stats[3]); a device
// wait that gives up is reported in *status (the context's error word, read by glc_sync).
cudaError_t launch_pack(glc_dtype dt, const void* values, glc_column* c, int64_t parts_per_tile, int* status,
                        cudaStream_t s);
// decode.cu: values (or residuals when residual_out) of positions [lo, hi) to out_base[lo..hi)
cudaError_t launch_decode(glc_ctx* ctx, const glc_column* c, int plain_src, int residual_out, int64_t lo,
                          int64_t hi, void* out_base, cudaStream_t s);
// decode.cu: the same with an explicit ring depth and unroll depth (the tuner's candidates)
cudaError_t launch_decode_shape(glc_ctx* ctx, const glc_column* c, int plain_src, int residual_out, int64_t lo,
                                int64_t hi, void* out_base, int stages, int unroll, int cap_words, int warps,
                                cudaStream_t s);
constexpr int kStageCapWordsMax = 8192 + 16;  // a whole tile of 64-bit fields
// decode.cu: packed-source value decode with caller-supplied scratch; the counter must be zero.
cudaError_t launch_decode_scratch(const glc_column* c, int64_t lo, int64_t hi, void* out_base, int* counter,
                                  int* err, int num_sms, cudaStream_t s);
// decode.cu: batched decode over a device work list (many columns, mixed element types)
struct BatchColumn {
  const PartDesc* desc;
  const int32_t* starts;
  const TileInfo* tiles;
  const uint32_t* words;
  int64_t n;
  int32_t dtype;
  int32_t max_bits;
};
struct BatchWork {
  int32_t col;
  int32_t tile;    // tile of that column
  int64_t lo, hi;  // element range of the column decoded by this item (clipped to the tile)
  void* out_base;  // element e of the column is written to out_base[e] (16-byte aligned)
};
// decode.cu: range pieces (one BatchWork each, `tile` = its first tile) -> per-tile work items;
// tile_base[p] = tiles of the pieces before p (npieces + 1 entries)
cudaError_t launch_expand_pieces(const BatchWork* pieces, const int64_t* tile_base, int npieces, int64_t ntiles,
                                 BatchWork* work, int num_sms, cudaStream_t s);
struct BatchDecodeArgs {
  const BatchColumn* cols;
  const BatchWork* work;
  int64_t nwork;
  int64_t group_begin[5];       // items of element type d: [group_begin[d], group_begin[d + 1])
  int32_t grid_begin[5];        // CTAs of element type d (set by the launcher)
  unsigned long long* counter;  // 4 work-item counters (one per type), zeroed per launch
  int* err;
  int stage_bytes;
};
// decode.cu: stable grouping of a work list by element type (col_dtype[c] = type of column c)
void group_work_by_type(std::vector<BatchWork>& w, const std::vector<int32_t>& col_dtype, int64_t group_begin[5]);
cudaError_t launch_batch_decode(const BatchDecodeArgs& b, int num_sms, cudaStream_t s);
// Same launch without zeroing the work counter first (the caller's stream has zeroed it).
cudaError_t launch_batch_decode_zeroed(const BatchDecodeArgs& b, int num_sms, cudaStream_t s);
int batch_stage_bytes(int max_bits);
// random_access.cu
cudaError_t launch_random_access(glc_ctx* ctx, const glc_column* c, int plain_src, const int32_t* pos,
                                 int64_t q, void* out, int32_t fixed_len, cudaStream_t s);
cudaError_t launch_random_access_shape(glc_ctx* ctx, const glc_column* c, int plain_src, const int32_t* pos, int64_t q,
                                       void* out, int32_t fixed_len, int shape, cudaStream_t s);
// api.cu: glc_deserialize with the column's arrays allocated from `pool` (nullptr: cudaMalloc);
// defer_words leaves the bitstream zeroed (the caller uploads it).
glc_status deserialize_column(glc_ctx* ctx, glc_dtype dtype, const void* blob, uint64_t size, int flags, int crc32c,
                              int pre_unpack, glc_column** out, glc_stream stream, cudaMemPool_t pool,
                              bool defer_words = false);
// api.cu: glc_attach_blob; with own_copy the blob is first copied into memory the column owns
// (from `pool`, or cudaMalloc when pool is null), whether it lies in host or device memory.
glc_status attach_column(glc_ctx* ctx, glc_dtype dtype, const void* blob, uint64_t size, int flags, int crc32c,
                         glc_column** out, glc_stream stream, cudaMemPool_t pool, bool own_copy);
// random_access.cu: lookups of many requests into many columns (serving)
struct RAColumn {
  const PartDesc* desc;
  const int32_t* starts;
  const uint32_t* words;
  int64_t P, n;
  int32_t fixed_len;  // > 0: partition = pos / fixed_len
  int32_t dtype;
};
struct RARequest {
  int64_t base;         // first lookup of the request in the launch
  int32_t col;          // index into the launch's column table
  int32_t pad;
  const int32_t* pos;   // the request's positions
  uint8_t* out;         // value k goes to out + k * element size
};
cudaError_t launch_multi_lookup(const RAColumn* cols, const RARequest* reqs, int nreq, int64_t total, int num_sms,
                                cudaStream_t s);
// partition.cu: allocates *d_starts / *d_ends (and, when d_err is given, *d_err: each partition's
// max |delta| against its exact least-squares line) from the context's pool on s
cudaError_t launch_partition_variable(glc_ctx* ctx, glc_dtype dt, const void* values, int64_t n,
                                      int32_t** d_starts, int32_t** d_ends, int64_t* P, cudaStream_t s,
                                      std::string* err, long long** d_err = nullptr);
// partition_v6.cu: the reference's GPU partitioner boundaries (pool-allocated starts/ends)
constexpr int32_t kV6Base = 2048;  // base size compress passes (api/G-LeCo.cuh:384-387)
cudaError_t launch_partition_v6(glc_ctx* ctx, glc_dtype dt, const void* values, int64_t n, int32_t base,
                                int32_t** d_starts, int32_t** d_ends, int64_t* P, cudaStream_t s);

}  // namespace glc
