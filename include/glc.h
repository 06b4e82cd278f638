/* glc.h -- C ABI of the B200-native G-LeCo learned integer-column compression path.
 *
 * Every entry point replaces a method of the reference's header-only C++ class
 * `template<typename T> class LeCoGPU` (api/G-LeCo.cuh:39-2304); the comment above each one
 * names the reference method (file:line) whose behaviour it keeps.  Plain pointers, sizes and
 * integer codes only: no C++ or framework types cross this boundary.
 *
 * Conventions
 *  - Every call returns a glc_status; nothing exits the process (the reference's CUDA_CHECK
 *    calls exit(), core/CudaUtils.cuh:5-13).  glc_last_error() gives a message.
 *  - Device work is stream-ordered on the `stream` argument (a cudaStream_t; NULL = the
 *    context's own stream).  Calls that read or write HOST buffers synchronise that stream
 *    before returning, like the reference's methods; calls on device buffers do not.
 *  - `flags` bit GLC_HOST_IN / GLC_HOST_OUT say that an input / output pointer is host memory
 *    (pageable or pinned); otherwise it is device memory of the context's device.
 *  - A column owns device memory in the reference's SoA layout (CompressedData<T>,
 *    api/G-LeCo_Types.cuh:18-42) plus derived lookup tables.
 *  - A context may be shared by several host threads (the reference's instances may not,
 *    api/G-LeCo.cuh:46-85, :103-107): calls that read results back to the host (compress,
 *    partition, deserialize) take the context's lock, and pageable host buffers of 4 MB or more
 *    share its two pinned 32 MB chunks one transfer at a time.
 */
#ifndef GLC_H_
#define GLC_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GLC_API __attribute__((visibility("default")))
#else
#define GLC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  GLC_OK = 0,
  GLC_ERR_INVALID_ARG = 1, /* bad pointer, size, mode or dtype                       */
  GLC_ERR_BAD_BLOB = 2,    /* blob rejected: magic, version, type size, checksum, size */
  GLC_ERR_OOM = 3,         /* device or host allocation failed                        */
  GLC_ERR_CUDA = 4,        /* a CUDA runtime call failed (message in glc_last_error)  */
  GLC_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up                       */
  GLC_ERR_BUDGET = 6,      /* admission refused: memory budget exceeded                */
  GLC_ERR_UNSUPPORTED = 7  /* the column lacks what the call needs (e.g. no residuals) */
} glc_status;

/* Element types: int32 / int64 / uint64 / uint32 (the reference instantiates LeCoGPU for
 * int, long long, unsigned long long and unsigned int, app/Main.cu:875-987). */
typedef enum { GLC_I32 = 0, GLC_I64 = 1, GLC_U64 = 2, GLC_U32 = 3 } glc_dtype;

/* Partitioning: fixed length (api/G-LeCo.cuh:401-416); variable by model cost
 * (api/G-LeCo.cuh:390-398, compression/CpuPartitioner.cuh: the reference's default variable
 * mode); or the reference's GPU partitioner, compress(..., use_gpu_partitioning = true)
 * (api/G-LeCo.cuh:382-389, compression/GpuPartitioner.cuh:34-214): blocks of 16,384 values get
 * partitions of 8192 / 4096 / 2048 / 1024 values by the quartile of a per-block variance. */
typedef enum { GLC_PART_FIXED = 0, GLC_PART_VARIABLE = 1, GLC_PART_VARIABLE_V6 = 2 } glc_partitioning;

/* Residual source for decoding: the packed bitstream, or the pre-unpacked int64 residual per
 * value (the reference's "high-throughput" mode, d_plain_deltas). AUTO picks pre-unpacked when
 * present, like decompressFullFile (api/G-LeCo.cuh:680-693). */
typedef enum { GLC_SRC_AUTO = 0, GLC_SRC_PACKED = 1, GLC_SRC_PREUNPACKED = 2 } glc_source;

enum { GLC_HOST_IN = 1, GLC_HOST_OUT = 2 };

typedef struct glc_ctx glc_ctx;
typedef struct glc_column glc_column;
typedef struct CUstream_st* glc_stream; /* == cudaStream_t */

/* Read-only view of a column's device arrays (the CompressedData<T> fields). */
typedef struct {
  glc_dtype dtype;
  int64_t total_values;           /* CompressedData::total_values                 */
  int64_t num_partitions;         /* CompressedData::num_partitions               */
  int64_t total_bits;             /* end of the last partition's bit range        */
  int64_t compressed_size_bytes;  /* size compress() reports, api/G-LeCo.cuh:589-603 */
  int32_t fixed_partition_len;    /* > 0 when every partition but the last has this length */
  int32_t has_packed;             /* delta_array present                           */
  int32_t has_preunpacked;        /* d_plain_deltas present                        */
  const int32_t* d_start_indices;
  const int32_t* d_end_indices;
  const int32_t* d_model_types;
  const double* d_model_params;   /* 4 per partition: theta0, theta1, 0, 0 */
  const int32_t* d_delta_bits;
  const int64_t* d_delta_array_bit_offsets;
  const int64_t* d_error_bounds;
  const uint32_t* delta_array;    /* ceil(total_bits/32) words (+ zero padding)   */
  const int64_t* d_plain_deltas;  /* total_values residuals, or NULL               */
  int32_t max_delta_bits;         /* widest residual field (selects the tuned launch shapes) */
} glc_column_info;

/* ---- context ------------------------------------------------------------------------ */

/* Replaces LeCoGPU() (api/G-LeCo.cuh:103-107): binds a device and creates the context's
 * stream.  device < 0 means the current device. */
GLC_API glc_status glc_create(glc_ctx** out, int device);
/* Replaces ~LeCoGPU() (api/G-LeCo.cuh:109-113). */
GLC_API glc_status glc_destroy(glc_ctx* ctx);
GLC_API const char* glc_last_error(const glc_ctx* ctx);
GLC_API const char* glc_status_string(glc_status s);
/* Synchronise the stream and report device-side error flags (bounded waits that gave up). */
GLC_API glc_status glc_sync(glc_ctx* ctx, glc_stream stream);

/* ---- compression -------------------------------------------------------------------- */

/* Replaces LeCoGPU::compress (api/G-LeCo.cuh:349-614).  `values` holds n elements of dtype
 * (host memory when flags & GLC_HOST_IN).  GLC_PART_FIXED uses partitions of
 * `fixed_partition_len` values (the reference's TILE_SIZE = 4096, core/CudaUtils.cuh:18);
 * GLC_PART_VARIABLE runs the device split/merge partitioner (the reference runs
 * VariableLengthPartitioner on the host, compression/CpuPartitioner.cuh:342-422).
 * *compressed_size_bytes (may be NULL) receives the size the reference reports
 * (64 B per partition + 120 B header + ceil(total_bits/8)). n == 0 gives an empty column.
 * Device `values` must be aligned to the element size (GLC_ERR_INVALID_ARG otherwise).  The
 * column's arrays come from the context's memory pool; glc_column_free synchronises the device
 * before releasing them, as the reference's cleanup() (cudaFree) does. */
GLC_API glc_status glc_compress(glc_ctx* ctx, glc_dtype dtype, const void* values, int64_t n, int flags,
                        glc_partitioning mode, int32_t fixed_partition_len, glc_column** out,
                        int64_t* compressed_size_bytes, glc_stream stream);

/* Only the partitioner: start/end arrays of the variable partitioning (device or host
 * buffers of capacity `cap`).  *num_partitions receives P; GLC_ERR_INVALID_ARG when cap < P.
 * Replaces VariableLengthPartitioner<T>::partition (compression/CpuPartitioner.cuh:342). */
GLC_API glc_status glc_partition_variable(glc_ctx* ctx, glc_dtype dtype, const void* values, int64_t n,
                                  int flags, int32_t* starts, int32_t* ends, int64_t cap,
                                  int64_t* num_partitions, glc_stream stream);

/* Only the reference's GPU partitioner (GPUVariableLengthPartitionerV6<T>::partition,
 * compression/GpuPartitioner.cuh:34-214) with its base size (compress uses 2048; even, 2..2^26):
 * the same boundaries, without the reference's per-partition fit (compress refits them).  Where the
 * reference would write more partitions than n / (base / 2) (n <= 8 * base and not a multiple of
 * base / 2) it leaves the last ones unwritten; here every partition is written. */
GLC_API glc_status glc_partition_v6(glc_ctx* ctx, glc_dtype dtype, const void* values, int64_t n, int flags,
                                    int32_t base_size, int32_t* starts, int32_t* ends, int64_t cap,
                                    int64_t* num_partitions, glc_stream stream);

/* Replaces LeCoGPU::cleanup (api/G-LeCo.cuh:793-821).  Like its cudaFree calls, it waits for all
 * work on the device before the column's memory is released (compressed and deserialized columns),
 * so a decode still running on any stream finishes first.  Free columns before glc_destroy. */
GLC_API glc_status glc_column_free(glc_column* col);
GLC_API glc_status glc_column_get_info(const glc_column* col, glc_column_info* info);

/* ---- decompression ------------------------------------------------------------------ */

/* Full decode into `out` (total_values elements).  Replaces decompressFullFile
 * (api/G-LeCo.cuh:680-693) and its variants _BitPacked (:1739), _PreUnpacked (:1790),
 * _OnTheFly_Optimized_V2 (:1842), _WorkStealing (:166), _WorkStealingAdvanced (:220) and
 * _Fix (:768): all are one persistent work-stealing kernel here, reading the residuals from
 * `source`. */
GLC_API glc_status glc_decompress_full(glc_ctx* ctx, const glc_column* col, glc_source source, void* out,
                               int flags, glc_stream stream);

/* Decode the values of the position range [first, first + count) (a range decode).  Same
 * kernel as glc_decompress_full on a sub-range of tiles. */
GLC_API glc_status glc_decompress_range(glc_ctx* ctx, const glc_column* col, glc_source source, int64_t first,
                                int64_t count, void* out, int flags, glc_stream stream);

/* Random access: out[k] = value at positions[k] (0 for positions outside the column).
 * Replaces decompress (random access, api/G-LeCo.cuh:615-678), randomAccessPreUnpacked
 * (:696-766), randomAccessFixed (:1878-1928) and randomAccessFixedPreUnpacked (:1931-1996).
 * fixed_partition_len > 0 asserts fixed partitions of that length (O(1) partition lookup, as
 * the reference's Fixed variants); 0 uses the column's own layout. */
GLC_API glc_status glc_random_access(glc_ctx* ctx, const glc_column* col, glc_source source,
                             const int32_t* positions, int64_t count, void* out, int flags,
                             int32_t fixed_partition_len, glc_stream stream);

/* Build the pre-unpacked int64 residual array (decompression/UnpackKernel.cuh:31-98, called
 * by deserializeGPU(..., true), api/G-LeCo.cuh:2249-2288).  drop_packed != 0 frees the
 * bitstream afterwards, as the reference does; such a column can no longer be serialized. */
GLC_API glc_status glc_preunpack(glc_ctx* ctx, glc_column* col, int drop_packed, glc_stream stream);

/* ---- serialization (blob version 5) --------------------------------------------------- */

/* Exact byte size of the column's blob (api/G-LeCo.cuh:895-960). */
GLC_API glc_status glc_blob_size(const glc_column* col, uint64_t* size);

/* Replaces serialize / serializeGPU (api/G-LeCo.cuh:826-1016, :1999-2152): writes the blob
 * into `blob` (capacity `cap`, host memory when flags & GLC_HOST_OUT).  The header checksum is
 * the rotate-add sum the reference computes without SSE4.2 (api/G-LeCo.cuh:87-100);
 * crc32c != 0 selects its CRC32C variant. */
GLC_API glc_status glc_serialize(glc_ctx* ctx, const glc_column* col, void* blob, uint64_t cap, int flags,
                         int crc32c, uint64_t* written, glc_stream stream);

/* Replaces deserialize / deserializeGPU(blob, preUnpackDeltas) (api/G-LeCo.cuh:1019-1154,
 * :2157-2302).  Accepts versions 4 and 5; rejects (GLC_ERR_BAD_BLOB) a wrong magic, version,
 * type size or checksum, a short blob, or any array outside the blob. */
GLC_API glc_status glc_deserialize(glc_ctx* ctx, glc_dtype dtype, const void* blob, uint64_t size, int flags,
                           int crc32c, int pre_unpack, glc_column** out, glc_stream stream);

/* Decode a serialized column held in HOST memory straight into host memory `out` (total_values
 * elements), streaming: the bitstream is uploaded, decoded and the values downloaded in chunks of
 * about 64 MB on three streams, so upload, decode and download overlap (PCIe carries both
 * directions at once) and the call takes about the download time.  The same checks as
 * glc_deserialize; the values equal glc_deserialize + glc_decompress_full(..., GLC_HOST_OUT),
 * which is the reference's deserializeGPU + decompressFullFile (api/G-LeCo.cuh:2157, :680).
 * col_out (may be NULL) receives the deserialized column, which then stays on the device;
 * out may be NULL when col_out is not.  Pinned `out` gives the full PCIe rate. */
GLC_API glc_status glc_decode_blob_to_host(glc_ctx* ctx, glc_dtype dtype, const void* blob, uint64_t size,
                                           int crc32c, void* out, glc_column** col_out, glc_stream stream);

/* Replaces createDirectAccessHandle(blob, size, copy_to_device) (api/G-LeCo.cuh:1157-1255),
 * whose handle directRandomAccessGPU reads in place (:1257-1334,
 * decompression/RandomAccessKernels.cuh:173-333): a column that reads a serialized blob where it
 * lies, with no deserialize.  Only the partition descriptors and the decode tile table (48 bytes
 * per partition and per 4096 values) are built; random access, range and full decode, the batch
 * and the server read the blob's own arrays and bitstream.  Same checks as glc_deserialize.
 *  - GLC_HOST_IN: the host blob is copied once into device memory the column owns (the
 *    reference's copy_to_device = true).
 *  - otherwise `blob` is device memory of the context's device, 8-byte aligned, BORROWED: it must
 *    stay valid and unchanged until glc_column_free.  When the allocation holding it ends less
 *    than 64 bytes after the bitstream (the decoders read ahead in 16-byte pieces), only the
 *    bitstream is copied into memory the column owns.
 * The column cannot drop its bitstream (glc_preunpack with drop_packed). */
GLC_API glc_status glc_attach_blob(glc_ctx* ctx, glc_dtype dtype, const void* blob, uint64_t size, int flags,
                                   int crc32c, glc_column** out, glc_stream stream);

/* ---- batches: many columns per launch (no counterpart in the reference) ----------------- */

typedef struct glc_batch glc_batch;

/* A batch over existing columns (not owned; they must outlive the batch). */
GLC_API glc_status glc_batch_create(glc_ctx* ctx, glc_column* const* cols, int32_t ncols, glc_batch** out);

/* Compress ncols device columns (values[i]: ns[i] elements of dtypes[i]) with fixed-length
 * partitions in a fixed number of launches.  fixed_partition_len = 0 picks, per column, the length
 * among 1024 / 2048 / 4096 with the smallest compressed size; otherwise 1..8192 for all.  Each
 * column equals glc_compress of the same values with the same length.  The batch owns the
 * columns (glc_batch_column); *compressed_size_bytes receives the sum of their reported sizes. */
GLC_API glc_status glc_batch_compress(glc_ctx* ctx, const glc_dtype* dtypes, const void* const* values,
                                      const int64_t* ns, int32_t ncols, int32_t fixed_partition_len,
                                      glc_batch** out, int64_t* compressed_size_bytes, glc_stream stream);

/* Borrowed handle of column i (valid while the batch lives; freed with it). */
GLC_API glc_status glc_batch_column(const glc_batch* batch, int32_t i, glc_column** col);

/* Decode every column of the batch (outs[i]: 16-byte aligned device buffer for column i) in ONE
 * persistent launch over a device work list.  use_graph != 0 captures the launch in a CUDA graph
 * on the first call and replays it while the outputs stay the same. */
GLC_API glc_status glc_batch_decompress(glc_ctx* ctx, glc_batch* batch, void* const* outs, int use_graph,
                                        glc_stream stream);

/* Compress new values into a batch that glc_batch_compress made at lengths 1024 / 2048 / 4096
 * (fixed_partition_len 0, 1024, 2048 or 4096): the same columns -- element types and sizes in the
 * same order -- with values at new device addresses (aligned to the element size), every column
 * at the partition length the batch chose for it.  Nothing is read back to the host and nothing is
 * allocated after the first call (which gives the batch word arrays for the widest fields of each
 * element type), so the call is stream-ordered; with use_graph != 0 it is captured in a CUDA graph
 * on the first such call and replayed while `values` stay the same.  The columns' device arrays are
 * rewritten in place; their host-side sizes (glc_column_get_info, glc_blob_size, glc_serialize,
 * the compressed size) are brought up to date by glc_batch_sync.  No counterpart in the reference,
 * whose every compress is one host round trip per column (api/G-LeCo.cuh:349-614). */
GLC_API glc_status glc_batch_recompress(glc_ctx* ctx, glc_batch* batch, const void* const* values, int use_graph,
                                        glc_stream stream);

/* Wait for the batch's work on `stream`, then read the columns' sizes written by the last
 * glc_batch_recompress (GLC_ERR_TIMEOUT if a bounded wait of it gave up); *compressed_size_bytes
 * (may be NULL) receives the sum of the columns' reported sizes. */
GLC_API glc_status glc_batch_sync(glc_ctx* ctx, glc_batch* batch, glc_stream stream, int64_t* compressed_size_bytes);

GLC_API glc_status glc_batch_free(glc_batch* batch);

/* ---- allocation-free range decode (no counterpart in the reference) --------------------- */

/* Largest output, in bytes, of one glc_decompress_range_noalloc call:
 * 1,048,576 int32/uint32 values or 524,288 int64/uint64 values. */
#define GLC_NOALLOC_MAX_OUTPUT_BYTES (4u << 20)

/* Decode the values of positions [first, first + count) of `col` into host memory `host_out`
 * without allocating anything: no context is created and no cudaMalloc, cudaFree or pool
 * allocation happens.  It is meant for callers that cannot allocate device memory while they
 * run -- request handlers working under a fixed device-memory budget, or code that must not block
 * on the allocator or trigger its device-wide synchronisation.  glc_decompress_range with
 * GLC_HOST_OUT gives the same values but takes a device staging buffer on every call.
 *
 * The decode kernel's scratch (its work counter and error word) and the device staging of the
 * values live in one static device array of GLC_NOALLOC_MAX_OUTPUT_BYTES + 272 bytes, which
 * every GPU that loads this library holds until the process exits.
 *  - count * element size above GLC_NOALLOC_MAX_OUTPUT_BYTES is rejected (GLC_ERR_INVALID_ARG);
 *    decode larger ranges in several calls.
 *  - The first call on a device looks up the array's device address (cudaGetSymbolAddress);
 *    make that first call before any stream capture.
 *  - All calls share the array: calls that overlap on the GPU race, so serialise them (one
 *    stream, or one call at a time).  Each call clears the counter and error word it needs.
 *  - The column must hold its packed bitstream (GLC_ERR_UNSUPPORTED otherwise).
 *  - stream NULL = the stream of the context that made the column.  Returns after the values
 *    are in host_out; GLC_ERR_TIMEOUT if a bounded device-side wait gave up. */
GLC_API glc_status glc_decompress_range_noalloc(const glc_column* col, int64_t first, int64_t count,
                                                void* host_out, glc_stream stream);

/* ---- launch-shape tuning (no counterpart in the reference, whose launch shapes are
 * compile-time constants, core/CudaUtils.cuh:16-21) ---------------------------------------- */

typedef struct glc_tune_entry {
  int32_t decode_stages;  /* TMA ring depth of the decode kernel: 2, 3 or 4 */
  int32_t decode_unroll;  /* unroll depth of the decode's full-tile loop: 1, 2 or 4 */
  int32_t ra_shape;       /* random-access shape 0..4: (lookups per thread, CTAs per SM) =
                             (4,1), (4,5), (2,8), (8,2), (2,6) */
  int32_t measured;       /* 1 when chosen by glc_autotune, 0 for the built-in default */
  int32_t decode_cap_words; /* largest tile staged in shared memory, in 32-bit words: 0 = 6160
                             (48-bit fields), up to 8208 (a whole tile of 64-bit fields) */
  int32_t decode_warps;   /* consumer warps per CTA of the packed decode (the threads that share a
                             4096-value tile): 4 or 8 (0 = 8) */
  float decode_gbs;       /* decoded GB/s of the chosen shape on the tuning column */
  float ra_glookups;      /* G lookups/s of the chosen random-access shape */
  int32_t partition_len;  /* fixed partition length (1024, 2048, 4096) whose column decoded fastest;
                             glc_batch_compress prefers it between lengths of equal size (0 = none) */
  int32_t reserved;       /* 0 */
} glc_tune_entry;

enum { GLC_TUNE_FORCE = 1 };

/* Time every candidate decode shape (ring depth x unroll depth x consumer warps x stage capacity)
 * and random-access shape on this context's device, per element type, widest-field bucket (<= 8,
 * 16, 24, 32, 48, 64 bits) and residual source (packed, pre-unpacked), each on a synthetic
 * fixed-partitioned column of 48M values with fields of that width, and the partition length
 * (1024, 2048, 4096) whose column decodes fastest; keep the fastest in the context (a few seconds).  With
 * cache_path, results already stored there for this device (name, SM count, compute capability)
 * are loaded instead (unless GLC_TUNE_FORCE), and new results are written there.  A context also
 * loads the file named by the GLC_TUNE_CACHE environment variable when it is created. */
GLC_API glc_status glc_autotune(glc_ctx* ctx, const char* cache_path, int32_t flags);

/* The shapes used for columns of `dtype` whose widest field has `field_bits` bits. */
GLC_API glc_status glc_tune_get(const glc_ctx* ctx, glc_dtype dtype, int32_t field_bits, int32_t preunpacked,
                                glc_tune_entry* out);
GLC_API glc_status glc_tune_set(glc_ctx* ctx, glc_dtype dtype, int32_t field_bits, int32_t preunpacked,
                                const glc_tune_entry* entry);

/* ---- serving: resident columns and continuously batched requests (no counterpart in the
 * reference, whose every call is a blocking host round trip) ------------------------------ */

typedef struct glc_server glc_server;

typedef enum { GLC_REQ_LOOKUP = 0, GLC_REQ_RANGE = 1 } glc_request_kind;

/* One request against a resident column.  Inputs and outputs are device memory of the server's
 * device and must stay valid until the request's completion is reported.
 *  LOOKUP: out[k] = value at positions[k] for k < count (0 outside the column), as
 *          glc_random_access.
 *  RANGE:  out[k] = value at first + k for k < count, as glc_decompress_range; [first,
 *          first + count) must lie inside the column.  When (out - first * element size) is
 *          16-byte aligned the values are written in place, otherwise through the server's
 *          staging and one device copy per piece. */
typedef struct glc_request {
  int32_t kind;              /* glc_request_kind */
  int32_t column;            /* id from glc_server_admit */
  int64_t first;             /* RANGE: first position */
  int64_t count;             /* LOOKUP: positions; RANGE: values (>= 1) */
  const int32_t* positions;  /* LOOKUP: device array of count positions */
  void* out;                 /* device output of count values */
  int64_t tag;               /* caller's identifier, returned in the completion */
  int64_t not_before_ns;     /* arrival time on glc_server_now_ns()'s clock; the request is not
                                scheduled earlier and its latency counts from then.  0 = now. */
} glc_request;

typedef struct glc_completion {
  int64_t tag;
  int32_t status;      /* GLC_OK, or GLC_ERR_TIMEOUT / GLC_ERR_CUDA from its launches */
  int32_t launches;    /* shared launches that carried a piece of the request */
  int64_t arrival_ns;  /* max(not_before_ns, submission time) */
  int64_t done_ns;     /* when the server saw the request's last launch complete */
} glc_completion;

typedef struct glc_server_config {
  uint64_t budget_bytes;     /* device bytes the resident columns may hold (> 0) */
  int32_t slots;             /* shared launches in flight at once (0 = 4, at most 16) */
  int32_t max_requests;      /* lookup requests per launch (0 = 4096) */
  int64_t max_lookups;       /* positions per launch (0 = 4,194,304); one larger request runs alone */
  int64_t max_range_values;  /* range values per launch (0 = 16,777,216); longer ranges are split
                                into pieces so that they cannot hold back small requests */
  int32_t flags;             /* GLC_SERVER_RESERVE: reserve budget_bytes of device memory for
                                glc_server_admit_blob at creation */
  int32_t reserved;          /* 0 */
} glc_server_config;

enum { GLC_SERVER_RESERVE = 1 };

typedef struct glc_server_stats {
  uint64_t resident_bytes;   /* device bytes of admitted columns not yet freed */
  int32_t resident_columns;
  int32_t in_flight;         /* launches on the GPU now */
  int64_t launches, submitted, completed, lookups, range_values, evictions, admissions_refused;
} glc_server_stats;

/* A server on ctx's device: a worker thread takes submitted requests once they have arrived and
 * packs every request that is waiting into the next free launch slot (one lookup launch over all
 * of the slot's lookup requests and one persistent decode launch over all of its range pieces,
 * whatever their columns and element types), while up to `slots` launches run on the GPU. */
GLC_API glc_status glc_server_create(glc_ctx* ctx, const glc_server_config* config, glc_server** out);

/* Waits for every submitted request, stops the worker and frees every resident column. */
GLC_API glc_status glc_server_destroy(glc_server* server);

/* Make `col` resident and give it an id; the server takes ownership on success.  When the budget
 * would be exceeded, idle columns are evicted least recently used first; if that cannot make room
 * the call fails with GLC_ERR_BUDGET, evicts nothing and the caller keeps the column.  The column
 * must hold its packed bitstream (GLC_ERR_UNSUPPORTED otherwise), and its device data must be
 * complete: synchronise the stream that produced it first (calls with host buffers, and
 * glc_server_admit_blob, return with their stream synchronised). */
GLC_API glc_status glc_server_admit(glc_server* server, glc_column* col, int32_t* id);

/* Admit a serialized column (host or device memory; the same checks as glc_deserialize).  The blob
 * itself is copied once into the server's stream-ordered pool and read in place there, as
 * glc_attach_blob reads it (no deserialize; the caller may free its blob afterwards), so neither
 * this admission nor the column's later eviction calls cudaMalloc or cudaFree, which would stall
 * the launches in flight; with GLC_SERVER_RESERVE the pool holds budget_bytes from creation on. */
GLC_API glc_status glc_server_admit_blob(glc_server* server, glc_dtype dtype, const void* blob, uint64_t size,
                                         int flags, int32_t* id, glc_stream stream);

/* Remove a column: no new requests are accepted for it and its memory is freed once its
 * submitted requests have completed. */
GLC_API glc_status glc_server_evict(glc_server* server, int32_t id);

/* Queue requests (thread-safe).  Every request is checked first; if one is invalid (unknown or
 * evicted column, count < 1, range outside the column, null pointer) none is queued and the call
 * returns GLC_ERR_INVALID_ARG. */
GLC_API glc_status glc_server_submit(glc_server* server, const glc_request* requests, int32_t count);

/* Take up to `max` completion records (in completion order); *got receives how many. */
GLC_API glc_status glc_server_poll(glc_server* server, glc_completion* out, int32_t max, int32_t* got);

/* Wait until every submitted request has completed; GLC_ERR_TIMEOUT after timeout_ms (< 0 = no
 * limit). */
GLC_API glc_status glc_server_drain(glc_server* server, int64_t timeout_ms);

GLC_API glc_status glc_server_get_stats(glc_server* server, glc_server_stats* stats);

/* Ids of the columns that accept requests (admitted, not evicted), ascending; *got receives how
 * many were written (at most max). */
GLC_API glc_status glc_server_columns(glc_server* server, int32_t* ids, int32_t max, int32_t* got);

/* The server's clock (CLOCK_MONOTONIC, nanoseconds). */
GLC_API int64_t glc_server_now_ns(void);

#ifdef __cplusplus
}
#endif
#endif /* GLC_H_ */
