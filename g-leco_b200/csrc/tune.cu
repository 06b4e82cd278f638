// tune.cu -- measured choice of launch shapes per element type and field width.
//
// The reference fixes its launch shapes at compile time (core/CudaUtils.cuh:16-21).  Here each
// context holds a table, indexed by element type, widest-field bucket (<= 8, 16, 24, 32, 48, 64
// bits) and residual source (packed / pre-unpacked), of
//   - the decode kernel's TMA ring depth (2, 3, 4) and the unroll depth of its full-tile loop
//     (1, 2, 4): the values each CTA keeps in flight per tile; for fields wider than 32 bits also
//     the largest tile staged in shared memory (6160 words, or a whole tile of 64-bit fields at
//     the cost of fewer CTAs per SM; larger tiles are read from global memory);
//   - the consumer warps per CTA of the packed decode (4 or 8: the threads that share a tile);
//   - the random-access launch shape (lookups per thread x CTAs per SM, five candidates);
//   - the fixed partition length (1024, 2048, 4096) whose column decodes fastest; the batched
//     compress prefers it when two lengths give the same size (the length is otherwise chosen per
//     column by the exact compressed size).
// glc_autotune times every candidate on a synthetic fixed-partitioned column whose fields have the
// bucket's width (48M values, larger than L2) and keeps the fastest; the table can be written to
// and read from a text file keyed by the device (name, SM count, compute capability).
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <string>

#include "glc_internal.h"

using namespace glc;

namespace {

constexpr int kTuneVersion = 3;
constexpr int64_t kTuneValues = 48ll << 20;
constexpr int64_t kTuneLookups = 16ll << 20;
constexpr int kNoiseBits[kTuneBuckets] = {5, 13, 21, 29, 45, 59};  // fields of 6..60 bits

__device__ __forceinline__ uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

// v[i] = base + slope * i + noise, noise uniform over `noise_bits` bits.
template <typename T>
__global__ void fill_line_noise(T* v, int64_t n, int noise_bits, uint64_t seed) {
  const bool wide = sizeof(T) == 8;
  const uint64_t base = wide ? (1ull << 40) : 1000ull, slope = wide ? 1000ull : 3ull;
  const uint64_t mask = (1ull << noise_bits) - 1;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (T)(base + slope * (uint64_t)i + (mix64((uint64_t)i ^ seed) & mask));
}

__global__ void fill_positions(int32_t* pos, int64_t q, int64_t n, uint64_t seed) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < q; i += (int64_t)gridDim.x * blockDim.x)
    pos[i] = (int32_t)(mix64((uint64_t)i * 0x9e3779b97f4a7c15ull + seed) % (uint64_t)n);
}

std::string device_key(const glc_ctx* ctx) {
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, ctx->device) != cudaSuccess) return "unknown";
  std::string name = p.name;
  for (char& ch : name)
    if (ch == ' ') ch = '_';
  char buf[256];
  snprintf(buf, sizeof buf, "glc-tune %d %d %d.%d %s", kTuneVersion, p.multiProcessorCount, p.major, p.minor,
           name.c_str());
  return buf;
}

// Written to a private temporary file and renamed over `path`, so processes tuning at the same
// time (one per GPU) never read a half-written table.
bool tune_save(const glc_ctx* ctx, const char* path) {
  const std::string tmp = std::string(path) + ".tmp." + std::to_string((long long)getpid());
  FILE* f = fopen(tmp.c_str(), "w");
  if (!f) return false;
  fprintf(f, "%s\n", device_key(ctx).c_str());
  for (int d = 0; d < 4; d++)
    for (int b = 0; b < kTuneBuckets; b++)
      for (int p = 0; p < 2; p++) {
        const TuneEntry& t = ctx->tune[d][b][p];
        fprintf(f, "%d %d %d %d %d %d %d %d %d %.3f %.4f\n", d, b, p, t.decode_stages, t.decode_unroll, t.ra_shape,
                t.decode_cap_words, t.decode_warps, t.partition_len, t.decode_gbs, t.ra_glookups);
      }
  if (fclose(f) != 0) {
    remove(tmp.c_str());
    return false;
  }
  if (rename(tmp.c_str(), path) != 0) {
    remove(tmp.c_str());
    return false;
  }
  return true;
}

// Mean device time of `reps` launches after two warm-up launches, in milliseconds (< 0: failure).
template <typename F>
float time_launches(F launch, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1, int reps = 5) {
  for (int i = 0; i < 2; i++)
    if (launch() != cudaSuccess) return -1.f;
  if (cudaEventRecord(e0, s) != cudaSuccess) return -1.f;
  for (int i = 0; i < reps; i++)
    if (launch() != cudaSuccess) return -1.f;
  if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) return -1.f;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) return -1.f;
  return ms / reps;
}

glc_status tfail(glc_ctx* ctx, glc_status st, const std::string& msg) {
  ctx->err = msg;
  return st;
}

}  // namespace

// Built-in shapes for contexts that never tune: the choices glc_autotune made on a B200 (148 SMs),
// rounded to one rule per element size -- 4-byte outputs: ring depth 3, unroll 2; 8-byte outputs:
// depth 2, unroll 4 on packed fields (2 on pre-unpacked residuals), a whole tile staged for 64-bit
// fields; random access: shape 4 up to 32-bit fields, 0 at 48, 3 at 64, 3 for pre-unpacked.
void glc::tune_defaults(glc_ctx* ctx) {
  for (int d = 0; d < 4; d++)
    for (int b = 0; b < kTuneBuckets; b++)
      for (int p = 0; p < 2; p++) {
        TuneEntry& t = ctx->tune[d][b][p];
        const bool wide_type = d == GLC_I64 || d == GLC_U64;
        t.decode_stages = wide_type ? 2 : 3;
        t.decode_unroll = (wide_type && !p) ? 4 : 2;
        t.ra_shape = p ? 3 : (b <= 3 ? 4 : (b == 4 ? 0 : 3));
        t.measured = 0;
        t.decode_cap_words = (wide_type && !p && b == kTuneBuckets - 1) ? kStageCapWordsMax : 0;
        t.decode_warps = 0;
        t.partition_len = 0;
        t.reserved = 0;
        t.decode_gbs = 0.f;
        t.ra_glookups = 0.f;
      }
}

bool glc::tune_load(glc_ctx* ctx, const char* path) {
  FILE* f = fopen(path, "r");
  if (!f) return false;
  char line[512];
  bool ok = fgets(line, sizeof line, f) != nullptr;
  if (ok) {
    line[strcspn(line, "\n")] = 0;
    ok = device_key(ctx) == line;
  }
  TuneEntry tab[4][kTuneBuckets][2];
  int seen = 0;
  while (ok && fgets(line, sizeof line, f)) {
    int d, b, p, st, un, ra, cap, wp, pl;
    float gbs, gl;
    if (sscanf(line, "%d %d %d %d %d %d %d %d %d %f %f", &d, &b, &p, &st, &un, &ra, &cap, &wp, &pl, &gbs, &gl) != 11) {
      ok = false;
      break;
    }
    if (d < 0 || d > 3 || b < 0 || b >= kTuneBuckets || p < 0 || p > 1 || st < 2 || st > 4 ||
        (un != 1 && un != 2 && un != 4) || ra < 0 || ra > 4 || cap < 0 || cap > kStageCapWordsMax ||
        (wp != 0 && wp != 4 && wp != 8) || (pl != 0 && pl != 1024 && pl != 2048 && pl != 4096)) { ok = false; break; }
    tab[d][b][p] = TuneEntry{st, un, ra, 1, cap, wp, gbs, gl, pl, 0};
    seen++;
  }
  fclose(f);
  if (!ok || seen != 4 * kTuneBuckets * 2) return false;
  std::memcpy(ctx->tune, tab, sizeof tab);
  return true;
}

extern "C" {

glc_status glc_tune_get(const glc_ctx* ctx, glc_dtype dtype, int32_t field_bits, int32_t preunpacked,
                        glc_tune_entry* out) {
  if (!ctx || !out || (int)dtype < 0 || (int)dtype > 3 || field_bits < 0 || field_bits > 64) return GLC_ERR_INVALID_ARG;
  const TuneEntry& t = tune_entry(ctx, dtype, field_bits, preunpacked);
  *out = glc_tune_entry{t.decode_stages, t.decode_unroll, t.ra_shape, t.measured, t.decode_cap_words,
                        t.decode_warps, t.decode_gbs, t.ra_glookups, t.partition_len, 0};
  return GLC_OK;
}

glc_status glc_tune_set(glc_ctx* ctx, glc_dtype dtype, int32_t field_bits, int32_t preunpacked,
                        const glc_tune_entry* e) {
  if (!ctx || !e || (int)dtype < 0 || (int)dtype > 3 || field_bits < 0 || field_bits > 64) return GLC_ERR_INVALID_ARG;
  if (e->decode_stages < 2 || e->decode_stages > 4 || (e->decode_unroll != 1 && e->decode_unroll != 2 &&
      e->decode_unroll != 4) || e->ra_shape < 0 || e->ra_shape > 4 || e->decode_cap_words < 0 ||
      e->decode_cap_words > kStageCapWordsMax || (e->decode_warps != 0 && e->decode_warps != 4 &&
      e->decode_warps != 8) || (e->partition_len != 0 && e->partition_len != 1024 && e->partition_len != 2048 &&
      e->partition_len != 4096))
    return tfail(ctx, GLC_ERR_INVALID_ARG, "tune entry out of range");
  ctx->tune[(int)dtype][tune_bucket(field_bits)][preunpacked ? 1 : 0] =
      TuneEntry{e->decode_stages, e->decode_unroll, e->ra_shape, e->measured, e->decode_cap_words, e->decode_warps,
                e->decode_gbs, e->ra_glookups, e->partition_len, 0};
  return GLC_OK;
}

glc_status glc_autotune(glc_ctx* ctx, const char* cache_path, int32_t flags) {
  if (!ctx || (flags & ~GLC_TUNE_FORCE) != 0) return GLC_ERR_INVALID_ARG;
  if (cache_path && !(flags & GLC_TUNE_FORCE) && tune_load(ctx, cache_path)) return GLC_OK;
  glc::DeviceScope device_scope(ctx->device);
  cudaStream_t s = ctx->own_stream;
  void* vals = nullptr;
  void* out = nullptr;
  int32_t* pos = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  TuneEntry tab[4][kTuneBuckets][2];
  std::memcpy(tab, ctx->tune, sizeof tab);
  glc_status st = GLC_OK;
  cudaError_t e;
  if ((e = cudaMalloc(&vals, 8 * kTuneValues)) != cudaSuccess || (e = cudaMalloc(&out, 8 * kTuneValues + 16)) != cudaSuccess ||
      (e = cudaMalloc((void**)&pos, 4 * kTuneLookups)) != cudaSuccess || (e = cudaEventCreate(&e0)) != cudaSuccess ||
      (e = cudaEventCreate(&e1)) != cudaSuccess) {
    st = tfail(ctx, GLC_ERR_OOM, std::string("autotune: ") + cudaGetErrorString(e));
  }
  if (st == GLC_OK) fill_positions<<<ctx->num_sms * 8, 256, 0, s>>>(pos, kTuneLookups, kTuneValues, 7);
  for (int d = 0; d < 4 && st == GLC_OK; d++) {
    const glc_dtype dt = (glc_dtype)d;
    const int nb = dtype_size(dt) == 8 ? kTuneBuckets : 4;  // 32-bit fields at most for 4-byte types
    for (int b = 0; b < nb && st == GLC_OK; b++) {
      const int grid = ctx->num_sms * 8;
      switch (dt) {
        case GLC_I32: fill_line_noise<<<grid, 256, 0, s>>>((int32_t*)vals, kTuneValues, kNoiseBits[b], 11 + b); break;
        case GLC_U32: fill_line_noise<<<grid, 256, 0, s>>>((uint32_t*)vals, kTuneValues, kNoiseBits[b], 11 + b); break;
        case GLC_I64: fill_line_noise<<<grid, 256, 0, s>>>((int64_t*)vals, kTuneValues, kNoiseBits[b], 11 + b); break;
        default: fill_line_noise<<<grid, 256, 0, s>>>((uint64_t*)vals, kTuneValues, kNoiseBits[b], 11 + b); break;
      }
      glc_column* col = nullptr;
      st = glc_compress(ctx, dt, vals, kTuneValues, 0, GLC_PART_FIXED, 4096, &col, nullptr, s);
      if (st != GLC_OK) break;
      const int bucket = tune_bucket(col->max_bits);
      for (int plain = 0; plain < 2 && st == GLC_OK; plain++) {
        if (plain && (st = glc_preunpack(ctx, col, 0, s)) != GLC_OK) break;
        TuneEntry best = tab[d][bucket][plain];
        float best_ms = 1e30f;
        for (int cap : {0, kStageCapWordsMax}) {
          if (cap && (plain || col->max_bits <= 32)) continue;  // only tiles of wide fields exceed the default
          for (int warps : {8, 4}) {
            if (plain && warps != 8) continue;  // the pre-unpacked decode keeps 8 warps
            for (int stages = 2; stages <= 4; stages++)
              for (int unroll : {1, 2, 4}) {
                if (plain && unroll != 2) continue;  // the pre-unpacked decode has no unroll choice
                const float ms = time_launches([&] {
                  return launch_decode_shape(ctx, col, plain, 0, 0, kTuneValues, out, stages, unroll, cap, warps, s);
                }, s, e0, e1);
                if (ms < 0.f) { st = tfail(ctx, GLC_ERR_CUDA, "autotune: decode launch failed"); break; }
                if (ms < best_ms) {
                  best_ms = ms;
                  best.decode_stages = stages;
                  best.decode_unroll = unroll;
                  best.decode_cap_words = cap;
                  best.decode_warps = warps;
                  best.decode_gbs = (float)(dtype_size(dt) * (double)kTuneValues / (ms * 1e6));
                }
              }
          }
        }
        float best_ra = 1e30f;
        for (int shape = 0; shape < 5 && st == GLC_OK; shape++) {
          const float ms = time_launches([&] {
            return launch_random_access_shape(ctx, col, plain, pos, kTuneLookups, out, col->fixed_len, shape, s);
          }, s, e0, e1);
          if (ms < 0.f) { st = tfail(ctx, GLC_ERR_CUDA, "autotune: random-access launch failed"); break; }
          if (ms < best_ra) {
            best_ra = ms;
            best.ra_shape = shape;
            best.ra_glookups = (float)(kTuneLookups / (ms * 1e6));
          }
        }
        best.measured = 1;
        tab[d][bucket][plain] = best;
      }
      glc_column_free(col);
      // partition length: the same column at 1024 and 2048 values per partition, decoded with the
      // packed shape just chosen; the fastest of the three lengths is kept
      if (st == GLC_OK) {
        TuneEntry& tp = tab[d][bucket][0];
        int best_len = 4096;
        float best_len_ms = (float)(dtype_size(dt) * (double)kTuneValues / (tp.decode_gbs * 1e6));
        for (int L : {2048, 1024}) {
          glc_column* cl = nullptr;
          if ((st = glc_compress(ctx, dt, vals, kTuneValues, 0, GLC_PART_FIXED, L, &cl, nullptr, s)) != GLC_OK) break;
          const float ms = time_launches([&] {
            return launch_decode_shape(ctx, cl, 0, 0, 0, kTuneValues, out, tp.decode_stages, tp.decode_unroll,
                                       tp.decode_cap_words, tp.decode_warps, s);
          }, s, e0, e1);
          glc_column_free(cl);
          if (ms < 0.f) { st = tfail(ctx, GLC_ERR_CUDA, "autotune: decode launch failed"); break; }
          if (ms < best_len_ms) { best_len_ms = ms; best_len = L; }
        }
        tp.partition_len = best_len;
        tab[d][bucket][1].partition_len = best_len;
      }
      if (st == GLC_OK) st = glc_sync(ctx, s);  // a device-side wait that gave up fails the tuning
    }
    if (st == GLC_OK && nb < kTuneBuckets)  // wider buckets of 4-byte types reuse the 32-bit choice
      for (int b = nb; b < kTuneBuckets; b++)
        for (int p = 0; p < 2; p++) tab[d][b][p] = tab[d][nb - 1][p];
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(vals);
  cudaFree(out);
  cudaFree(pos);
  if (st != GLC_OK) return st;
  std::memcpy(ctx->tune, tab, sizeof tab);
  if (cache_path && !tune_save(ctx, cache_path)) return tfail(ctx, GLC_ERR_INVALID_ARG, "autotune: cannot write the cache file");
  return GLC_OK;
}

}  // extern "C"
