// decode.cu -- persistent work-stealing full / range decode with a TMA producer warp.
//
// Replaces the reference's full-decode kernels, which all do the same arithmetic with
// different work layouts: decompressFullFile_BitPacked / _PreUnpacked (grid-stride, a binary
// search per value, decompression/FullDecompressionKernels.cuh:47-288), _OnTheFly_Optimized_V2
// (one CTA per partition, :292-378), decompressFullFileFix (:382-476), and the work-stealing
// kernels (atomic batches of partitions, WorkStealingDecompressionKernels.cuh:331-619).  The
// pre-unpack kernel (decompression/UnpackKernel.cuh:31-98) is the same walk with a residual
// epilogue, so it is a mode of this kernel too.
//
// Work unit: a TILE of 4096 consecutive output values, independent of partition sizes, so every
// unit writes the same number of bytes.  A table built once per column gives each tile's first
// bit and first/last partition; no per-value search is needed.
//
// CTA = 1 producer warp + 8 consumer warps, persistent (grid = resident CTAs on all SMs):
//   producer (one lane): claims the next tile from a global counter (work stealing), waits until
//     the consumers released the ring stage, then issues 1-D TMA bulk copies (cp.async.bulk,
//     non-multicast) of the tile's packed words (or pre-unpacked residuals) AND of the tile's
//     32-byte partition descriptors into that stage, completing on the stage's "full" mbarrier.
//     Two stages keep up to two tiles in flight per CTA (2-4 measured; two leave room for more
//     resident CTAs).
//   consumers: wait on "full", decode the tile from shared memory and write 16-byte vector
//     stores, then arrive on the stage's "empty" mbarrier.  The common case (a vector whose
//     values all lie in one partition, fields <= 32 bits) uses 32-bit bit arithmetic relative to
//     the stage, one funnel shift per field, a two-shift sign extension and the FP64 prediction
//     fma(theta1, i, theta0) -> round -> saturating convert, exactly as the reference computes it.
// No CTA-wide barrier runs inside the loop.  A tile whose packed words exceed a stage is decoded
// straight from global memory (rare: fields averaging more than 48 bits over a tile).
// Every mbarrier wait is bounded by wall time; on expiry the kernel records an error code and
// returns after a second bounded wait for its own copies.
#include <atomic>
#include <vector>
#include <climits>
#include <cstdlib>
#include <type_traits>
#include "glc_internal.h"
#include "glc_tma.cuh"

namespace glc {

constexpr int kDefaultStages = 2;  // ring depth; measured best on the 200M uint64 column (2-4 swept)
constexpr int kTileDescs = 40;  // descriptors staged per tile (a 4096-value tile of >= 128-value partitions spans <= 34)
constexpr int kConsumerWarps = 8;
constexpr int kConsumers = kConsumerWarps * 32;
constexpr int kPCThreads = kConsumers + 32;
constexpr int kStageCapWords = 6144 + 16;  // 48 bits per value on average over a tile (1040-6160 swept)

struct DecodeArgs {
  const PartDesc* desc;
  const int32_t* starts;
  const TileInfo* tiles;
  const uint32_t* words;
  const int64_t* plain;
  int64_t P, n;
  int64_t lo, hi;            // element range
  int64_t t_begin, t_end;    // tile range
  void* out_base;            // element e goes to out_base[e]
  int* counter;
  int* err;
  int stage_bytes;
  // >= 0: the consumers' FIRST wait for a stage gives up after this many non-blocking tests
  // (0: at once) -- a test hook that makes a bounded wait run out on a healthy copy; -1: normal
  int first_wait_tests;
};

struct StageInfo {
  int64_t tile;
  int64_t bit_lo;
  int32_t pf, pl;
  int32_t big;     // words read from global memory instead of the stage
  int32_t cached;  // descriptors are in the stage
};

__device__ __forceinline__ PartDesc load_desc_g(const PartDesc* d) {
  const double2 x = __ldg(reinterpret_cast<const double2*>(d));
  const longlong2 y = __ldg(reinterpret_cast<const longlong2*>(d) + 1);
  PartDesc r;
  r.theta0 = x.x;
  r.theta1 = x.y;
  r.bit_off = y.x;
  r.start = (int32_t)(y.y & 0xffffffffll);
  r.bits_type = (int32_t)(y.y >> 32);
  return r;
}

// Field of 0..64 bits at 32-bit bit position `pos` of a word array (shared or global).
__device__ __forceinline__ uint64_t field_at(const uint32_t* w, uint32_t pos, int bits) {
  const uint32_t wi = pos >> 5, sh = pos & 31;
  uint64_t f = (((uint64_t)w[wi + 1] << 32) | w[wi]) >> sh;
  if (bits + (int)sh > 64) f |= (uint64_t)w[wi + 2] << (64 - sh);
  return bits >= 64 ? f : (f & ((1ull << bits) - 1ull));
}

template <typename T> __device__ __forceinline__ T predict_x(double t0, double t1, double x) {
  return predict_from<T>(__fma_rn(t1, x, t0));
}

// Partition cursor of one consumer thread inside a tile.
struct Cursor {
  double t0, t1;
  uint32_t base;  // bit of value e (relative to the stage) = base + e * bits  (mod 2^32)
  int start, next, bits, type, idx;
  bool nonneg;    // theta0 >= 0 and theta1 >= 0: predictions at x >= 0 are never negative
  bool small;     // nonneg, and every prediction of the partition in this tile inside
                  // pred_fp64_safe's bounds: the prediction needs no conversion instruction
};

// SMALL: 4-byte outputs may take the conversion-free prediction (off in the batch kernel, whose
// one body serves every element type and would otherwise need more registers than its occupancy
// allows).
template <typename T, bool PLAIN, bool RESID, int kUnroll = 2, int CW = kConsumerWarps, bool SMALL = true>
__device__ __forceinline__ void decode_tile(const DecodeArgs& a, const StageInfo& si, const uint8_t* stage,
                                            const PartDesc* sdesc) {
  constexpr int kThreads = CW * 32;  // consumer threads of the CTA
  typedef typename std::conditional<RESID, int64_t, T>::type OutT;
  // values per thread-vector: 32 bytes for 4-byte outputs (two 16-byte stores; the per-vector
  // cursor and address work is then shared by 8 values), 16 bytes for 8-byte outputs
  constexpr int kVecBytes = sizeof(OutT) == 4 ? 32 : 16;
  constexpr int V = kVecBytes / (int)sizeof(OutT);
  OutT* out = reinterpret_cast<OutT*>(a.out_base);
  const int tid = threadIdx.x;
  const int64_t tile_e0 = si.tile * kDecodeTile;
  const int E0 = (int)(tile_e0 > a.lo ? tile_e0 : a.lo);
  const int E1 = (int)((tile_e0 + kDecodeTile < a.hi) ? tile_e0 + kDecodeTile : a.hi);
  const int Ea = (E0 / V) * V;
  const int nvec = (E1 - Ea + V - 1) / V;
  const int64_t w0 = (si.bit_lo >> 5) & ~3ll;
  const int64_t stage_bit0 = w0 * 32;
  const uint32_t* src = si.big ? a.words + w0 : reinterpret_cast<const uint32_t*>(stage);
  const int64_t* sp = reinterpret_cast<const int64_t*>(stage);
  const int pf = si.pf, np = si.pl - si.pf + 1;
  const bool cached = si.cached != 0;

  Cursor c;
  c.idx = -1;
  c.next = INT_MIN;
  c.start = 0;
  auto load = [&](int k) {
    const PartDesc d = cached ? sdesc[k] : load_desc_g(a.desc + pf + k);
    c.t0 = d.theta0;
    c.t1 = d.theta1;
    c.nonneg = d.theta0 >= 0.0 && d.theta1 >= 0.0;
    c.bits = d.bits_type & 0xff;
    c.type = d.bits_type >> 8;
    c.start = d.start;
    c.base = (uint32_t)(d.bit_off - stage_bit0) - (uint32_t)d.start * (uint32_t)c.bits;
    c.next = (k + 1 < np) ? (cached ? sdesc[k + 1].start : __ldg(a.starts + pf + k + 1)) : INT_MAX;
    c.idx = k;
    // 4-byte outputs (8 values per vector, so the conversions dominate): the partition's last index
    // in this tile; with theta0, theta1 >= 0 its prediction is the largest
    if (SMALL && sizeof(T) == 4) {
      const int hi = (c.next < E1 ? c.next : E1) - 1 - c.start;
      c.small = c.nonneg && pred_fp64_safe<T>(__fma_rn(c.t1, (double)(hi > 0 ? hi : 0), c.t0));
    } else {
      c.small = false;
    }
  };
  auto seek = [&](int e) {  // position the cursor on the partition holding value e
    int k;
    if (cached) {
      k = c.idx < 0 ? 0 : c.idx;
      while (k + 1 < np && sdesc[k + 1].start <= e) k++;
    } else {
      int lo = 0, hi = np - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(a.starts + pf + mid) <= e) lo = mid; else hi = mid - 1;
      }
      k = lo;
    }
    load(k);
  };
  auto one = [&](int e) -> OutT {  // any value, any width
    const int local = e - c.start;
    long long r;
    if (PLAIN) {
      r = sp[e - tile_e0];
    } else {
      const uint64_t f = c.bits > 0 ? field_at(src, c.base + (uint32_t)e * (uint32_t)c.bits, c.bits) : 0ull;
      r = (c.type == MODEL_DIRECT_COPY) ? (long long)f : sign_extend(f, c.bits);
    }
    if (RESID) return (OutT)r;
    if (c.type == MODEL_DIRECT_COPY) return (OutT)(T)r;
    return (OutT)apply_delta<T>(predict_x<T>(c.t0, c.t1, (double)local), r);
  };

  // Fast path for a vector whose values all lie in the cursor's partition: packed fields of at
  // most 32 bits, 32-bit positions relative to the stage, one funnel shift per field.
  auto fast_vec = [&](int e) {
    OutT vals[V];
    const double x0 = (double)(e - c.start);
    if (!PLAIN && c.bits <= 32 && c.type != MODEL_DIRECT_COPY) {
      // fields of the vector, sign-extended (zero-width fields read nothing)
      int32_t rr[V];
      if (c.bits == 0) {
#pragma unroll
        for (int u = 0; u < V; u++) rr[u] = 0;
      } else {
        const uint32_t pos = c.base + (uint32_t)e * (uint32_t)c.bits;
        const uint32_t shl = (uint32_t)(32 - c.bits) & 31u;
        const int b = c.bits;
        if (V % 4 == 0 && b <= 8) {
          // the 32-bit window at field u holds fields u .. u+3 whole (4b <= 32): one window per 4
#pragma unroll
          for (int g = 0; g < V; g += 4) {
            const uint32_t p = pos + (uint32_t)(g * b);
            const uint32_t wi = p >> 5;
            const uint32_t f = __funnelshift_r(src[wi], src[wi + 1], p & 31);
#pragma unroll
            for (int h = 0; h < 4; h++) rr[g + h] = (int32_t)(f << (uint32_t)(32 - (h + 1) * b)) >> shl;
          }
        } else if (V % 2 == 0 && b <= 16) {  // two fields per window (2b <= 32)
#pragma unroll
          for (int g = 0; g < V; g += 2) {
            const uint32_t p = pos + (uint32_t)(g * b);
            const uint32_t wi = p >> 5;
            const uint32_t f = __funnelshift_r(src[wi], src[wi + 1], p & 31);
            rr[g] = (int32_t)(f << shl) >> shl;
            rr[g + 1] = (int32_t)(f << (uint32_t)(32 - 2 * b)) >> shl;
          }
        } else {
#pragma unroll
          for (int u = 0; u < V; u++) {
            const uint32_t p = pos + (uint32_t)(u * c.bits);
            const uint32_t wi = p >> 5;
            const uint32_t f = __funnelshift_r(src[wi], src[wi + 1], p & 31);
            rr[u] = (int32_t)(f << shl) >> shl;
          }
        }
      }
      if (RESID) {
#pragma unroll
        for (int u = 0; u < V; u++) vals[u] = (OutT)rr[u];
      } else if (SMALL && sizeof(T) == 4 && c.small) {
        // theta0, theta1 >= 0 and predictions below 2^51 (and inside the type): round half away
        // by the constant bias, truncate by adding 2^52 rounded toward zero (trunc_small) and
        // read the integer from the sum's low bits -- no conversion instruction
        const double bias = __longlong_as_double(0x3FDFFFFFFFFFFFFFll);
#pragma unroll
        for (int u = 0; u < V; u++) {
          const double pr = __fma_rn(c.t1, u ? x0 + (double)u : x0, c.t0);
          const long long m = __double_as_longlong(__dadd_rz(__dadd_rn(pr, bias), 4503599627370496.0));
          const T pred = sizeof(T) == 8 ? (T)(m & 0xFFFFFFFFFFFFFll) : (T)(uint32_t)m;
          vals[u] = (OutT)apply_delta<T>(pred, (long long)rr[u]);
        }
      } else if (c.nonneg) {  // theta0, theta1 >= 0: every prediction is >= 0, one rounding bias
        const double bias = __longlong_as_double(0x3FDFFFFFFFFFFFFFll);
#pragma unroll
        for (int u = 0; u < V; u++) {
          const double pr = __fma_rn(c.t1, u ? x0 + (double)u : x0, c.t0);
          vals[u] = (OutT)apply_delta<T>(sat_cast<T>(__dadd_rn(pr, bias)), (long long)rr[u]);
        }
      } else {
#pragma unroll
        for (int u = 0; u < V; u++)
          vals[u] = (OutT)apply_delta<T>(predict_x<T>(c.t0, c.t1, u ? x0 + (double)u : x0), (long long)rr[u]);
      }
    } else {
#pragma unroll
      for (int u = 0; u < V; u++) vals[u] = one(e + u);
    }
#pragma unroll
    for (int h = 0; h < kVecBytes / 16; h++) {
      uint4 pk;
      memcpy(&pk, reinterpret_cast<const uint8_t*>(vals) + 16 * h, 16);
      *reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(out + e) + 16 * h) = pk;
    }
  };
  auto general_vec = [&](int e) {  // partition boundary inside the vector, or a partial tile
#pragma unroll
    for (int u = 0; u < V; u++) {
      const int ee = e + u;
      if (ee < E0 || ee >= E1) continue;
      if (c.idx < 0 || ee >= c.next) seek(ee);
      out[ee] = one(ee);
    }
  };

  if (E0 == tile_e0 && E1 - E0 == kDecodeTile) {  // full tile: every vector is in range
    constexpr int kIters = kDecodeTile / V / kThreads;
#pragma unroll kUnroll
    for (int it = 0; it < kIters; it++) {
      const int e = Ea + (it * kThreads + tid) * V;
      if (c.idx < 0 || e >= c.next) seek(e);
      if (e <= c.next - V) fast_vec(e); else general_vec(e);  // e + V - 1 < next, without overflow
    }
  } else {
    for (int j = tid; j < nvec; j += kThreads) {
      const int e = Ea + j * V;
      // e + V <= E1 and e + V - 1 < next, written so that they cannot overflow at n = 2^31 - 1
      if (e >= E0 && e <= E1 - V) {
        if (c.idx < 0 || e >= c.next) seek(e);
        if (e <= c.next - V) { fast_vec(e); continue; }
      }
      general_vec(e);
    }
  }
}

// CW consumer warps per CTA (8, or 4 for a tuned choice of the packed decode) + one producer warp.
// HOOK: the instantiation that honours DecodeArgs::first_wait_tests (the test hook); the others
// carry no trace of it.
template <typename T, bool PLAIN, bool RESID, int kStages, int kUnroll, int CW = kConsumerWarps, bool HOOK = false>
__global__ void __launch_bounds__(CW * 32 + 32) decode_kernel(DecodeArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(128) PartDesc s_desc[kStages][kTileDescs];
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages];
  __shared__ StageInfo s_info[kStages];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], CW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (warp == CW) {  // ---- producer ----
    if (lane != 0) return;
    for (int k = 0;; k++) {
      const int s = k % kStages;
      if (k >= kStages && !mbar_wait_bounded(&empty[s], (uint32_t)((k / kStages) - 1) & 1u)) {
        atomicExch(a.err, DEVERR_TIMEOUT);
        break;
      }
      StageInfo si;
      si.tile = a.t_begin + atomicAdd(a.counter, 1);
      if (si.tile >= a.t_end) {
        s_info[s] = si;
        mbar_arrive(&full[s]);  // no copy: completes the phase, consumers see the end
        break;
      }
      const TileInfo ti = a.tiles[si.tile];
      si.bit_lo = ti.bit_lo;
      si.pf = ti.p_first;
      si.pl = ti.p_last;
      const int np = si.pl - si.pf + 1;
      si.cached = np <= kTileDescs;
      const void* src;
      uint32_t bytes;
      if (PLAIN) {
        const int64_t e0 = si.tile * kDecodeTile;
        const int64_t e1 = (e0 + kDecodeTile < a.n) ? e0 + kDecodeTile : a.n;
        src = a.plain + e0;
        bytes = (uint32_t)((((e1 - e0) * 8) + 15) & ~15ll);
        si.big = 0;
      } else {
        const int64_t bh = a.tiles[si.tile + 1].bit_lo;
        const int64_t w0 = (ti.bit_lo >> 5) & ~3ll;
        const int64_t w1 = (((bh >> 5) + 3) + 3) & ~3ll;
        src = a.words + w0;
        bytes = (uint32_t)((w1 - w0) * 4);
        si.big = bytes > (uint32_t)a.stage_bytes;
      }
      s_info[s] = si;
      const uint32_t dbytes = si.cached ? (uint32_t)np * (uint32_t)sizeof(PartDesc) : 0u;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive_expect_tx(&full[s], (si.big ? 0u : bytes) + dbytes);
      if (!si.big) tma_bulk_load(smem + (size_t)s * a.stage_bytes, src, bytes, &full[s]);
      if (dbytes) tma_bulk_load(&s_desc[s][0], a.desc + si.pf, dbytes, &full[s]);
    }
    return;
  }

  // ---- consumers ----
  for (int k = 0;; k++) {
    const int s = k % kStages;
    const bool got = (HOOK && k == 0 && a.first_wait_tests >= 0)
                         ? mbar_test_n(&full[s], 0u, a.first_wait_tests)
                         : mbar_wait_bounded(&full[s], (uint32_t)(k / kStages) & 1u);
    if (!got) {
      if (lane == 0) atomicExch(a.err, DEVERR_TIMEOUT);
      mbar_wait_bounded(&full[s], (uint32_t)(k / kStages) & 1u);  // copies in flight land first
      break;
    }
    const StageInfo si = s_info[s];
    if (si.tile >= a.t_end) break;
    decode_tile<T, PLAIN, RESID, kUnroll, CW>(a, si, smem + (size_t)s * a.stage_bytes, &s_desc[s][0]);
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
}

// ---------------------------------------------------------------------------------------
// Batched decode: one persistent launch over a device work list spanning many columns of mixed
// element types.  A work item is one tile of one column, clipped to an element range, with its
// own output base, so the same launch serves full decodes of thousands of columns and range
// requests of different sizes.  The producer stages each item exactly like a single-column tile;
// consumers switch on the item's element type (uniform per tile) and reuse decode_tile.
// ---------------------------------------------------------------------------------------
// The work list is grouped by element type ([int32 items][int64][uint64][uint32]) and so is the
// grid: a CTA decodes items of one type for its whole life, from its group's own counter, so the
// hot loop is one type's (a per-item type switch doubles the registers and thrashes the
// instruction cache).  Groups follow one another in block order: as the CTAs of one type run
// out of items and exit, CTAs of the next type take their place.
template <typename T, int kStages>
__device__ __forceinline__ void batch_body(const BatchDecodeArgs& b, int g, uint8_t* smem,
                                           PartDesc (*s_desc)[kTileDescs], uint64_t* full, uint64_t* empty,
                                           StageInfo* s_info, BatchWork* s_work, BatchColumn* s_col) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t first = b.group_begin[g], last = b.group_begin[g + 1];
  if (warp == kConsumerWarps) {  // ---- producer ----
    if (lane != 0) return;
    for (int k = 0;; k++) {
      const int s = k % kStages;
      if (k >= kStages && !mbar_wait_bounded(&empty[s], (uint32_t)((k / kStages) - 1) & 1u)) {
        *(volatile int*)b.err = DEVERR_TIMEOUT;  // may be mapped host memory
        break;
      }
      const int64_t item = first + (int64_t)atomicAdd(b.counter + g, 1ull);
      StageInfo si;
      if (item >= last) {
        si.tile = -1;
        s_info[s] = si;
        mbar_arrive(&full[s]);
        break;
      }
      const BatchWork w = b.work[item];
      const BatchColumn col = b.cols[w.col];
      s_work[s] = w;  // the consumers read the item and its column from the stage, not from global memory
      s_col[s] = col;
      const TileInfo ti = col.tiles[w.tile];
      const int64_t bh = col.tiles[w.tile + 1].bit_lo;
      si.tile = w.tile;
      si.bit_lo = ti.bit_lo;
      si.pf = ti.p_first;
      si.pl = ti.p_last;
      const int np = si.pl - si.pf + 1;
      si.cached = np <= kTileDescs;
      const int64_t w0 = (ti.bit_lo >> 5) & ~3ll;
      const int64_t w1 = (((bh >> 5) + 3) + 3) & ~3ll;
      const uint32_t bytes = (uint32_t)((w1 - w0) * 4);
      si.big = bytes > (uint32_t)b.stage_bytes;
      s_info[s] = si;
      const uint32_t dbytes = si.cached ? (uint32_t)np * (uint32_t)sizeof(PartDesc) : 0u;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive_expect_tx(&full[s], (si.big ? 0u : bytes) + dbytes);
      if (!si.big) tma_bulk_load(smem + (size_t)s * b.stage_bytes, col.words + w0, bytes, &full[s]);
      if (dbytes) tma_bulk_load(&s_desc[s][0], col.desc + si.pf, dbytes, &full[s]);
    }
    return;
  }

  for (int k = 0;; k++) {  // ---- consumers ----
    const int s = k % kStages;
    if (!mbar_wait_bounded(&full[s], (uint32_t)(k / kStages) & 1u)) {
      if (lane == 0) *(volatile int*)b.err = DEVERR_TIMEOUT;
      mbar_wait_bounded(&full[s], (uint32_t)(k / kStages) & 1u);
      break;
    }
    const StageInfo si = s_info[s];
    if (si.tile < 0) break;
    const BatchWork w = s_work[s];
    const BatchColumn col = s_col[s];
    DecodeArgs a;
    a.desc = col.desc;
    a.starts = col.starts;
    a.tiles = col.tiles;
    a.words = col.words;
    a.plain = nullptr;
    a.P = 0;
    a.n = col.n;
    a.lo = w.lo;
    a.hi = w.hi;
    a.out_base = w.out_base;
    a.stage_bytes = b.stage_bytes;
    a.first_wait_tests = -1;
    decode_tile<T, false, false, 2, kConsumerWarps, false>(a, si, smem + (size_t)s * b.stage_bytes, &s_desc[s][0]);
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
}

template <int kStages>
__global__ void __launch_bounds__(kPCThreads) batch_decode_kernel(BatchDecodeArgs b) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(128) PartDesc s_desc[kStages][kTileDescs];
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages];
  __shared__ StageInfo s_info[kStages];
  __shared__ BatchWork s_work[kStages];
  __shared__ BatchColumn s_col[kStages];

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumerWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  int g = 0;
  while (g < 3 && (int)blockIdx.x >= b.grid_begin[g + 1]) g++;
  switch (g) {  // the group's element type: GLC_I32, GLC_I64, GLC_U64, GLC_U32
    case 0: batch_body<int32_t, kStages>(b, g, smem, s_desc, full, empty, s_info, s_work, s_col); break;
    case 1: batch_body<int64_t, kStages>(b, g, smem, s_desc, full, empty, s_info, s_work, s_col); break;
    case 2: batch_body<uint64_t, kStages>(b, g, smem, s_desc, full, empty, s_info, s_work, s_col); break;
    default: batch_body<uint32_t, kStages>(b, g, smem, s_desc, full, empty, s_info, s_work, s_col); break;
  }
}

// Stable grouping of a work list by element type; group_begin[d] .. group_begin[d + 1] are the
// items of type d afterwards.
void group_work_by_type(std::vector<BatchWork>& w, const std::vector<int32_t>& col_dtype, int64_t group_begin[5]) {
  int64_t cnt[4] = {0, 0, 0, 0};
  for (const BatchWork& x : w) cnt[col_dtype[x.col] & 3]++;
  group_begin[0] = 0;
  for (int d = 0; d < 4; d++) group_begin[d + 1] = group_begin[d] + cnt[d];
  bool sorted = true;
  for (size_t i = 1; i < w.size() && sorted; i++) sorted = (col_dtype[w[i - 1].col] & 3) <= (col_dtype[w[i].col] & 3);
  if (sorted) return;
  std::vector<BatchWork> out(w.size());
  int64_t pos[4] = {group_begin[0], group_begin[1], group_begin[2], group_begin[3]};
  for (const BatchWork& x : w) out[(size_t)pos[col_dtype[x.col] & 3]++] = x;
  w.swap(out);
}

// Range pieces -> per-tile work items, on the device: item t (in the pieces' order, grouped by
// element type) is tile (t - tile_base[p]) of piece p, the last piece with tile_base[p] <= t.  A
// piece is one BatchWork whose `tile` is its first tile; the host builds one per range piece
// instead of one per tile.
__global__ void expand_pieces_kernel(const BatchWork* __restrict__ pieces, const int64_t* __restrict__ tile_base,
                                     int npieces, int64_t ntiles, BatchWork* __restrict__ work) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = npieces - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tile_base[mid] <= t) lo = mid; else hi = mid - 1;
    }
    BatchWork w = pieces[lo];
    w.tile += (int32_t)(t - tile_base[lo]);
    work[t] = w;
  }
}

cudaError_t launch_expand_pieces(const BatchWork* pieces, const int64_t* tile_base, int npieces, int64_t ntiles,
                                 BatchWork* work, int num_sms, cudaStream_t s) {
  if (ntiles <= 0 || npieces <= 0) return cudaSuccess;
  int64_t grid = (ntiles + 255) / 256;
  if (grid > 4ll * num_sms) grid = 4ll * num_sms;
  expand_pieces_kernel<<<(unsigned)grid, 256, 0, s>>>(pieces, tile_base, npieces, ntiles, work);
  return cudaGetLastError();
}

// Launch configuration of the batched decode, per device: the shared-memory attribute is raised
// once to the largest stage ring, and the resident CTAs per SM are kept per stage size (these
// queries cost microseconds, and the serving loop launches tens of thousands of times a second).
constexpr int kMaxDevices = 16;
static std::atomic<int> g_batch_attr[kMaxDevices][2];  // [device][ring depth 2 or 3]
static std::atomic<int> g_batch_per_sm[kMaxDevices][2][kStageCapWords / 4 + 1];

// Ring depth of the batched decode: 3 (measured on 4096 mixed int32/int64/uint64 columns: 0.548-0.550
// ms per launch with 3 stages, 0.572 ms with 2), or GLC_BATCH_STAGES (2 or 3) for sweeps.
constexpr int kBatchStages = 3;
static int batch_stages() {
  static const int st = [] {
    const char* v = getenv("GLC_BATCH_STAGES");
    const int x = (v && *v) ? atoi(v) : kBatchStages;
    return (x == 2 || x == 3) ? x : kBatchStages;
  }();
  return st;
}

static cudaError_t batch_decode_go(const BatchDecodeArgs& b, int num_sms, bool zero, cudaStream_t s) {
  if (b.nwork <= 0) return cudaSuccess;
  const int stages = batch_stages();
  const int si = stages - 2;
  void (*kern)(BatchDecodeArgs) = stages == 3 ? batch_decode_kernel<3> : batch_decode_kernel<2>;
  const size_t smem = (size_t)stages * b.stage_bytes;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const bool cached = dev >= 0 && dev < kMaxDevices && b.stage_bytes % 16 == 0 && b.stage_bytes <= kStageCapWords * 4;
  int per_sm = 0;
  if (cached) {
    if (!g_batch_attr[dev][si].load(std::memory_order_acquire)) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, stages * kStageCapWords * 4);
      if (e != cudaSuccess) return e;
      g_batch_attr[dev][si].store(1, std::memory_order_release);
    }
    per_sm = g_batch_per_sm[dev][si][b.stage_bytes / 16].load(std::memory_order_relaxed);
  } else if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) {
    return e;
  }
  if (per_sm == 0) {
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPCThreads, smem)) != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    if (cached) g_batch_per_sm[dev][si][b.stage_bytes / 16].store(per_sm, std::memory_order_relaxed);
  }
  BatchDecodeArgs a = b;
  a.grid_begin[0] = 0;
  for (int d = 0; d < 4; d++) {
    const int64_t items = b.group_begin[d + 1] - b.group_begin[d];
    const int64_t g = items < (int64_t)per_sm * num_sms ? items : (int64_t)per_sm * num_sms;
    a.grid_begin[d + 1] = a.grid_begin[d] + (int32_t)g;
  }
  if (a.grid_begin[4] <= 0) return cudaSuccess;
  if (zero && (e = cudaMemsetAsync(b.counter, 0, 4 * sizeof(unsigned long long), s)) != cudaSuccess) return e;
  kern<<<(unsigned)a.grid_begin[4], kPCThreads, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_batch_decode(const BatchDecodeArgs& b, int num_sms, cudaStream_t s) {
  return batch_decode_go(b, num_sms, true, s);
}

cudaError_t launch_batch_decode_zeroed(const BatchDecodeArgs& b, int num_sms, cudaStream_t s) {
  return batch_decode_go(b, num_sms, false, s);
}

int batch_stage_bytes(int max_bits) {
  int64_t words = ((int64_t)kDecodeTile * max_bits + 31) / 32 + 16;
  words = (words + 3) & ~3ll;
  if (words > kStageCapWords) words = kStageCapWords;
  return (int)(words * 4);
}

template <typename T, bool PLAIN, bool RESID, int kStages, int kUnroll, int CW = kConsumerWarps, bool HOOK = false>
static cudaError_t run_decode(glc_ctx* ctx, const DecodeArgs& a, cudaStream_t s) {
  const size_t smem = (size_t)kStages * a.stage_bytes;
  constexpr int kBlock = CW * 32 + 32;
  void (*kern)(DecodeArgs) = decode_kernel<T, PLAIN, RESID, kStages, kUnroll, CW, HOOK>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  const int64_t ntile = a.t_end - a.t_begin;
  int64_t grid = (int64_t)per_sm * ctx->num_sms;
  if (grid > ntile) grid = ntile;
  if (grid < 1) return cudaSuccess;
  if ((e = cudaMemsetAsync(a.counter, 0, sizeof(int), s)) != cudaSuccess) return e;
  kern<<<(unsigned)grid, kBlock, smem, s>>>(a);
  return cudaGetLastError();
}

// The unroll depth and the consumer warps per CTA (threads per tile) are tuning choices of the
// packed value decode (the path every full and range decode takes); the residual and pre-unpacked
// variants keep depth 2 and 8 warps.
template <typename T, int kStages, int CW>
static cudaError_t decode_packed(glc_ctx* ctx, const DecodeArgs& a, int unroll, cudaStream_t s) {
  if (unroll == 1) return run_decode<T, false, false, kStages, 1, CW>(ctx, a, s);
  if (unroll == 4) return run_decode<T, false, false, kStages, 4, CW>(ctx, a, s);
  return run_decode<T, false, false, kStages, 2, CW>(ctx, a, s);
}

template <typename T, int kStages>
static cudaError_t decode_staged(glc_ctx* ctx, const DecodeArgs& a, int plain, int resid, int unroll, int warps,
                                 cudaStream_t s) {
  // the armed test hook: one instantiation per element type, whatever the tuned shape
  if (a.first_wait_tests >= 0) return run_decode<T, false, false, kDefaultStages, 2, kConsumerWarps, true>(ctx, a, s);
  if (plain) return resid ? run_decode<T, true, true, kStages, 2>(ctx, a, s) : run_decode<T, true, false, kStages, 2>(ctx, a, s);
  if (resid) return run_decode<T, false, true, kStages, 2>(ctx, a, s);
  if (warps == 4) return decode_packed<T, kStages, 4>(ctx, a, unroll, s);
  return decode_packed<T, kStages, kConsumerWarps>(ctx, a, unroll, s);
}

template <typename T>
static cudaError_t decode_typed(glc_ctx* ctx, const DecodeArgs& a, int plain, int resid, int stages, int unroll,
                                int warps, cudaStream_t s) {
  if (stages == 2) return decode_staged<T, 2>(ctx, a, plain, resid, unroll, warps, s);
  if (stages == 4) return decode_staged<T, 4>(ctx, a, plain, resid, unroll, warps, s);
  return decode_staged<T, 3>(ctx, a, plain, resid, unroll, warps, s);
}

// Launch shape overrides for tuning sweeps (ring depth, stage capacity in words).
static int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  return (v && *v) ? atoi(v) : dflt;
}

// Same kernel with caller-supplied scratch (work counter, error word) and SM count, for the
// allocation-free entry point (noalloc.cu).  The counter must be zero at launch.
cudaError_t launch_decode_scratch(const glc_column* c, int64_t lo, int64_t hi, void* out_base, int* counter, int* err,
                                  int num_sms, cudaStream_t s) {
  if (hi <= lo || c->n <= 0) return cudaSuccess;
  if (((uintptr_t)out_base & 15) != 0) return cudaErrorMisalignedAddress;
  DecodeArgs a;
  a.desc = c->d_desc;
  a.starts = c->d_start;
  a.tiles = c->d_tiles;
  a.words = c->d_words;
  a.plain = c->d_plain;
  a.P = c->P;
  a.n = c->n;
  a.lo = lo;
  a.hi = hi;
  a.t_begin = lo / kDecodeTile;
  a.t_end = (hi + kDecodeTile - 1) / kDecodeTile;
  a.out_base = out_base;
  a.counter = counter;
  a.err = err;
  a.first_wait_tests = -1;
  int64_t words = ((int64_t)kDecodeTile * c->max_bits + 31) / 32 + 16;
  words = (words + 3) & ~3ll;
  if (words > kStageCapWords) words = kStageCapWords;
  a.stage_bytes = (int)(words * 4);
  void (*kern)(DecodeArgs) = nullptr;
  switch (c->dtype) {
    case GLC_I32: kern = decode_kernel<int32_t, false, false, kDefaultStages, 2>; break;
    case GLC_I64: kern = decode_kernel<int64_t, false, false, kDefaultStages, 2>; break;
    case GLC_U64: kern = decode_kernel<uint64_t, false, false, kDefaultStages, 2>; break;
    case GLC_U32: kern = decode_kernel<uint32_t, false, false, kDefaultStages, 2>; break;
    default: return cudaErrorInvalidValue;
  }
  const size_t smem = (size_t)kDefaultStages * a.stage_bytes;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPCThreads, smem)) != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * num_sms;
  if (grid > a.t_end - a.t_begin) grid = a.t_end - a.t_begin;
  kern<<<(unsigned)grid, kPCThreads, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_decode_shape(glc_ctx* ctx, const glc_column* c, int plain_src, int residual_out, int64_t lo,
                                int64_t hi, void* out_base, int stages, int unroll, int cap_words, int warps,
                                cudaStream_t s) {
  if (hi <= lo || c->n <= 0) return cudaSuccess;
  if (((uintptr_t)out_base & 15) != 0) return cudaErrorMisalignedAddress;  // 16-byte vector stores
  DecodeArgs a;
  a.desc = c->d_desc;
  a.starts = c->d_start;
  a.tiles = c->d_tiles;
  a.words = c->d_words;
  a.plain = c->d_plain;
  a.P = c->P;
  a.n = c->n;
  a.lo = lo;
  a.hi = hi;
  a.t_begin = lo / kDecodeTile;
  a.t_end = (hi + kDecodeTile - 1) / kDecodeTile;
  a.out_base = out_base;
  a.counter = ctx->d_flags + (ctx->next_slot.fetch_add(1u) % kCounterSlots);
  a.err = ctx->d_flags + kFlagError;
  a.first_wait_tests = ctx->expire_next_wait.exchange(0) ? 0 : -1;  // test hook, one launch
  if (plain_src) {
    a.stage_bytes = kDecodeTile * 8 + 16;
  } else {
    int64_t words = ((int64_t)kDecodeTile * c->max_bits + 31) / 32 + 16;
    words = (words + 3) & ~3ll;
    int64_t cap = (cap_words > 0 ? cap_words : kStageCapWords) & ~3;
    if (cap > kStageCapWordsMax) cap = kStageCapWordsMax;
    if (words > cap) words = cap < 32 ? 32 : cap;
    a.stage_bytes = (int)(words * 4);
  }
  switch (c->dtype) {
    case GLC_I32: return decode_typed<int32_t>(ctx, a, plain_src, residual_out, stages, unroll, warps, s);
    case GLC_I64: return decode_typed<int64_t>(ctx, a, plain_src, residual_out, stages, unroll, warps, s);
    case GLC_U64: return decode_typed<uint64_t>(ctx, a, plain_src, residual_out, stages, unroll, warps, s);
    case GLC_U32: return decode_typed<uint32_t>(ctx, a, plain_src, residual_out, stages, unroll, warps, s);
  }
  return cudaErrorInvalidValue;
}

// Ring depth, unroll depth, stage capacity and consumer warps from the context's tuning table for
// the column's element type and widest field (GLC_DECODE_STAGES / _UNROLL / _CAP_WORDS / _WARPS
// override them, for sweeps).
cudaError_t launch_decode(glc_ctx* ctx, const glc_column* c, int plain_src, int residual_out, int64_t lo, int64_t hi,
                          void* out_base, cudaStream_t s) {
  const TuneEntry& t = tune_entry(ctx, c->dtype, c->max_bits, plain_src);
  const int stages = env_int("GLC_DECODE_STAGES", t.decode_stages);
  const int unroll = env_int("GLC_DECODE_UNROLL", t.decode_unroll);
  const int cap = env_int("GLC_DECODE_CAP_WORDS", t.decode_cap_words);
  const int warps = env_int("GLC_DECODE_WARPS", t.decode_warps);
  return launch_decode_shape(ctx, c, plain_src, residual_out, lo, hi, out_base, stages, unroll, cap, warps, s);
}

}  // namespace glc
