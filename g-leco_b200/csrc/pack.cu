// pack.cu -- bit-packer: residuals per value into shared memory, then words per thread.
//
// Replaces compression/CompressionKernels.cuh:242-372 (packDeltasKernelOptimized: one value per
// thread, a binary search over partitions per value and 1-3 atomicOr per value into a word
// array that a separate memset pass zeroed first).
//
// Here the OUTPUT words are the unit of work.  A CTA owns a tile of 2048 consecutive words
// (8 KB) and builds it in shared memory:
//   * the CTA finds the first partition whose bit range reaches the tile with a 256-way search
//     (every thread probes one bound per level; two levels for 65K partitions);
//   * the CTA walks partitions while their bit ranges start inside the tile; the values whose
//     fields touch the tile are taken in segments of kPackSeg;
//   * phase 1: one thread per value (coalesced loads) computes the residual field and stores it
//     in shared memory;
//   * phase 2: one thread per output word finds the first field that overlaps the word (a
//     multiply-high by the reciprocal of the width, exact for these magnitudes) and ORs the
//     fields that overlap it into place with 32-bit shifts (64-bit only for fields wider than
//     32 bits); a word shared with the previous segment or partition is merged with one shared
//     atomicOr;
//   * the finished tile is written with coalesced 128-bit stores, padding words included, so
//     every word of the array is written exactly once and no memset pass is needed.
// Values whose fields straddle two tiles are computed by both CTAs; each keeps its own bits.
#include "glc_internal.h"
#include "glc_tma.cuh"

namespace glc {

constexpr int kPackWords = 2048;
constexpr int kPackThreads = 256;
constexpr int kPackSeg = 2048;  // residual fields per segment in shared memory

__device__ __forceinline__ int64_t end_bit(const PackArgs& a, int64_t p) {
  return a.offs[p] + ((int64_t)a.ends[p] - a.starts[p]) * (int64_t)a.bits[p];
}

struct PackSmem {
  uint32_t tile[kPackWords];
  uint64_t res[kPackSeg];
};

// Builds output word tile `tile` (kPackWords words) of one column; every thread of the CTA calls it.
template <typename T> __device__ __forceinline__ void pack_word_tile(const T* __restrict__ v, const PackArgs& a,
                                                                    int64_t tile, PackSmem& sm) {
  uint32_t* const s_tile = sm.tile;
  uint64_t* const s_res = sm.res;
  uint32_t* const s_res32 = reinterpret_cast<uint32_t*>(s_res);
  const int64_t W0 = tile * kPackWords;
  const int64_t W1 = (W0 + kPackWords < a.nwords_alloc) ? W0 + kPackWords : a.nwords_alloc;
  const int tile_words = (int)(W1 - W0);
  const int64_t B0 = W0 * 32, B1 = W1 * 32;

  for (int k = threadIdx.x; k < kPackWords; k += kPackThreads) s_tile[k] = 0u;
  // First partition whose bit range ends after B0 = the number of partitions ending at or before
  // B0 (end bits are non-decreasing).  The answer stays in [lo, hi]; each level probes 256 bounds.
  int64_t lo = 0, hi = a.P;
  while (lo < hi) {
    const int64_t step = (hi - lo + kPackThreads - 1) / kPackThreads;
    const int64_t q = lo + (int64_t)(threadIdx.x + 1) * step - 1;
    const int c = __syncthreads_count(q < hi && end_bit(a, q) <= B0);
    const int64_t nhi = lo + (int64_t)(c + 1) * step - 1;
    lo += (int64_t)c * step;
    if (nhi < hi) hi = nhi;
  }
  __syncthreads();

  for (int64_t p = lo; p < a.P; p++) {
    const int64_t off = a.offs[p];
    if (off >= B1) break;
    const int b = a.bits[p];
    if (b <= 0) continue;
    const int64_t start = a.starts[p];
    const int64_t len = (int64_t)a.ends[p] - start;
    const bool direct = a.types[p] == MODEL_DIRECT_COPY;
    const double t0 = a.params[4 * p], t1 = a.params[4 * p + 1];
    const int64_t i_lo = (B0 > off) ? (B0 - off) / b : 0;
    int64_t i_hi = (B1 - off + b - 1) / b;
    if (i_hi > len) i_hi = len;
    // floor(x / b) = umulhi(x, mb) for 0 <= x < 2^26 (x * (mb * b - 2^32) < 2^32)
    const uint32_t mb = b > 1 ? 0xffffffffu / (uint32_t)b + 1u : 0u;
    for (int64_t s0 = i_lo; s0 < i_hi; s0 += kPackSeg) {
      const int cnt = (int)((i_hi - s0) < kPackSeg ? (i_hi - s0) : kPackSeg);
      // phase 1: residual fields of values s0 .. s0 + cnt - 1
#pragma unroll 4
      for (int j = threadIdx.x; j < cnt; j += kPackThreads) {
        const int64_t i = s0 + j;
        const T x = __ldg(v + start + i);
        const uint64_t f = low_bits(direct ? (uint64_t)x : (uint64_t)calc_delta<T>(x, predict<T>(t0, t1, i)), b);
        if (b <= 32) s_res32[j] = (uint32_t)f; else s_res[j] = f;
      }
      __syncthreads();
      // phase 2: the tile words these fields touch.  R0 = tile-relative bit of field s0, in
      // (-b, 2^16 + 2b): every quantity below fits in 32 bits.
      const int R0 = (int)(off + s0 * b - B0);
      const int R1 = R0 + cnt * b;
      const int w_lo = R0 > 0 ? (R0 >> 5) : 0;
      const int w_hi = min(tile_words, (R1 + 31) >> 5);
      for (int w = w_lo + (int)threadIdx.x; w < w_hi; w += kPackThreads) {
        const int x = 32 * w - R0;  // word start, relative to the first bit of field s0
        int j = x <= 0 ? 0 : (b > 1 ? (int)__umulhi((uint32_t)x, mb) : x);
        int sh = j * b - x;         // bit of field j relative to the word start, in (-b, 0] or j = 0
        uint32_t word = 0u;
        if (b <= 32) {
          for (; j < cnt && sh < 32; j++, sh += b) {
            const uint32_t f = s_res32[j];
            word |= sh >= 0 ? (f << sh) : (f >> -sh);
          }
        } else {
          for (; j < cnt && sh < 32; j++, sh += b) {
            const uint64_t f = s_res[j];
            word |= sh >= 0 ? (uint32_t)(f << sh) : (uint32_t)(f >> -sh);
          }
        }
        if (word != 0u) atomicOr(&s_tile[w], word);
      }
      __syncthreads();
    }
  }
  uint4* dst = reinterpret_cast<uint4*>(a.words + W0);
  const uint4* src = reinterpret_cast<const uint4*>(s_tile);
  for (int k = threadIdx.x; k < tile_words / 4; k += kPackThreads) dst[k] = src[k];
}

template <typename T> __global__ void __launch_bounds__(kPackThreads) pack_kernel(const T* __restrict__ v, PackArgs a) {
  __shared__ __align__(16) PackSmem sm;
  pack_word_tile<T>(v, a, blockIdx.x, sm);
}

// ---------------------------------------------------------------------------------------
// Single-column pack over VALUE tiles (the decode tiles: 4096 values, their first bit and
// partitions from the column's tile table).  Persistent CTAs of 8 compute warps + 1 producer
// warp; the producer stages each tile's values and partition descriptors in shared memory with
// bulk copies (cp.async.bulk, non-multicast; the value source rounded down and its length up
// to 16 bytes, within the same 16-byte blocks), two tiles ahead on full/empty mbarriers.
//   phase 1: one thread per value computes its residual field from the staged value into a
//            shared field array (coalesced shared-memory traffic, HBM read once);
//   phase 2: one thread per output word the tile touches assembles it from the fields (a
//            multiply-high by the width's reciprocal finds the first field, then 32-bit shifts).
// Words wholly inside a tile's bit range are written with plain stores; the first and last word
// of a tile, shared with the neighbouring tile, are merged with atomicOr into words that
// pack_edge_zero_kernel cleared first (the two kinds never meet: a word wholly inside one tile's
// range has no bits from another tile).  Needs at most kPackTileParts partitions per tile.
// ---------------------------------------------------------------------------------------
constexpr int kPackTileParts = kPackTilePartsMax;
constexpr int kPackCompute = 256;
constexpr int kPackCTA = kPackCompute + 32;
constexpr int kPackStages = 2;

struct PackTileArgs {
  PackTileCol col;           // single column (BATCH = false)
  const PackTileCol* cols;   // batch: the columns of one element type
  const int32_t* owner;      // batch: work item -> column
  const int64_t* item_base;  // batch: column -> its first work item (its tiles follow)
  int64_t nitems;            // batch: work items (tiles of all the columns)
  int* status;  // DEVERR_* (the context's device error word)
};

struct PackStage {
  int64_t tile;    // -1 = no more work
  int64_t e0;      // first value of the tile
  int64_t bit_lo, bit_hi;
  uint32_t* words; // the tile's column's word array
  int32_t cnt;     // values in the tile
  int32_t head;    // byte offset of the first value in the stage
  int32_t pf, np;  // partitions of the tile
};

struct PackPart {  // one partition of the current tile, tile-relative
  double t0, t1;
  int64_t start;   // first value of the partition (absolute)
  int32_t j0;      // first in-tile value (tile-relative)
  int32_t bl;      // bit of that value's field (tile-relative)
  int32_t bend;    // end of the partition's in-tile bits (tile-relative)
  int32_t b, type;
  uint32_t mb;     // floor(x / b) = umulhi(x, mb) for x < 2^26
};

template <typename T> __host__ __device__ constexpr int pack_stage_bytes() {
  return kDecodeTile * (int)sizeof(T) + 32 + kPackTileParts * (int)sizeof(PartDesc);
}

__device__ __forceinline__ void pack_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kPackCompute) : "memory"); }

// Zero the words that two tiles share (the word holding each tile's first bit when that bit is
// not word-aligned; entry ntiles holds total_bits) and the padding words after the stream.
__global__ void pack_edge_zero_kernel(const TileInfo* __restrict__ tiles, int64_t ntiles, int64_t nwords,
                                      int64_t nwords_alloc, uint32_t* __restrict__ words) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t <= ntiles) {
    const int64_t b = tiles[t].bit_lo;
    if (b & 31) words[b >> 5] = 0u;
  }
  const int64_t w = nwords + t;
  if (w < nwords_alloc) words[w] = 0u;
}

template <typename T, bool BATCH> __global__ void __launch_bounds__(kPackCTA)
pack_tile_kernel(PackTileArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];  // [stages][values | descriptors] (+ fields for 4-byte types)
  __shared__ __align__(8) uint64_t full[kPackStages], empty[kPackStages];
  __shared__ PackStage s_meta[kPackStages];
  __shared__ PackPart s_part[kPackTileParts];
  __shared__ int s_ok;
  // Fields replace the values in place for 8-byte types (a thread reads value j, then writes field
  // j into the same 8 bytes; a field of <= 32 bits in the low half); 4-byte types use a separate
  // 64-bit array after the stages (a 4-byte value cannot hold a 33-bit field).
  constexpr int NS = sizeof(T) == 8 ? 2 : 1;  // 32-bit field j lives at f32[NS * j]
  if (threadIdx.x == 0) {
    for (int st = 0; st < kPackStages; st++) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (threadIdx.x >= kPackCompute) {  // ---- producer ----
    if (threadIdx.x != kPackCompute) return;
    const int64_t nitems = BATCH ? a.nitems : a.col.ntiles;
    int64_t item = blockIdx.x;
    for (int k = 0;; k++, item += gridDim.x) {
      const int st = k % kPackStages;
      if (k >= kPackStages && !mbar_wait_bounded(&empty[st], (uint32_t)((k / kPackStages) - 1) & 1u)) {
        atomicExch(a.status, DEVERR_TIMEOUT);
        s_meta[st].tile = -1;
        mbar_arrive(&full[st]);
        return;
      }
      if (item >= nitems) {
        s_meta[st].tile = -1;
        mbar_arrive(&full[st]);  // no copy: completes the phase, the compute warps see the end
        return;
      }
      PackTileCol c;
      int64_t t = item;
      if (BATCH) {
        const int32_t ci = a.owner[item];
        c = a.cols[ci];
        t = item - a.item_base[ci];
      } else {
        c = a.col;
      }
      const TileInfo ti = c.tiles[t];
      PackStage m;
      m.tile = t;
      m.e0 = t * kDecodeTile;
      m.cnt = (int)((c.n - m.e0) < kDecodeTile ? (c.n - m.e0) : kDecodeTile);
      m.bit_lo = ti.bit_lo;
      m.bit_hi = c.tiles[t + 1].bit_lo;
      m.words = c.words;
      m.pf = ti.p_first;
      m.np = ti.p_last - ti.p_first + 1;
      const uintptr_t addr = reinterpret_cast<uintptr_t>(reinterpret_cast<const T*>(c.v) + m.e0);
      m.head = (int)(addr & 15);
      s_meta[st] = m;
      const uint32_t vbytes = (uint32_t)((m.head + (int64_t)m.cnt * (int64_t)sizeof(T) + 15) & ~15ll);
      const uint32_t dbytes = m.np <= kPackTileParts ? (uint32_t)m.np * (uint32_t)sizeof(PartDesc) : 0u;
      uint8_t* stage = smem + (size_t)st * pack_stage_bytes<T>();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive_expect_tx(&full[st], vbytes + dbytes);
      tma_bulk_load(stage, reinterpret_cast<const uint8_t*>(addr - m.head), vbytes, &full[st]);
      if (dbytes) tma_bulk_load(stage + kDecodeTile * sizeof(T) + 32, c.desc + m.pf, dbytes, &full[st]);
    }
  }

  // ---- compute warps ----
  const int tid = threadIdx.x;
  for (int k = 0;; k++) {
    const int st = k % kPackStages;
    const uint32_t par = (uint32_t)(k / kPackStages) & 1u;
    if (tid == 0) {
      s_ok = mbar_wait_bounded(&full[st], par);
      if (!s_ok) {
        atomicExch(a.status, DEVERR_TIMEOUT);
        mbar_wait_bounded(&full[st], par);  // a copy in flight lands before the CTA exits
      }
    }
    pack_sync();
    if (!s_ok) return;
    mbar_try_wait(&full[st], par);  // the phase is complete: orders this thread's reads after the copy
    const PackStage m = s_meta[st];
    if (m.tile < 0) return;
    if (m.np > kPackTileParts) {  // excluded by the host (partitions of >= 108 values); never packed wrong
      if (tid == 0) atomicExch(a.status, DEVERR_BOUNDS);
    } else {
      uint8_t* stage = smem + (size_t)st * pack_stage_bytes<T>();
      const T* x = reinterpret_cast<const T*>(stage + m.head);
      const PartDesc* sd = reinterpret_cast<const PartDesc*>(stage + kDecodeTile * sizeof(T) + 32);
      uint64_t* fields = sizeof(T) == 8 ? reinterpret_cast<uint64_t*>(stage + m.head)
                                        : reinterpret_cast<uint64_t*>(smem + (size_t)kPackStages * pack_stage_bytes<T>());
      if (tid < m.np) {  // the tile's partitions, tile-relative
        const PartDesc d = sd[tid];
        PackPart q;
        q.t0 = d.theta0;
        q.t1 = d.theta1;
        q.start = d.start;
        q.b = d.bits_type & 0xff;
        q.type = d.bits_type >> 8;
        const int64_t first = q.start > m.e0 ? q.start : m.e0;
        const int64_t nxt = tid + 1 < m.np ? (int64_t)sd[tid + 1].start : m.e0 + m.cnt;
        const int64_t last = nxt < m.e0 + m.cnt ? nxt : m.e0 + m.cnt;
        q.j0 = (int)(first - m.e0);
        q.bl = (int)(d.bit_off + (first - q.start) * q.b - m.bit_lo);
        q.bend = q.bl + (int)(last - first) * q.b;
        q.mb = q.b > 1 ? 0xffffffffu / (uint32_t)q.b + 1u : 0u;
        s_part[tid] = q;
      }
      pack_sync();
      bool m_wide = false;  // fields wider than 32 bits anywhere in the tile: 64-bit field array
      for (int i = 0; i < m.np; i++) m_wide |= s_part[i].b > 32;
      // phase 1: fields of the tile's values, partition by partition (parameters in registers;
      // the index advances as an exact double).  For fields of at most 32 bits the residual's
      // low 32 bits are the difference of the low 32 bits (no saturation can reach such a field).
      uint32_t* f32 = reinterpret_cast<uint32_t*>(fields);
      for (int i = 0; i < m.np; i++) {
        const PackPart q = s_part[i];
        const int jend = i + 1 < m.np ? s_part[i + 1].j0 : m.cnt;
        int j = q.j0 + (((tid - q.j0) % kPackCompute) + kPackCompute) % kPackCompute;
        double xd = (double)(m.e0 + j - q.start);
        if (q.b == 0) continue;
        if (!m_wide) {
          const uint32_t mask = q.b >= 32 ? 0xffffffffu : ((1u << q.b) - 1u);
          if (q.type == MODEL_DIRECT_COPY) {
            for (; j < jend; j += kPackCompute) f32[NS * j] = (uint32_t)x[j] & mask;
          } else {
#pragma unroll 4
            for (; j < jend; j += kPackCompute, xd += (double)kPackCompute) {
              const T p = predict_from<T>(__fma_rn(q.t1, xd, q.t0));
              f32[NS * j] = ((uint32_t)x[j] - (uint32_t)p) & mask;
            }
          }
        } else {
#pragma unroll 2
          for (; j < jend; j += kPackCompute, xd += (double)kPackCompute) {
            const T xv = x[j];
            const uint64_t f = q.type == MODEL_DIRECT_COPY
                                   ? (uint64_t)xv
                                   : (uint64_t)calc_delta<T>(xv, predict_from<T>(__fma_rn(q.t1, xd, q.t0)));
            fields[j] = low_bits(f, q.b);
          }
        }
      }
      pack_sync();
      // phase 2: words.  Word k covers tile-relative bits [32k - sh0, 32k - sh0 + 32).
      const int sh0 = (int)(m.bit_lo & 31);
      const int bh = (int)(m.bit_hi - m.bit_lo);
      const int nw = bh > 0 ? (sh0 + bh + 31) >> 5 : 0;
      const bool last_partial = (m.bit_hi & 31) != 0;
      const int64_t W0 = m.bit_lo >> 5;
      if (m.np == 1 && !m_wide) {
        // one partition of width 1..32 over the whole tile (the common case): its parameters in
        // registers; the first field of a word may start before it, the rest start inside it
        const int qb = s_part[0].b, qj0 = s_part[0].j0;
        const uint32_t qmb = s_part[0].mb;
        for (int w = tid; w < nw; w += kPackCompute) {
          const int wb = 32 * w - sh0;
          const int pos = wb > 0 ? wb : 0;
          const int wend = wb + 32 < bh ? wb + 32 : bh;
          const int jj = qb > 1 ? (int)__umulhi((uint32_t)pos, qmb) : pos;
          int fb = jj * qb;  // start of the field holding bit pos (the partition starts at tile bit 0)
          int j = qj0 + jj;
          int sh = fb - wb;
          uint32_t word = sh >= 0 ? (f32[NS * j] << sh) : (f32[NS * j] >> -sh);
          for (fb += qb, sh += qb, j++; fb < wend; fb += qb, sh += qb, j++) word |= f32[NS * j] << sh;
          const bool partial = (w == 0 && sh0 != 0) || (w == nw - 1 && last_partial);
          if (partial) atomicOr(m.words + W0 + w, word);
          else m.words[W0 + w] = word;
        }
      } else {
      int qi = 0;
      for (int w = tid; w < nw; w += kPackCompute) {
        const int wb = 32 * w - sh0;  // tile-relative bit of the word's bit 0
        int pos = wb > 0 ? wb : 0;
        const int wend = wb + 32 < bh ? wb + 32 : bh;
        uint32_t word = 0u;
        while (qi + 1 < m.np && s_part[qi + 1].bl <= pos) qi++;  // bl never decreases
        while (pos < wend) {
          while (qi + 1 < m.np && s_part[qi].bend <= pos) qi++;  // past this partition (or an empty one)
          const int qbl = s_part[qi].bl, qbend = s_part[qi].bend, qb = s_part[qi].b;
          if (qbend <= pos) break;  // the table ends before bit pos (cannot happen for a consistent column)
          const uint32_t xo = (uint32_t)(pos - qbl);
          const int jj = qb > 1 ? (int)__umulhi(xo, s_part[qi].mb) : (int)xo;
          int fb = qbl + jj * qb;  // start of the field holding bit pos
          int j = s_part[qi].j0 + jj;
          const int qend = qbend < wend ? qbend : wend;
          if (!m_wide) {
            for (; fb < qend; fb += qb, j++) {
              const uint32_t f = f32[NS * j];
              const int sh = fb - wb;
              word |= sh >= 0 ? (f << sh) : (f >> -sh);
            }
          } else {
            for (; fb < qend; fb += qb, j++) {
              const uint64_t f = fields[j];
              const int sh = fb - wb;
              word |= sh >= 0 ? (uint32_t)(f << sh) : (uint32_t)(f >> -sh);
            }
          }
          pos = qend;
        }
        const bool partial = (w == 0 && sh0 != 0) || (w == nw - 1 && last_partial);
        if (partial) atomicOr(m.words + W0 + w, word);
        else m.words[W0 + w] = word;
      }
      }
    }
    pack_sync();  // every compute thread is done with stage st and the field array
    if (tid == 0) mbar_arrive(&empty[st]);
  }
}

template <typename T, bool BATCH>
static cudaError_t launch_pack_tile_kernel(const PackTileArgs& a, int64_t nitems, int num_sms, cudaStream_t s) {
  const int smem = kPackStages * pack_stage_bytes<T>() + (sizeof(T) == 4 ? kDecodeTile * 8 : 0);
  static PerDeviceFlag attr_set;  // per instantiation and device
  const int dev = current_device();
  cudaError_t e;
  if (!attr_set.test(dev)) {
    if ((e = cudaFuncSetAttribute(pack_tile_kernel<T, BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) !=
        cudaSuccess)
      return e;
    attr_set.set(dev);
  }
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pack_tile_kernel<T, BATCH>, kPackCTA, smem)) !=
      cudaSuccess)
    return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * num_sms;
  if (grid > nitems) grid = nitems;
  if (grid < 1) grid = 1;
  pack_tile_kernel<T, BATCH><<<(unsigned)grid, kPackCTA, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T>
static cudaError_t launch_pack_tiles(const T* v, glc_column* c, int* status, cudaStream_t s) {
  const int64_t zthreads = (c->ntiles + 1) > (c->nwords_alloc - c->nwords) ? c->ntiles + 1 : c->nwords_alloc - c->nwords;
  pack_edge_zero_kernel<<<(unsigned)((zthreads + 255) / 256), 256, 0, s>>>(c->d_tiles, c->ntiles, c->nwords,
                                                                          c->nwords_alloc, c->d_words);
  PackTileArgs a{};
  a.col = PackTileCol{v, c->d_desc, c->d_tiles, c->n, c->ntiles, c->d_words};
  a.status = status;
  return launch_pack_tile_kernel<T, false>(a, c->ntiles, c->ctx->num_sms, s);
}

// Batched value-tile pack over the columns of one element type: cols[i] (device), item_base[i] =
// its first work item, owner[item] = its column, nitems = all their tiles.  The word arrays must be
// zero (interior words are stored, the edge words merged with atomicOr).
cudaError_t launch_batch_pack_tiles(glc_dtype dt, const PackTileCol* cols, const int32_t* owner,
                                    const int64_t* item_base, int64_t nitems, int* status, int num_sms, cudaStream_t s) {
  if (nitems <= 0) return cudaSuccess;
  PackTileArgs a{};
  a.cols = cols;
  a.owner = owner;
  a.item_base = item_base;
  a.nitems = nitems;
  a.status = status;
  switch (dt) {
    case GLC_I32: return launch_pack_tile_kernel<int32_t, true>(a, nitems, num_sms, s);
    case GLC_I64: return launch_pack_tile_kernel<int64_t, true>(a, nitems, num_sms, s);
    case GLC_U64: return launch_pack_tile_kernel<uint64_t, true>(a, nitems, num_sms, s);
    case GLC_U32: return launch_pack_tile_kernel<uint32_t, true>(a, nitems, num_sms, s);
  }
  return cudaErrorInvalidValue;
}

// owner[item] = i for the items of column i (one thread per column).
__global__ void pack_item_owner_kernel(const int64_t* __restrict__ item_base, int ncols, int32_t* __restrict__ owner) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncols) return;
  for (int64_t k = item_base[i]; k < item_base[i + 1]; k++) owner[k] = i;
}

cudaError_t launch_pack_item_owner(const int64_t* item_base, int ncols, int32_t* owner, cudaStream_t s) {
  if (ncols <= 0) return cudaSuccess;
  pack_item_owner_kernel<<<(unsigned)((ncols + 255) / 256), 256, 0, s>>>(item_base, ncols, owner);
  return cudaGetLastError();
}

cudaError_t launch_pack(glc_dtype dt, const void* values, glc_column* c, int64_t parts_per_tile, int* status,
                        cudaStream_t s) {
  if (c->nwords_alloc <= 0) return cudaSuccess;
  if (parts_per_tile + 2 <= kPackTileParts && c->d_tiles && c->d_desc && c->ntiles > 0) {
    switch (dt) {
      case GLC_I32: return launch_pack_tiles<int32_t>((const int32_t*)values, c, status, s);
      case GLC_I64: return launch_pack_tiles<int64_t>((const int64_t*)values, c, status, s);
      case GLC_U64: return launch_pack_tiles<uint64_t>((const uint64_t*)values, c, status, s);
      case GLC_U32: return launch_pack_tiles<uint32_t>((const uint32_t*)values, c, status, s);
    }
    return cudaErrorInvalidValue;
  }
  // short partitions (more than kPackTileParts per tile): output word tiles
  PackArgs a{c->d_start, c->d_end, c->d_types, c->d_params, c->d_bits, c->d_offs, c->P, c->d_words, c->nwords_alloc};
  const unsigned grid = (unsigned)((c->nwords_alloc + kPackWords - 1) / kPackWords);
  switch (dt) {
    case GLC_I32: pack_kernel<int32_t><<<grid, kPackThreads, 0, s>>>((const int32_t*)values, a); break;
    case GLC_I64: pack_kernel<int64_t><<<grid, kPackThreads, 0, s>>>((const int64_t*)values, a); break;
    case GLC_U64: pack_kernel<uint64_t><<<grid, kPackThreads, 0, s>>>((const uint64_t*)values, a); break;
    case GLC_U32: pack_kernel<uint32_t><<<grid, kPackThreads, 0, s>>>((const uint32_t*)values, a); break;
  }
  return cudaGetLastError();
}

}  // namespace glc
