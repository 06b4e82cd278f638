// decode.cu -- persistent work-stealing full / range decode with TMA-staged input.
//
// Replaces the reference's full-decode kernels, which all do the same arithmetic with
// different work layouts: decompressFullFile_BitPacked / _PreUnpacked (grid-stride, a binary
// search per value, decompression/FullDecompressionKernels.cuh:47-288), _OnTheFly_Optimized_V2
// (one CTA per partition, :292-378), decompressFullFileFix (:382-476), and the work-stealing
// kernels (atomic batches of partitions, WorkStealingDecompressionKernels.cuh:331-619).  The
// pre-unpack kernel (decompression/UnpackKernel.cuh:31-98) is the same walk with a residual
// epilogue, so it is a mode of this kernel too.
//
// Work unit: a TILE of 4096 consecutive output values (independent of partition sizes, so
// every unit writes the same number of bytes).  A table built once per column holds each
// tile's first bit and first/last partition, so no per-value search is needed.
// Per CTA (persistent, grid = resident CTAs on all SMs):
//   thread 0 claims tiles from a global counter one ahead of the CTA, and for each claimed
//   tile issues a 1-D TMA bulk copy (cp.async.bulk, non-multicast) of the tile's packed words
//   (or its pre-unpacked residuals) into one of two shared-memory stages, completing on that
//   stage's mbarrier; while that copy flies, the CTA decodes the previous tile from the other
//   stage: each thread walks its values with a partition cursor over the tile's descriptors
//   (cached in shared memory), extracts the field from shared memory, recomputes the FP64
//   prediction exactly as the reference does and writes 16-byte vector stores.
// Every mbarrier wait is bounded by wall time; on expiry the kernel records an error code,
// waits (bounded) for its own copies in flight and returns.
#include <type_traits>
#include "glc_internal.h"

namespace glc {

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
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for `parity` on `bar`, giving up after ~2 s of wall time.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (long long it = 0; it < kSpinLimit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255) == 0 && global_ns() - t0 > 2000000000ull) return false;
  }
  return false;
}

template <bool PLAIN> __device__ __forceinline__ void issue_tile(const DecodeArgs& a, int64_t t, void* stage, uint64_t* bar) {
  const void* src;
  uint32_t bytes;
  if (PLAIN) {
    const int64_t e0 = t * kDecodeTile;
    const int64_t e1 = (e0 + kDecodeTile < a.n) ? e0 + kDecodeTile : a.n;
    src = a.plain + e0;
    bytes = (uint32_t)((((e1 - e0) * 8) + 15) & ~15ll);
  } else {
    const int64_t bl = a.tiles[t].bit_lo, bh = a.tiles[t + 1].bit_lo;
    const int64_t w0 = (bl >> 5) & ~3ll;
    const int64_t w1 = (((bh >> 5) + 3) + 3) & ~3ll;
    src = a.words + w0;
    bytes = (uint32_t)((w1 - w0) * 4);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_arrive_expect_tx(bar, bytes);
  tma_bulk_load(stage, src, bytes, bar);
}

struct Cursor {
  double t0, t1;
  int64_t bit_rel;  // descriptor bit offset minus the stage's first bit
  int64_t start;
  int64_t next_start;
  int bits, type;
  int idx;
};

__device__ __forceinline__ void cursor_load(Cursor& c, const PartDesc& d, int64_t next_start, int64_t stage_bit0) {
  c.t0 = d.theta0;
  c.t1 = d.theta1;
  c.bit_rel = d.bit_off - stage_bit0;
  c.start = d.start;
  c.bits = d.bits_type & 0xff;
  c.type = d.bits_type >> 8;
  c.next_start = next_start;
}

template <typename T, bool PLAIN, bool RESID, bool VEC>
__global__ void __launch_bounds__(kDecodeThreads) decode_kernel(DecodeArgs a) {
  typedef typename std::conditional<RESID, int64_t, T>::type OutT;
  constexpr int V = 16 / (int)sizeof(OutT);
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ int64_t s_tile[2];
  __shared__ PartDesc s_desc[kDescCache];

  uint8_t* stage_ptr[2] = {smem, smem + a.stage_bytes};
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    const int64_t t = a.t_begin + atomicAdd(a.counter, 1);
    s_tile[0] = t;
    if (t < a.t_end) issue_tile<PLAIN>(a, t, stage_ptr[0], &bars[0]);
  }
  __syncthreads();

  uint32_t phase[2] = {0u, 0u};
  int st = 0;
  OutT* out = reinterpret_cast<OutT*>(a.out_base);
  bool failed = false;
  while (true) {
    const int64_t cur = s_tile[st];
    if (cur >= a.t_end) break;
    if (tid == 0) {
      const int64_t nt = a.t_begin + atomicAdd(a.counter, 1);
      s_tile[st ^ 1] = nt;
      if (nt < a.t_end) issue_tile<PLAIN>(a, nt, stage_ptr[st ^ 1], &bars[st ^ 1]);
    }
    const TileInfo ti = a.tiles[cur];
    const int64_t pf = ti.p_first, pl = ti.p_last;
    const int np = (int)(pl - pf + 1);
    const bool cached = np <= kDescCache;
    if (cached)
      for (int k = tid; k < np; k += kDecodeThreads) s_desc[k] = a.desc[pf + k];
    const bool ok = mbar_wait_bounded(&bars[st], phase[st]);
    phase[st] ^= 1u;
    if (__syncthreads_or(!ok)) { failed = true; break; }

    const int64_t tile_e0 = cur * kDecodeTile;
    const int64_t E0 = tile_e0 > a.lo ? tile_e0 : a.lo;
    const int64_t E1 = (tile_e0 + kDecodeTile < a.hi) ? tile_e0 + kDecodeTile : a.hi;
    const int64_t Ea = (E0 / V) * V;
    const int64_t nvec = (E1 - Ea + V - 1) / V;
    const int64_t stage_bit0 = ((ti.bit_lo >> 5) & ~3ll) * 32;
    const uint32_t* sw = reinterpret_cast<const uint32_t*>(stage_ptr[st]);
    const int64_t* sp = reinterpret_cast<const int64_t*>(stage_ptr[st]);

    Cursor c;
    c.idx = -1;
    c.next_start = INT64_MIN;
    for (int64_t j = tid; j < nvec; j += kDecodeThreads) {
      const int64_t e = Ea + j * V;
      OutT vals[V];
#pragma unroll
      for (int u = 0; u < V; u++) {
        const int64_t ee = e + u;
        vals[u] = OutT(0);
        if (ee < E0 || ee >= E1) continue;
        if (c.idx < 0 || ee >= c.next_start) {
          int k;
          if (cached) {
            k = c.idx < 0 ? 0 : c.idx;
            while (k + 1 < np && (int64_t)s_desc[k + 1].start <= ee) k++;
            cursor_load(c, s_desc[k], (k + 1 < np) ? (int64_t)s_desc[k + 1].start : INT64_MAX, stage_bit0);
          } else {
            int64_t lo = pf, hi = pl;
            while (lo < hi) {
              int64_t mid = (lo + hi + 1) >> 1;
              if ((int64_t)__ldg(a.starts + mid) <= ee) lo = mid; else hi = mid - 1;
            }
            k = (int)(lo - pf);
            cursor_load(c, a.desc[lo], (lo + 1 <= pl) ? (int64_t)__ldg(a.starts + lo + 1) : INT64_MAX, stage_bit0);
          }
          c.idx = k;
        }
        const int64_t local = ee - c.start;
        long long resid;
        if (PLAIN) {
          resid = sp[ee - tile_e0];
        } else {
          uint64_t f = (c.bits > 0) ? read_field(sw, c.bit_rel + local * c.bits, c.bits) : 0ull;
          resid = (c.type == MODEL_DIRECT_COPY) ? (long long)f : sign_extend(f, c.bits);
        }
        if (RESID) {
          vals[u] = (OutT)resid;
        } else if (c.type == MODEL_DIRECT_COPY) {
          vals[u] = (OutT)(T)resid;
        } else {
          vals[u] = (OutT)apply_delta<T>(predict<T>(c.t0, c.t1, local), resid);
        }
      }
      if (VEC && e >= E0 && e + V <= E1) {
        uint4 pk;
        static_assert(sizeof(vals) == 16, "vector of 16 bytes");
        memcpy(&pk, vals, 16);
        *reinterpret_cast<uint4*>(out + e) = pk;
      } else {
#pragma unroll
        for (int u = 0; u < V; u++)
          if (e + u >= E0 && e + u < E1) out[e + u] = vals[u];
      }
    }
    __syncthreads();
    st ^= 1;
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(a.err, DEVERR_TIMEOUT);
      // the copy for the other stage may still be in flight: wait for it (bounded) before exit
      if (s_tile[st ^ 1] < a.t_end) mbar_wait_bounded(&bars[st ^ 1], phase[st ^ 1]);
    }
    __syncthreads();
  }
}

template <typename T, bool PLAIN, bool RESID>
static cudaError_t run_decode(glc_ctx* ctx, const DecodeArgs& a0, bool vec, cudaStream_t s) {
  DecodeArgs a = a0;
  const size_t smem = 2 * (size_t)a.stage_bytes;
  void (*kern)(DecodeArgs) = vec ? decode_kernel<T, PLAIN, RESID, true> : decode_kernel<T, PLAIN, RESID, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kDecodeThreads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  const int64_t ntile = a.t_end - a.t_begin;
  int64_t grid = (int64_t)per_sm * ctx->num_sms;
  if (grid > ntile) grid = ntile;
  if (grid < 1) return cudaSuccess;
  if ((e = cudaMemsetAsync(a.counter, 0, sizeof(int), s)) != cudaSuccess) return e;
  kern<<<(unsigned)grid, kDecodeThreads, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T>
static cudaError_t decode_typed(glc_ctx* ctx, const DecodeArgs& a, int plain, int resid, bool vec, cudaStream_t s) {
  if (plain) return resid ? run_decode<T, true, true>(ctx, a, vec, s) : run_decode<T, true, false>(ctx, a, vec, s);
  return resid ? run_decode<T, false, true>(ctx, a, vec, s) : run_decode<T, false, false>(ctx, a, vec, s);
}

cudaError_t launch_decode(glc_ctx* ctx, const glc_column* c, int plain_src, int residual_out, int64_t lo, int64_t hi,
                          void* out_base, cudaStream_t s) {
  if (hi <= lo || c->n <= 0) return cudaSuccess;
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
  if (plain_src) {
    a.stage_bytes = kDecodeTile * 8 + 16;
  } else {
    int64_t words = ((int64_t)kDecodeTile * c->max_bits + 31) / 32 + 16;
    a.stage_bytes = (int)(((words + 3) & ~3ll) * 4);
  }
  const bool vec = ((uintptr_t)out_base % 16) == 0;
  switch (c->dtype) {
    case GLC_I32: return decode_typed<int32_t>(ctx, a, plain_src, residual_out, vec, s);
    case GLC_I64: return decode_typed<int64_t>(ctx, a, plain_src, residual_out, vec, s);
    case GLC_U64: return decode_typed<uint64_t>(ctx, a, plain_src, residual_out, vec, s);
    case GLC_U32: return decode_typed<uint32_t>(ctx, a, plain_src, residual_out, vec, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace glc
