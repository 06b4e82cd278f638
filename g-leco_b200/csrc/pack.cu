// pack.cu -- warp-cooperative bit-packer.
//
// Replaces compression/CompressionKernels.cuh:242-372 (packDeltasKernelOptimized: one value per
// thread, a binary search over partitions per value and 1-3 atomicOr per value into a word
// array that a separate memset pass zeroed first).
//
// Here the OUTPUT words are the unit of work.  A CTA owns a tile of 2048 consecutive words
// (8 KB) and builds it in shared memory:
//   * a binary search finds the first partition whose bit range reaches the tile; the CTA
//     walks partitions while their bit ranges start inside the tile;
//   * for each partition, the values whose fields touch the tile are taken in groups of 32
//     consecutive values, one per lane (coalesced loads); each lane computes its residual field;
//   * the group's fields occupy a contiguous run of 32*b bits, i.e. at most b+1 words.  Lane l
//     builds word l of that run by pulling the (at most ceil(32/b)+1) fields that overlap it
//     with __shfl_sync and shifting each into place (funnel shifts), so every word is
//     assembled in registers and reaches shared memory with one conflict-free atomicOr
//     (atomics only reconcile words shared by adjacent groups or partitions);
//   * the finished tile is written with coalesced 128-bit stores, padding words included, so
//     every word of the array is written exactly once and no memset pass is needed.
// Values whose fields straddle two tiles are computed by both CTAs; each keeps its own bits.
#include "glc_internal.h"

namespace glc {

constexpr int kPackWords = 2048;
constexpr int kPackThreads = 256;
constexpr int kPackWarps = kPackThreads / 32;

__device__ __forceinline__ int64_t end_bit(const PackArgs& a, int64_t p) {
  return a.offs[p] + ((int64_t)a.ends[p] - a.starts[p]) * (int64_t)a.bits[p];
}

// Builds output word tile `tile` (kPackWords words) of one column; every thread of the CTA calls it.
template <typename T> __device__ __forceinline__ void pack_word_tile(const T* __restrict__ v, const PackArgs& a,
                                                                    int64_t tile) {
  __shared__ __align__(16) uint32_t s_tile[kPackWords];
  __shared__ int64_t s_plo;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t W0 = tile * kPackWords;
  const int64_t W1 = (W0 + kPackWords < a.nwords_alloc) ? W0 + kPackWords : a.nwords_alloc;
  const int tile_words = (int)(W1 - W0);
  const int64_t B0 = W0 * 32, B1 = W1 * 32;

  for (int k = threadIdx.x; k < kPackWords; k += kPackThreads) s_tile[k] = 0u;
  if (threadIdx.x == 0) {
    // first partition whose bit range ends after B0
    int64_t lo = 0, hi = a.P;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (end_bit(a, mid) > B0) hi = mid; else lo = mid + 1;
    }
    s_plo = lo;
  }
  __syncthreads();

  for (int64_t p = s_plo; p < a.P; p++) {
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
    if (i_lo >= i_hi) continue;
    const int64_t ngroups = (i_hi - i_lo + 31) >> 5;
    const int nj = min(32, (31 + b) / b + 1);  // fields that can overlap one word

    for (int64_t g = warp; g < ngroups; g += kPackWarps) {
      const int64_t gi = i_lo + (g << 5);
      const int64_t i = gi + lane;
      const int nvalid = (i_hi - gi) < 32 ? (int)(i_hi - gi) : 32;
      uint64_t field = 0;
      if (lane < nvalid) {
        T x = __ldg(v + start + i);
        field = direct ? (uint64_t)x : (uint64_t)calc_delta<T>(x, predict<T>(t0, t1, i));
        field = low_bits(field, b);
      }
      const int64_t R0 = off + gi * b - B0;               // bit of lane 0's field, tile-relative
      const int64_t wf = R0 >> 5;                          // floor
      const int64_t wl = (R0 + (int64_t)nvalid * b - 1) >> 5;
      const int nw = (int)(wl - wf + 1);
      for (int r = 0; r < nw; r += 32) {
        const int64_t wrel = wf + r + lane;
        const bool wvalid = wrel <= wl;
        const int64_t x = 32 * wrel - R0;                  // word start, group-relative bit
        int k0 = (x <= 0 || !wvalid) ? 0 : (int)(x / b);
        uint32_t word = 0u;
        if (b <= 32) {
          const uint32_t f32 = (uint32_t)field;
          for (int j = 0; j < nj; j++) {
            const int k = k0 + j;
            const uint32_t val = __shfl_sync(FULL_MASK, f32, k & 31);
            const int64_t sh = R0 + (int64_t)k * b - 32 * wrel;
            if (wvalid && k < nvalid && sh > -b && sh < 32)
              word |= (sh >= 0) ? __funnelshift_l(0u, val, (int)sh) : __funnelshift_r(val, 0u, (int)-sh);
          }
        } else {
          const uint32_t flo = (uint32_t)field, fhi = (uint32_t)(field >> 32);
          for (int j = 0; j < nj; j++) {
            const int k = k0 + j;
            const uint32_t vlo = __shfl_sync(FULL_MASK, flo, k & 31);
            const uint32_t vhi = __shfl_sync(FULL_MASK, fhi, k & 31);
            const int64_t sh = R0 + (int64_t)k * b - 32 * wrel;
            if (wvalid && k < nvalid && sh > -b && sh < 32) {
              const uint64_t val = ((uint64_t)vhi << 32) | vlo;
              word |= (sh >= 0) ? (uint32_t)(val << sh) : (uint32_t)(val >> (-sh));
            }
          }
        }
        if (wvalid && wrel >= 0 && wrel < tile_words && word != 0u) atomicOr(&s_tile[wrel], word);
      }
    }
  }
  __syncthreads();
  uint4* dst = reinterpret_cast<uint4*>(a.words + W0);
  const uint4* src = reinterpret_cast<const uint4*>(s_tile);
  for (int k = threadIdx.x; k < tile_words / 4; k += kPackThreads) dst[k] = src[k];
}

template <typename T> __global__ void __launch_bounds__(kPackThreads) pack_kernel(const T* __restrict__ v, PackArgs a) {
  pack_word_tile<T>(v, a, blockIdx.x);
}

cudaError_t launch_pack(glc_dtype dt, const void* values, glc_column* c, cudaStream_t s) {
  if (c->nwords_alloc <= 0) return cudaSuccess;
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

// Batched pack: one CTA per output word tile of any column of a batch (PackArgs per column).
__global__ void __launch_bounds__(kPackThreads)
batch_pack_kernel(const PackArgs* __restrict__ cols, const void* const* __restrict__ values,
                  const int32_t* __restrict__ dtypes, const int64_t* __restrict__ tile_base, int ncols) {
  const int64_t t = blockIdx.x;
  int lo = 0, hi = ncols - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile_base[mid] <= t) lo = mid; else hi = mid - 1;
  }
  const PackArgs a = cols[lo];
  const int64_t tile = t - tile_base[lo];
  switch (dtypes[lo]) {
    case GLC_I32: pack_word_tile<int32_t>((const int32_t*)values[lo], a, tile); break;
    case GLC_I64: pack_word_tile<int64_t>((const int64_t*)values[lo], a, tile); break;
    case GLC_U64: pack_word_tile<uint64_t>((const uint64_t*)values[lo], a, tile); break;
    default: pack_word_tile<uint32_t>((const uint32_t*)values[lo], a, tile); break;
  }
}

int64_t pack_tiles(int64_t nwords_alloc) { return (nwords_alloc + kPackWords - 1) / kPackWords; }

cudaError_t launch_batch_pack(const PackArgs* cols, const void* const* values, const int32_t* dtypes,
                              const int64_t* tile_base, int ncols, int64_t total_tiles, cudaStream_t s) {
  if (total_tiles <= 0) return cudaSuccess;
  batch_pack_kernel<<<(unsigned)total_tiles, kPackThreads, 0, s>>>(cols, values, dtypes, tile_base, ncols);
  return cudaGetLastError();
}

}  // namespace glc
