// compress_fixed.cu -- one-pass compression of a column with fixed partitions whose length L
// divides the 4096-value tile and is at least 256 (L = 256, 512, 1024, 2048, 4096; the
// reference's TILE_SIZE is 4096, core/CudaUtils.cuh:18).
//
// Replaces, for those columns, the separate fit, bit-offset scan, table build and pack passes
// (fit.cu, glc_scan.cuh, pack.cu; in the reference wprocessPartitionsKernel,
// setBitOffsetsKernel and packDeltasKernelOptimized, compression/CompressionKernels.cuh:45-372,
// which read the values four times) with ONE persistent kernel that reads every value once:
//
//   producer warp   stages tile t's values in shared memory with cp.async.bulk, three stages
//                   (full/empty mbarriers, bounded waits that sleep in the barrier);
//   solver warp     fits the lines of tile k + 1 from its exact sums (one lane per partition, the
//                   same arithmetic as fit.cu, so the result is identical bit for bit) and picks
//                   each partition's residual mode, while the compute warps work on tile k;
//   compute warps   per step, with every partition inside the tile (L divides 4096):
//     A  exact sums of tile k + 1 per partition from 64-bit partials of 32-bit halves, and the
//        range flags (direct copy; FP64-safe values); a group of L/16 threads owns a partition,
//        16 values each;
//     B  the residual of every value of tile k (fma prediction, round half away from zero,
//        saturating cast; calculateDelta -- in FP64 without conversion instructions where the
//        line and the values allow it) and max |residual| per partition -> the bit widths;
//     C  the tile's words into its own slot of a scratch array (slots of the worst-case size of
//        a tile, bit offsets relative to the tile), the partitions' descriptors with
//        tile-relative offsets and their max errors, and the tile's bit count;
//   then an exclusive scan of the tiles' bit counts gives every tile's first bit, and
//   fixed_place_kernel (one CTA per tile) copies each tile's words to their place in the column
//   and writes the metadata arrays from the descriptors.  No tile waits for another.
//
// The column's word array is allocated at its exact size between the two kernels (the scan gives
// the total); the slots cost one extra write and read of the compressed bits.
#include <type_traits>
#include "glc_internal.h"
#include "glc_scan.cuh"
#include "glc_tma.cuh"

namespace glc {

constexpr int kCfThreads = 256;                       // compute threads (8 warps)
constexpr int kCfMinLen = 256;
constexpr int kCfMaxParts = kDecodeTile / kCfMinLen;  // 16 partitions per tile at L = 256
constexpr int kCfPerThread = kDecodeTile / kCfThreads;  // 16 values per thread
constexpr int kCfMaxSegs = 16;                        // reduction segments (half-warps at L = 256)

// The work area of the packing: the transposed fields (32 x 129 words) and the staged words (4096
// plus a pad word per 32), or the 64-bit residuals of the wide-field path (4096 x 8 bytes).
constexpr int kCfWorkBytes = (32 * 129 + kDecodeTile + kDecodeTile / 32) * 4;
static_assert(kCfWorkBytes >= kDecodeTile * 8, "the work area holds a tile's 64-bit residuals");
// A stage holds a tile's values from the 16-byte block of the first one; for 8-byte types it is
// also the work area of its tile.
template <typename T> __host__ __device__ constexpr int cf_stage_bytes() {
  return sizeof(T) == 8 ? kCfWorkBytes : kDecodeTile * (int)sizeof(T) + 16;
}

// A launch: work item i = one 4096-value tile of column owner[i] (every column of one element
// type, tiles in order), or of `single` when cols is null.
struct FixedCompressArgs {
  const CfColumn* cols;
  const int32_t* owner;
  CfColumn single;
  int64_t nitems;
  uint32_t* slots;            // item i's words at slots + i * slot_words (tile-relative bits)
  int64_t slot_words;
  int64_t* tile_bits;         // per item: bits of the tile (nitems + 1 entries: the scan's input)
  const int64_t* tile_first;  // per item: exclusive scan of tile_bits over the launch (nitems + 1)
  unsigned long long* status; // DEVERR_* when a bounded wait gave up or a column's words overflow
  PartDesc* tdesc;            // the length choice that also packs at 4096: per item, the tile's one
  long long* terr;            // partition's descriptor (tile-relative offset) and max error
};

__device__ __forceinline__ void cf_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kCfThreads) : "memory"); }
// cf_sync that also returns whether any compute thread passed true.
__device__ __forceinline__ bool cf_sync_or(bool v) {
  uint32_t r;
  asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 q, %1, 0;\n bar.red.or.pred p, 1, %2, q;\n selp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(r)
               : "r"((uint32_t)v), "n"(kCfThreads)
               : "memory");
  return r != 0;
}

// The producer lane of a launch: stages item blockIdx.x + k * gridDim.x of the work list into stage
// k % S (its values, from the 16-byte block that holds the first one), with the item, its
// column and the offset of its first value in the stage; an item of -1 marks the end.
template <typename T, int S>
__device__ __forceinline__ void cf_produce(const FixedCompressArgs& a, uint8_t* smem, uint64_t* full, uint64_t* empty,
                                           int64_t* s_stile, int* s_shead, int* s_scol) {
  int64_t item = blockIdx.x;
  for (int k = 0;; k++, item += gridDim.x) {
    const int st = k % S;
    if (k >= S && !mbar_wait_sleep(&empty[st], (uint32_t)((k / S) - 1) & 1u)) {
      atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
      s_stile[st] = -1;  // the compute warps stop at this stage (or time out on it)
      mbar_arrive(&full[st]);
      return;
    }
    if (item >= a.nitems) {
      s_stile[st] = -1;
      mbar_arrive(&full[st]);  // no copy: completes the phase, the compute warps see the end
      return;
    }
    const int c = a.owner ? a.owner[item] : 0;
    const CfColumn& col = a.cols ? a.cols[c] : a.single;
    const int64_t e0 = (item - col.item_base) * kDecodeTile;
    const int cnt = (int)((col.n - e0) < kDecodeTile ? (col.n - e0) : kDecodeTile);
    const uintptr_t addr = reinterpret_cast<uintptr_t>(reinterpret_cast<const T*>(col.values) + e0);
    const int head = (int)(addr & 15);
    s_stile[st] = item;
    s_shead[st] = head;
    s_scol[st] = c;
    // the copy covers the 16-byte blocks that hold the tile's values, never another page
    const uint32_t bytes = (uint32_t)((head + (int64_t)cnt * (int64_t)sizeof(T) + 15) & ~15ll);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive_expect_tx(&full[st], bytes);
    tma_bulk_load(smem + (size_t)st * cf_stage_bytes<T>(), reinterpret_cast<const void*>(addr - head), bytes,
                  &full[st]);
  }
}

// ---- pieces of the compute warps -----------------------------------------------------------

constexpr double kMagic = 6755399441055744.0;        // K = 1.5 * 2^52: the bits of K + v are 0x4338... + v, |v| <= 2^51
constexpr double kHalfBias = 0x1.fffffffffffffp-2;    // 0.5 - 2^-54
constexpr int kFtStride = 129;                        // transposed fields: field f of 32-value group G at f * 129 + G
constexpr int kFtWords = 32 * kFtStride;
constexpr int kStgWords = kDecodeTile + kDecodeTile / 32;  // a tile's words, one pad word after every 32

// How a partition's residuals are computed (uniform per partition, so per thread):
//   CF_DIRECT   direct copy (a uint64 value above 2^53): the field is the value;
//   CF_NONNEG   |y| < 2^51 and predictions in [-0.25, 2^51] (4-byte types: inside the type): in
//               FP64 with K: K + y from the bits, K + pred = (x + (0.5 - 2^-54)) + K rounded toward
//               zero, their difference is y - pred exactly;
//   CF_NONPOS   the mirror for signed types, predictions in [-2^51, 0.25]: K - pred =
//               ((0.5 - 2^-54) - x) + K rounded toward zero;
//   CF_OFFSET   8-byte types with predictions in [2^50, 2^62] within 2^50 of c = trunc(theta0):
//               x - c and x - c + 0.5 are exact, pred = c + floor(x - c + 0.5), y - c by integer
//               arithmetic (a thread whose |y - c| reaches 2^51 recomputes its values in general);
//   CF_GENERAL  predict_from / calc_delta / abs_ref per value.
// Each gives calc_delta<T>(y, predict_from<T>(fma(theta1, i, theta0))) exactly; the field is its
// low 32 bits (the low bits of (y - pred) + K), which is all the packing of a width <= 31 reads.
enum : int { CF_DIRECT = 0, CF_NONNEG = 1, CF_NONPOS = 2, CF_GENERAL = 3, CF_OFFSET = 4 };

// Exact sum over a reduction segment of W lanes (32, or 16 at L = 256) of values |v| < 2^48: for a
// whole warp two redux sums of the 24-bit limbs (each limb's sum stays below 2^29).
__device__ __forceinline__ long long seg_sum48(long long v, int W) {
  if (W == 32) {
    const unsigned lo = __reduce_add_sync(FULL_MASK, (unsigned)v & 0xFFFFFFu);
    const int hi = __reduce_add_sync(FULL_MASK, (int)(v >> 24));
    return (long long)hi * 16777216ll + (long long)lo;
  }
  for (int msk = W >> 1; msk > 0; msk >>= 1) v += __shfl_xor_sync(FULL_MASK, v, msk);
  return v;
}
__device__ __forceinline__ unsigned seg_max_u32(unsigned v, int W) {
  if (W == 32) return __reduce_max_sync(FULL_MASK, v);
  for (int msk = W >> 1; msk > 0; msk >>= 1) {
    const unsigned o = __shfl_xor_sync(FULL_MASK, v, msk);
    v = o > v ? o : v;
  }
  return v;
}
__device__ __forceinline__ unsigned seg_or_u32(unsigned v, int W) {
  if (W == 32) return __reduce_or_sync(FULL_MASK, v);
  for (int msk = W >> 1; msk > 0; msk >>= 1) v |= __shfl_xor_sync(FULL_MASK, v, msk);
  return v;
}
__device__ __forceinline__ unsigned long long seg_max_u64(unsigned long long v, int W) {
  const unsigned hi = seg_max_u32((unsigned)(v >> 32), W);
  const unsigned lo = seg_max_u32((unsigned)(v >> 32) == hi ? (unsigned)v : 0u, W);
  return ((unsigned long long)hi << 32) | lo;
}

// Per value, for the range tests of the partition: uint64 keeps the max of the high words, above
// 2^21 when some value exceeds 2^53 (direct copy; exactly 2^21 is decided by a rescan of the
// partition, cf_any_above_2_53) and below 2^19 iff every value is below 2^51; int64 keeps the OR of
// hi ^ (hi >> 31), below 2^19 iff every value is in [-2^51, 2^51); 4-byte values always fit.
template <typename T> __device__ __forceinline__ void value_flag(uint32_t& f, T y) {
  if (sizeof(T) == 8) {
    const uint32_t hi = (uint32_t)((uint64_t)y >> 32);
    if (TypeTraits<T>::is_signed) f |= hi ^ (uint32_t)((int32_t)hi >> 31);
    else f = hi > f ? hi : f;
  }
}
// Whether a uint64 partition whose largest high word is exactly 2^21 holds a value above 2^53.
template <typename T> __device__ __noinline__ bool cf_any_above_2_53(const T* __restrict__ xp, int len) {
  for (int i = 0; i < len; i++)
    if ((uint64_t)xp[i] > (1ull << 53)) return true;
  return false;
}
// Direct copy for the range flag of a partition (the reference copies a uint64 partition with a
// value above 2^53 directly).
template <typename T> __device__ __forceinline__ bool cf_overflows(uint32_t flag, const T* __restrict__ xp, int len) {
  if (TypeTraits<T>::is_signed || sizeof(T) != 8) return false;
  return flag > 0x200000u || (flag == 0x200000u && cf_any_above_2_53<T>(xp, len));
}

// K + y as a double from the bits of y (|y| <= 2^51).
template <typename T> __device__ __forceinline__ double magic_of(T y) {
  if (sizeof(T) == 8) {
    const uint64_t u = (uint64_t)y;
    return __hiloint2double((int)((uint32_t)(u >> 32) + 0x43380000u), (int)(uint32_t)u);
  } else if (TypeTraits<T>::is_signed) {
    return __hiloint2double((int)(0x43380000u + (uint32_t)((int32_t)y >> 31)), (int)y);
  } else {
    return __hiloint2double(0x43380000, (int)(uint32_t)y);
  }
}
__device__ __forceinline__ uint32_t low_field(double d) { return (uint32_t)__double2loint(__dadd_rn(d, kMagic)); }

__device__ __forceinline__ uint64_t madw_u(uint32_t a, uint32_t b, uint64_t c) {
  uint64_t d;
  asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"(b), "l"(c));
  return d;
}
__device__ __forceinline__ int64_t madw_s(int32_t a, int32_t b, int64_t c) {
  int64_t d;
  asm("mad.wide.s32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"(b), "l"(c));
  return d;
}

// The HalfSums of a thread's values y_m = xp[r + g m] (m < 16), without the index per value:
// sum (r + g m) y_m = r sum y_m + g sum m y_m, each sum accumulated by one 32 x 32 -> 64-bit
// multiply-add per value and half (m is a compile-time constant); every partial stays below 2^48.
template <typename T, bool FULL>
__device__ __forceinline__ void cf_sums(const T* __restrict__ xp, int r, int g, int len, HalfSums<T>& hs,
                                        uint32_t& flag) {
  typedef typename HalfSums<T>::Acc Acc;
  Acc s_lo = 0, s_hi = 0, t_lo = 0, t_hi = 0;
  const T* p = xp + r;
#pragma unroll
  for (int m = 0; m < kCfPerThread; m++) {
    if (FULL || r + g * m < len) {
      const T y = p[g * m];
      value_flag<T>(flag, y);
      if (sizeof(T) == 8) {
        const uint32_t yl = (uint32_t)(uint64_t)y, yh = (uint32_t)((uint64_t)y >> 32);
        s_lo = (Acc)madw_u(yl, 1u, (uint64_t)s_lo);
        if (m) t_lo = (Acc)madw_u(yl, (uint32_t)m, (uint64_t)t_lo);
        if (TypeTraits<T>::is_signed) {
          s_hi = (Acc)madw_s((int32_t)yh, 1, (int64_t)s_hi);
          if (m) t_hi = (Acc)madw_s((int32_t)yh, m, (int64_t)t_hi);
        } else {
          s_hi = (Acc)madw_u(yh, 1u, (uint64_t)s_hi);
          if (m) t_hi = (Acc)madw_u(yh, (uint32_t)m, (uint64_t)t_hi);
        }
      } else if (TypeTraits<T>::is_signed) {
        s_lo = (Acc)madw_s((int32_t)y, 1, (int64_t)s_lo);
        if (m) t_lo = (Acc)madw_s((int32_t)y, m, (int64_t)t_lo);
      } else {
        s_lo = (Acc)madw_u((uint32_t)y, 1u, (uint64_t)s_lo);
        if (m) t_lo = (Acc)madw_u((uint32_t)y, (uint32_t)m, (uint64_t)t_lo);
      }
    }
  }
  hs.s_lo += s_lo;
  hs.s_hi += s_hi;
  hs.x_lo += (Acc)r * s_lo + (Acc)g * t_lo;
  hs.x_hi += (Acc)r * s_hi + (Acc)g * t_hi;
}

template <typename T, bool FULL, bool NEG>
__device__ __forceinline__ unsigned long long cf_resid_sign(const T* __restrict__ xp, int r, int g, int len,
                                                            double t0, double t1, uint32_t (&fl)[kCfPerThread]) {
  double dm = 0.0, xd = (double)r;
  const double gd = (double)g;
#pragma unroll
  for (int m = 0; m < kCfPerThread; m++) {
    const int i = r + g * m;
    fl[m] = 0u;
    if (FULL || i < len) {
      const double yc = magic_of<T>(xp[i]);
      const double x = __fma_rn(t1, xd, t0);
      double d;
      if (!NEG) {
        d = __dsub_rn(yc, __dadd_rz(__dadd_rn(x, kHalfBias), kMagic));  // (K + y) - (K + pred)
      } else {
        d = __dadd_rn(__dsub_rn(yc, 2.0 * kMagic), __dadd_rz(__dsub_rn(kHalfBias, x), kMagic));  // (y - K) + (K - pred)
      }
      dm = fmax(dm, fabs(d));
      fl[m] = low_field(d);
    }
    xd = __dadd_rn(xd, gd);
  }
  return (unsigned long long)dm;
}

template <typename T, bool FULL>
__device__ __forceinline__ bool cf_resid_offset(const T* __restrict__ xp, int r, int g, int len, double t0,
                                                double t1, double c, long long ci, uint32_t (&fl)[kCfPerThread],
                                                unsigned long long& mx) {
  double dm = 0.0, xd = (double)r;
  const double gd = (double)g;
  uint32_t range = 0u;
#pragma unroll
  for (int m = 0; m < kCfPerThread; m++) {
    const int i = r + g * m;
    fl[m] = 0u;
    if (FULL || i < len) {
      const uint64_t yo = (uint64_t)xp[i] - (uint64_t)ci;  // y - c
      const uint32_t yh = (uint32_t)(yo >> 32);
      range |= yh ^ (uint32_t)((int32_t)yh >> 31);
      const double yk = __hiloint2double((int)(yh + 0x43380000u), (int)(uint32_t)yo);  // K + (y - c)
      const double v = __dadd_rn(__dsub_rn(__fma_rn(t1, xd, t0), c), 0.5);          // x - c + 0.5
      const double d = __dsub_rn(yk, __dadd_rz(v, kMagic));                          // - (K + pred - c)
      dm = fmax(dm, fabs(d));
      fl[m] = low_field(d);
    }
    xd = __dadd_rn(xd, gd);
  }
  mx = (unsigned long long)dm;
  return range < 0x80000u;  // every |y - c| below 2^51 (y - c in [-2^51, 2^51))
}

template <typename T>
__device__ __forceinline__ unsigned long long cf_resid_general(const T* __restrict__ xp, int r, int g, int len,
                                                               double t0, double t1, uint32_t (&fl)[kCfPerThread]) {
  unsigned long long mx = 0;
#pragma unroll
  for (int m = 0; m < kCfPerThread; m++) {
    const int i = r + g * m;
    fl[m] = 0u;
    if (i < len) {
      const long long d = calc_delta<T>(xp[i], predict_from<T>(__fma_rn(t1, (double)i, t0)));
      fl[m] = (uint32_t)d;
      const unsigned long long ad = (unsigned long long)abs_ref(d);
      mx = ad > mx ? ad : mx;
    }
  }
  return mx;
}

// The residual mode of a partition from its line and the range test of its values.
template <typename T>
__device__ __forceinline__ int cf_mode(double t0, double t1, int len, bool vsafe, double& c, long long& ci) {
  const double xa = t0, xb = __fma_rn(t1, (double)(len - 1), t0);  // the ends (fma is monotone in i)
  const double lo = fmin(xa, xb), hi = fmax(xa, xb);
  constexpr double kS = 2251799813685248.0;  // 2^51
  const double hi_ok = sizeof(T) == 4 ? (TypeTraits<T>::is_signed ? 2147483646.0 : 4294967294.0) : kS;
  const double lo_ok = sizeof(T) == 4 ? -2147483647.0 : -kS;
  if (vsafe && lo >= -0.25 && hi <= hi_ok) return CF_NONNEG;
  if (TypeTraits<T>::is_signed && vsafe && hi <= 0.25 && lo >= lo_ok) return CF_NONPOS;
  if (sizeof(T) == 8 && lo >= 1125899906842624.0 && hi <= 4611686018427387904.0) {  // [2^50, 2^62]
    c = trunc(t0);
    if (fabs(__dsub_rn(xb, c)) < 562949953421312.0) {  // 2^49
      ci = __double2ll_rz(c);
      return CF_OFFSET;
    }
  }
  return CF_GENERAL;
}

// Packs the 32 fields of one group (width B, 1..31, at fg[f * kFtStride]) into B words at staged
// word o onward (staged word k at stg[k + k / 32]).
template <int B>
__device__ __forceinline__ void cf_pack_group(const uint32_t* __restrict__ fg, uint32_t* __restrict__ stg, int o) {
  constexpr uint32_t kMask = (1u << B) - 1u;
  uint32_t w = 0u;
#pragma unroll
  for (int f = 0; f < 32; f++) {
    const uint32_t v = fg[f * kFtStride] & kMask;
    const int sh = (f * B) & 31;
    w |= v << sh;
    if (sh + B >= 32) {
      const int k = o + ((f * B) >> 5);
      stg[k + (k >> 5)] = w;
      w = sh + B > 32 ? v >> (32 - sh) : 0u;
    }
  }
}

__device__ __forceinline__ void cf_pack_dispatch(int b, const uint32_t* __restrict__ fg, uint32_t* __restrict__ stg,
                                              int o) {
  switch (b) {
#define GLC_CF_PACK(B) \
  case B: cf_pack_group<B>(fg, stg, o); break;
    GLC_CF_PACK(1) GLC_CF_PACK(2) GLC_CF_PACK(3) GLC_CF_PACK(4) GLC_CF_PACK(5) GLC_CF_PACK(6) GLC_CF_PACK(7)
    GLC_CF_PACK(8) GLC_CF_PACK(9) GLC_CF_PACK(10) GLC_CF_PACK(11) GLC_CF_PACK(12) GLC_CF_PACK(13) GLC_CF_PACK(14)
    GLC_CF_PACK(15) GLC_CF_PACK(16) GLC_CF_PACK(17) GLC_CF_PACK(18) GLC_CF_PACK(19) GLC_CF_PACK(20)
    GLC_CF_PACK(21) GLC_CF_PACK(22) GLC_CF_PACK(23) GLC_CF_PACK(24) GLC_CF_PACK(25) GLC_CF_PACK(26)
    GLC_CF_PACK(27) GLC_CF_PACK(28) GLC_CF_PACK(29) GLC_CF_PACK(30) GLC_CF_PACK(31)
#undef GLC_CF_PACK
    default: break;  // width 0: no words
  }
}

// The words of a partition of width b (1..64) whose exact residuals are rp[0, len), one thread per
// word: word w holds the partition's bits [32 w, 32 w + 32), from the field holding bit 32 w and
// the following ones (fields past len are zero).  One routine for every width (the wide-field path
// is taken by a few tiles; a copy per width made the kernels' code several times larger than the
// instruction cache).
__device__ __noinline__ void cf_words_dispatch(int b, const long long* rp, int len, uint32_t* __restrict__ out,
                                               int tid) {
  if (b <= 0) return;
  const int nwp = (int)(((long long)len * b + 31) >> 5);
  const uint32_t mb = 0xffffffffu / (uint32_t)b + 1u;  // 32 w / b by a multiply-high (32 w < 2^18)
  const uint64_t mask = b >= 64 ? ~0ull : ((1ull << b) - 1ull);
  for (int w = tid; w < nwp; w += kCfThreads) {
    int j = b > 1 ? (int)__umulhi((uint32_t)(32 * w), mb) : 32 * w;
    const int s = 32 * w - j * b;
    uint64_t v = ((uint64_t)rp[j] & mask) >> s;
    int have = b - s;
    while (have < 32 && ++j < len) {
      v |= ((uint64_t)rp[j] & mask) << have;
      have += b;
    }
    out[w] = (uint32_t)v;
  }
}

// The exact residuals of one thread's values (value i of its partition at xp[i], written to rp[i];
// for 8-byte types rp is xp, each value read before its residual replaces it).  The FP64 modes give
// y - pred as an exact integer-valued double, converted once; the others use the integer formula.
template <typename T>
__device__ __forceinline__ void cf_store_resid(const T* xp, long long* rp, int r, int g, int len, int mode, double t0,
                                               double t1) {
  for (int m = 0; m < kCfPerThread; m++) {
    const int i = r + g * m;
    if (i >= len) break;
    const T y = xp[i];
    long long d;
    if (mode == CF_DIRECT) {
      d = (long long)(uint64_t)y;  // the field is the value itself (zero-extended)
    } else if (mode == CF_NONNEG) {
      const double x = __fma_rn(t1, (double)i, t0);
      d = __double2ll_rn(__dsub_rn(magic_of<T>(y), __dadd_rz(__dadd_rn(x, kHalfBias), kMagic)));
    } else if (TypeTraits<T>::is_signed && mode == CF_NONPOS) {
      const double x = __fma_rn(t1, (double)i, t0);
      d = __double2ll_rn(
          __dadd_rn(__dsub_rn(magic_of<T>(y), 2.0 * kMagic), __dadd_rz(__dsub_rn(kHalfBias, x), kMagic)));
    } else {
      d = calc_delta<T>(y, predict_from<T>(__fma_rn(t1, (double)i, t0)));
    }
    rp[i] = d;
  }
}

// The compress kernel's CTA: eight compute warps, the producer warp and the solver warp.  Per step
// k the compute warps take the sums of tile k + 1 and the residuals, widths and words of tile k,
// while the solver warp fits the lines of tile k + 1 (one lane per partition) and the producer
// stages the next tile as soon as a stage is free: the fit's long dependency chain (128-bit
// arithmetic, two divisions) runs beside the compute warps instead of between two of their
// barriers.  Every wait is bounded.  The compress kernel runs two stages at three CTAs per SM (64
// registers; measured 5 % faster than three stages at two CTAs per SM: other CTAs cover the load
// of the next tile); the length choice, with heavier per-value work, three stages at two (two
// stages at three CTAs per SM fit its registers too, but measured 3 % slower).
constexpr int kCfCompressStages = 2;
constexpr int kCfChooseStages = 3;
constexpr int kCfFixCTA = kCfThreads + 64;

template <typename T> __host__ __device__ constexpr int cf_fix_smem_bytes(int stages) {
  return stages * cf_stage_bytes<T>() + (sizeof(T) == 4 ? kCfWorkBytes : 0);
}

// A tile as a step sees it.
struct CfGeom {
  const CfColumn* col;
  int64_t t, e0;
  int L, g, W, cnt, np, segs_per_part;
  int lg_L, lg_g, lg_W;  // L, g and W are powers of two: divisions are shifts
};
__device__ __forceinline__ CfGeom cf_geom(const FixedCompressArgs& a, int64_t item, int c) {
  CfGeom q;
  q.col = a.cols ? a.cols + c : &a.single;
  q.t = item - q.col->item_base;
  q.e0 = q.t * kDecodeTile;
  const int64_t left = q.col->n - q.e0;
  q.cnt = (int)(left < kDecodeTile ? left : kDecodeTile);
  q.L = q.col->L;
  q.lg_L = 31 - __clz(q.L);
  q.g = q.L >> 4;
  q.lg_g = q.lg_L - 4;
  q.W = q.g < 32 ? q.g : 32;
  q.lg_W = q.lg_g < 5 ? q.lg_g : 5;
  q.np = (q.cnt + q.L - 1) >> q.lg_L;
  q.segs_per_part = q.g >> q.lg_W;
  return q;
}

template <typename T> __global__ void __launch_bounds__(kCfFixCTA, 3)
fixed_compress_kernel(const __grid_constant__ FixedCompressArgs a) {
  constexpr int S = kCfCompressStages;
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t full[S], empty[S], sums[S], lines[S];
  __shared__ int64_t s_stile[S];   // work item staged in each stage (-1: the end)
  __shared__ int s_shead[S];
  __shared__ int s_scol[S];
  __shared__ long long s_acc[S][kCfMaxSegs][4];   // per stage: the segments' exact partial sums
  __shared__ uint32_t s_flag[S][kCfMaxSegs];      // and range flags
  __shared__ double s_t0[S][kCfMaxParts], s_t1[S][kCfMaxParts], s_c[S][kCfMaxParts];  // the solver's lines
  __shared__ long long s_ci[S][kCfMaxParts];
  __shared__ int s_mode[S][kCfMaxParts];
  __shared__ unsigned long long s_mx[kCfMaxSegs];
  __shared__ int s_b[kCfMaxParts];
  __shared__ int s_bl[kCfMaxParts + 1];
  __shared__ int s_ok;

  if (threadIdx.x == 0) {
    for (int st = 0; st < S; st++) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
      mbar_init(&sums[st], kCfThreads / 32);
      mbar_init(&lines[st], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  const int tid = threadIdx.x, lane = tid & 31;
  if (tid >= kCfThreads + 32) {  // ---- solver warp ----
    for (int k = 0;; k++) {
      const int st = k % S;
      int ok = 1;
      if (lane == 0) {
        ok = mbar_wait_sleep(&sums[st], (uint32_t)(k / S) & 1u);
        if (!ok) atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
      }
      if (!__shfl_sync(FULL_MASK, ok, 0)) return;
      const int64_t item = s_stile[st];
      if (item < 0) return;
      const CfGeom q = cf_geom(a, item, s_scol[st]);
      if (lane < q.np) {  // lane p fits partition p (fit.cu's arithmetic) and picks its residual mode
        const int p = lane;
        long long a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        uint32_t flag = 0;
        for (int s = p * q.segs_per_part; s < (p + 1) * q.segs_per_part; s++) {
          a0 += s_acc[st][s][0];
          a1 += s_acc[st][s][1];
          a2 += s_acc[st][s][2];
          a3 += s_acc[st][s][3];
          flag = TypeTraits<T>::is_signed ? (flag | s_flag[st][s]) : (s_flag[st][s] > flag ? s_flag[st][s] : flag);
        }
        const int len = (q.cnt - p * q.L) < q.L ? (q.cnt - p * q.L) : q.L;
        const T* xp = reinterpret_cast<const T*>(smem + (size_t)st * cf_stage_bytes<T>() + s_shead[st]) + p * q.L;
        const bool ovf = cf_overflows<T>(flag, xp, len);  // a value above 2^53: direct copy
        const bool vsafe = sizeof(T) == 4 || flag < 0x80000u;
        double t0 = 0.0, t1 = 0.0, c = 0.0;
        long long ci = 0;
        int mode = CF_DIRECT;
        if (!ovf) {
          solve_line(len, (i128)a0 + (i128)a1 * ((i128)1 << 32), (i128)a2 + (i128)a3 * ((i128)1 << 32), t0, t1);
          mode = cf_mode<T>(t0, t1, len, vsafe, c, ci);
        }
        s_t0[st][p] = t0;
        s_t1[st][p] = t1;
        s_c[st][p] = c;
        s_ci[st][p] = ci;
        s_mode[st][p] = mode;
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&lines[st]);
    }
  }
  if (tid >= kCfThreads) {  // ---- producer ----
    if (tid == kCfThreads) cf_produce<T, S>(a, smem, full, empty, s_stile, s_shead, s_scol);
    return;
  }

  // ---- compute warps ----
  // the exact sums of the tile in stage st into s_acc[st] / s_flag[st], then each warp arrives on
  // sums[st] (an end marker is passed on unsummed, so the solver sees the end too)
  auto stage_sums = [&](int st) {
    const int64_t item = s_stile[st];
    if (item >= 0) {
      const CfGeom q = cf_geom(a, item, s_scol[st]);
      const int p_me = tid >> q.lg_g, r_me = tid & (q.g - 1);
      const int my_len = p_me < q.np ? ((q.cnt - p_me * q.L) < q.L ? (q.cnt - p_me * q.L) : q.L) : 0;
      const T* xp = reinterpret_cast<const T*>(smem + (size_t)st * cf_stage_bytes<T>() + s_shead[st]) + p_me * q.L;
      HalfSums<T> hs;
      uint32_t flag = 0;
      if (my_len == q.L) cf_sums<T, true>(xp, r_me, q.g, q.L, hs, flag);
      else if (my_len > 0) cf_sums<T, false>(xp, r_me, q.g, my_len, hs, flag);
      // every partial is below 2^48 in magnitude (16 values, i < 2^12, 32-bit halves)
      const long long c0 = seg_sum48((long long)hs.s_lo, q.W);
      const long long c1 = sizeof(T) == 8 ? seg_sum48((long long)hs.s_hi, q.W) : 0;
      const long long c2 = seg_sum48((long long)hs.x_lo, q.W);
      const long long c3 = sizeof(T) == 8 ? seg_sum48((long long)hs.x_hi, q.W) : 0;
      flag = TypeTraits<T>::is_signed ? seg_or_u32(flag, q.W) : seg_max_u32(flag, q.W);
      if ((tid & (q.W - 1)) == 0) {
        const int seg = tid >> q.lg_W;
        s_acc[st][seg][0] = c0;
        s_acc[st][seg][1] = c1;
        s_acc[st][seg][2] = c2;
        s_acc[st][seg][3] = c3;
        s_flag[st][seg] = flag;
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&sums[st]);
  };
  // tid 0 waits for a phase; every compute thread learns the outcome after the barrier
  auto wait_all = [&](uint64_t* bar, uint32_t par) {
    if (tid == 0) {
      s_ok = mbar_wait_sleep(bar, par);
      if (!s_ok) atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
    }
  };

  if (tid == 0) {
    s_ok = mbar_wait_sleep(&full[0], 0);
    if (!s_ok) {
      atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
      mbar_wait_bounded(&full[0], 0);  // a copy in flight lands before the CTA exits
    }
  }
  cf_sync();
  if (!s_ok) return;
  mbar_try_wait(&full[0], 0);  // the phase is complete: orders this thread's reads after the copy
  if (s_stile[0] < 0) return;
  stage_sums(0);

  for (int k = 0;; k++) {
    const int st = k % S, st1 = (k + 1) % S;
    const uint32_t par = (uint32_t)(k / S) & 1u, par1 = (uint32_t)((k + 1) / S) & 1u;
    // the next tile's values and this tile's lines
    if (tid == 0) {
      s_ok = mbar_wait_sleep(&full[st1], par1);
      if (!s_ok) {
        atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
        mbar_wait_bounded(&full[st1], par1);  // a copy in flight lands before the CTA exits
      } else {
        wait_all(&lines[st], par);
      }
    }
    cf_sync();
    if (!s_ok) return;
    mbar_try_wait(&full[st1], par1);
    mbar_try_wait(&lines[st], par);
    const int64_t item1 = s_stile[st1];
    stage_sums(st1);

    const int64_t item = s_stile[st];
    const CfGeom q = cf_geom(a, item, s_scol[st]);
    const CfColumn& col = *q.col;
    const int L = q.L, g = q.g, W = q.W, np = q.np, cnt = q.cnt;
    const int64_t t = q.t, e0 = q.e0;
    const int seg = tid >> q.lg_W, segs_per_part = q.segs_per_part;
    const int p_me = tid >> q.lg_g, r_me = tid & (g - 1);
    uint8_t* stage = smem + (size_t)st * cf_stage_bytes<T>();
    T* x = reinterpret_cast<T*>(stage + s_shead[st]);
    // the fields and staged words of the fast packing: over the stage for 8-byte types (its values
    // are dead by then), in the work area for 4-byte types
    uint8_t* work = sizeof(T) == 8 ? stage : smem + (size_t)S * cf_stage_bytes<T>();
    const int my_len = p_me < np ? ((cnt - p_me * L) < L ? (cnt - p_me * L) : L) : 0;
    const T* xp = x + p_me * L;

    // ---- B: residual of every value: its low 32 bits kept, max |residual| per partition ----
    uint32_t fl[kCfPerThread];
    bool wide;
    {
      unsigned long long mx = 0;
#pragma unroll
      for (int m = 0; m < kCfPerThread; m++) fl[m] = 0u;
      if (my_len > 0) {
        const int mode = s_mode[st][p_me];
        const double t0 = s_t0[st][p_me], t1 = s_t1[st][p_me];
        bool general = mode == CF_GENERAL;
        if (mode == CF_NONNEG) {
          mx = my_len == L ? cf_resid_sign<T, true, false>(xp, r_me, g, L, t0, t1, fl)
                           : cf_resid_sign<T, false, false>(xp, r_me, g, my_len, t0, t1, fl);
        } else if (TypeTraits<T>::is_signed && mode == CF_NONPOS) {
          mx = my_len == L ? cf_resid_sign<T, true, true>(xp, r_me, g, L, t0, t1, fl)
                           : cf_resid_sign<T, false, true>(xp, r_me, g, my_len, t0, t1, fl);
        } else if (sizeof(T) == 8 && mode == CF_OFFSET) {
          const double c = s_c[st][p_me];
          const long long ci = s_ci[st][p_me];
          general = !(my_len == L ? cf_resid_offset<T, true>(xp, r_me, g, L, t0, t1, c, ci, fl, mx)
                                  : cf_resid_offset<T, false>(xp, r_me, g, my_len, t0, t1, c, ci, fl, mx));
        }
        if (general) mx = cf_resid_general<T>(xp, r_me, g, my_len, t0, t1, fl);
      }
      mx = seg_max_u64(mx, W);
      if ((tid & (W - 1)) == 0) s_mx[seg] = mx;
      // a width above 31 anywhere in the tile (a max |residual| of 2^30 or more, or direct copy)
      wide = my_len > 0 && (s_mode[st][p_me] == CF_DIRECT || mx >= (1ull << 30));
    }
    wide = cf_sync_or(wide);
    if (tid < 32) {  // widths, tile-relative bit ranges (a warp scan), descriptors, the tile's bits
      const int p = lane;
      int b = 0, nb = 0;
      unsigned long long err = 0;
      if (p < np) {
        unsigned long long m = 0;
        for (int s = p * segs_per_part; s < (p + 1) * segs_per_part; s++) m = s_mx[s] > m ? s_mx[s] : m;
        const bool direct = s_mode[st][p] == CF_DIRECT;
        b = direct ? (int)sizeof(T) * 8 : bits_for((long long)m);
        err = direct ? 0 : m;
        nb = ((cnt - p * L) < L ? (cnt - p * L) : L) * b;
      }
      int inc = nb;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(FULL_MASK, inc, o);
        if (lane >= o) inc += v;
      }
      const int bl = inc - nb;
      const int bmax = (int)__reduce_max_sync(FULL_MASK, (unsigned)b);
      const int total = __shfl_sync(FULL_MASK, inc, 31);
      if (p < np) {
        s_bl[p] = bl;
        s_b[p] = b;
        // the descriptor with the tile-relative offset and the max error; fixed_place_kernel
        // completes the offset and writes the other metadata arrays from the descriptor
        const int64_t gp = t * col.parts_per_tile + p;
        PartDesc d;
        d.theta0 = s_t0[st][p];
        d.theta1 = s_t1[st][p];
        d.bit_off = bl;
        d.start = (int32_t)(e0 + (int64_t)p * L);
        d.bits_type = (b & 0xff) | ((s_mode[st][p] == CF_DIRECT ? MODEL_DIRECT_COPY : MODEL_LINEAR) << 8);
        col.desc[gp] = d;
        col.err[gp] = (long long)err;
      }
      if (lane == 0) {
        s_bl[np] = total;
        a.tile_bits[item] = total;
        if (bmax > 0) atomicMax(col.stats + 1, (unsigned long long)bmax);
      }
    }
    // (the widths are not needed by the field writes or the residual recompute below: they run
    // beside warp 0's section and one barrier covers both)

    uint32_t* out = a.slots + item * a.slot_words;
    if (!wide) {
      // ---- C (every width <= 31): fields transposed, one thread packs each 32-value group into
      // its `width` words (every partition starts on a word: L is a multiple of 32), staged, then
      // copied to the slot with coalesced stores ----
      uint32_t* fT = reinterpret_cast<uint32_t*>(work);
      uint32_t* stg = fT + kFtWords;
      if (g >= 32) {  // g a multiple of 32: position j = p_me L + r_me + g m has j % 32 = lane
        uint32_t* fp = fT + lane * kFtStride + ((p_me * L + r_me) >> 5);
        const int step = g >> 5;
#pragma unroll
        for (int m = 0; m < kCfPerThread; m++) fp[m * step] = fl[m];
      } else {
#pragma unroll
        for (int m = 0; m < kCfPerThread; m++) {
          const int j = p_me * L + r_me + g * m;  // position in the tile (the threads cover all 4096)
          fT[(j & 31) * kFtStride + (j >> 5)] = fl[m];
        }
      }
      cf_sync();
      if (tid < ((cnt + 31) >> 5)) {
        const int G = tid, p = G >> (q.lg_L - 5);  // L / 32 groups per partition
        cf_pack_dispatch(s_b[p], fT + G, stg, (s_bl[p] >> 5) + (G - (p << (q.lg_L - 5))) * s_b[p]);
      }
      cf_sync();
      const int nw = (s_bl[np] + 31) >> 5;
      for (int w = tid; w < nw; w += kCfThreads) out[w] = stg[w + (w >> 5)];
    } else {
      // ---- C (a width above 31): the exact 64-bit residuals over the values (8-byte types) or in
      // the work area, then per partition one thread per word of the slot ----
      long long* res = sizeof(T) == 8 ? reinterpret_cast<long long*>(x) : reinterpret_cast<long long*>(work);
      if (my_len > 0)
        cf_store_resid<T>(xp, res + p_me * L, r_me, g, my_len, s_mode[st][p_me], s_t0[st][p_me], s_t1[st][p_me]);
      cf_sync();
      for (int p = 0; p < np; p++)
        cf_words_dispatch(s_b[p], res + p * L, (cnt - p * L) < L ? (cnt - p * L) : L, out + (s_bl[p] >> 5), tid);
    }
    cf_sync();  // every compute thread is done with stage st and the work area
    if (tid == 0) mbar_arrive(&empty[st]);
    if (item1 < 0) return;
  }
}

// The partition-length choice of the batched compress, one tile per step with the CTA layout of
// fixed_compress_kernel (eight compute warps, a producer warp staging tiles three ahead, a solver
// warp): the tile's four 1024-value quarters, its two halves and the whole tile are fitted from
// exact per-quarter sums (the index offsets of a half or the tile added exactly) by the solver warp
// while the compute warps measure the previous tile; every value's residual is measured against the
// three lines that cover it (with the residual modes of fixed_compress_kernel), and the bits of each
// candidate length are added into the column's choice_bits[0..2] (1024, 2048, 4096).  The widths
// are the ones the compress at that length computes, so the column's size is exact.  With PACK the
// tile is also compressed at length 4096 -- the usual choice -- exactly as fixed_compress_kernel
// would (the tile's line from the same exact sums, the same residual modes and packing): its words
// into its slot, its descriptor and max error into tdesc / terr, its bits into tile_bits.
template <typename T, bool PACK> __global__ void __launch_bounds__(kCfFixCTA, 2)
choose_lengths_kernel(const __grid_constant__ FixedCompressArgs a) {
  constexpr int S = kCfChooseStages;
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t full[S], empty[S], sums[S], lines[S];
  __shared__ int64_t s_stile[S];
  __shared__ int s_shead[S];
  __shared__ int s_scol[S];
  __shared__ long long s_acc[S][8][4];
  __shared__ uint32_t s_flag[S][8];
  __shared__ double s_t0[S][7], s_t1[S][7], s_c[S][7];
  __shared__ long long s_ci[S][7];
  __shared__ int s_mode[S][7], s_len[S][7];
  __shared__ unsigned long long s_m[8][3];
  __shared__ int s_ok, s_b0;
  if (threadIdx.x == 0) {
    for (int st = 0; st < S; st++) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
      mbar_init(&sums[st], kCfThreads / 32);
      mbar_init(&lines[st], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid >= kCfThreads + 32) {  // ---- solver warp: line l = 0 the tile, 1-2 its halves, 3-6 its quarters ----
    for (int k = 0;; k++) {
      const int st = k % S;
      int ok = 1;
      if (lane == 0) {
        ok = mbar_wait_sleep(&sums[st], (uint32_t)(k / S) & 1u);
        if (!ok) atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
      }
      if (!__shfl_sync(FULL_MASK, ok, 0)) return;
      const int64_t item = s_stile[st];
      if (item < 0) return;
      if (lane < 7) {
        const CfColumn& col = a.cols[s_scol[st]];
        const int64_t e0 = (item - col.item_base) * kDecodeTile;
        const int cnt = (int)((col.n - e0) < kDecodeTile ? (col.n - e0) : kDecodeTile);
        const int l = lane;
        const int q0 = l == 0 ? 0 : (l < 3 ? (l - 1) * 2 : l - 3);
        const int q1 = l == 0 ? 4 : (l < 3 ? q0 + 2 : q0 + 1);
        i128 sy = 0, sxy = 0;
        uint32_t flag = 0;
        for (int qq = q0; qq < q1; qq++) {
          long long a0 = 0, a1 = 0, a2 = 0, a3 = 0;
          for (int w = 2 * qq; w < 2 * qq + 2; w++) {
            a0 += s_acc[st][w][0];
            a1 += s_acc[st][w][1];
            a2 += s_acc[st][w][2];
            a3 += s_acc[st][w][3];
            flag = TypeTraits<T>::is_signed ? (flag | s_flag[st][w]) : (s_flag[st][w] > flag ? s_flag[st][w] : flag);
          }
          const i128 qy = (i128)a0 + (i128)a1 * ((i128)1 << 32);
          sy += qy;
          sxy += (i128)a2 + (i128)a3 * ((i128)1 << 32) + (i128)(1024 * (qq - q0)) * qy;  // quarter index -> line index
        }
        int len = cnt - 1024 * q0;
        len = len < 0 ? 0 : (len < 1024 * (q1 - q0) ? len : 1024 * (q1 - q0));
        const T* x = reinterpret_cast<const T*>(smem + (size_t)st * cf_stage_bytes<T>() + s_shead[st]);
        const bool ovf = len > 0 && cf_overflows<T>(flag, x + 1024 * q0, len);
        const bool vsafe = sizeof(T) == 4 || flag < 0x80000u;
        double t0 = 0.0, t1 = 0.0, c = 0.0;
        long long ci = 0;
        int mode = CF_DIRECT;
        if (len > 0 && !ovf) {
          solve_line(len, sy, sxy, t0, t1);
          mode = cf_mode<T>(t0, t1, len, vsafe, c, ci);
        }
        s_t0[st][l] = t0;
        s_t1[st][l] = t1;
        s_c[st][l] = c;
        s_ci[st][l] = ci;
        s_mode[st][l] = mode;
        s_len[st][l] = len;
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&lines[st]);
    }
  }
  if (tid >= kCfThreads) {  // ---- producer ----
    if (tid == kCfThreads) cf_produce<T, S>(a, smem, full, empty, s_stile, s_shead, s_scol);
    return;
  }
  // ---- compute warps: thread tid measures values r + 64 m of quarter q ----
  const int q = tid >> 6, r = tid & 63;
  auto stage_sums = [&](int st) {  // exact sums per quarter (two warps each) and the range flags
    const int64_t item = s_stile[st];
    if (item >= 0) {
      const CfColumn& col = a.cols[s_scol[st]];
      const int64_t e0 = (item - col.item_base) * kDecodeTile;
      const int cnt = (int)((col.n - e0) < kDecodeTile ? (col.n - e0) : kDecodeTile);
      const int qlen = (cnt - 1024 * q) < 0 ? 0 : ((cnt - 1024 * q) < 1024 ? (cnt - 1024 * q) : 1024);
      const T* xq = reinterpret_cast<const T*>(smem + (size_t)st * cf_stage_bytes<T>() + s_shead[st]) + 1024 * q;
      HalfSums<T> hs;
      uint32_t flag = 0;
      if (qlen == 1024) cf_sums<T, true>(xq, r, 64, 1024, hs, flag);
      else if (qlen > 0) cf_sums<T, false>(xq, r, 64, qlen, hs, flag);
      const long long c0 = seg_sum48((long long)hs.s_lo, 32);
      const long long c1 = sizeof(T) == 8 ? seg_sum48((long long)hs.s_hi, 32) : 0;
      const long long c2 = seg_sum48((long long)hs.x_lo, 32);
      const long long c3 = sizeof(T) == 8 ? seg_sum48((long long)hs.x_hi, 32) : 0;
      flag = TypeTraits<T>::is_signed ? seg_or_u32(flag, 32) : seg_max_u32(flag, 32);
      if (lane == 0) {
        s_acc[st][warp][0] = c0;
        s_acc[st][warp][1] = c1;
        s_acc[st][warp][2] = c2;
        s_acc[st][warp][3] = c3;
        s_flag[st][warp] = flag;
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&sums[st]);
  };

  if (tid == 0) {
    s_ok = mbar_wait_sleep(&full[0], 0);
    if (!s_ok) {
      atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
      mbar_wait_bounded(&full[0], 0);  // a copy in flight lands before the CTA exits
    }
  }
  cf_sync();
  if (!s_ok) return;
  mbar_try_wait(&full[0], 0);
  if (s_stile[0] < 0) return;
  stage_sums(0);

  for (int k = 0;; k++) {
    const int st = k % S, st1 = (k + 1) % S;
    const uint32_t par = (uint32_t)(k / S) & 1u, par1 = (uint32_t)((k + 1) / S) & 1u;
    if (tid == 0) {
      s_ok = mbar_wait_sleep(&full[st1], par1);
      if (!s_ok) {
        atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
        mbar_wait_bounded(&full[st1], par1);  // a copy in flight lands before the CTA exits
      } else {
        s_ok = mbar_wait_sleep(&lines[st], par);
        if (!s_ok) atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
      }
    }
    cf_sync();
    if (!s_ok) return;
    mbar_try_wait(&full[st1], par1);
    mbar_try_wait(&lines[st], par);
    const int64_t item1 = s_stile[st1];
    stage_sums(st1);

    const int64_t item = s_stile[st];
    const CfColumn& col = a.cols[s_scol[st]];
    const int64_t e0 = (item - col.item_base) * kDecodeTile;
    const int cnt = (int)((col.n - e0) < kDecodeTile ? (col.n - e0) : kDecodeTile);
    const T* x = reinterpret_cast<const T*>(smem + (size_t)st * cf_stage_bytes<T>() + s_shead[st]);
    const int qlen = (cnt - 1024 * q) < 0 ? 0 : ((cnt - 1024 * q) < 1024 ? (cnt - 1024 * q) : 1024);
    const T* xq = x + 1024 * q;
    uint32_t fl[kCfPerThread];  // PACK: the low 32 bits of each value's residual against the tile's line
#pragma unroll
    for (int m = 0; m < kCfPerThread; m++) fl[m] = 0u;
    {  // max |residual| of each value against its quarter's, its half's and the tile's line
      const int ls[3] = {3 + q, 1 + (q >> 1), 0};
      const int off[3] = {0, 1024 * (q & 1), 1024 * q};
      unsigned long long mx[3] = {0, 0, 0};
      if (qlen > 0) {
        if (s_mode[st][ls[0]] == CF_NONNEG && s_mode[st][ls[1]] == CF_NONNEG && s_mode[st][ls[2]] == CF_NONNEG) {
          // the common case in one pass: each value read once, K + y shared by the three lines.  A
          // width needs only the bit length of the largest |residual|, i.e. its FP64 exponent: the
          // largest high word of |d| (sign cleared) for the lines that only count bits; the tile's
          // line keeps the exact maximum when it is packed (its max error is stored)
          double t0[3], t1[3], xd[3], dm = 0.0;
          uint32_t mh[3] = {0u, 0u, 0u};
#pragma unroll
          for (int c = 0; c < 3; c++) {
            t0[c] = s_t0[st][ls[c]];
            t1[c] = s_t1[st][ls[c]];
            xd[c] = (double)(r + off[c]);
          }
#pragma unroll
          for (int m = 0; m < kCfPerThread; m++) {
            const int i = r + 64 * m;
            if (i < qlen) {
              const double yc = magic_of<T>(xq[i]);
#pragma unroll
              for (int c = 0; c < 3; c++) {
                const double d = __dsub_rn(yc, __dadd_rz(__dadd_rn(__fma_rn(t1[c], xd[c], t0[c]), kHalfBias), kMagic));
                if (PACK && c == 2) {
                  dm = fmax(dm, fabs(d));
                  fl[m] = low_field(d);
                } else {
                  const uint32_t h = (uint32_t)__double2hiint(d) & 0x7fffffffu;
                  mh[c] = h > mh[c] ? h : mh[c];
                }
              }
            }
#pragma unroll
            for (int c = 0; c < 3; c++) xd[c] = __dadd_rn(xd[c], 64.0);
          }
#pragma unroll
          for (int c = 0; c < 3; c++) {
            // an integer with the same bit length as the largest |residual| (|d| < 2^53, integral)
            mx[c] = mh[c] ? (1ull << ((mh[c] >> 20) - 1023)) : 0ull;
          }
          if (PACK) mx[2] = (unsigned long long)dm;
        } else {
#pragma unroll
          for (int c = 0; c < 3; c++) {
            // the line's index of value i of the quarter is i + off: read through a pointer moved back by off
            const int l = ls[c], mode = s_mode[st][l];
            const T* xl = xq - off[c];
            const int rl = r + off[c], ll = qlen + off[c];
            const double t0 = s_t0[st][l], t1 = s_t1[st][l];
            uint32_t fd[kCfPerThread];  // the quarter's and the half's fields are not kept
            uint32_t (&f)[kCfPerThread] = (PACK && c == 2) ? fl : fd;
            bool general = mode == CF_GENERAL;
            if (mode == CF_NONNEG) {
              mx[c] = cf_resid_sign<T, false, false>(xl, rl, 64, ll, t0, t1, f);
            } else if (TypeTraits<T>::is_signed && mode == CF_NONPOS) {
              mx[c] = cf_resid_sign<T, false, true>(xl, rl, 64, ll, t0, t1, f);
            } else if (sizeof(T) == 8 && mode == CF_OFFSET) {
              general = !cf_resid_offset<T, false>(xl, rl, 64, ll, t0, t1, s_c[st][l], s_ci[st][l], f, mx[c]);
            }
            if (general) mx[c] = cf_resid_general<T>(xl, rl, 64, ll, t0, t1, f);
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 3; c++) mx[c] = seg_max_u64(mx[c], 32);
      if (lane == 0) {
        s_m[warp][0] = mx[0];
        s_m[warp][1] = mx[1];
        s_m[warp][2] = mx[2];
      }
    }
    cf_sync();
    if (tid < 32) {  // lane l < 7: line l's width and bits; the three lengths' sums by shuffles
      const int l = lane;
      unsigned long long add[3] = {0, 0, 0};
      int b_line = 0;
      unsigned long long m_line = 0;
      if (l < 7 && s_len[st][l] > 0) {
        const int c = l == 0 ? 2 : (l < 3 ? 1 : 0);                      // index into s_m's lines
        const int w0 = l == 0 ? 0 : (l < 3 ? 4 * (l - 1) : 2 * (l - 3));  // the line's warps
        const int w1 = l == 0 ? 8 : (l < 3 ? w0 + 4 : w0 + 2);
        for (int w = w0; w < w1; w++) m_line = s_m[w][c] > m_line ? s_m[w][c] : m_line;
        b_line = s_mode[st][l] == CF_DIRECT ? (int)sizeof(T) * 8 : bits_for((long long)m_line);
        add[c] = (unsigned long long)s_len[st][l] * (unsigned long long)b_line;
      }
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) add[c] += __shfl_xor_sync(FULL_MASK, add[c], o);  // lanes 0-7
      if (lane == 0) {
        for (int c = 0; c < 3; c++)
          if (add[c]) atomicAdd(col.choice_bits + c, add[c]);
        if (PACK) {  // the tile as one partition of 4096 (line 0): width, descriptor, max error, bits
          const bool direct = s_mode[st][0] == CF_DIRECT;
          const int b = b_line;
          PartDesc d;
          d.theta0 = s_t0[st][0];
          d.theta1 = s_t1[st][0];
          d.bit_off = 0;
          d.start = (int32_t)e0;
          d.bits_type = (b & 0xff) | ((direct ? MODEL_DIRECT_COPY : MODEL_LINEAR) << 8);
          a.tdesc[item] = d;
          a.terr[item] = direct ? 0 : (long long)m_line;
          a.tile_bits[item] = (int64_t)cnt * b;
          if (b > 0) atomicMax(col.stats + 1, (unsigned long long)b);
          s_b0 = b;
        }
      }
    }
    cf_sync();  // every compute thread is done with s_m (and, without PACK, with stage st)
    if (PACK) {  // the tile's words at length 4096 into its slot (as fixed_compress_kernel)
      const int b = s_b0;
      uint8_t* stage = smem + (size_t)st * cf_stage_bytes<T>();
      uint8_t* work = sizeof(T) == 8 ? stage : smem + (size_t)S * cf_stage_bytes<T>();
      uint32_t* out = a.slots + item * a.slot_words;
      if (b <= 31) {
        uint32_t* fT = reinterpret_cast<uint32_t*>(work);
        uint32_t* stg = fT + kFtWords;
        uint32_t* fp = fT + lane * kFtStride + ((1024 * q + r) >> 5);  // position 1024 q + r + 64 m: j % 32 = lane
#pragma unroll
        for (int m = 0; m < kCfPerThread; m++) fp[2 * m] = fl[m];
        cf_sync();
        if (tid < ((cnt + 31) >> 5)) cf_pack_dispatch(b, fT + tid, stg, tid * b);
        cf_sync();
        const int nw = (int)(((long long)cnt * b + 31) >> 5);
        for (int w = tid; w < nw; w += kCfThreads) out[w] = stg[w + (w >> 5)];
      } else {
        long long* res = sizeof(T) == 8 ? reinterpret_cast<long long*>(const_cast<T*>(x))
                                        : reinterpret_cast<long long*>(work);
        if (qlen > 0)
          cf_store_resid<T>(x, res, 1024 * q + r, 64, cnt, s_mode[st][0], s_t0[st][0], s_t1[st][0]);
        cf_sync();
        cf_words_dispatch(b, res, cnt, out, tid);
      }
      cf_sync();  // every compute thread is done with stage st and the work area
    }
    if (tid == 0) mbar_arrive(&empty[st]);
    if (item1 < 0) return;
  }
}

// Places every tile of the launch in its column, one CTA per tile: the tile's first bit F (the
// scan of the tiles' bits, relative to the column's first tile) is added to its partitions'
// descriptors, whose fields also fill the other metadata arrays (starts, ends, types, params,
// bits, offsets), the tile's decode-table entry is written, and the words whose first bit lies in the
// tile are written -- from the tile's slot with a funnel shift, ORed with the first bits of every
// later tile of the column that starts inside the same word (tiles without bits are skipped).  The
// column's last tile writes the final decode-table entry and the total, and zeroes the padding.
//
// Word w of the column, when its bits all lie in the tile, is funnelshift(slot[i], slot[i + 1], r)
// with i = w - (first word the tile owns) and r = -F mod 32: each thread loads kPlaceUnroll slot
// words before it uses one (the copy is bound by memory latency, so many loads are kept in
// flight), and takes slot[i + 1] from the next lane.
constexpr int kPlaceThreads = 128;
constexpr int kPlaceUnroll = 4;
constexpr int kPlaceVec = 4;

__global__ void __launch_bounds__(kPlaceThreads, 8) fixed_place_kernel(FixedCompressArgs a) {
  const int tid = threadIdx.x, lane = tid & 31;
  for (int64_t item = blockIdx.x; item < a.nitems; item += gridDim.x) {
    const CfColumn& col = a.cols ? a.cols[a.owner ? a.owner[item] : 0] : a.single;
    if (!col.words) continue;  // a column this launch does not place
    const int64_t t = item - col.item_base;
    const int64_t col_end = col.item_base + col.ntiles;  // the column's items are [item_base, col_end)
    const int64_t base = a.tile_first[col.item_base];
    const int64_t first = a.tile_first[item] - base;
    const int64_t bits = a.tile_bits[item];
    uint32_t* __restrict__ words = col.words;
    const int64_t e0 = t * kDecodeTile;
    const int cnt = (int)((col.n - e0) < kDecodeTile ? (col.n - e0) : kDecodeTile);
    const int np = (cnt + col.L - 1) / col.L;
    if (tid < np) {  // the tile's partitions: their metadata arrays from the descriptor
      const int64_t gp = t * col.parts_per_tile + tid;
      PartDesc d;
      if (a.tdesc) {  // packed by the length choice: the tile is one partition
        d = a.tdesc[item];
        col.err[gp] = a.terr[item];
      } else {
        d = col.desc[gp];
      }
      const int64_t off = d.bit_off + first;
      const int len = (cnt - tid * col.L) < col.L ? (cnt - tid * col.L) : col.L;
      d.bit_off = off;
      col.desc[gp] = d;
      col.starts[gp] = d.start;
      col.ends[gp] = d.start + len;
      col.types[gp] = d.bits_type >> 8;
      col.params[4 * gp] = d.theta0;
      col.params[4 * gp + 1] = d.theta1;
      col.params[4 * gp + 2] = 0.0;
      col.params[4 * gp + 3] = 0.0;
      col.bits[gp] = d.bits_type & 0xff;
      col.offs[gp] = off;
    }
    const int64_t total = a.tile_first[col_end - 1] - base + a.tile_bits[col_end - 1];
    if (tid == 0) {
      TileInfo ti;
      ti.bit_lo = first;
      ti.p_first = (int32_t)(t * col.parts_per_tile);
      ti.p_last = (int32_t)(t * col.parts_per_tile + np - 1);
      col.tiles[t] = ti;
      if (t == col.ntiles - 1) {
        TileInfo te;
        te.bit_lo = total;
        te.p_first = te.p_last = (int32_t)(col.P - 1);
        col.tiles[col.ntiles] = te;
        col.stats[0] = (unsigned long long)total;
      }
    }
    // words [w_begin, w_end) have their first bit in the tile; [w_begin, w_begin + nfull) lie in it
    const int64_t w_begin = (first + 31) >> 5, w_end = (first + bits + 31) >> 5;
    if (w_end > col.words_cap) {  // the caller sized the array from another count: report, write nothing
      if (tid == 0) atomicExch(a.status, (unsigned long long)DEVERR_BOUNDS);
      continue;
    }
    const uint32_t* __restrict__ slot = a.slots + item * a.slot_words;
    if ((first & 127) == 0 && ((bits & 31) == 0 || item == col_end - 1) &&
        (reinterpret_cast<uintptr_t>(words + w_begin) & 15) == 0) {
      // the usual case: every partition holds L * width bits with L a multiple of 256, so every
      // tile starts on a 16-byte boundary of its column and only a column's last tile ends inside
      // a word -- a vector copy of the slot's first nw words
      const int64_t nw = w_end - w_begin;
      const uint4* __restrict__ src = reinterpret_cast<const uint4*>(slot);
      uint4* __restrict__ dst = reinterpret_cast<uint4*>(words + w_begin);
      const int64_t n4 = nw >> 2;
      for (int64_t i0 = 0; i0 < n4; i0 += (int64_t)kPlaceThreads * kPlaceVec) {
        uint4 v[kPlaceVec];
#pragma unroll
        for (int u = 0; u < kPlaceVec; u++) {
          const int64_t i = i0 + tid + u * kPlaceThreads;
          if (i < n4) v[u] = __ldg(src + i);
        }
#pragma unroll
        for (int u = 0; u < kPlaceVec; u++) {
          const int64_t i = i0 + tid + u * kPlaceThreads;
          if (i < n4) dst[i] = v[u];
        }
      }
      if (tid < (int)(nw & 3)) words[w_begin + 4 * n4 + tid] = slot[4 * n4 + tid];
    } else {
      const int64_t nfull = ((first + bits) >> 5) - w_begin;  // may be negative: the tile owns no full word
      const int r = (int)((32 * w_begin - first) & 31);
      // slot words [0, nfull] are read (the one after the last full word feeds its funnel shift; the
      // slot holds one word more than the widest tile's bits)
      for (int64_t i0 = 0; i0 < nfull; i0 += (int64_t)kPlaceThreads * kPlaceUnroll) {
        uint32_t lo[kPlaceUnroll], hi[kPlaceUnroll];
#pragma unroll
        for (int u = 0; u < kPlaceUnroll; u++) {
          const int64_t i = i0 + tid + u * kPlaceThreads;
          lo[u] = i <= nfull ? __ldg(slot + i) : 0u;
          hi[u] = (lane == 31 && i + 1 <= nfull) ? __ldg(slot + i + 1) : 0u;
        }
#pragma unroll
        for (int u = 0; u < kPlaceUnroll; u++) {
          const uint32_t nx = __shfl_down_sync(FULL_MASK, lo[u], 1);
          const uint32_t h = lane == 31 ? hi[u] : nx;
          const int64_t i = i0 + tid + u * kPlaceThreads;
          if (i < nfull) words[w_begin + i] = __funnelshift_r(lo[u], h, r);
        }
      }
      if (tid == 0 && w_end > w_begin && ((first + bits) & 31) != 0) {
        // the tile ends inside its last word: that word's tile bits, then the next tiles' first bits
        const int64_t w = w_end - 1, i = w - w_begin;
        const int64_t avail = first + bits - 32 * w;  // 1..31 tile bits in the word
        uint32_t v = __funnelshift_r(slot[i], slot[i + 1], r) & ((1u << avail) - 1u);
        int64_t pos = first + bits;  // column bit where the next tile starts
        for (int64_t u = item + 1; u < col_end && pos < 32 * w + 32; u++) {
          const int64_t ub = a.tile_bits[u];
          if (ub == 0) continue;
          const int64_t take = (32 * w + 32 - pos) < ub ? (32 * w + 32 - pos) : ub;
          uint32_t f = a.slots[u * a.slot_words];
          if (take < 32) f &= (1u << take) - 1u;
          v |= f << (pos - 32 * w);
          pos += ub;
        }
        words[w] = v;
      }
    }
    if (t == col.ntiles - 1 && col.nwords_alloc > 0) {  // the decoders' zeroed read-ahead after the bitstream
      const int64_t wt = (total + 31) >> 5;
      int64_t pad_end = ((wt + 3) & ~3ll) + 8;
      pad_end = pad_end < col.nwords_alloc ? pad_end : col.nwords_alloc;
      for (int64_t w = wt + tid; w < pad_end && w < col.words_cap; w += kPlaceThreads) words[w] = 0u;
    }
  }
}

template <typename T> static cudaError_t launch_fixed_compress_t(const FixedCompressArgs& a, int num_sms, cudaStream_t s) {
  constexpr int smem = cf_fix_smem_bytes<T>(kCfCompressStages);
  static PerDeviceFlag attr_set;  // per instantiation and device
  const int dev = current_device();
  cudaError_t e;
  if (!attr_set.test(dev)) {
    if ((e = cudaFuncSetAttribute(fixed_compress_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) !=
        cudaSuccess)
      return e;
    attr_set.set(dev);
  }
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fixed_compress_kernel<T>, kCfFixCTA, smem)) !=
      cudaSuccess)
    return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * num_sms;
  if (grid > a.nitems) grid = a.nitems;
  if (grid < 1) grid = 1;
  fixed_compress_kernel<T><<<(unsigned)grid, kCfFixCTA, smem, s>>>(a);
  return cudaGetLastError();
}

static cudaError_t launch_fixed_compress_dt(glc_dtype dt, const FixedCompressArgs& a, int num_sms, cudaStream_t s) {
  switch (dt) {
    case GLC_I32: return launch_fixed_compress_t<int32_t>(a, num_sms, s);
    case GLC_I64: return launch_fixed_compress_t<int64_t>(a, num_sms, s);
    case GLC_U64: return launch_fixed_compress_t<uint64_t>(a, num_sms, s);
    case GLC_U32: return launch_fixed_compress_t<uint32_t>(a, num_sms, s);
  }
  return cudaErrorInvalidValue;
}

template <typename T, bool PACK> static cudaError_t launch_choose_t(const FixedCompressArgs& a, int num_sms, cudaStream_t s) {
  constexpr int smem = PACK ? cf_fix_smem_bytes<T>(kCfChooseStages) : kCfChooseStages * cf_stage_bytes<T>();
  static PerDeviceFlag attr_set;
  const int dev = current_device();
  cudaError_t e;
  if (!attr_set.test(dev)) {
    if ((e = cudaFuncSetAttribute(choose_lengths_kernel<T, PACK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  smem)) != cudaSuccess)
      return e;
    attr_set.set(dev);
  }
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, choose_lengths_kernel<T, PACK>, kCfFixCTA, smem)) !=
      cudaSuccess)
    return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * num_sms;
  if (grid > a.nitems) grid = a.nitems;
  if (grid < 1) grid = 1;
  choose_lengths_kernel<T, PACK><<<(unsigned)grid, kCfFixCTA, smem, s>>>(a);
  return cudaGetLastError();
}

static void carve(FixedCompressArgs& a, glc_dtype dt, void* scratch);

cudaError_t launch_choose_lengths(glc_dtype dt, const CfColumn* cols, const int32_t* owner, int64_t nitems,
                                  unsigned long long* status, int num_sms, cudaStream_t s, void* scratch,
                                  PartDesc* tdesc, long long* terr) {
  if (nitems <= 0) return cudaSuccess;
  FixedCompressArgs a{};
  a.cols = cols;
  a.owner = owner;
  a.nitems = nitems;
  a.status = status;
  const bool pack = scratch != nullptr;
  if (pack) {
    carve(a, dt, scratch);
    a.tdesc = tdesc;
    a.terr = terr;
  }
  switch (dt) {
    case GLC_I32: return pack ? launch_choose_t<int32_t, true>(a, num_sms, s) : launch_choose_t<int32_t, false>(a, num_sms, s);
    case GLC_I64: return pack ? launch_choose_t<int64_t, true>(a, num_sms, s) : launch_choose_t<int64_t, false>(a, num_sms, s);
    case GLC_U64: return pack ? launch_choose_t<uint64_t, true>(a, num_sms, s) : launch_choose_t<uint64_t, false>(a, num_sms, s);
    case GLC_U32: return pack ? launch_choose_t<uint32_t, true>(a, num_sms, s) : launch_choose_t<uint32_t, false>(a, num_sms, s);
  }
  return cudaErrorInvalidValue;
}

int64_t fixed_compress_worst_words(glc_dtype dt, int64_t n) {
  const int64_t per_value = (dt == GLC_I64 || dt == GLC_U64) ? 64 : 33;  // widest field of the type
  return (n * per_value + 31) / 32 + 12;  // + the decoders' zeroed read-ahead
}

bool fixed_compress_supported(int64_t n, int32_t L) {
  return n > 0 && L >= kCfMinLen && L <= kDecodeTile && (kDecodeTile % L) == 0;
}

// Words of one tile's slot: the widest fields of the type (64 bits for 8-byte types, 33 for 4-byte
// ones) plus the word the placing funnel shift reads after the last, rounded to 16 bytes.
int64_t fixed_compress_slot_words(glc_dtype dt) {
  const int64_t per_value = (dt == GLC_I64 || dt == GLC_U64) ? 64 : 33;
  return ((kDecodeTile * per_value + 31) / 32 + 1 + 3) & ~3ll;
}

// Scratch of a launch over nitems tiles: slots, the tiles' bits, their scan and its tile sums.
size_t fixed_compress_scratch_bytes(glc_dtype dt, int64_t nitems) {
  return (size_t)nitems * fixed_compress_slot_words(dt) * 4 + (size_t)(nitems + 1) * 16 +
         (size_t)(scan_num_tiles(nitems + 1) + 1) * 8 + 256;
}

static void carve(FixedCompressArgs& a, glc_dtype dt, void* scratch) {
  uint8_t* sp = reinterpret_cast<uint8_t*>(scratch);
  a.slot_words = fixed_compress_slot_words(dt);
  a.slots = reinterpret_cast<uint32_t*>(sp);
  sp += (size_t)a.nitems * a.slot_words * 4;
  a.tile_bits = reinterpret_cast<int64_t*>(sp);
  sp += (size_t)(a.nitems + 1) * 8;
  a.tile_first = reinterpret_cast<int64_t*>(sp);
}

// Pass 1 for one launch: fit, residuals and each tile's words into its slot, the tiles' bits, and
// their exclusive scan (tile_first[nitems] = all the launch's bits).
static cudaError_t compress_pass(glc_dtype dt, FixedCompressArgs& a, void* scratch, int num_sms, cudaStream_t s) {
  carve(a, dt, scratch);
  cudaError_t e;
  if ((e = launch_fixed_compress_dt(dt, a, num_sms, s)) != cudaSuccess) return e;
  int64_t* first = const_cast<int64_t*>(a.tile_first);
  int64_t* tmp = first + a.nitems + 1;
  return exclusive_scan<int64_t>(a.tile_bits, first, a.nitems, first + a.nitems, tmp, s);
}

static cudaError_t place_pass(const FixedCompressArgs& a, int num_sms, cudaStream_t s) {
  const int64_t cap = (int64_t)num_sms * 8;  // eight CTAs of 128 threads per SM (twice the tiles in flight of four of 256: 33 -> 26 us per 32M values)
  int64_t grid = a.nitems < cap ? a.nitems : cap;
  if (grid < 1) grid = 1;
  fixed_place_kernel<<<(unsigned)grid, kPlaceThreads, 0, s>>>(a);
  return cudaGetLastError();
}

// One column: values (n of dt, fixed partitions of L) into c's metadata arrays and tables
// (allocated by the caller for P = ceil(n / L) partitions); scratch holds
// fixed_compress_scratch_bytes(dt, ntiles) bytes.  Pass 1 leaves stats[0] = the column's total bits,
// stats[1] = its widest field, stats[2] = a DEVERR_* code (stats[0..3] zeroed here); the caller
// reads them, allocates the words and calls launch_fixed_place.
cudaError_t launch_fixed_compress(glc_dtype dt, const void* values, glc_column* c, int32_t L, void* scratch,
                                  unsigned long long* stats, cudaStream_t s) {
  FixedCompressArgs a{};
  CfColumn& col = a.single;
  col.values = values;
  col.n = c->n;
  col.L = L;
  col.parts_per_tile = kDecodeTile / L;
  col.P = c->P;
  col.ntiles = c->ntiles;
  col.item_base = 0;
  col.starts = c->d_start;
  col.ends = c->d_end;
  col.types = c->d_types;
  col.params = c->d_params;
  col.bits = c->d_bits;
  col.offs = c->d_offs;
  col.err = c->d_err;
  col.desc = c->d_desc;
  col.tiles = c->d_tiles;
  col.stats = stats;
  a.nitems = c->ntiles;
  a.status = stats + 2;
  cudaError_t e;
  if ((e = cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned long long), s)) != cudaSuccess) return e;
  if ((e = compress_pass(dt, a, scratch, c->ctx ? c->ctx->num_sms : 148, s)) != cudaSuccess) return e;
  // the total: the scan's grand total (the column is the whole launch)
  return cudaMemcpyAsync(stats, a.tile_first + a.nitems, sizeof(int64_t), cudaMemcpyDeviceToDevice, s);
}

// Pass 2 for one column: its words into c->d_words (c->nwords_alloc words), its offsets, descriptors
// and decode-table entries completed.  Same arguments as launch_fixed_compress.
cudaError_t launch_fixed_place(glc_dtype dt, glc_column* c, int32_t L, void* scratch, unsigned long long* stats,
                               cudaStream_t s) {
  FixedCompressArgs a{};
  CfColumn& col = a.single;
  col.n = c->n;
  col.L = L;
  col.parts_per_tile = kDecodeTile / L;
  col.P = c->P;
  col.ntiles = c->ntiles;
  col.item_base = 0;
  col.nwords_alloc = c->nwords_alloc;
  col.words_cap = c->nwords_alloc;
  col.starts = c->d_start;
  col.ends = c->d_end;
  col.types = c->d_types;
  col.params = c->d_params;
  col.bits = c->d_bits;
  col.offs = c->d_offs;
  col.desc = c->d_desc;
  col.tiles = c->d_tiles;
  col.words = c->d_words;
  col.stats = stats;
  a.nitems = c->ntiles;
  a.status = stats + 2;
  carve(a, dt, scratch);
  return place_pass(a, c->ctx ? c->ctx->num_sms : 148, s);
}

// The columns packed at 4096 by launch_choose_lengths (same cols layout and owner list, same
// scratch, tdesc and terr): the scan of the tiles' bits and the place of every column whose words
// are set in cols (the others are skipped).
cudaError_t launch_place_prepacked(glc_dtype dt, const CfColumn* cols, const int32_t* owner, int64_t nitems,
                                   void* scratch, PartDesc* tdesc, long long* terr, unsigned long long* status,
                                   int num_sms, cudaStream_t s) {
  if (nitems <= 0) return cudaSuccess;
  FixedCompressArgs a{};
  a.cols = cols;
  a.owner = owner;
  a.nitems = nitems;
  a.status = status;
  a.tdesc = tdesc;
  a.terr = terr;
  carve(a, dt, scratch);
  int64_t* first = const_cast<int64_t*>(a.tile_first);
  cudaError_t e = exclusive_scan<int64_t>(a.tile_bits, first, a.nitems, first + a.nitems, first + a.nitems + 1, s);
  if (e != cudaSuccess) return e;
  return place_pass(a, num_sms, s);
}

// Many columns of one element type: cols (device, each with its own arrays, its exact word array
// and words_cap, stats zeroed) and owner (device, nitems entries: the column of each item, items in
// column order); both passes in stream order.  scratch: fixed_compress_scratch_bytes(dt, nitems).
cudaError_t launch_fixed_compress_batch(glc_dtype dt, const CfColumn* cols, const int32_t* owner, int64_t nitems,
                                        void* scratch, unsigned long long* status, int num_sms, cudaStream_t s) {
  if (nitems <= 0) return cudaSuccess;
  FixedCompressArgs a{};
  a.cols = cols;
  a.owner = owner;
  a.nitems = nitems;
  a.status = status;
  cudaError_t e;
  if ((e = compress_pass(dt, a, scratch, num_sms, s)) != cudaSuccess) return e;
  return place_pass(a, num_sms, s);
}

}  // namespace glc
