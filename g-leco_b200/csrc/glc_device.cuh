// glc_device.cuh -- device-side arithmetic of the G-LeCo format (sm_100a).
//
// The format contract (identical to the reference, so reference-made blobs decode here and
// blobs made here decode with the reference):
//   prediction  pred = sat_cast<T>(round(fma(theta1, (double)i, theta0)))
//               decompression/FullDecompressionKernels.cuh:161,177-187; the encoder
//               compression/CompressionKernels.cuh:318-324 computes the same value because the
//               GPU double->int conversion saturates (negative -> 0 for unsigned types).
//   residual    core/MathHelpers.cuh:22-53 calculateDelta (u64: saturating signed difference)
//   apply       core/MathHelpers.cuh:55-84 applyDelta (wraparound)
//   bit width   bitlen(max|delta|) + 1, capped at 64 (CompressionKernels.cuh:190-207)
//   bitstream   field i of partition p at bit offset[p] + i*bits, LSB first in uint32 words,
//               sign-extended on read; direct-copy fields zero-extended
//               (core/BitManipulation.cuh:80-200)
//
// The model fit is this implementation's own: least squares from EXACT 128-bit integer sums,
// converted to double with one correctly rounded step, so any summation order gives the
// same theta (the reference's theta depends on its reduction order).
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

namespace glc {

typedef __int128 i128;
typedef unsigned __int128 u128;

enum : int { MODEL_CONSTANT = 0, MODEL_LINEAR = 1, MODEL_POLY2 = 2, MODEL_POLY3 = 3, MODEL_DIRECT_COPY = 4 };
constexpr unsigned FULL_MASK = 0xffffffffu;
constexpr int kMinPart = 128;        // core/CudaUtils.cuh:20 MIN_PARTITION_SIZE
constexpr double kModelBytes = 80.0; // compression/CpuPartitioner.cuh:18 sizeof(PartitionInfo)

// 32-byte packed partition descriptor: one sector per lookup in random access.
// bits_type = delta_bits | (model_type << 8).
struct __align__(32) PartDesc {
  double theta0;
  double theta1;
  int64_t bit_off;
  int32_t start;
  int32_t bits_type;
};

template <typename T> struct TypeTraits;
template <> struct TypeTraits<int32_t>  { static constexpr bool is_signed = true;  };
template <> struct TypeTraits<int64_t>  { static constexpr bool is_signed = true;  };
template <> struct TypeTraits<uint64_t> { static constexpr bool is_signed = false; };
template <> struct TypeTraits<uint32_t> { static constexpr bool is_signed = false; };

// ---------------------------------------------------------------------------------------
// Saturating cast of an integral double.  The PTX float-to-integer conversion (cvt.rzi) clamps
// to the destination range by default and maps NaN to 0, which is exactly the reference's
// static_cast<T>(round(x)) on the GPU and its decoders' clamp of unsigned predictions to
// [0, max] (decompression/FullDecompressionKernels.cuh:177-186).
// ---------------------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T sat_cast(double r);
template <> __device__ __forceinline__ int32_t sat_cast<int32_t>(double r) { return __double2int_rz(r); }
template <> __device__ __forceinline__ int64_t sat_cast<int64_t>(double r) { return __double2ll_rz(r); }
template <> __device__ __forceinline__ uint64_t sat_cast<uint64_t>(double r) { return __double2ull_rz(r); }
template <> __device__ __forceinline__ uint32_t sat_cast<uint32_t>(double r) { return __double2uint_rz(r); }

// Rounding half away from zero by adding the predecessor of 0.5 and truncating: the method of the
// fix of Java's Math.round (OpenJDK bug 6430675, floor(x + 0.49999999999999994)), applied here to
// both signs.  round-half-away-from-zero(x) == trunc(x + copysign(0.5 - 2^-54, x)) for every double x under
// round-to-nearest-even addition: with k = trunc(|x|) and f = |x| - k, the sum stays below k + 1
// when f < 0.5 (it falls short of k + 1 by more than half an ulp) and reaches k + 1 when
// f >= 0.5 (at f = 0.5 in [0.5, 1) it is the tie 1 - 2^-54, which rounds to even, 1.0); values of
// magnitude >= 2^52 are integers and the addend is below half an ulp.  The truncation is folded
// into the saturating round-toward-zero conversion, so prediction = one fma, one add, one convert.
__device__ __forceinline__ double half_away_bias(double x) {
  return __longlong_as_double((__double_as_longlong(x) & (long long)0x8000000000000000ull) |
                              0x3FDFFFFFFFFFFFFFll);  // +-(0.5 - 2^-54)
}

template <typename T> __device__ __forceinline__ T predict_from(double p) {
  return sat_cast<T>(__dadd_rn(p, half_away_bias(p)));
}

// trunc(t) for |t| < 2^52 without a conversion instruction (conversions between 64-bit integers
// and doubles issue on the narrow XU pipe): the magic-number method -- adding 2^52 with t's sign,
// rounded toward zero, lands in [2^52, 2^53), where doubles are the integers, so the low 52 bits
// of the sum hold |trunc(t)| exactly.
__device__ __forceinline__ long long trunc_small(double t) {
  const double m = __dadd_rz(t, copysign(4503599627370496.0, t));
  const long long mag = __double_as_longlong(m) & 0xFFFFFFFFFFFFFll;
  return t < 0.0 ? -mag : mag;
}

// predict_from<T>(p) for a prediction argument inside pred_fp64_safe's bounds (then |p| < 2^51
// and the result needs no saturation): round half away from zero, by trunc_small.
__device__ __forceinline__ long long predict_small(double p) { return trunc_small(__dadd_rn(p, half_away_bias(p))); }

template <typename T> __device__ __forceinline__ T predict(double theta0, double theta1, int64_t i) {
  return predict_from<T>(__fma_rn(theta1, __ll2double_rn(i), theta0));
}

// ---- exact residual magnitudes in FP64 -------------------------------------------------
// For a value with |y| < 2^51 and a prediction argument x inside pred_fp64_safe's bounds, the
// prediction round_half_away(x) = trunc(x + copysign(0.5 - 2^-54, x)) is an FP64 integer that
// the saturating conversion leaves unchanged, y - pred is below 2^52 in magnitude (no
// saturation, no wraparound), and every step is exact: abs_resid_fp64 equals
// abs_ref(calc_delta<T>(y, predict<T>(...))).  fma(theta1, i, theta0) is monotone in i, so a
// line is safe over [i0, i1] when its two ends are.
template <typename T> __device__ __forceinline__ bool value_fp64_safe(T y) {
  return TypeTraits<T>::is_signed ? ((long long)y > -(1ll << 51) && (long long)y < (1ll << 51))
                                  : ((uint64_t)y < (1ull << 51));
}
template <typename T> __device__ __forceinline__ bool pred_fp64_safe(double x) {
  constexpr double kSafe = 2251799813685248.0;  // 2^51
  const double lo = TypeTraits<T>::is_signed ? (sizeof(T) == 4 ? -2147483647.0 : -kSafe) : -0.25;
  const double hi = sizeof(T) == 4 ? (TypeTraits<T>::is_signed ? 2147483646.0 : 4294967294.0) : kSafe;
  return x >= lo && x <= hi;
}
template <typename T> __device__ __forceinline__ bool line_fp64_safe(double t0, double t1, int64_t i0, int64_t i1) {
  return pred_fp64_safe<T>(__fma_rn(t1, (double)i0, t0)) && pred_fp64_safe<T>(__fma_rn(t1, (double)i1, t0));
}
__device__ __forceinline__ double abs_resid_fp64(double yd, double x) {
  // trunc(t) by the magic number c = +-2^52 (trunc_small): m = t + c rounded toward zero is
  // c + trunc(t) exactly, and (yd + c) - m = yd - trunc(t) is exact (|yd| < 2^51), so no
  // rounding instruction is needed
  const double t = __dadd_rn(x, half_away_bias(x));
  const double c = copysign(4503599627370496.0, t);
  return fabs(__dsub_rn(__dadd_rn(yd, c), __dadd_rz(t, c)));
}

// Exact sums of y and j * y over the values a thread adds (j < 2^14, at most 2^10 values per
// thread) from 64-bit partials of the 32-bit halves of y; sum(y) and sum(j * y) as 128-bit.
template <typename T> struct HalfSums {
  typedef typename std::conditional<TypeTraits<T>::is_signed, int64_t, uint64_t>::type Acc;
  Acc s_lo = 0, s_hi = 0, x_lo = 0, x_hi = 0;
  __device__ __forceinline__ void add(T y, int j) {
    if (sizeof(T) == 8) {  // j >= 0: 32 x 32 -> 64-bit products
      const uint32_t yl = (uint32_t)(uint64_t)y, yh = (uint32_t)((uint64_t)y >> 32);
      s_lo += (Acc)yl;
      x_lo += (Acc)((uint64_t)(uint32_t)j * (uint64_t)yl);
      if (TypeTraits<T>::is_signed) {
        s_hi += (Acc)(int32_t)yh;
        x_hi += (Acc)((long long)j * (long long)(int32_t)yh);
      } else {
        s_hi += (Acc)yh;
        x_hi += (Acc)((uint64_t)(uint32_t)j * (uint64_t)yh);
      }
    } else {
      s_lo += (Acc)y;
      x_lo += (Acc)j * (Acc)y;
    }
  }
  __device__ __forceinline__ i128 sy() const { return (i128)s_lo + (i128)s_hi * ((i128)1 << 32); }
  __device__ __forceinline__ i128 sxy() const { return (i128)x_lo + (i128)x_hi * ((i128)1 << 32); }
};

template <typename T> __device__ __forceinline__ long long calc_delta(T actual, T pred) {
  if (TypeTraits<T>::is_signed) {
    return (long long)((unsigned long long)(long long)actual - (unsigned long long)(long long)pred);
  } else if (sizeof(T) == 8) {
    unsigned long long a = (unsigned long long)actual, p = (unsigned long long)pred;
    if (a >= p) {
      unsigned long long d = a - p;
      return d <= 0x7fffffffffffffffull ? (long long)d : (long long)0x7fffffffffffffffull;
    }
    unsigned long long d = p - a;
    return d <= 0x7fffffffffffffffull ? -(long long)d : (long long)0x8000000000000000ull;
  } else {
    return (long long)actual - (long long)pred;
  }
}

template <typename T> __device__ __forceinline__ T apply_delta(T pred, long long delta) {
  if (sizeof(T) == 8) return (T)((unsigned long long)pred + (unsigned long long)delta);
  return (T)((uint32_t)pred + (uint32_t)delta);
}

// |d| for the bit width; |LLONG_MIN| counts as LLONG_MAX so that residual gets a 64-bit field
// (the reference's (d < 0) ? -d : d leaves it negative and truncates it,
// compression/CompressionKernels.cuh:171-174).
__device__ __forceinline__ long long abs_ref(long long d) {
  if (d == (long long)0x8000000000000000ull) return 0x7fffffffffffffffll;
  return d < 0 ? -d : d;
}

__device__ __forceinline__ int bits_for(long long max_err) {
  if (max_err <= 0) return 0;
  int b = 64 - __clzll(max_err);
  return b + 1 < 64 ? b + 1 : 64;
}

template <typename T> __device__ __forceinline__ bool overflows_double(T v) {
  if (TypeTraits<T>::is_signed) return false;
  return (uint64_t)v > (1ull << 53);
}

// Field of `bits` bits (1..64), masked.
__device__ __forceinline__ uint64_t low_bits(uint64_t x, int bits) {
  return bits >= 64 ? x : (x & ((1ull << bits) - 1ull));
}

__device__ __forceinline__ long long sign_extend(uint64_t f, int bits) {
  if (bits <= 0) return 0;
  if (bits >= 64) return (long long)f;
  uint64_t sign = 1ull << (bits - 1);
  return (long long)((f ^ sign) - sign);
}

// Read `bits` (1..64) bits starting at bit `pos` from a word array (global or shared).
// Reads up to three consecutive words; callers guarantee those words exist (padding).
__device__ __forceinline__ uint64_t read_field(const uint32_t* w, int64_t pos, int bits) {
  int64_t wi = pos >> 5;
  int sh = (int)(pos & 31);
  uint64_t lo = (uint64_t)w[wi] | ((uint64_t)w[wi + 1] << 32);
  uint64_t f = lo >> sh;
  if (bits + sh > 64) f |= (uint64_t)w[wi + 2] << (64 - sh);
  return low_bits(f, bits);
}

// ---------------------------------------------------------------------------------------
// Exact sums -> least-squares line.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double pow2_exact(int e) {
  return __longlong_as_double((long long)(1023 + e) << 52);
}

// Correctly rounded (nearest-even) conversion of a 128-bit integer.
__device__ __forceinline__ double i128_to_double(i128 v) {
  if (v == 0) return 0.0;
  bool neg = v < 0;
  u128 u = neg ? (u128)0 - (u128)v : (u128)v;
  uint64_t hi = (uint64_t)(u >> 64);
  double r;
  if (hi == 0) {
    r = __ull2double_rn((uint64_t)u);
  } else {
    int sh = 64 - __clzll((long long)hi);
    uint64_t m = (uint64_t)(u >> sh);
    uint64_t mask = (sh == 64) ? ~0ull : ((1ull << sh) - 1ull);
    if (((uint64_t)u & mask) != 0) m |= 1ull;
    r = __dmul_rn(__ull2double_rn(m), pow2_exact(sh));
  }
  return neg ? -r : r;
}

// n(n^2-1)/6 exactly, without 128-bit division.
__device__ __forceinline__ i128 den6_exact(int64_t n) {
  int64_t a = n - 1, b = n, c = n + 1;
  if (a % 3 == 0) a /= 3; else if (b % 3 == 0) b /= 3; else c /= 3;
  if ((a & 1) == 0) a /= 2; else if ((b & 1) == 0) b /= 2; else c /= 2;
  return (i128)a * (i128)b * (i128)c;
}

// theta1 = (2 Sxy - (n-1) Sy) / (n(n^2-1)/6);  theta0 = (Sy - theta1 * n(n-1)/2) / n.
__device__ __forceinline__ void solve_line(int64_t n, i128 sy, i128 sxy, double& theta0, double& theta1) {
  if (n <= 0) { theta0 = 0.0; theta1 = 0.0; return; }
  if (n == 1) { theta1 = 0.0; theta0 = i128_to_double(sy); return; }
  i128 num = (i128)2 * sxy - (i128)(n - 1) * sy;
  double t1 = __ddiv_rn(i128_to_double(num), i128_to_double(den6_exact(n)));
  double sx = __ll2double_rn((n * (n - 1)) / 2);
  double diff = __dsub_rn(i128_to_double(sy), __dmul_rn(t1, sx));
  theta1 = t1;
  theta0 = __ddiv_rn(diff, __ll2double_rn(n));
}

// ---------------------------------------------------------------------------------------
// Warp reductions.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ i128 shfl_xor_i128(i128 v, int m) {
  unsigned long long lo = (unsigned long long)v;
  long long hi = (long long)(v >> 64);
  lo = __shfl_xor_sync(FULL_MASK, lo, m);
  hi = __shfl_xor_sync(FULL_MASK, hi, m);
  return ((i128)hi << 64) | (i128)lo;
}

__device__ __forceinline__ i128 warp_sum_i128(i128 v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v += shfl_xor_i128(v, m);
  return v;
}

__device__ __forceinline__ long long warp_max_ll(long long v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) {
    long long o = __shfl_xor_sync(FULL_MASK, v, m);
    v = o > v ? o : v;
  }
  return v;
}

// Bounded spin limit for every wait in these kernels (an mbarrier phase); after it the kernel
// records an error code and returns instead of spinning forever.
constexpr long long kSpinLimit = 1ll << 26;

enum : int { DEVERR_NONE = 0, DEVERR_TIMEOUT = 1, DEVERR_BOUNDS = 2 };

}  // namespace glc
