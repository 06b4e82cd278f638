// glc_oracle.cpp -- CPU restatement of G-LeCo's learned integer-column compression path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product is compared
// against.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
// legs may load it; the product library never links, calls or falls back to it.
//
// Every function names the reference code it restates (paths are relative to the
// G-LeCo source tree).  Two groups of functions live here:
//
//   (1) The format and arithmetic contract shared with the reference: the prediction
//       fma(theta1, i, theta0) -> round half away from zero -> saturating cast, the residual
//       rules of calculateDelta/applyDelta, the residual bit width, the LSB-first bitstream,
//       the exclusive bit-offset prefix, the reported compressed size and the serialized
//       blob (version 5, rotate-add header checksum).  These are bit-for-bit the reference's.
//
//   (2) The partitioning and model-fit arithmetic of THIS implementation.  The reference
//       fits with order-dependent floating-point sums (strided per-thread sums and a
//       shared-memory tree on the GPU, prefix-sum differences on the CPU), so its theta
//       is an artefact of summation order.  This implementation fits from EXACT 128-bit
//       integer sums, which any summation order reproduces.  The restatement below follows
//       that definition so the device output can be compared byte for byte.
//
//   (3) A faithful restatement of the reference's own CPU partitioner
//       (compression/CpuPartitioner.cuh), with its prefix-sum arithmetic and quirks, used
//       for the compressed-size parity check and as the CPU baseline.
//
// Build: g++ -O2 -std=c++17 -ffp-contract=off -fPIC -shared (see oracle/Makefile).
// -ffp-contract=off matters: every multiply-add below is either an explicit std::fma
// (mirroring the device's __fma_rn) or two separately rounded operations.

#include <cstdint>
#include <cstring>
#include <cmath>
#include <climits>
#include <cstdlib>
#include <vector>
#include <limits>
#include <algorithm>
#include <type_traits>

typedef __int128 i128;
typedef unsigned __int128 u128;

namespace {

enum DType { DT_I32 = 0, DT_I64 = 1, DT_U64 = 2, DT_U32 = 3 };
// api/G-LeCo_Types.cuh:8-14
enum Model { M_CONSTANT = 0, M_LINEAR = 1, M_POLY2 = 2, M_POLY3 = 3, M_DIRECT = 4 };

const int kMinPart = 128;          // core/CudaUtils.cuh:20 MIN_PARTITION_SIZE
const int kMaxDeltaBits = 64;      // core/CudaUtils.cuh:19 MAX_DELTA_BITS
const double kModelBytes = 80.0;   // compression/CpuPartitioner.cuh:18 sizeof(PartitionInfo)

// ---------------------------------------------------------------------------------------
// Exact integer -> double conversion, round to nearest even.  The product uses the same
// definition on the device; both sides convert a 128-bit exact sum with one rounding.
// ---------------------------------------------------------------------------------------
double pow2(int e) {  // exact 2^e for 0 <= e <= 1023
  uint64_t bits = (uint64_t)(1023 + e) << 52;
  double d;
  std::memcpy(&d, &bits, 8);
  return d;
}

double i128_to_double(i128 v) {
  if (v == 0) return 0.0;
  bool neg = v < 0;
  u128 u = neg ? (u128)0 - (u128)v : (u128)v;
  uint64_t hi = (uint64_t)(u >> 64);
  double r;
  if (hi == 0) {
    r = (double)(uint64_t)u;  // correctly rounded u64 -> f64
  } else {
    int sh = 64 - __builtin_clzll(hi);  // bits to drop so the leading 1 sits at bit 63
    uint64_t m = (uint64_t)(u >> sh);
    uint64_t mask = (sh == 64) ? ~0ULL : ((1ULL << sh) - 1ULL);
    if (((uint64_t)u & mask) != 0) m |= 1ULL;  // sticky bit, below the rounding position
    r = (double)m * pow2(sh);
  }
  return neg ? -r : r;
}

// ---------------------------------------------------------------------------------------
// Typed helpers: the reference's per-type rules.
// ---------------------------------------------------------------------------------------
template <typename T> struct TypeInfo;
template <> struct TypeInfo<int32_t>  { static const bool is_signed = true;  };
template <> struct TypeInfo<int64_t>  { static const bool is_signed = true;  };
template <> struct TypeInfo<uint64_t> { static const bool is_signed = false; };
template <> struct TypeInfo<uint32_t> { static const bool is_signed = false; };

// Saturating double -> T of an already integral value.  On the GPU the reference's
// static_cast<T>(round(x)) is a cvt.rzi that clamps to T's range (NaN -> 0); the decoders
// additionally clamp unsigned predictions to [0, max] first
// (decompression/FullDecompressionKernels.cuh:177-186).  Both give this function.
template <typename T> T sat_cast(double r);
template <> int32_t sat_cast<int32_t>(double r) {
  if (r != r) return 0;
  if (r >= 2147483648.0) return INT32_MAX;
  if (r <= -2147483648.0) return INT32_MIN;
  return (int32_t)r;
}
template <> int64_t sat_cast<int64_t>(double r) {
  if (r != r) return 0;
  if (r >= 9223372036854775808.0) return INT64_MAX;
  if (r <= -9223372036854775808.0) return INT64_MIN;
  return (int64_t)r;
}
template <> uint64_t sat_cast<uint64_t>(double r) {
  if (!(r > 0.0)) return 0;
  if (r >= 18446744073709551616.0) return UINT64_MAX;
  return (uint64_t)r;
}
template <> uint32_t sat_cast<uint32_t>(double r) {
  if (!(r > 0.0)) return 0;
  if (r >= 4294967296.0) return UINT32_MAX;
  return (uint32_t)r;
}

// Prediction of local index i: decompression/FullDecompressionKernels.cuh:161 (fma),
// :187 (round, half away from zero), and the encoder compression/CompressionKernels.cuh:318-324.
template <typename T> T predict(double theta0, double theta1, int64_t i) {
  double p = std::fma(theta1, (double)i, theta0);
  return sat_cast<T>(std::round(p));
}

// core/MathHelpers.cuh:22-53 calculateDelta
template <typename T> long long calc_delta(T actual, T pred) {
  if (TypeInfo<T>::is_signed) {
    // signed: (ll)a - (ll)p; wraps on the GPU when it overflows
    return (long long)((unsigned long long)(long long)actual - (unsigned long long)(long long)pred);
  }
  if (sizeof(T) == 8) {
    unsigned long long a = (unsigned long long)actual, p = (unsigned long long)pred;
    if (a >= p) {
      unsigned long long d = a - p;
      return d <= (unsigned long long)LLONG_MAX ? (long long)d : LLONG_MAX;
    }
    unsigned long long d = p - a;
    return d <= (unsigned long long)LLONG_MAX ? -(long long)d : LLONG_MIN;
  }
  return (long long)actual - (long long)pred;
}

// core/MathHelpers.cuh:55-84 applyDelta (wraparound)
template <typename T> T apply_delta(T pred, long long delta) {
  if (sizeof(T) == 8) return (T)((unsigned long long)pred + (unsigned long long)delta);
  return (T)((uint32_t)pred + (uint32_t)delta);
}

// |delta| for the bit width.  The reference computes (d < 0) ? -d : d
// (compression/CompressionKernels.cuh:171-174), which leaves LLONG_MIN negative, so such a
// residual never raises the maximum and is later truncated (the value does not round-trip).
// Here |LLONG_MIN| counts as LLONG_MAX, which forces 64-bit fields; every other residual gets
// the reference's width.
long long abs_ref(long long d) {
  if (d == LLONG_MIN) return LLONG_MAX;
  return d < 0 ? -d : d;
}

// compression/CompressionKernels.cuh:194-206: bits = bitlen(max|delta|) + 1, capped at 64.
int bits_for(long long max_err) {
  if (max_err <= 0) return 0;
  int b = 64 - __builtin_clzll((unsigned long long)max_err);
  return std::min(b + 1, kMaxDeltaBits);
}

// core/MathHelpers.cuh:10-19 mightOverflowDoublePrecision
template <typename T> bool overflows_double(T v) {
  if (TypeInfo<T>::is_signed) return false;
  return (uint64_t)v > (1ULL << 53);
}

// ---------------------------------------------------------------------------------------
// Least-squares line from exact sums.  x = local index 0..n-1, y = value.
//   theta1 = sum((x - xbar) * y) / sum((x - xbar)^2)
//          = (2*Sxy - (n-1)*Sy) / (n*(n^2-1)/6)      numerator and denominator exact
//   theta0 = (Sy - theta1 * Sx) / n,  Sx = n(n-1)/2
// For n == 1 the reference falls back to theta1 = 0, theta0 = Sy / n
// (compression/CompressionKernels.cuh:142-151, same normal equations).
// ---------------------------------------------------------------------------------------
void solve_line(int64_t n, i128 sy, i128 sxy, double* theta0, double* theta1) {
  if (n <= 0) { *theta0 = 0.0; *theta1 = 0.0; return; }
  if (n == 1) { *theta1 = 0.0; *theta0 = i128_to_double(sy); return; }
  i128 N = n;
  i128 num = 2 * sxy - (N - 1) * sy;
  i128 den6 = N * (N * N - 1) / 6;
  double t1 = i128_to_double(num) / i128_to_double(den6);
  double sx = i128_to_double(N * (N - 1) / 2);
  double prod = t1 * sx;
  double diff = i128_to_double(sy) - prod;
  *theta1 = t1;
  *theta0 = diff / (double)n;
}

template <typename T> struct Fit {
  int type; double theta0, theta1; int bits; long long err;
};

// Max |delta| of values v[0..n) under (theta0, theta1).
template <typename T> long long max_err(const T* v, int64_t n, double th0, double th1) {
  long long m = 0;
  for (int64_t i = 0; i < n; i++) {
    long long a = abs_ref(calc_delta<T>(v[i], predict<T>(th0, th1, i)));
    if (a > m) m = a;
  }
  return m;
}

// Fit of one partition: compression/CompressionKernels.cuh:45-218 (overflow check -> direct
// copy, linear fit, max error, bit width), with exact sums as described above.
template <typename T> Fit<T> fit_partition(const T* v, int64_t n) {
  Fit<T> f;
  bool over = false;
  for (int64_t i = 0; i < n && !over; i++) over = overflows_double<T>(v[i]);
  if (over) {  // CompressionKernels.cuh:95-105
    f.type = M_DIRECT; f.theta0 = 0.0; f.theta1 = 0.0; f.err = 0; f.bits = (int)sizeof(T) * 8;
    return f;
  }
  i128 sy = 0, sxy = 0;
  for (int64_t i = 0; i < n; i++) { sy += (i128)v[i]; sxy += (i128)i * (i128)v[i]; }
  solve_line(n, sy, sxy, &f.theta0, &f.theta1);
  f.type = M_LINEAR;
  f.err = max_err<T>(v, n, f.theta0, f.theta1);
  f.bits = bits_for(f.err);
  return f;
}

// ---------------------------------------------------------------------------------------
// Bitstream: core/BitManipulation.cuh:80-200 (extract), CompressionKernels.cuh:287-368 (pack).
// Field of element i of partition p at bit offset[p] + i*bits, LSB first in uint32 words.
// ---------------------------------------------------------------------------------------
void put_bits(uint32_t* w, int64_t bitpos, int nbits, uint64_t field) {
  while (nbits > 0) {
    int64_t wi = bitpos >> 5; int off = (int)(bitpos & 31);
    int take = std::min(nbits, 32 - off);
    uint64_t mask = (take == 64) ? ~0ULL : ((1ULL << take) - 1ULL);
    w[wi] |= (uint32_t)((field & mask) << off);
    field >>= take; nbits -= take; bitpos += take;
  }
}

uint64_t get_bits(const uint32_t* w, int64_t nwords, int64_t bitpos, int nbits) {
  uint64_t r = 0; int shift = 0;
  while (nbits > 0) {
    int64_t wi = bitpos >> 5; int off = (int)(bitpos & 31);
    int take = std::min(nbits, 32 - off);
    uint32_t word = (wi < nwords) ? w[wi] : 0u;
    uint64_t part = (uint64_t)(word >> off) & ((take == 32) ? 0xFFFFFFFFULL : ((1ULL << take) - 1ULL));
    r |= part << shift;
    shift += take; nbits -= take; bitpos += take;
  }
  return r;
}

long long sign_extend(uint64_t f, int bits) {
  if (bits <= 0) return 0;
  if (bits >= 64) return (long long)f;
  uint64_t sign = 1ULL << (bits - 1);
  return (long long)((f ^ sign) - sign);
}

template <typename T> T decode_one(const int32_t* starts, const int32_t* types, const double* params,
                                   const int32_t* bits, const int64_t* offs, const uint32_t* words,
                                   int64_t nwords, int p, int64_t pos) {
  int64_t local = pos - starts[p];
  int b = bits[p];
  if (types[p] == M_DIRECT) {  // BitManipulation.cuh:155-200 zero-extended raw value
    if (b <= 0) return (T)0;
    return (T)get_bits(words, nwords, offs[p] + local * b, b);
  }
  long long d = 0;
  if (b > 0) d = sign_extend(get_bits(words, nwords, offs[p] + local * b, b), b);
  T pred = predict<T>(params[4 * (int64_t)p], params[4 * (int64_t)p + 1], local);
  return apply_delta<T>(pred, d);
}

// Prediction variants of the reference's decoders that depart from the format's contract
// (fma, round half away from zero).  They exist only to predict, value for value, what those
// decoders return on a blob, so that a test can compare the reference's output exactly.
enum PredVariant {
  PV_FMA_HALF_AWAY = 0,  // every full decoder and packed random access (the contract, predict<T>)
  // directRandomAccessCPU (api/G-LeCo.cuh:1470-1646): theta0 + theta1 * i as two separately
  // rounded operations (x86-64 host code, no fma unit assumed), clamps for 4-byte types and
  // unsigned types below zero, then static_cast<T>(std::round(p)).
  PV_SUM_HALF_AWAY = 1,
  // randomAccessFixedPreUnpackedKernel (decompression/FixedPartitionKernels.cuh:185-206):
  // __fma_rn, then __double2int_rn / __double2uint_rn after clamping (4-byte types) or
  // __double2ll_rn (8-byte types): round half to EVEN, saturating.
  PV_FMA_HALF_EVEN = 2,
};

template <typename T> T predict_variant(double theta0, double theta1, int64_t i, int variant) {
  if (variant == PV_FMA_HALF_AWAY) return predict<T>(theta0, theta1, i);
  if (variant == PV_SUM_HALF_AWAY) {
    double p = theta0 + theta1 * (double)i;  // -ffp-contract=off: two roundings
    if (!TypeInfo<T>::is_signed) {
      if (p < 0) p = 0;
      else if (sizeof(T) == 4 && p > 4294967295.0) p = 4294967295.0;
    } else if (sizeof(T) == 4) {
      if (p > 2147483647.0) p = 2147483647.0;
      else if (p < -2147483648.0) p = -2147483648.0;
    }
    // out-of-range 8-byte casts are undefined in C++; in-range values are exact either way
    return sat_cast<T>(std::round(p));
  }
  double p = std::fma(theta1, (double)i, theta0);
  double r = std::nearbyint(p);  // default rounding mode: nearest, ties to even
  if (sizeof(T) == 4) {
    if (!TypeInfo<T>::is_signed) return (T)sat_cast<uint32_t>(std::nearbyint(std::fmax(0.0, std::fmin(p, 4294967295.0))));
    return (T)sat_cast<int32_t>(std::nearbyint(std::fmax(-2147483648.0, std::fmin(p, 2147483647.0))));
  }
  return (T)sat_cast<int64_t>(r);  // __double2ll_rn saturates to the int64 range, then static_cast<T>
}

// Partition of a position by binary search over [start, end) (RandomAccessKernels.cuh:55-169).
int find_partition(const int32_t* starts, const int32_t* ends, int P, int64_t pos) {
  int lo = 0, hi = P - 1;
  while (lo <= hi) {
    int mid = lo + (hi - lo) / 2;
    if (pos >= starts[mid] && pos < ends[mid]) return mid;
    if (pos < starts[mid]) hi = mid - 1; else lo = mid + 1;
  }
  return -1;
}

// ---------------------------------------------------------------------------------------
// Variable partitioning of THIS implementation (device algorithm, restated).
//
// Split (the reference's greedy walk, compression/CpuPartitioner.cuh:141-195): from a start s,
// try sizes 128..3712 in the reference's stepping (128 up to 640, then 256 up to 2176, then
// 512), keep the size with the smallest cost per element (first minimum wins), jump there.
// Every start on the walk is a multiple of 128, so the best end of every 128-aligned start
// can be evaluated independently and the walk from 0 follows those pointers.
// Cost = 80 + len * bits / 8 (CpuPartitioner.cuh:128-138), bits from the exact-sum fit.
//
// Merge: the reference merges left to right, absorbing right neighbours while the merged
// cost is below the sum (CpuPartitioner.cuh:198-242).  Here merging runs in rounds: each
// round evaluates every adjacent pair, and merges the profitable pairs whose index k has
// (k + round) even, so chosen pairs never overlap; rounds stop when no pair is profitable
// (or after kMaxMergeRounds).
// ---------------------------------------------------------------------------------------
const int kSplitSizes[14] = {128, 256, 384, 512, 640, 896, 1152, 1408, 1664, 1920, 2176, 2688, 3200, 3712};
const int kMaxMergeRounds = 64;

template <typename T> struct VarPartitioner {
  const T* v; int64_t n; int64_t nb;
  std::vector<i128> py, piy;  // exclusive block prefix of y and of (global index * y)

  VarPartitioner(const T* v_, int64_t n_) : v(v_), n(n_) {
    nb = (n + kMinPart - 1) / kMinPart;
    py.assign(nb + 1, 0); piy.assign(nb + 1, 0);
    for (int64_t j = 0; j < nb; j++) {
      i128 sy = 0, siy = 0;
      int64_t e = std::min(n, (j + 1) * kMinPart);
      for (int64_t i = j * kMinPart; i < e; i++) { sy += (i128)v[i]; siy += (i128)i * (i128)v[i]; }
      py[j + 1] = py[j] + sy; piy[j + 1] = piy[j] + siy;
    }
  }
  int64_t blk(int64_t pos) const { return (pos >= n) ? nb : pos / kMinPart; }
  int range_bits(int64_t a, int64_t b) const {
    int64_t len = b - a;
    if (len <= 0) return 0;
    i128 sy = py[blk(b)] - py[blk(a)];
    i128 sxy = (piy[blk(b)] - piy[blk(a)]) - (i128)a * sy;
    double t0, t1;
    solve_line(len, sy, sxy, &t0, &t1);
    return bits_for(max_err<T>(v + a, len, t0, t1));
  }
  double cost(int64_t a, int64_t b) const {
    return kModelBytes + (double)(b - a) * (double)range_bits(a, b) / 8.0;
  }
  int64_t best_end(int64_t s) const {
    int64_t max_size = std::min<int64_t>(n - s, (int64_t)kMinPart * 32);
    int64_t best = std::min<int64_t>(s + kMinPart, n);
    double best_cpe = std::numeric_limits<double>::max();
    for (int k = 0; k < 14; k++) {
      int64_t size = kSplitSizes[k];
      if (size > max_size) break;
      double cpe = cost(s, s + size) / (double)size;
      if (cpe < best_cpe) { best_cpe = cpe; best = s + size; }
    }
    return best;
  }
  void run(std::vector<int32_t>& starts, std::vector<int32_t>& ends) {
    starts.clear(); ends.clear();
    if (n <= 0) return;
    std::vector<int64_t> ps, pe; std::vector<double> pc;
    for (int64_t s = 0; s < n;) {
      int64_t e = best_end(s);
      ps.push_back(s); pe.push_back(e); pc.push_back(cost(s, e));
      s = e;
    }
    for (int r = 0; r < kMaxMergeRounds; r++) {
      size_t m = ps.size();
      if (m < 2) break;
      std::vector<char> prof(m - 1, 0); std::vector<double> mc(m - 1, 0.0);
      bool any = false;
      for (size_t k = 0; k + 1 < m; k++) {
        mc[k] = cost(ps[k], pe[k + 1]);
        double sum = pc[k] + pc[k + 1];
        prof[k] = mc[k] < sum;
        any = any || prof[k];
      }
      if (!any) break;
      std::vector<int64_t> ns, ne; std::vector<double> nc;
      for (size_t k = 0; k < m;) {
        if (k + 1 < m && prof[k] && ((k + (size_t)r) % 2 == 0)) {
          ns.push_back(ps[k]); ne.push_back(pe[k + 1]); nc.push_back(mc[k]); k += 2;
        } else {
          ns.push_back(ps[k]); ne.push_back(pe[k]); nc.push_back(pc[k]); k += 1;
        }
      }
      ps.swap(ns); pe.swap(ne); pc.swap(nc);
    }
    for (size_t k = 0; k < ps.size(); k++) { starts.push_back((int32_t)ps[k]); ends.push_back((int32_t)pe[k]); }
  }
};

// ---------------------------------------------------------------------------------------
// The reference's CPU partitioner, restated with its own arithmetic
// (compression/CpuPartitioner.cuh:33-422): sequential double prefix sums of y, range sums
// from prefix differences, sum_x = n*(n-1)/2.0 computed in int (wraps for n >= 46342),
// prediction theta0 + theta1*i without fma, host casts, greedy split, sequential merge with
// at most 10 passes.  Used for compressed-size parity and as the CPU baseline.
// ---------------------------------------------------------------------------------------
template <typename T> struct RefCpuPartitioner {
  const T* v; int n;
  std::vector<double> prefix_y;
  struct Cand { int s, e; double t0, t1; long long err; int bits; double cost; };

  RefCpuPartitioner(const T* v_, int n_) : v(v_), n(n_) {}

  void sums(int start, int end, double& sx, double& sy, double& sxx, double& sxy) const {
    int len = end - start;
    int prod = (int)((unsigned)len * (unsigned)(len - 1));  // int overflow wraps (CpuPartitioner.cuh:60)
    sx = prod / 2.0;
    sy = prefix_y[end] - prefix_y[start];
    sxx = 0.0; sxy = 0.0;
    for (int i = 0; i < len; i++) {
      double lx = i; int gx = start + i;
      double a = lx * lx; sxx = sxx + a;
      double b = lx * (prefix_y[gx + 1] - prefix_y[gx]); sxy = sxy + b;
    }
  }
  void fit(int start, int end, double& t0, double& t1, long long& err, int& bits) const {
    int len = end - start;
    if (len <= 0) { t0 = t1 = 0.0; err = 0; bits = 0; return; }
    double sx, sy, sxx, sxy;
    sums(start, end, sx, sy, sxx, sxy);
    double a = len * sxx; double b = sx * sx; double det = a - b;
    if (std::abs(det) > 1e-10) {
      double c = len * sxy; double d = sx * sy;
      t1 = (c - d) / det;
      double e = t1 * sx;
      t0 = (sy - e) / len;
    } else {
      t1 = 0.0; t0 = sy / len;
    }
    err = 0;
    for (int i = 0; i < len; i++) {
      double m = t1 * i; double pred = t0 + m;
      T pt = static_cast<T>(std::round(pred));  // host cast, as in CpuPartitioner.cuh:106
      long long dlt = calc_delta<T>(v[start + i], pt);
      long long ad = dlt < 0 ? (long long)(0ULL - (unsigned long long)dlt) : dlt;
      err = std::max(err, ad);
    }
    bits = bits_for(err);
  }
  double cost(int start, int end) const {
    double t0, t1; long long err; int bits;
    fit(start, end, t0, t1, err, bits);
    return kModelBytes + static_cast<double>(end - start) * bits / 8.0;
  }
  void run(std::vector<int32_t>& starts, std::vector<int32_t>& ends) {
    starts.clear(); ends.clear();
    if (n <= 0) return;
    prefix_y.assign((size_t)n + 1, 0.0);
    for (int i = 0; i < n; i++) prefix_y[i + 1] = prefix_y[i] + static_cast<double>(v[i]);
    std::vector<Cand> c;
    int cur = 0;
    while (cur < n) {  // CpuPartitioner.cuh:150-194
      int best_end = std::min(cur + kMinPart, n);
      double best_cpe = std::numeric_limits<double>::max();
      int step = kMinPart;
      int max_size = std::min(n - cur, kMinPart * 32);
      for (int size = kMinPart; size <= max_size; size += step) {
        int end = std::min(cur + size, n);
        double cpe = cost(cur, end) / (end - cur);
        if (cpe < best_cpe) { best_cpe = cpe; best_end = end; }
        if (size > kMinPart * 4) step = kMinPart * 2;
        if (size > kMinPart * 16) step = kMinPart * 4;
      }
      Cand k; k.s = cur; k.e = best_end;
      fit(cur, best_end, k.t0, k.t1, k.err, k.bits);
      k.cost = cost(cur, best_end);
      c.push_back(k);
      cur = best_end;
    }
    bool changed = true; int it = 0;  // CpuPartitioner.cuh:198-242
    while (changed && it < 10) {
      changed = false; it++;
      for (int i = 0; i < (int)c.size() - 1;) {
        double comb = c[i].cost + c[i + 1].cost;
        double merged = cost(c[i].s, c[i + 1].e);
        if (merged < comb) {
          c[i].e = c[i + 1].e;
          fit(c[i].s, c[i].e, c[i].t0, c[i].t1, c[i].err, c[i].bits);
          c[i].cost = merged;
          c.erase(c.begin() + i + 1);
          changed = true;
        } else {
          i++;
        }
      }
    }
    for (auto& k : c) { starts.push_back(k.s); ends.push_back(k.e); }
  }
};

// ---------------------------------------------------------------------------------------
// Serialized blob, version 5: api/G-LeCo.cuh:826-1016 (CPU) and :1999-2152 (GPU, same bytes).
// Header layout core/InternalTypes.cuh:39-63 (120 bytes; 4 trailing pad bytes are zero).
// ---------------------------------------------------------------------------------------
#pragma pack(push, 1)
struct BlobHeader {
  uint32_t magic, version, total_values, num_partitions;
  uint64_t start_off, end_off, types_off, params_off, bits_off, offsets_off, errb_off, delta_off;
  uint64_t params_size, delta_size;
  uint32_t type_size, checksum;
  uint32_t reserved[3];
  uint32_t pad;
};
#pragma pack(pop)
static_assert(sizeof(BlobHeader) == 120, "blob header is 120 bytes");

const uint32_t kMagic = 0x4F43454C;

// api/G-LeCo.cuh:87-100 (rotate-add branch, taken when the host compiler lacks SSE4.2) and
// the CRC32C branch (byte-wise, Castagnoli polynomial, reflected 0x82F63B78, initial value 0,
// no final xor -- exactly what _mm_crc32_u8 accumulates from 0).
uint32_t checksum(const uint8_t* p, size_t n, int crc32c) {
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

uint64_t align8(uint64_t x) { return (x + 7) & ~7ULL; }

}  // namespace

// =======================================================================================
// (4) The reference's GPU partitioner (use_gpu_partitioning = true):
//     GPUVariableLengthPartitionerV6<T>::partition, compression/GpuPartitioner.cuh:34-214, with
//     analyzeDataVarianceFast and createPartitionsFast, compression/PartitioningKernels.cuh:647-727.
//     Only its boundaries matter: compress refits every partition (api/G-LeCo.cuh:512-530).
// =======================================================================================

// PartitioningKernels.cuh:647-692: 128 threads per variance block; thread t Kahan-sums v and v^2
// over positions start + t + 128k (v*v - c contracted to one fma by the reference's compiler);
// each warp reduces with __shfl_down over 16, 8, 4, 2, 1 (MathHelpers.cuh:91-95), and lane 0 adds
// float(S2/n - (S1/n)^2) (again one fma) into the block's value.  The reference adds the four
// warp values with float atomics in completion order; this restatement adds them in warp order.
template <typename T>
static float v6_block_variance(const T* v, int64_t start, int64_t end) {
  double s1[128], s2[128];
  for (int t = 0; t < 128; t++) {
    double a = 0.0, b = 0.0, c1 = 0.0, c2 = 0.0;
    for (int64_t i = start + t; i < end; i += 128) {
      const double x = (double)v[i];
      const double y1 = x - c1;
      const double t1 = a + y1;
      c1 = (t1 - a) - y1;
      a = t1;
      const double y2 = std::fma(x, x, -c2);
      const double t2 = b + y2;
      c2 = (t2 - b) - y2;
      b = t2;
    }
    s1[t] = a;
    s2[t] = b;
  }
  const double dn = (double)(end - start);
  float acc = 0.0f;
  for (int w = 0; w < 4; w++) {
    double a[32], b[32];
    for (int l = 0; l < 32; l++) { a[l] = s1[32 * w + l]; b[l] = s2[32 * w + l]; }
    for (int off = 16; off > 0; off >>= 1)  // lanes whose source is past the warp keep their value
      for (int l = 0; l < 32; l++) {
        const double ya = l + off < 32 ? a[l + off] : a[l];
        const double yb = l + off < 32 ? b[l + off] : b[l];
        // lane l reads lane l + off's value from before this step: walk lanes upwards
        a[l] = a[l] + ya;
        b[l] = b[l] + yb;
      }
    const double m = a[0] / dn;
    acc = acc + (float)std::fma(-m, m, b[0] / dn);
  }
  return acc;
}

// GpuPartitioner.cuh:44-84 and PartitioningKernels.cuh:695-727: the thresholds are the values of
// rank nb/4, nb/2, 3nb/4 of the sorted block values.  thrust::sort sorts the value array IN PLACE
// (GpuPartitioner.cuh:60-61) before createPartitionsFast reads it, so block i is sized by the i-th
// smallest value, not by its own: 4*base, 2*base, base or base/2 by the first threshold that value
// is below (with distinct values: the first quarter of the blocks by position get 4*base, and so
// on).  The last partition of a block ends at the block's end.
template <typename T>
static void v6_partition(const T* v, int64_t n, int64_t base, std::vector<int32_t>& starts,
                         std::vector<int32_t>& ends, std::vector<float>* variances) {
  starts.clear();
  ends.clear();
  if (n <= 0) return;
  const int64_t blen = 8 * base, nb = (n + blen - 1) / blen;
  std::vector<float> var((size_t)nb);
  for (int64_t b = 0; b < nb; b++) var[b] = v6_block_variance(v, b * blen, std::min(n, (b + 1) * blen));
  std::vector<float> sorted = var;
  std::sort(sorted.begin(), sorted.end());
  const float t0 = sorted[nb / 4], t1 = sorted[nb / 2], t2 = sorted[3 * nb / 4];
  for (int64_t b = 0; b < nb; b++) {
    const float x = sorted[b];
    const int64_t size = x < t0 ? 4 * base : (x < t1 ? 2 * base : (x < t2 ? base : base / 2));
    const int64_t bs = b * blen, be = std::min(n, bs + blen);
    for (int64_t j = bs; j < be; j += size) {
      starts.push_back((int32_t)j);
      ends.push_back((int32_t)std::min(j + size, be));
    }
  }
  if (variances) *variances = var;
}

// =======================================================================================
// extern "C" surface used by tests/ through ctypes.
// =======================================================================================
#define DISPATCH(dtype, CALL)                                   \
  switch (dtype) {                                              \
    case DT_I32: { typedef int32_t T; CALL; break; }            \
    case DT_I64: { typedef int64_t T; CALL; break; }            \
    case DT_U64: { typedef uint64_t T; CALL; break; }           \
    case DT_U32: { typedef uint32_t T; CALL; break; }           \
    default: return -1;                                         \
  }

extern "C" {

double orc_i128_to_double(int64_t hi, uint64_t lo) {
  i128 v = ((i128)hi << 64) | (i128)lo;
  return i128_to_double(v);
}

void orc_solve_line(int64_t n, int64_t sy_hi, uint64_t sy_lo, int64_t sxy_hi, uint64_t sxy_lo,
                    double* theta0, double* theta1) {
  i128 sy = ((i128)sy_hi << 64) | (i128)sy_lo;
  i128 sxy = ((i128)sxy_hi << 64) | (i128)sxy_lo;
  solve_line(n, sy, sxy, theta0, theta1);
}

uint32_t orc_checksum(const uint8_t* p, uint64_t n, int crc32c) { return checksum(p, (size_t)n, crc32c); }

// Fixed partitions: api/G-LeCo.cuh:401-416 (partition size L, last one short).
int64_t orc_partition_fixed(int64_t n, int32_t L, int32_t* starts, int32_t* ends, int64_t cap) {
  if (n <= 0 || L <= 0) return 0;
  int64_t P = (n + L - 1) / L;
  if (P > cap) return -P;
  for (int64_t p = 0; p < P; p++) { starts[p] = (int32_t)(p * L); ends[p] = (int32_t)std::min<int64_t>(n, (p + 1) * L); }
  return P;
}

// Variable partitions of this implementation (see VarPartitioner).  Returns P, or -P if cap is short.
int64_t orc_partition_variable(int dtype, const void* values, int64_t n, int32_t* starts, int32_t* ends, int64_t cap) {
  std::vector<int32_t> s, e;
  DISPATCH(dtype, { VarPartitioner<T> vp((const T*)values, n); vp.run(s, e); });
  if ((int64_t)s.size() > cap) return -(int64_t)s.size();
  for (size_t i = 0; i < s.size(); i++) { starts[i] = s[i]; ends[i] = e[i]; }
  return (int64_t)s.size();
}

// The reference's GPU partitioner boundaries (restated).  Returns P, or -P if cap is short.
int64_t orc_partition_v6(int dtype, const void* values, int64_t n, int32_t base, int32_t* starts, int32_t* ends,
                         int64_t cap) {
  std::vector<int32_t> s, e;
  DISPATCH(dtype, { v6_partition<T>((const T*)values, n, base, s, e, nullptr); });
  if ((int64_t)s.size() > cap) return -(int64_t)s.size();
  for (size_t i = 0; i < s.size(); i++) { starts[i] = s[i]; ends[i] = e[i]; }
  return (int64_t)s.size();
}

// The per-block values the V6 thresholds are taken from.  Returns the block count.
int64_t orc_v6_variances(int dtype, const void* values, int64_t n, int32_t base, float* out, int64_t cap) {
  std::vector<int32_t> s, e;
  std::vector<float> var;
  DISPATCH(dtype, { v6_partition<T>((const T*)values, n, base, s, e, &var); });
  if ((int64_t)var.size() > cap) return -(int64_t)var.size();
  for (size_t i = 0; i < var.size(); i++) out[i] = var[i];
  return (int64_t)var.size();
}

// Best split end of one 128-aligned start (one entry of the device's split table).
int64_t orc_split_best_end(int dtype, const void* values, int64_t n, int64_t start) {
  int64_t r = 0;
  DISPATCH(dtype, { VarPartitioner<T> vp((const T*)values, n); r = vp.best_end(start); });
  return r;
}

// Bits of one range under this implementation's exact-sum fit (no direct-copy check).
int orc_range_bits(int dtype, const void* values, int64_t n, int64_t a, int64_t b) {
  int r = 0;
  DISPATCH(dtype, { VarPartitioner<T> vp((const T*)values, n); r = vp.range_bits(a, b); });
  return r;
}

// The reference's CPU partitioner (restated).  Returns P, or -P if cap is short.
int64_t orc_ref_partition_cpu(int dtype, const void* values, int64_t n, int32_t* starts, int32_t* ends, int64_t cap) {
  std::vector<int32_t> s, e;
  DISPATCH(dtype, { RefCpuPartitioner<T> rp((const T*)values, (int)n); rp.run(s, e); });
  if ((int64_t)s.size() > cap) return -(int64_t)s.size();
  for (size_t i = 0; i < s.size(); i++) { starts[i] = s[i]; ends[i] = e[i]; }
  return (int64_t)s.size();
}

// Fit every partition (CompressionKernels.cuh:45-218).  params is 4*P doubles {t0, t1, 0, 0}.
int orc_fit(int dtype, const void* values, const int32_t* starts, const int32_t* ends, int64_t P,
            int32_t* types, double* params, int32_t* bits, int64_t* err) {
  DISPATCH(dtype, {
    const T* v = (const T*)values;
    for (int64_t p = 0; p < P; p++) {
      Fit<T> f = fit_partition<T>(v + starts[p], (int64_t)ends[p] - starts[p]);
      types[p] = f.type; bits[p] = f.bits; err[p] = f.err;
      params[4 * p] = f.theta0; params[4 * p + 1] = f.theta1; params[4 * p + 2] = 0.0; params[4 * p + 3] = 0.0;
    }
  });
  return 0;
}

// Max |delta| of values under a given line (for columns with chosen parameters).
int64_t orc_max_err_for_line(int dtype, const void* values, int64_t n, double theta0, double theta1) {
  int64_t r = 0;
  DISPATCH(dtype, { r = max_err<T>((const T*)values, n, theta0, theta1); });
  return r;
}

int orc_bits_for(int64_t max_err) { return bits_for(max_err); }

// Exclusive prefix of len*bits (CompressionKernels.cuh:222-238); returns total bits.
int64_t orc_bit_offsets(const int32_t* starts, const int32_t* ends, const int32_t* bits, int64_t P, int64_t* offs) {
  int64_t acc = 0;
  for (int64_t p = 0; p < P; p++) { offs[p] = acc; acc += (int64_t)(ends[p] - starts[p]) * bits[p]; }
  return acc;
}

// Reported compressed size (api/G-LeCo.cuh:589-603): 64 B per partition + 120 B header + ceil(bits/8).
int64_t orc_reported_size(int64_t P, int64_t total_bits) { return 64 * P + 120 + (total_bits + 7) / 8; }

// Pack residuals (CompressionKernels.cuh:242-372) into words (zeroed here first).
int orc_pack(int dtype, const void* values, const int32_t* starts, const int32_t* ends, const int32_t* types,
             const double* params, const int32_t* bits, const int64_t* offs, int64_t P, uint32_t* words, int64_t nwords) {
  std::memset(words, 0, (size_t)nwords * 4);
  DISPATCH(dtype, {
    const T* v = (const T*)values;
    for (int64_t p = 0; p < P; p++) {
      int b = bits[p];
      if (b <= 0) continue;
      for (int64_t i = 0; i < (int64_t)ends[p] - starts[p]; i++) {
        T x = v[starts[p] + i];
        uint64_t field;
        if (types[p] == M_DIRECT) {
          field = (uint64_t)x;
        } else {
          long long d = calc_delta<T>(x, predict<T>(params[4 * p], params[4 * p + 1], i));
          field = (uint64_t)d;
        }
        if (b < 64) field &= (1ULL << b) - 1ULL;
        put_bits(words, offs[p] + i * b, b, field);
      }
    }
  });
  return 0;
}

// Full decode (FullDecompressionKernels.cuh:47-192; every variant computes the same values).
int orc_decode_full(int dtype, const int32_t* starts, const int32_t* ends, const int32_t* types, const double* params,
                    const int32_t* bits, const int64_t* offs, int64_t P, const uint32_t* words, int64_t nwords,
                    int64_t n, void* out) {
  DISPATCH(dtype, {
    T* o = (T*)out;
    for (int64_t i = 0; i < n; i++) o[i] = (T)0;
    for (int64_t p = 0; p < P; p++)
      for (int64_t i = starts[p]; i < ends[p] && i < n; i++)
        o[i] = decode_one<T>(starts, types, params, bits, offs, words, nwords, (int)p, i);
  });
  return 0;
}

// Random access (RandomAccessKernels.cuh:55-169): binary search, 0 for positions outside.
int orc_random_access(int dtype, const int32_t* starts, const int32_t* ends, const int32_t* types, const double* params,
                      const int32_t* bits, const int64_t* offs, int64_t P, const uint32_t* words, int64_t nwords,
                      const int32_t* pos, int64_t q, void* out) {
  DISPATCH(dtype, {
    T* o = (T*)out;
    for (int64_t k = 0; k < q; k++) {
      int p = find_partition(starts, ends, (int)P, pos[k]);
      o[k] = (p < 0) ? (T)0 : decode_one<T>(starts, types, params, bits, offs, words, nwords, p, pos[k]);
    }
  });
  return 0;
}

// What one of the reference's decoders returns at each position (see PredVariant): the same
// residual field and direct-copy rule as decode_one, with that decoder's prediction.  0 for
// positions outside the column.
int orc_decode_variant(int dtype, const int32_t* starts, const int32_t* ends, const int32_t* types,
                       const double* params, const int32_t* bits, const int64_t* offs, int64_t P,
                       const uint32_t* words, int64_t nwords, const int32_t* pos, int64_t q, int variant, void* out) {
  DISPATCH(dtype, {
    T* o = (T*)out;
    for (int64_t k = 0; k < q; k++) {
      int p = find_partition(starts, ends, (int)P, pos[k]);
      if (p < 0) { o[k] = (T)0; continue; }
      int64_t local = (int64_t)pos[k] - starts[p];
      int b = bits[p];
      if (types[p] == M_DIRECT) {
        o[k] = b <= 0 ? (T)0 : (T)get_bits(words, nwords, offs[p] + local * b, b);
        continue;
      }
      long long d = b > 0 ? sign_extend(get_bits(words, nwords, offs[p] + local * b, b), b) : 0;
      o[k] = apply_delta<T>(predict_variant<T>(params[4 * (int64_t)p], params[4 * (int64_t)p + 1], local, variant), d);
    }
  });
  return 0;
}

// Residuals as int64 per value (decompression/UnpackKernel.cuh:31-98): sign-extended
// residual, or the zero-extended raw value for direct-copy partitions.
int orc_unpack_deltas(int dtype, const int32_t* starts, const int32_t* ends, const int32_t* types,
                      const int32_t* bits, const int64_t* offs, int64_t P, const uint32_t* words, int64_t nwords,
                      int64_t n, int64_t* plain) {
  (void)dtype;
  for (int64_t i = 0; i < n; i++) plain[i] = 0;
  for (int64_t p = 0; p < P; p++) {
    int b = bits[p];
    for (int64_t i = starts[p]; i < ends[p] && i < n; i++) {
      int64_t local = i - starts[p];
      if (b <= 0) { plain[i] = 0; continue; }
      uint64_t f = get_bits(words, nwords, offs[p] + local * b, b);
      plain[i] = (types[p] == M_DIRECT) ? (int64_t)f : sign_extend(f, b);
    }
  }
  return 0;
}

// Decode from pre-unpacked residuals (FullDecompressionKernels.cuh:196-288).
int orc_decode_preunpacked(int dtype, const int32_t* starts, const int32_t* ends, const int32_t* types,
                           const double* params, int64_t P, const int64_t* plain, int64_t n, void* out) {
  DISPATCH(dtype, {
    T* o = (T*)out;
    for (int64_t i = 0; i < n; i++) o[i] = (T)0;
    for (int64_t p = 0; p < P; p++)
      for (int64_t i = starts[p]; i < ends[p] && i < n; i++) {
        if (types[p] == M_DIRECT) { o[i] = (T)plain[i]; continue; }
        T pred = predict<T>(params[4 * p], params[4 * p + 1], i - starts[p]);
        o[i] = apply_delta<T>(pred, plain[i]);
      }
  });
  return 0;
}

// Blob size for P partitions and total_bits (api/G-LeCo.cuh:895-960).
uint64_t orc_blob_size(int64_t P, int64_t total_bits) {
  uint64_t off = 120;
  off = align8(off) + 4 * P; off = align8(off) + 4 * P; off = align8(off) + 4 * P;
  off = align8(off) + 32 * P; off = align8(off) + 4 * P; off = align8(off) + 8 * P;
  off = align8(off) + 8 * P; off = align8(off);
  return align8(off + (uint64_t)(total_bits + 7) / 8);
}

// Serialize to a blob of exactly orc_blob_size() bytes (api/G-LeCo.cuh:826-1016).
int64_t orc_serialize(int type_size, int64_t total_values, const int32_t* starts, const int32_t* ends,
                      const int32_t* types, const double* params, const int32_t* bits, const int64_t* offs,
                      const int64_t* err, int64_t P, const uint32_t* words, uint8_t* blob, uint64_t cap,
                      int crc32c) {
  uint64_t max_end = 0;
  for (int64_t p = 0; p < P; p++) {
    int64_t len = std::max<int64_t>(0, (int64_t)ends[p] - starts[p]);
    max_end = std::max<uint64_t>(max_end, (uint64_t)offs[p] + (uint64_t)len * (uint64_t)bits[p]);
  }
  uint64_t dbytes = (max_end + 7) / 8;
  BlobHeader h; std::memset(&h, 0, sizeof h);
  h.magic = kMagic; h.version = 5; h.total_values = (uint32_t)total_values; h.num_partitions = (uint32_t)P;
  uint64_t off = sizeof(BlobHeader);
  off = align8(off); h.start_off = off; off += 4 * P;
  off = align8(off); h.end_off = off; off += 4 * P;
  off = align8(off); h.types_off = off; off += 4 * P;
  off = align8(off); h.params_off = off; h.params_size = 32 * P; off += 32 * P;
  off = align8(off); h.bits_off = off; off += 4 * P;
  off = align8(off); h.offsets_off = off; off += 8 * P;
  off = align8(off); h.errb_off = off; off += 8 * P;
  off = align8(off); h.delta_off = off; h.delta_size = dbytes;
  h.type_size = (uint32_t)type_size;
  h.checksum = 0;
  h.checksum = checksum((const uint8_t*)&h, sizeof h, crc32c);
  uint64_t total = align8(off + dbytes);
  if (total > cap) return -(int64_t)total;
  std::memset(blob, 0, total);
  std::memcpy(blob, &h, sizeof h);
  if (P > 0) {
    std::memcpy(blob + h.start_off, starts, 4 * P);
    std::memcpy(blob + h.end_off, ends, 4 * P);
    std::memcpy(blob + h.types_off, types, 4 * P);
    std::memcpy(blob + h.params_off, params, 32 * P);
    std::memcpy(blob + h.bits_off, bits, 4 * P);
    std::memcpy(blob + h.offsets_off, offs, 8 * P);
    std::memcpy(blob + h.errb_off, err, 8 * P);
  }
  if (dbytes > 0) std::memcpy(blob + h.delta_off, words, dbytes);
  return (int64_t)total;
}

// Header validation of deserialize (api/G-LeCo.cuh:1019-1049), extended with bounds checks on
// every array.  Returns 0 when the blob is acceptable for a type of type_size bytes, else a
// nonzero reason code: 1 short, 2 magic/version, 3 type size, 4 checksum, 5 size, 6 array bounds.
int orc_blob_check(const uint8_t* blob, uint64_t size, int type_size, int crc32c,
                   int64_t* total_values, int64_t* P, uint64_t* delta_bytes) {
  if (!blob || size < sizeof(BlobHeader)) return 1;
  BlobHeader h; std::memcpy(&h, blob, sizeof h);
  if (h.magic != kMagic || (h.version != 4 && h.version != 5)) return 2;
  if ((int)h.type_size != type_size) return 3;
  BlobHeader t = h; t.checksum = 0;
  if (checksum((const uint8_t*)&t, sizeof t, crc32c) != h.checksum) return 4;
  uint64_t expected = h.delta_off + h.delta_size;
  if (h.version == 5) expected = align8(expected);
  if (h.delta_off > size || expected > size) return 5;
  uint64_t np = h.num_partitions;
  const uint64_t offs[7] = {h.start_off, h.end_off, h.types_off, h.params_off, h.bits_off, h.offsets_off, h.errb_off};
  const uint64_t lens[7] = {4 * np, 4 * np, 4 * np, 32 * np, 4 * np, 8 * np, 8 * np};
  for (int k = 0; k < 7; k++) if (offs[k] > size || lens[k] > size - offs[k]) return 6;
  *total_values = h.total_values; *P = (int64_t)np; *delta_bytes = h.delta_size;
  return 0;
}

// Copy the arrays out of a checked blob.  words must hold ceil(delta_bytes/4) words.
int orc_deserialize(const uint8_t* blob, int32_t* starts, int32_t* ends, int32_t* types, double* params,
                    int32_t* bits, int64_t* offs, int64_t* err, uint32_t* words) {
  BlobHeader h; std::memcpy(&h, blob, sizeof h);
  uint64_t P = h.num_partitions;
  if (P > 0) {
    std::memcpy(starts, blob + h.start_off, 4 * P);
    std::memcpy(ends, blob + h.end_off, 4 * P);
    std::memcpy(types, blob + h.types_off, 4 * P);
    std::memcpy(params, blob + h.params_off, 32 * P);
    std::memcpy(bits, blob + h.bits_off, 4 * P);
    std::memcpy(offs, blob + h.offsets_off, 8 * P);
    std::memcpy(err, blob + h.errb_off, 8 * P);
  }
  uint64_t nw = (h.delta_size + 3) / 4;
  if (nw) { words[nw - 1] = 0; std::memcpy(words, blob + h.delta_off, h.delta_size); }
  return 0;
}

}  // extern "C"
