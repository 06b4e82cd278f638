// partition.cu -- variable-length partitioning by model cost, on the device.
//
// Replaces VariableLengthPartitioner<T>::partition (compression/CpuPartitioner.cuh:342-422),
// which the reference runs single-threaded on the host (its GPU alternative,
// GPUVariableLengthPartitionerV6, sizes partitions by a variance heuristic and never merges).
//
// Cost of a partition [a, b): 80 + (b - a) * bits / 8 bytes (CpuPartitioner.cuh:128-138), with
// bits from the exact-sum least-squares fit of [a, b) (glc_device.cuh).
//
// Split.  The reference walks from 0: at start s it tries sizes 128..3712 (steps of 128 up to
// 640, then 256 up to 2176, then 512; CpuPartitioner.cuh:150-175), keeps the first size with
// the lowest cost per value and jumps there.  Every start on that walk is a multiple of 128 and
// the best end of a start depends on nothing else, so the walk is cut into ranges of 2048
// blocks: each range is walked from its first block and from the block where the previous
// range's first walk leaves it (one warp per range, each start's best end evaluated on the way:
// each value of its reach scored against all candidate lines that contain it), one warp chains
// the ranges through the exits of the visited starts, and each range marks its walk.  When the
// walk from 0 enters a range at a start no walk visited, the best end of every start is
// evaluated (one warp per start) and the ranges are chained through the exits of all their
// possible entry points instead.  The max |delta| each evaluation measured for the partition it
// chose is kept, so the split partitions' costs need no second pass over the values.
//
// Merge.  The reference absorbs right neighbours left to right while the merged cost is lower
// (CpuPartitioner.cuh:198-242).  Here merging runs in rounds: every adjacent pair is scored,
// and the profitable pairs with (index + round) even merge, so the chosen pairs never overlap;
// rounds stop when no pair is profitable (at most 64 rounds).  A pair whose two partitions did
// not change keeps its score from the previous round.
//
// Fits use exact 128-bit sums from a prefix over 128-value blocks (every boundary here is a
// multiple of 128 or n), so each candidate's line costs O(1) and only its max |delta| needs a
// pass over the values.  The CPU oracle restates this algorithm step for step.
#include "glc_internal.h"
#include "glc_scan.cuh"

namespace glc {

constexpr int kNumSizes = 14;
__constant__ int c_sizes[kNumSizes] = {128, 256, 384, 512, 640, 896, 1152, 1408, 1664, 1920, 2176, 2688, 3200, 3712};
__host__ __device__ constexpr int split_size(int k) {
  return k < 5 ? 128 * (k + 1) : k < 11 ? 640 + 256 * (k - 4) : 2176 + 512 * (k - 10);
}
static_assert(split_size(0) == 128 && split_size(4) == 640 && split_size(5) == 896 && split_size(10) == 2176 &&
              split_size(11) == 2688 && split_size(13) == 3712, "candidate sizes");
constexpr int kMaxJumpBlocks = 29;  // 3712 / 128
constexpr int kRangeBlocks = 2048;
constexpr int kMaxMergeRounds = 64;
constexpr int kPairChunk = 4096;
constexpr int32_t kUnknown = -1;  // best end of a start not evaluated

struct SumPair {  // trivially constructible: SumPair() value-initialises to zero
  i128 y;
  i128 iy;
  __device__ __forceinline__ SumPair operator+(const SumPair& o) const {
    SumPair r;
    r.y = y + o.y;
    r.iy = iy + o.iy;
    return r;
  }
};

// ---- block sums -----------------------------------------------------------------------
template <typename T> __global__ void block_sums_kernel(const T* __restrict__ v, int64_t n, int64_t nb, SumPair* __restrict__ out) {
  const int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= nb) return;
  i128 sy = 0, siy = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int64_t i = j * kMinPart + k * 32 + lane;
    if (i < n) {
      const i128 y = (i128)__ldg(v + i);
      sy += y;
      siy += (i128)i * y;
    }
  }
  sy = warp_sum_i128(sy);
  siy = warp_sum_i128(siy);
  if (lane == 0) {
    SumPair s;
    s.y = sy;
    s.iy = siy;
    out[j] = s;
  }
}

struct RangeSums {
  const SumPair* pre;  // nb + 1 entries
  int64_t n, nb;
  __device__ __forceinline__ int64_t blk(int64_t pos) const { return pos >= n ? nb : pos / kMinPart; }
  // exact sums of [a, b): sum y and sum (i - a) * y
  __device__ __forceinline__ void get(int64_t a, int64_t b, i128& sy, i128& sxy) const {
    const SumPair pb = pre[blk(b)], pa = pre[blk(a)];
    sy = pb.y - pa.y;
    sxy = (pb.iy - pa.iy) - (i128)a * sy;
  }
  __device__ __forceinline__ void line(int64_t a, int64_t b, double& t0, double& t1) const {
    i128 sy, sxy;
    get(a, b, sy, sxy);
    solve_line(b - a, sy, sxy, t0, t1);
  }
};

__device__ __forceinline__ double part_cost(int64_t len, int bits) {
  return __dadd_rn(kModelBytes, __ddiv_rn(__dmul_rn(__ll2double_rn(len), (double)bits), 8.0));
}

// ---- split: best end of every 128-aligned start ------------------------------------------
// Offsets [size(B-1), size(B)) lie in candidates B..13 only: one loop per band with the candidate
// range known at compile time, no per-candidate test.  Used when all 14 candidates exist and every
// prediction is >= -0.25 (so round-half-away is trunc(x + 0.5 - 2^-54) with a constant addend)
// and the values are below 2^51: all quantities are exact integers in FP64.
// A value of the start's reach: from global memory (read-only path) or from the warp's staged copy.
template <bool SMEM, typename T> __device__ __forceinline__ T ld_val(const T* p) {
  if constexpr (SMEM) return *p;
  else return __ldg(p);
}

// Copies vals[0, count) to win[0, count) with asynchronous copies (cp.async, element-sized, so any
// element-aligned input works); the caller waits with cp_async_wait_all + __syncwarp.
template <typename T>
__device__ __forceinline__ void stage_reach(const T* __restrict__ vals, T* win, int count, int lane) {
  for (int o = lane; o < count; o += 32) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(win + o);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dst), "l"(vals + o), "n"((int)sizeof(T))
                 : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <int B, bool SMEM, typename T>
__device__ __forceinline__ void split_bands(const T* __restrict__ vs, int lane, const double (*th)[2],
                                            double (&md)[kNumSizes], bool& vals_ok) {
  if constexpr (B < kNumSizes) {
    constexpr int lo = B == 0 ? 0 : split_size(B - 1), hi = split_size(B);
    constexpr double kBias = 0x1.fffffffffffffp-2;  // 0.5 - 2^-54
    double od = (double)(lo + lane);
#pragma unroll 2
    for (int o0 = lo; o0 < hi; o0 += 32, od += 32.0) {
      const T y = ld_val<SMEM>(vs + o0 + lane);
      vals_ok &= TypeTraits<T>::is_signed ? ((long long)y > -(1ll << 51) && (long long)y < (1ll << 51))
                                          : ((uint64_t)y < (1ull << 51));
      // yd + 2^52 (exact for |y| < 2^51); with predictions >= -0.25 the truncation is the sum
      // with 2^52 rounded toward zero (trunc_small), and their difference is y - pred exactly
      const double yc = __dadd_rn((double)(long long)y, 4503599627370496.0);
#pragma unroll
      for (int k = B; k < kNumSizes; k++) {
        const double2 t = *reinterpret_cast<const double2*>(th[k]);  // broadcast shared-memory load
        const double m = __dadd_rz(__dadd_rn(__fma_rn(t.y, od, t.x), kBias), 4503599627370496.0);
        md[k] = fmax(md[k], fabs(__dsub_rn(yc, m)));
      }
    }
    split_bands<B + 1, SMEM, T>(vs, lane, th, md, vals_ok);
  }
}


// The same band loops for 8-byte values beyond 2^51, measured from an offset: with every
// prediction argument x in [2^51, 2^62] (a multiple of 0.5 there, and no saturation) and within
// 2^50 of the integer d = c, and every value within 2^50 of c, the prediction is
// round_half_away(x) = floor(x + 0.5) (trunc(x + 0.5 - 2^-54) at a spacing of 0.5 or more), so
// pred - c = floor((x - d) + 0.5), where x - d and the + 0.5 are exact and the floor is the sum
// with 1.5 * 2^52 rounded down; y - c is an exact 64-bit difference below 2^50.
template <int B, bool SMEM, typename T>
__device__ __forceinline__ void split_bands_off(const T* __restrict__ vs, int lane, const double (*th)[2], double d,
                                                long long c, double (&md)[kNumSizes], bool& vals_ok) {
  if constexpr (B < kNumSizes) {
    constexpr int lo = B == 0 ? 0 : split_size(B - 1), hi = split_size(B);
    constexpr double kM = 6755399441055744.0;  // 1.5 * 2^52
    double od = (double)(lo + lane);
#pragma unroll 2
    for (int o0 = lo; o0 < hi; o0 += 32, od += 32.0) {
      const long long yv = (long long)ld_val<SMEM>(vs + o0 + lane);
      const long long dy = yv - c;  // no overflow: c in [2^51, 2^62], checked values >= 0
      vals_ok &= yv >= 0 && dy > -(1ll << 50) && dy < (1ll << 50);
      const double yc = __dadd_rn((double)dy, kM);
#pragma unroll
      for (int k = B; k < kNumSizes; k++) {
        const double2 t = *reinterpret_cast<const double2*>(th[k]);
        const double x = __fma_rn(t.y, od, t.x);
        const double m = __dadd_rd(__dadd_rn(__dsub_rn(x, d), 0.5), kM);
        md[k] = fmax(md[k], fabs(__dsub_rn(yc, m)));
      }
    }
    split_bands_off<B + 1, SMEM, T>(vs, lane, th, d, c, md, vals_ok);
  }
}

// Best end (as a block index; nb for the end of the column) of the start at block j.  One warp:
// every lane takes part and returns the same result; th is the warp's own table of lines.  SMEM:
// the start's reach (up to 3712 values) is first copied to win (the warp's own buffer) with all
// copies in flight at once, for walks where one warp evaluates starts one after another.
template <typename T, bool SMEM>
__device__ __forceinline__ int32_t split_best_block(const T* __restrict__ v, const RangeSums& rs, int64_t j, int lane,
                                                    double (*th)[2], T* win, long long& best_err) {
  const int64_t s = j * kMinPart;
  const int64_t max_size = (rs.n - s < kMinPart * 32) ? rs.n - s : kMinPart * 32;
  int ncand = 0;
#pragma unroll
  for (int k = 0; k < kNumSizes; k++) ncand += (c_sizes[k] <= max_size) ? 1 : 0;
  best_err = -1;  // not measured
  if (ncand == 0) return (int32_t)rs.nb;  // fewer than 128 values left: the rest is one partition
  __syncwarp();  // the previous start's lines and values are no longer read
  const T* vs = v + s;
  if constexpr (SMEM) {
    stage_reach<T>(v + s, win, c_sizes[ncand - 1], lane);
    vs = win;
  }
  // Fast path: when every value of the start's reach and every candidate's prediction (checked
  // at both ends of the candidate: fma(theta1, o, theta0) is monotone in o) lie well inside
  // (-2^51, 2^51) and inside T's range, the saturating conversion, the saturating or wrapping
  // difference and abs_ref all reduce to plain arithmetic: pred = trunc(x + bias) with one
  // conversion, delta = y - pred with one 64-bit subtraction.  Same results; any start that
  // leaves those bounds is measured by the exact loop below.
  constexpr double kSafe = 2251799813685248.0;  // 2^51
  const double lo_ok = TypeTraits<T>::is_signed ? (sizeof(T) == 4 ? -2147483647.0 : -kSafe) : -0.25;
  const double hi_ok = sizeof(T) == 4 ? (TypeTraits<T>::is_signed ? 2147483646.0 : 4294967294.0) : kSafe;
  bool cand_ok = true, cand_nonneg = true;
  double xa = 0.0, xb = 0.0;  // each candidate's prediction argument at its two ends
  if (lane < ncand) {
    double t0, t1;
    rs.line(s, s + c_sizes[lane], t0, t1);
    th[lane][0] = t0;
    th[lane][1] = t1;
    xa = t0;
    xb = __fma_rn(t1, (double)(c_sizes[lane] - 1), t0);
    cand_ok = xa >= lo_ok && xa <= hi_ok && xb >= lo_ok && xb <= hi_ok;
    cand_nonneg = xa >= -0.25 && xb >= -0.25;
  }
  if constexpr (SMEM) cp_async_wait_all();
  __syncwarp();
  long long m[kNumSizes];
#pragma unroll
  for (int k = 0; k < kNumSizes; k++) m[k] = 0;
  const int total = c_sizes[ncand - 1];
  bool fast = __all_sync(FULL_MASK, cand_ok);
  bool banded = false;
  if (fast && ncand == kNumSizes && __all_sync(FULL_MASK, cand_nonneg)) {
    double md[kNumSizes];
#pragma unroll
    for (int k = 0; k < kNumSizes; k++) md[k] = 0.0;
    bool vals_ok = true;
    split_bands<0, SMEM, T>(vs, lane, th, md, vals_ok);
    if (__all_sync(FULL_MASK, vals_ok)) {
#pragma unroll
      for (int k = 0; k < kNumSizes; k++) m[k] = (long long)md[k];
      banded = true;
    }
  }
  if constexpr (sizeof(T) == 8 && SMEM) {  // (walks only: it would cost the all-starts kernel occupancy)
    if (!fast && ncand == kNumSizes) {  // values beyond 2^51: the offset form, when it applies
      constexpr double kLo = 2251799813685248.0, kHi = 4611686018427387904.0, kNear = 1125899906842624.0;
      const double x0 = __shfl_sync(FULL_MASK, xa, 0);
      const bool d_ok = x0 >= kLo && x0 <= kHi;
      const double d = d_ok ? trunc(x0) : 0.0;
      const bool cand_off = lane >= ncand || (xa >= kLo && xa <= kHi && xb >= kLo && xb <= kHi &&
                                              fabs(xa - d) <= kNear && fabs(xb - d) <= kNear);
      if (__all_sync(FULL_MASK, d_ok && cand_off)) {
        double md[kNumSizes];
#pragma unroll
        for (int k = 0; k < kNumSizes; k++) md[k] = 0.0;
        bool vals_ok = true;
        split_bands_off<0, SMEM, T>(vs, lane, th, d, (long long)d, md, vals_ok);
        if (__all_sync(FULL_MASK, vals_ok)) {
#pragma unroll
          for (int k = 0; k < kNumSizes; k++) m[k] = (long long)md[k];
          banded = true;
          fast = true;  // measured
        }
      }
    }
  }
  if (fast && !banded) {
    // every quantity below is an integer of magnitude < 2^53, so FP64 holds it exactly: the
    // prediction trunc(x + bias), the residual y - pred, and the running max of |residual|
    double md[kNumSizes];
#pragma unroll
    for (int k = 0; k < kNumSizes; k++) md[k] = 0.0;
    bool vals_ok = true;
    int band = 0;  // first candidate whose size exceeds the offset (uniform: sizes are multiples of 128)
    double od = (double)lane;
    for (int o0 = 0; o0 < total; o0 += 32, od += 32.0) {
      while (c_sizes[band] <= o0) band++;
      const T y = ld_val<SMEM>(vs + o0 + lane);
      const long long yv = (long long)y;
      vals_ok &= TypeTraits<T>::is_signed ? (yv > -(1ll << 51) && yv < (1ll << 51)) : ((uint64_t)y < (1ull << 51));
      const double yd = (double)yv;  // exact when vals_ok (a start where it is not is measured again below)
#pragma unroll
      for (int k = 0; k < kNumSizes; k++) {
        if (k < band || k >= ncand) continue;
        const double2 tk = *reinterpret_cast<const double2*>(&th[k][0]);
        md[k] = fmax(md[k], abs_resid_fp64(yd, __fma_rn(tk.y, od, tk.x)));
      }
    }
    fast = __all_sync(FULL_MASK, vals_ok);
    if (fast) {
#pragma unroll
      for (int k = 0; k < kNumSizes; k++) m[k] = (long long)md[k];
    }
  }
  if (!fast && !banded) {
    int band = 0;
    for (int o0 = 0; o0 < total; o0 += 32) {
      while (c_sizes[band] <= o0) band++;
      const int o = o0 + lane;
      const T y = ld_val<SMEM>(vs + o);
#pragma unroll
      for (int k = 0; k < kNumSizes; k++) {
        if (k < band || k >= ncand) continue;
        const long long d = abs_ref(calc_delta<T>(y, predict<T>(th[k][0], th[k][1], o)));
        m[k] = d > m[k] ? d : m[k];
      }
    }
  }
  double best_cpe = 1.7976931348623157e308;
  int best = 0;
#pragma unroll
  for (int k = 0; k < kNumSizes; k++) {
    if (k >= ncand) continue;
    const long long mk = warp_max_ll(m[k]);
    const double cpe = __ddiv_rn(part_cost(c_sizes[k], bits_for(mk)), (double)c_sizes[k]);
    if (cpe < best_cpe) { best_cpe = cpe; best = k; best_err = mk; }
  }
  const int64_t e = s + c_sizes[best];
  return (int32_t)(e >= rs.n ? rs.nb : e / kMinPart);
}

// Best end of every 128-aligned start not evaluated yet (one warp per start), and the max |delta|
// of the partition it makes (nb_err: -1 where not measured).
template <typename T> __global__ void __launch_bounds__(256)
split_kernel(const T* __restrict__ v, RangeSums rs, int32_t* __restrict__ nb_next, long long* __restrict__ nb_err) {
  __shared__ __align__(16) double s_th[8][kNumSizes][2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t j = (int64_t)blockIdx.x * 8 + warp;
  if (j >= rs.nb || nb_next[j] != kUnknown) return;
  long long err;
  const int32_t e = split_best_block<T, false>(v, rs, j, lane, s_th[warp], nullptr, err);
  if (lane == 0) {
    nb_next[j] = e;
    nb_err[j] = err;
  }
}

// ---- walk from 0 ---------------------------------------------------------------------------
constexpr int32_t kEnd = -1;

__global__ void chain_exit_kernel(const int32_t* __restrict__ nb_next, int64_t nb, int64_t nr, int32_t* __restrict__ exits) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nr * kMaxJumpBlocks) return;
  const int64_t r = t / kMaxJumpBlocks, x = t % kMaxJumpBlocks;
  const int64_t lim = (r + 1) * kRangeBlocks;
  int64_t node = r * kRangeBlocks + x;
  while (node < lim && node < nb) node = nb_next[node];
  exits[t] = (node >= nb) ? kEnd : (int32_t)(node - lim);
}

// ---- lazy walk: evaluate only the starts a walk can reach --------------------------------------
// The walk from 0 visits one start in ~25 on piecewise-linear data.  Each range is walked from its
// first block, and again from the block where the previous range's first walk leaves it (the
// walk from 0 usually enters there: walks from nearby starts meet where the data changes
// slope).  The ranges are then chained through the exits of the starts these walks visited; if
// the walk from 0 enters a range at a start no walk visited, every start is evaluated instead.

constexpr int kWalkWarps = 1;  // one warp per CTA: the few range walks spread evenly over the SMs

// Walk of each range from its first block (one warp per range).
template <typename T> __global__ void __launch_bounds__(kWalkWarps * 32)
walk_first_kernel(const T* __restrict__ v, RangeSums rs, int64_t nr, int32_t* __restrict__ nb_next,
                  long long* __restrict__ nb_err, int32_t* __restrict__ exit_first) {
  __shared__ __align__(16) double s_th[kWalkWarps][kNumSizes][2];
  __shared__ __align__(16) T s_win[kWalkWarps][kMinPart * kMaxJumpBlocks];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r = (int64_t)blockIdx.x * kWalkWarps + warp;
  if (r >= nr) return;
  const int64_t lim = (r + 1) * kRangeBlocks < rs.nb ? (r + 1) * kRangeBlocks : rs.nb;
  int64_t node = r * kRangeBlocks;
  while (node < lim) {
    long long err;
    const int32_t nx = split_best_block<T, true>(v, rs, node, lane, s_th[warp], s_win[warp], err);
    if (lane == 0) {
      nb_next[node] = nx;
      nb_err[node] = err;
    }
    node = nx;
  }
  if (lane == 0) exit_first[r] = (int32_t)node;
}

// The exit block of every start on the first walk of each range, then the walk from the block
// where the previous range's first walk leaves, evaluated until it meets the first walk (whose
// starts are the only ones of the range evaluated so far), and the exit of its starts.
template <typename T> __global__ void __launch_bounds__(kWalkWarps * 32)
walk_entry_kernel(const T* __restrict__ v, RangeSums rs, int64_t nr, int32_t* __restrict__ nb_next,
                  long long* __restrict__ nb_err, const int32_t* __restrict__ exit_first, int32_t* __restrict__ cexit) {
  __shared__ __align__(16) double s_th[kWalkWarps][kNumSizes][2];
  __shared__ __align__(16) T s_win[kWalkWarps][kMinPart * kMaxJumpBlocks];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r = (int64_t)blockIdx.x * kWalkWarps + warp;
  if (r >= nr) return;
  const int64_t lim = (r + 1) * kRangeBlocks < rs.nb ? (r + 1) * kRangeBlocks : rs.nb;
  const int32_t ex0 = exit_first[r];
  if (lane == 0)
    for (int64_t p = r * kRangeBlocks; p < lim; p = nb_next[p]) cexit[p] = ex0;
  if (r == 0) return;
  const int64_t x = exit_first[r - 1];  // in [r * kRangeBlocks, r * kRangeBlocks + 29) or past the end
  if (x >= lim) return;
  int64_t node = x;
  while (node < lim) {
    int32_t nx = lane == 0 ? nb_next[node] : 0;
    nx = __shfl_sync(FULL_MASK, nx, 0);
    if (nx != kUnknown) break;  // met the first walk
    long long err;
    nx = split_best_block<T, true>(v, rs, node, lane, s_th[warp], s_win[warp], err);
    if (lane == 0) {
      nb_next[node] = nx;
      nb_err[node] = err;
    }
    node = nx;
  }
  const int32_t exb = node < lim ? ex0 : (int32_t)node;
  if (lane == 0)
    for (int64_t p = x; p < lim && cexit[p] == kUnknown; p = nb_next[p]) cexit[p] = exb;
}

// Chains the ranges (one warp): entries[r] = the block offset at which the walk from 0 enters
// range r (kEnd past the end of the column).  LAZY: exits from cexit (absolute blocks, kUnknown
// where no walk passed; *fail = the first range entered at such a start, or -1); otherwise from
// the exit table of every entry offset (relative offsets, kEnd).  The exits of 32 ranges.
// 29 entry offsets are loaded together, one lane per offset, ahead of the dependent chain.
template <bool LAZY>
__global__ void chain_link_kernel(const int32_t* __restrict__ exits, int64_t nb, int64_t nr,
                                  int32_t* __restrict__ entries, int64_t* __restrict__ fail) {
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  constexpr int kAhead = 32;
  int32_t e = 0;
  for (int64_t r0 = 0; r0 < nr; r0 += kAhead) {
    int32_t c[kAhead];
#pragma unroll
    for (int q = 0; q < kAhead; q++) {
      const int64_t r = r0 + q;
      c[q] = kUnknown;
      if (r < nr && lane < kMaxJumpBlocks) {
        if (LAZY) {
          const int64_t b = r * kRangeBlocks + lane;
          if (b < nb) c[q] = exits[b];
        } else {
          c[q] = exits[r * kMaxJumpBlocks + lane];
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kAhead; q++) {
      const int64_t r = r0 + q;
      if (r >= nr) break;
      if (lane == 0) entries[r] = e;
      if (e == kEnd) continue;
      const int32_t ex = __shfl_sync(FULL_MASK, c[q], e);
      if (!LAZY) {
        e = ex;
        continue;
      }
      if (ex == kUnknown) {  // no walk passed this entry: the caller evaluates every start
        for (int64_t k = r + lane; k < nr; k += 32) entries[k] = kEnd;
        if (lane == 0) *fail = r;
        return;
      }
      e = (int64_t)ex >= nb ? kEnd : (int32_t)(ex - (r + 1) * kRangeBlocks);
    }
  }
  if (LAZY && lane == 0) *fail = -1;
}

__global__ void chain_mark_kernel(const int32_t* __restrict__ nb_next, const int32_t* __restrict__ entries, int64_t nb,
                                  int64_t nr, int64_t* __restrict__ flags) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nr) return;
  const int32_t e = entries[r];
  if (e == kEnd) return;
  const int64_t lim = (r + 1) * kRangeBlocks;
  int64_t node = r * kRangeBlocks + e;
  while (node < lim && node < nb) {
    flags[node] = 1;
    node = nb_next[node];
  }
}

// The walk's partitions in order, with the max |delta| their start's evaluation measured for them
// (-1 for a last partition of fewer than 128 values, which no evaluation measured).
__global__ void chain_compact_kernel(const int64_t* __restrict__ flags, const int64_t* __restrict__ idx,
                                     const int32_t* __restrict__ nb_next, const long long* __restrict__ nb_err,
                                     int64_t nb, int64_t n, int32_t* __restrict__ ps, int32_t* __restrict__ pe,
                                     long long* __restrict__ kerr) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nb || !flags[j]) return;
  const int64_t k = idx[j];
  ps[k] = (int32_t)(j * kMinPart);
  const int64_t e = (int64_t)nb_next[j] * kMinPart;
  pe[k] = (int32_t)(e > n ? n : e);
  kerr[k] = nb_err[j];
}

// ---- costs of partitions ---------------------------------------------------------------
struct LineJob {  // one range whose max |delta| is needed
  int32_t a, b;
  double t0, t1;
  double sum;  // pairs: the two partitions' costs (a merge must cost less); partitions: +inf
};

// chunks of each job (0 for jobs that are cached)
// known (partitions only): a max |delta| already measured (the split evaluation of the
// partition's start, same line and values), or -1.  A pair kept from the previous round (cached)
// keeps its max |delta| too (cached_err).
__global__ void job_setup_kernel(const int32_t* __restrict__ ps, const int32_t* __restrict__ pe, int64_t m, int pairs,
                                 const uint8_t* __restrict__ cached, const long long* __restrict__ cached_err,
                                 const long long* __restrict__ known, const double* __restrict__ pc, RangeSums rs,
                                 LineJob* __restrict__ jobs, int64_t* __restrict__ nch, long long* __restrict__ err) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t njobs = pairs ? m - 1 : m;
  if (k >= njobs) return;
  LineJob jb;
  jb.a = ps[k];
  jb.b = pairs ? pe[k + 1] : pe[k];
  rs.line(jb.a, jb.b, jb.t0, jb.t1);
  jb.sum = pairs ? __dadd_rn(pc[k], pc[k + 1]) : __longlong_as_double(0x7ff0000000000000ll);
  jobs[k] = jb;
  const long long kn = known ? known[k] : -1;
  const bool kept = cached && cached[k];
  err[k] = kn >= 0 ? kn : (kept ? cached_err[k] : 0);
  const bool skip = kept || kn >= 0;
  nch[k] = skip ? 0 : ((int64_t)jb.b - jb.a + kPairChunk - 1) / kPairChunk;
}

// Max |delta| of a job's line over chunk q of the job (256 threads, no CTA barrier: warps may
// skip a chunk independently), folded into *errk by each warp.
template <typename T>
__device__ __forceinline__ void job_chunk(const T* __restrict__ v, const LineJob& jb, int64_t q, long long* errk) {
  const int64_t off0 = q * kPairChunk;
  const int64_t len = (int64_t)jb.b - jb.a;
  const int64_t off1 = off0 + kPairChunk < len ? off0 + kPairChunk : len;
  long long mm = 0;
  bool exact = true;
  if (off1 > off0 && line_fp64_safe<T>(jb.t0, jb.t1, off0, off1 - 1)) {  // exact in FP64 (glc_device.cuh)
    static_assert(kPairChunk == 16 * 256, "16 values per thread");
    T ys[16];
#pragma unroll
    for (int u = 0; u < 16; u++) {  // all loads in flight before the arithmetic
      const int64_t o = off0 + threadIdx.x + u * 256;
      ys[u] = o < off1 ? __ldg(v + jb.a + o) : (T)0;
    }
    double md = 0.0;
    bool ok = true;
#pragma unroll
    for (int u = 0; u < 16; u++) {
      const int64_t o = off0 + threadIdx.x + u * 256;
      if (o < off1) {
        ok &= value_fp64_safe<T>(ys[u]);
        md = fmax(md, abs_resid_fp64((double)(long long)ys[u], __fma_rn(jb.t1, (double)o, jb.t0)));
      }
    }
    if (ok) {  // this thread's values were all inside the exact range
      mm = (long long)md;
      exact = false;
    }
  }
  if (exact)
    for (int64_t o = off0 + threadIdx.x; o < off1; o += 256) {
      const long long d = abs_ref(calc_delta<T>(__ldg(v + jb.a + o), predict<T>(jb.t0, jb.t1, o)));
      mm = d > mm ? d : mm;
    }
  mm = warp_max_ll(mm);
  if ((threadIdx.x & 31) == 0 && mm > 0) atomicMax(errk, mm);
}

// A pair whose partial max |delta| already makes the merge cost at least the two partitions'
// costs is not merged whatever the rest of it holds (the score stays unprofitable, also when it
// is kept for the next round), so its remaining chunks are skipped.  One warp decides.
__device__ __forceinline__ bool job_settled(const LineJob& jb, const long long* errk) {
  long long e = 0;
  if ((threadIdx.x & 31) == 0) e = *(const volatile long long*)errk;
  e = __shfl_sync(FULL_MASK, e, 0);
  return !(part_cost((int64_t)jb.b - jb.a, bits_for(e)) < jb.sum);
}

// Max |delta| of every job still to measure: persistent CTAs, one job at a time, its chunks in
// order (each warp stops at the first chunk after which the pair is settled).
template <typename T> __global__ void __launch_bounds__(256, 4)
job_err_kernel(const T* __restrict__ v, const LineJob* __restrict__ jobs, const int64_t* __restrict__ nch,
               int64_t njobs, long long* __restrict__ err) {
  for (int64_t k = blockIdx.x; k < njobs; k += gridDim.x) {
    const int64_t nc = nch[k];  // 0: kept from the previous round
    if (nc == 0) continue;
    const LineJob jb = jobs[k];
    for (int64_t q = 0; q < nc; q++) {
      if (q > 0 && job_settled(jb, err + k)) break;
      job_chunk<T>(v, jb, q, err + k);
    }
  }
}

// Initial part costs.
__global__ void part_cost_kernel(const LineJob* __restrict__ jobs, const long long* __restrict__ err, int64_t m,
                                 double* __restrict__ pc) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  pc[k] = part_cost((int64_t)jobs[k].b - jobs[k].a, bits_for(err[k]));
}

// Pair scores: merged cost (fresh or cached) and profitability; any profitable -> *any = 1.
__global__ void pair_score_kernel(const LineJob* __restrict__ jobs, const long long* __restrict__ err,
                                  const uint8_t* __restrict__ cached, const double* __restrict__ cached_mc,
                                  const double* __restrict__ pc, int64_t m, double* __restrict__ mc,
                                  uint8_t* __restrict__ prof, int* __restrict__ any) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m - 1) return;
  double c;
  if (cached && cached[k]) c = cached_mc[k];
  else c = part_cost((int64_t)jobs[k].b - jobs[k].a, bits_for(err[k]));
  mc[k] = c;
  const bool p = c < __dadd_rn(pc[k], pc[k + 1]);
  prof[k] = p ? 1 : 0;
  if (p) atomicOr(any, 1);
}

// heads: part k starts a new part unless pair k-1 merges.
__global__ void merge_heads_kernel(const uint8_t* __restrict__ prof, int64_t m, int round, int64_t* __restrict__ head) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const bool absorbed = k > 0 && prof[k - 1] && (((k - 1) + round) % 2 == 0);
  head[k] = absorbed ? 0 : 1;
}

__device__ __forceinline__ bool selected(const uint8_t* prof, int64_t m, int64_t k, int round) {
  return k >= 0 && k < m - 1 && prof[k] && ((k + round) % 2 == 0);
}

__global__ void merge_scatter_kernel(const int32_t* __restrict__ ps, const int32_t* __restrict__ pe,
                                     const double* __restrict__ pc, const double* __restrict__ mc,
                                     const uint8_t* __restrict__ prof, const int64_t* __restrict__ head,
                                     const int64_t* __restrict__ idx, int64_t m, int round,
                                     int32_t* __restrict__ ps2, int32_t* __restrict__ pe2, double* __restrict__ pc2,
                                     uint8_t* __restrict__ cached2, double* __restrict__ cmc2,
                                     const long long* __restrict__ pair_err, const long long* __restrict__ part_err,
                                     long long* __restrict__ part_err2, long long* __restrict__ cerr2) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m || !head[k]) return;
  const int64_t d = idx[k];
  const bool sel = selected(prof, m, k, round);
  ps2[d] = ps[k];
  pe2[d] = sel ? pe[k + 1] : pe[k];
  pc2[d] = sel ? mc[k] : pc[k];
  part_err2[d] = sel ? pair_err[k] : part_err[k];  // a merged pair was measured in full (never settled early)
  // the score of (this part, next part) survives when neither changed
  const int64_t nxt = sel ? k + 2 : k + 1;  // old index of the next head
  const bool keep = !sel && nxt < m && !selected(prof, m, nxt, round);
  cached2[d] = keep ? 1 : 0;
  cmc2[d] = keep ? mc[k] : 0.0;
  cerr2[d] = keep ? pair_err[k] : 0;
}

static inline size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

template <typename T>
static cudaError_t partition_typed(glc_ctx* ctx, const T* v, int64_t n, int32_t** out_s, int32_t** out_e, int64_t* outP,
                                   cudaStream_t s, std::string* err, long long** out_err) {
  cudaError_t e;
  *out_s = nullptr;
  *out_e = nullptr;
  *outP = 0;
  if (out_err) *out_err = nullptr;
  if (n <= 0) return cudaSuccess;
  const int64_t nb = (n + kMinPart - 1) / kMinPart;
  const int64_t nr = (nb + kRangeBlocks - 1) / kRangeBlocks;
  const int64_t mmax = nb;  // split partitions are >= 128 values except the last
  size_t bytes = 0;
  bytes += al(sizeof(SumPair) * (nb + 1));                     // prefix
  bytes += al(sizeof(SumPair) * (scan_num_tiles(nb) + 1));     // scan tiles (pair)
  bytes += al(sizeof(int32_t) * nb);                           // nb_next
  bytes += al(sizeof(int32_t) * nr * kMaxJumpBlocks);          // exits
  bytes += al(sizeof(int32_t) * nr) * 2;                       // entries, exit_first
  bytes += al(sizeof(int32_t) * nb);                           // cexit
  bytes += al(sizeof(long long) * nb);                         // nb_err
  bytes += al(sizeof(long long) * mmax);                       // kerr
  bytes += al(sizeof(long long) * mmax) * 4;                   // part_err, part_err2, cerr, cerr2
  bytes += al(sizeof(int64_t) * (nb + 1)) * 2;                 // flags, idx
  bytes += al(sizeof(int64_t) * (scan_num_tiles(nb) + 1));     // scan tiles (i64)
  bytes += al(sizeof(int32_t) * mmax) * 4;                     // ps, pe, ps2, pe2
  bytes += al(sizeof(double) * mmax) * 5;                      // pc, pc2, mc, cmc, cmc2
  bytes += al(sizeof(uint8_t) * mmax) * 3;                     // prof, cached, cached2
  bytes += al(sizeof(LineJob) * mmax);                         // jobs
  bytes += al(sizeof(int64_t) * (mmax + 1));                   // nch
  bytes += al(sizeof(long long) * mmax);                       // err
  bytes += al(sizeof(int64_t) * 4);                            // device scalars
  char* buf = nullptr;
  if ((e = pool_alloc(ctx, &buf, bytes, s)) != cudaSuccess) return e;
  char* sp = buf;
  auto take = [&](size_t b) { char* r = sp; sp += al(b); return (void*)r; };
  SumPair* pre = (SumPair*)take(sizeof(SumPair) * (nb + 1));
  SumPair* ptiles = (SumPair*)take(sizeof(SumPair) * (scan_num_tiles(nb) + 1));
  int32_t* nb_next = (int32_t*)take(sizeof(int32_t) * nb);
  int32_t* exits = (int32_t*)take(sizeof(int32_t) * nr * kMaxJumpBlocks);
  int32_t* entries = (int32_t*)take(sizeof(int32_t) * nr);
  int32_t* exit_first = (int32_t*)take(sizeof(int32_t) * nr);
  int32_t* cexit = (int32_t*)take(sizeof(int32_t) * nb);
  long long* nb_err = (long long*)take(sizeof(long long) * nb);
  long long* kerr = (long long*)take(sizeof(long long) * mmax);
  long long* part_err = (long long*)take(sizeof(long long) * mmax);
  long long* part_err2 = (long long*)take(sizeof(long long) * mmax);
  long long* cerr = (long long*)take(sizeof(long long) * mmax);
  long long* cerr2 = (long long*)take(sizeof(long long) * mmax);
  int64_t* flags = (int64_t*)take(sizeof(int64_t) * (nb + 1));
  int64_t* idx = (int64_t*)take(sizeof(int64_t) * (nb + 1));
  int64_t* itiles = (int64_t*)take(sizeof(int64_t) * (scan_num_tiles(nb) + 1));
  int32_t* ps = (int32_t*)take(sizeof(int32_t) * mmax);
  int32_t* pe = (int32_t*)take(sizeof(int32_t) * mmax);
  int32_t* ps2 = (int32_t*)take(sizeof(int32_t) * mmax);
  int32_t* pe2 = (int32_t*)take(sizeof(int32_t) * mmax);
  double* pc = (double*)take(sizeof(double) * mmax);
  double* pc2 = (double*)take(sizeof(double) * mmax);
  double* mc = (double*)take(sizeof(double) * mmax);
  double* cmc = (double*)take(sizeof(double) * mmax);
  double* cmc2 = (double*)take(sizeof(double) * mmax);
  uint8_t* prof = (uint8_t*)take(mmax);
  uint8_t* cached = (uint8_t*)take(mmax);
  uint8_t* cached2 = (uint8_t*)take(mmax);
  LineJob* jobs = (LineJob*)take(sizeof(LineJob) * mmax);
  int64_t* nch = (int64_t*)take(sizeof(int64_t) * (mmax + 1));
  long long* perr = (long long*)take(sizeof(long long) * mmax);
  int64_t* dsc = (int64_t*)take(sizeof(int64_t) * 4);  // [0] unused, [1] m, [2] any (int), [3] walk fail
  RangeSums rs{pre, n, nb};

  auto fail = [&](cudaError_t ee) { cudaFreeAsync(buf, s); return ee; };
  auto grid = [](int64_t x, int b) { return (unsigned)((x + b - 1) / b); };

  block_sums_kernel<T><<<grid(nb * 32, 256), 256, 0, s>>>(v, n, nb, pre);
  if ((e = exclusive_scan<SumPair>(pre, pre, nb, pre + nb, ptiles, s)) != cudaSuccess) return fail(e);
  // the walk from 0: first only the starts that the walks of the ranges visit
  if ((e = cudaMemsetAsync(nb_next, 0xff, sizeof(int32_t) * nb, s)) != cudaSuccess) return fail(e);
  if ((e = cudaMemsetAsync(cexit, 0xff, sizeof(int32_t) * nb, s)) != cudaSuccess) return fail(e);
  walk_first_kernel<T><<<grid(nr, kWalkWarps), kWalkWarps * 32, 0, s>>>(v, rs, nr, nb_next, nb_err, exit_first);
  walk_entry_kernel<T><<<grid(nr, kWalkWarps), kWalkWarps * 32, 0, s>>>(v, rs, nr, nb_next, nb_err, exit_first,
                                                                          cexit);
  chain_link_kernel<true><<<1, 32, 0, s>>>(cexit, nb, nr, entries, dsc + 3);
  auto mark_and_compact = [&]() -> cudaError_t {
    cudaError_t ee = cudaMemsetAsync(flags, 0, sizeof(int64_t) * (nb + 1), s);
    if (ee != cudaSuccess) return ee;
    chain_mark_kernel<<<grid(nr, 128), 128, 0, s>>>(nb_next, entries, nb, nr, flags);
    if ((ee = exclusive_scan<int64_t>(flags, idx, nb, dsc + 1, itiles, s)) != cudaSuccess) return ee;
    chain_compact_kernel<<<grid(nb, 256), 256, 0, s>>>(flags, idx, nb_next, nb_err, nb, n, ps, pe, kerr);
    if ((ee = cudaGetLastError()) != cudaSuccess) return ee;
    // dsc[1] = partitions, dsc[3] = first range the walks did not cover
    if ((ee = cudaMemcpyAsync(ctx->h_stats, dsc + 1, 3 * sizeof(int64_t), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      return ee;
    return cudaStreamSynchronize(s);
  };
  if ((e = mark_and_compact()) != cudaSuccess) return fail(e);
  if (ctx->h_stats[2] >= 0) {  // the walk from 0 left the visited starts: evaluate all of them
    split_kernel<T><<<grid(nb, 8), 256, 0, s>>>(v, rs, nb_next, nb_err);
    chain_exit_kernel<<<grid(nr * kMaxJumpBlocks, 128), 128, 0, s>>>(nb_next, nb, nr, exits);
    chain_link_kernel<false><<<1, 32, 0, s>>>(exits, nb, nr, entries, nullptr);
    if ((e = mark_and_compact()) != cudaSuccess) return fail(e);
  }
  int64_t m = ctx->h_stats[0];
  if (m <= 0 || m > mmax) {
    if (err) *err = "partitioner produced an invalid split";
    cudaFreeAsync(buf, s);
    return cudaErrorUnknown;
  }

  // max |delta| of each job's line (partitions, or adjacent pairs of the merge rounds)
  auto run_jobs = [&](int64_t cnt, int pairs, const uint8_t* cache, const long long* known) -> cudaError_t {
    job_setup_kernel<<<grid(cnt, 256), 256, 0, s>>>(ps, pe, m, pairs, cache, cerr, known, pc, rs, jobs, nch, perr);
    const int64_t resident = (int64_t)ctx->num_sms * 4;  // 256-thread CTAs, four per SM
    job_err_kernel<T><<<(unsigned)(cnt < resident ? cnt : resident), 256, 0, s>>>(v, jobs, nch, cnt, perr);
    return cudaGetLastError();
  };
  // costs of the split partitions: their max |delta| came with the split evaluation
  if ((e = run_jobs(m, 0, nullptr, kerr)) != cudaSuccess) return fail(e);
  part_cost_kernel<<<grid(m, 256), 256, 0, s>>>(jobs, perr, m, pc);
  // each partition's max |delta| travels with it through the merge rounds (for the fit)
  if ((e = cudaMemcpyAsync(part_err, perr, sizeof(long long) * m, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
    return fail(e);
  if ((e = cudaMemsetAsync(cached, 0, mmax, s)) != cudaSuccess) return fail(e);

  for (int round = 0; round < kMaxMergeRounds && m >= 2; round++) {
    if ((e = run_jobs(m - 1, 1, cached, nullptr)) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(dsc + 2, 0, sizeof(int64_t), s)) != cudaSuccess) return fail(e);
    pair_score_kernel<<<grid(m - 1, 256), 256, 0, s>>>(jobs, perr, cached, cmc, pc, m, mc, prof, (int*)(dsc + 2));
    merge_heads_kernel<<<grid(m, 256), 256, 0, s>>>(prof, m, round, flags);
    if ((e = exclusive_scan<int64_t>(flags, idx, m, dsc + 1, itiles, s)) != cudaSuccess) return fail(e);
    merge_scatter_kernel<<<grid(m, 256), 256, 0, s>>>(ps, pe, pc, mc, prof, flags, idx, m, round, ps2, pe2, pc2,
                                                       cached2, cmc2, perr, part_err, part_err2, cerr2);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpyAsync(ctx->h_stats, dsc + 1, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      return fail(e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(e);
    const int64_t m2 = ctx->h_stats[0];
    const int any = (int)(ctx->h_stats[1] & 0xffffffff);
    if (!any) break;  // nothing merged: the lists are unchanged
    std::swap(ps, ps2);
    std::swap(pe, pe2);
    std::swap(pc, pc2);
    std::swap(cached, cached2);
    std::swap(cmc, cmc2);
    std::swap(part_err, part_err2);
    std::swap(cerr, cerr2);
    m = m2;
  }

  int32_t* rs_out = nullptr;
  int32_t* re_out = nullptr;
  if ((e = pool_alloc(ctx, &rs_out, sizeof(int32_t) * m, s)) != cudaSuccess) return fail(e);
  if ((e = pool_alloc(ctx, &re_out, sizeof(int32_t) * m, s)) != cudaSuccess) {
    cudaFreeAsync(rs_out, s);
    return fail(e);
  }
  cudaMemcpyAsync(rs_out, ps, sizeof(int32_t) * m, cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(re_out, pe, sizeof(int32_t) * m, cudaMemcpyDeviceToDevice, s);
  if (out_err) {
    long long* er_out = nullptr;
    if ((e = pool_alloc(ctx, &er_out, sizeof(long long) * m, s)) != cudaSuccess) {
      cudaFreeAsync(rs_out, s);
      cudaFreeAsync(re_out, s);
      return fail(e);
    }
    cudaMemcpyAsync(er_out, part_err, sizeof(long long) * m, cudaMemcpyDeviceToDevice, s);
    *out_err = er_out;
  }
  cudaFreeAsync(buf, s);
  *out_s = rs_out;
  *out_e = re_out;
  *outP = m;
  return cudaGetLastError();
}

cudaError_t launch_partition_variable(glc_ctx* ctx, glc_dtype dt, const void* values, int64_t n, int32_t** d_starts,
                                      int32_t** d_ends, int64_t* P, cudaStream_t s, std::string* err,
                                      long long** d_err) {
  switch (dt) {
    case GLC_I32: return partition_typed<int32_t>(ctx, (const int32_t*)values, n, d_starts, d_ends, P, s, err, d_err);
    case GLC_I64: return partition_typed<int64_t>(ctx, (const int64_t*)values, n, d_starts, d_ends, P, s, err, d_err);
    case GLC_U64: return partition_typed<uint64_t>(ctx, (const uint64_t*)values, n, d_starts, d_ends, P, s, err, d_err);
    case GLC_U32: return partition_typed<uint32_t>(ctx, (const uint32_t*)values, n, d_starts, d_ends, P, s, err, d_err);
  }
  return cudaErrorInvalidValue;
}

}  // namespace glc
