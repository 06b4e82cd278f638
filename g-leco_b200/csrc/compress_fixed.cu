// compress_fixed.cu -- one-pass compression of a column with fixed partitions whose length L
// divides the 4096-value tile and is at least 256 (L = 256, 512, 1024, 2048, 4096; the
// reference's TILE_SIZE is 4096, core/CudaUtils.cuh:18).
//
// Replaces, for those columns, the separate fit, bit-offset scan, table build and pack passes
// (fit.cu, glc_scan.cuh, pack.cu; in the reference wprocessPartitionsKernel,
// setBitOffsetsKernel and packDeltasKernelOptimized, compression/CompressionKernels.cuh:45-372,
// which read the values four times) with ONE persistent kernel that reads every value once:
//
//   producer warp   stages tile t's values in shared memory with cp.async.bulk, two tiles ahead
//                   (full/empty mbarriers, bounded waits);
//   compute warps   per tile, with every partition inside the tile (L divides 4096):
//     A  exact sums per partition from 64-bit partials of 32-bit halves, and the overflow flag
//        that selects direct copy; a group of L/16 threads owns a partition, 16 values each,
//        so one reduction per group gives the partition's sums;
//     -  one thread per partition solves the line from the exact sums (the same arithmetic as
//        fit.cu, so the result is identical bit for bit);
//     B  the residual of every value (fma prediction, round half away from zero, saturating
//        cast; calculateDelta) written over the staged value (8-byte types) or into a residual
//        array (4-byte types), and max |residual| per partition -> the partition's bit width;
//     C  the tile's words from the residual fields, one thread per word, into the tile's own
//        slot of a scratch array (slots of the worst-case size of a tile, bit offsets relative to
//        the tile), with the partitions' metadata (the reference's SoA), their descriptors and
//        the tile's decode-table entry, all with tile-relative bit offsets, and the tile's bit
//        count;
//   then an exclusive scan of the tiles' bit counts gives every tile's first bit, and
//   fixed_place_kernel (one CTA per tile) writes each word of the column once -- the word holding
//   bit 32 W is built by the tile that holds that bit, from its slot with a funnel shift, ORed
//   with the first bits of any later tiles that start inside it -- and adds the tile's first bit
//   to its partitions' offsets, descriptors and decode-table entry.  No tile waits for another.
//
// The column's word array is allocated at its exact size between the two kernels (the scan gives
// the total); the slots cost one extra write and read of the compressed bits.
#include <type_traits>
#include "glc_internal.h"
#include "glc_scan.cuh"
#include "glc_tma.cuh"

namespace glc {

constexpr int kCfThreads = 256;                       // compute threads (8 warps)
constexpr int kCfCTA = kCfThreads + 32;               // + the producer warp
constexpr int kCfStages = 2;
constexpr int kCfMinLen = 256;
constexpr int kCfMaxParts = kDecodeTile / kCfMinLen;  // 16 partitions per tile at L = 256
constexpr int kCfPerThread = kDecodeTile / kCfThreads;  // 16 values per thread
constexpr int kCfMaxSegs = 16;                        // reduction segments (half-warps at L = 256)

template <typename T> __host__ __device__ constexpr int cf_stage_bytes() { return kDecodeTile * (int)sizeof(T) + 16; }
template <typename T> __host__ __device__ constexpr int cf_smem_bytes() {
  return kCfStages * cf_stage_bytes<T>() + (sizeof(T) == 4 ? kDecodeTile * 8 : 0);
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
};

__device__ __forceinline__ void cf_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kCfThreads) : "memory"); }

// The producer lane of a launch: stages item blockIdx.x + k * gridDim.x of the work list into stage
// k % kCfStages (its values, from the 16-byte block that holds the first one), with the item, its
// column and the offset of its first value in the stage; an item of -1 marks the end.
template <typename T>
__device__ __forceinline__ void cf_produce(const FixedCompressArgs& a, uint8_t* smem, uint64_t* full, uint64_t* empty,
                                           int64_t* s_stile, int* s_shead, int* s_scol) {
  int64_t item = blockIdx.x;
  for (int k = 0;; k++, item += gridDim.x) {
    const int st = k % kCfStages;
    if (k >= kCfStages && !mbar_wait_bounded(&empty[st], (uint32_t)((k / kCfStages) - 1) & 1u)) {
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

template <typename T> __global__ void __launch_bounds__(kCfCTA)
fixed_compress_kernel(FixedCompressArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t full[kCfStages], empty[kCfStages];
  __shared__ int64_t s_stile[kCfStages];   // work item staged in each stage (-1: the end)
  __shared__ int s_shead[kCfStages];
  __shared__ int s_scol[kCfStages];
  typedef typename HalfSums<T>::Acc Acc;
  __shared__ Acc s_acc[kCfMaxSegs][4];
  __shared__ int s_ovf[kCfMaxSegs];
  __shared__ unsigned long long s_mx[kCfMaxSegs];
  __shared__ double s_t0[kCfMaxParts], s_t1[kCfMaxParts];
  __shared__ int s_direct[kCfMaxParts], s_safe[kCfMaxParts], s_len[kCfMaxParts], s_b[kCfMaxParts];
  __shared__ uint32_t s_mb[kCfMaxParts];
  __shared__ long long s_err[kCfMaxParts];
  __shared__ int s_bl[kCfMaxParts + 1];
  __shared__ int s_ok;

  if (threadIdx.x == 0) {
    for (int st = 0; st < kCfStages; st++) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (threadIdx.x >= kCfThreads) {  // ---- producer ----
    if (threadIdx.x == kCfThreads) cf_produce<T>(a, smem, full, empty, s_stile, s_shead, s_scol);
    return;
  }

  // ---- compute warps ----
  const int tid = threadIdx.x;
  for (int k = 0;; k++) {
    const int st = k % kCfStages;
    const uint32_t par = (uint32_t)(k / kCfStages) & 1u;
    if (tid == 0) {
      s_ok = mbar_wait_bounded(&full[st], par);
      if (!s_ok) {
        atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
        mbar_wait_bounded(&full[st], par);  // a copy in flight lands before the CTA exits
      }
    }
    cf_sync();
    if (!s_ok) return;
    mbar_try_wait(&full[st], par);  // the phase is complete: orders this thread's reads after the copy
    const int64_t item = s_stile[st];
    if (item < 0) return;
    const CfColumn& col = a.cols ? a.cols[s_scol[st]] : a.single;
    const int64_t t = item - col.item_base;  // the tile within its column
    const int L = col.L;
    const int g = L >> 4;                     // threads per partition (16 values each)
    const int W = g < 32 ? g : 32;            // lanes of one reduction segment
    const int seg = tid / W;                  // reduction segment of this thread
    const int segs_per_part = g / W;
    const int p_me = tid / g;                 // this thread's partition within the tile
    const int r_me = tid - p_me * g;          // and its first value there
    uint8_t* stage = smem + (size_t)st * cf_stage_bytes<T>();
    T* x = reinterpret_cast<T*>(stage + s_shead[st]);
    // residuals: over the values for 8-byte types, in their own array for 4-byte types
    int64_t* res = sizeof(T) == 8 ? reinterpret_cast<int64_t*>(x)
                                  : reinterpret_cast<int64_t*>(smem + (size_t)kCfStages * cf_stage_bytes<T>());
    const int64_t e0 = t * kDecodeTile;
    const int cnt = (int)((col.n - e0) < kDecodeTile ? (col.n - e0) : kDecodeTile);
    const int np = (cnt + L - 1) / L;  // partitions in this tile (the last may be short)
    const int my_len = p_me < np ? ((cnt - p_me * L) < L ? (cnt - p_me * L) : L) : 0;
    const T* xp = x + p_me * L;

    // ---- A: exact sums of y and i * y (i = index within the partition), overflow flag ----
    {
      HalfSums<T> hs;
      int ovf = 0;
#pragma unroll 4
      for (int m = 0; m < kCfPerThread; m++) {
        const int i = r_me + g * m;
        if (i < my_len) {
          const T y = xp[i];
          ovf |= overflows_double<T>(y) ? 1 : 0;
          hs.add(y, i);
        }
      }
      Acc c0 = hs.s_lo, c1 = hs.s_hi, c2 = hs.x_lo, c3 = hs.x_hi;
      for (int msk = W >> 1; msk > 0; msk >>= 1) {
        c0 += __shfl_xor_sync(FULL_MASK, c0, msk);
        if (sizeof(T) == 8) c1 += __shfl_xor_sync(FULL_MASK, c1, msk);
        c2 += __shfl_xor_sync(FULL_MASK, c2, msk);
        if (sizeof(T) == 8) c3 += __shfl_xor_sync(FULL_MASK, c3, msk);
        ovf |= __shfl_xor_sync(FULL_MASK, ovf, msk);
      }
      if ((tid & (W - 1)) == 0) {
        s_acc[seg][0] = c0;
        s_acc[seg][1] = c1;
        s_acc[seg][2] = c2;
        s_acc[seg][3] = c3;
        s_ovf[seg] = ovf;
      }
    }
    cf_sync();
    if (tid < np) {  // one thread per partition: the line (fit.cu's arithmetic)
      const int p = tid;
      HalfSums<T> hs;
      int ovf = 0;
      for (int q = p * segs_per_part; q < (p + 1) * segs_per_part; q++) {
        hs.s_lo += s_acc[q][0];
        hs.s_hi += s_acc[q][1];
        hs.x_lo += s_acc[q][2];
        hs.x_hi += s_acc[q][3];
        ovf |= s_ovf[q];
      }
      const int len = (cnt - p * L) < L ? (cnt - p * L) : L;
      double t0 = 0.0, t1 = 0.0;
      if (!ovf) solve_line(len, hs.sy(), hs.sxy(), t0, t1);
      s_t0[p] = t0;
      s_t1[p] = t1;
      s_direct[p] = ovf;
      s_len[p] = len;
      s_safe[p] = !ovf && line_fp64_safe<T>(t0, t1, 0, len - 1);
    }
    cf_sync();

    // ---- B: residual of every value, max |residual| per partition ----
    {
      const int p = p_me;
      unsigned long long mx = 0;
      if (my_len > 0) {
        int64_t* rp = res + p_me * L;
        if (s_direct[p]) {  // direct copy: the field is the value itself (zero-extended)
          for (int m = 0; m < kCfPerThread; m++) {
            const int i = r_me + g * m;
            if (i < my_len) rp[i] = (int64_t)(uint64_t)xp[i];
          }
        } else {
          const double t0 = s_t0[p], t1 = s_t1[p];
          bool exact_fp64 = s_safe[p] != 0;
          if (exact_fp64) {
            // |y| < 2^51 and the predictions inside pred_fp64_safe's bounds: the prediction is
            // predict_small (no conversion instruction), y - pred is below 2^52 and is
            // calculateDelta; the index advances as an exact double
            long long dmax = 0, dmin = 0;
            double xd = (double)r_me;
            const double xstep = (double)g;
#pragma unroll 4
            for (int m = 0; m < kCfPerThread; m++, xd += xstep) {
              const int i = r_me + g * m;
              if (i < my_len) {
                const T y = xp[i];
                exact_fp64 &= value_fp64_safe<T>(y);
                const long long d = (long long)y - predict_small(__fma_rn(t1, xd, t0));
                rp[i] = d;
                dmax = d > dmax ? d : dmax;
                dmin = d < dmin ? d : dmin;
              }
            }
            mx = (unsigned long long)(dmax > -dmin ? dmax : -dmin);
          }
          if (!exact_fp64) {  // the general residual (saturating for uint64), and its exact magnitude
            mx = 0;
            for (int m = 0; m < kCfPerThread; m++) {
              const int i = r_me + g * m;
              if (i < my_len) {
                const T y = xp[i];
                const long long d = calc_delta<T>(y, predict_from<T>(__fma_rn(t1, (double)i, t0)));
                rp[i] = d;
                const unsigned long long ad = (unsigned long long)abs_ref(d);
                mx = ad > mx ? ad : mx;
              }
            }
          }
        }
      }
      for (int msk = W >> 1; msk > 0; msk >>= 1) {
        const unsigned long long o = __shfl_xor_sync(FULL_MASK, mx, msk);
        mx = o > mx ? o : mx;
      }
      if ((tid & (W - 1)) == 0) s_mx[seg] = mx;
    }
    cf_sync();
    if (tid < np) {
      const int p = tid;
      unsigned long long mx = 0;
      for (int q = p * segs_per_part; q < (p + 1) * segs_per_part; q++) mx = s_mx[q] > mx ? s_mx[q] : mx;
      const int b = s_direct[p] ? (int)sizeof(T) * 8 : bits_for((long long)mx);
      s_err[p] = s_direct[p] ? 0 : (long long)mx;
      s_b[p] = b;
      s_mb[p] = b > 1 ? 0xffffffffu / (uint32_t)b + 1u : 0u;
    }
    cf_sync();
    if (tid == 0) {  // tile-relative bit ranges, the tile's bit count and decode-table entry
      int acc = 0, bmax = 0;
      for (int p = 0; p < np; p++) {
        s_bl[p] = acc;
        acc += s_len[p] * s_b[p];
        bmax = s_b[p] > bmax ? s_b[p] : bmax;
      }
      s_bl[np] = acc;
      a.tile_bits[item] = acc;
      TileInfo ti;
      ti.bit_lo = 0;  // the tile's first bit is added by fixed_place_kernel
      ti.p_first = (int32_t)(t * col.parts_per_tile);
      ti.p_last = (int32_t)(t * col.parts_per_tile + np - 1);
      col.tiles[t] = ti;
      if (bmax > 0) atomicMax(col.stats + 1, (unsigned long long)bmax);
    }
    cf_sync();
    if (tid < np) {  // the partitions' metadata and descriptors (offsets relative to the tile)
      const int p = tid;
      const int64_t gp = t * col.parts_per_tile + p;
      const int32_t start = (int32_t)(e0 + (int64_t)p * L);
      const int type = s_direct[p] ? MODEL_DIRECT_COPY : MODEL_LINEAR;
      col.starts[gp] = start;
      col.ends[gp] = start + s_len[p];
      col.types[gp] = type;
      col.params[4 * gp] = s_t0[p];
      col.params[4 * gp + 1] = s_t1[p];
      col.params[4 * gp + 2] = 0.0;
      col.params[4 * gp + 3] = 0.0;
      col.bits[gp] = s_b[p];
      col.offs[gp] = s_bl[p];
      col.err[gp] = s_err[p];
      PartDesc d;
      d.theta0 = s_t0[p];
      d.theta1 = s_t1[p];
      d.bit_off = s_bl[p];
      d.start = start;
      d.bits_type = (s_b[p] & 0xff) | (type << 8);
      col.desc[gp] = d;
    }

    // ---- C: the tile's words into its slot; word w holds tile bits [32 w, 32 w + 32) ----
    {
      const int tb = s_bl[np];
      const int nw = (tb + 31) >> 5;
      const uint32_t* f32 = reinterpret_cast<const uint32_t*>(res);  // low half of residual j at 2 j
      uint32_t* out = a.slots + item * a.slot_words;
      int qi = 0;
      for (int w = tid; w < nw; w += kCfThreads) {
        const int wb = 32 * w;
        int pos = wb;
        const int wend = wb + 32 < tb ? wb + 32 : tb;
        uint32_t word = 0u;
        while (pos < wend) {
          while (s_bl[qi + 1] <= pos) qi++;  // the partition holding bit pos (empty ranges skipped)
          const int b = s_b[qi], bl = s_bl[qi];
          const int qend = s_bl[qi + 1] < wend ? s_bl[qi + 1] : wend;
          const int jj = b > 1 ? (int)__umulhi((uint32_t)(pos - bl), s_mb[qi]) : pos - bl;
          int fb = bl + jj * b;  // start of the field holding bit pos
          int j = qi * L + jj;
          if (b <= 32) {
            const uint32_t mask = b == 32 ? 0xffffffffu : ((1u << b) - 1u);
            for (; fb < qend; fb += b, j++) {
              const uint32_t f = f32[2 * j] & mask;
              const int sh = fb - wb;
              word |= sh >= 0 ? (f << sh) : (f >> -sh);
            }
          } else {
            for (; fb < qend; fb += b, j++) {
              const uint64_t f = low_bits((uint64_t)res[j], b);
              const int sh = fb - wb;
              word |= sh >= 0 ? (uint32_t)(f << sh) : (uint32_t)(f >> -sh);
            }
          }
          pos = qend;
        }
        out[w] = word;
      }
    }
    cf_sync();  // every compute thread is done with stage st and the residual array
    if (tid == 0) mbar_arrive(&empty[st]);
  }
}

// The partition-length choice of the batched compress, one tile per step (the same staging as
// fixed_compress_kernel): the tile's four 1024-value quarters, its two halves and the whole tile
// are fitted from exact per-quarter sums (the index offsets of a half or the tile added exactly),
// every value's residual is measured against the three lines that cover it, and the bits of each
// candidate length are added into the column's choice_bits[0..2] (1024, 2048, 4096).  The widths
// are the ones the compress at that length computes, so the column's size is exact.
template <typename T> __global__ void __launch_bounds__(kCfCTA)
choose_lengths_kernel(FixedCompressArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t full[kCfStages], empty[kCfStages];
  __shared__ int64_t s_stile[kCfStages];
  __shared__ int s_shead[kCfStages];
  __shared__ int s_scol[kCfStages];
  typedef typename HalfSums<T>::Acc Acc;
  __shared__ Acc s_acc[8][4];
  __shared__ int s_ovf[8];
  __shared__ unsigned long long s_m[8][3];
  __shared__ double s_t0[7], s_t1[7];
  __shared__ int s_dir[7], s_safe[7], s_len[7];
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    for (int st = 0; st < kCfStages; st++) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x >= kCfThreads) {  // ---- producer ----
    if (threadIdx.x == kCfThreads) cf_produce<T>(a, smem, full, empty, s_stile, s_shead, s_scol);
    return;
  }
  const int tid = threadIdx.x, warp = tid >> 5;
  const int q = tid >> 6;          // this thread's quarter (64 threads, 16 values each)
  const int r = tid & 63;
  for (int k = 0;; k++) {
    const int st = k % kCfStages;
    const uint32_t par = (uint32_t)(k / kCfStages) & 1u;
    if (tid == 0) {
      s_ok = mbar_wait_bounded(&full[st], par);
      if (!s_ok) {
        atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
        mbar_wait_bounded(&full[st], par);  // a copy in flight lands before the CTA exits
      }
    }
    cf_sync();
    if (!s_ok) return;
    mbar_try_wait(&full[st], par);
    const int64_t item = s_stile[st];
    if (item < 0) return;
    const CfColumn& col = a.cols[s_scol[st]];
    const int64_t e0 = (item - col.item_base) * kDecodeTile;
    const int cnt = (int)((col.n - e0) < kDecodeTile ? (col.n - e0) : kDecodeTile);
    const T* x = reinterpret_cast<const T*>(smem + (size_t)st * cf_stage_bytes<T>() + s_shead[st]);
    const int qlen = (cnt - 1024 * q) < 0 ? 0 : ((cnt - 1024 * q) < 1024 ? (cnt - 1024 * q) : 1024);
    const T* xq = x + 1024 * q;
    {  // exact sums per quarter (two warps each)
      HalfSums<T> hs;
      int ovf = 0;
#pragma unroll 4
      for (int m = 0; m < kCfPerThread; m++) {
        const int i = r + 64 * m;
        if (i < qlen) {
          const T y = xq[i];
          ovf |= overflows_double<T>(y) ? 1 : 0;
          hs.add(y, i);
        }
      }
      Acc c0 = hs.s_lo, c1 = hs.s_hi, c2 = hs.x_lo, c3 = hs.x_hi;
#pragma unroll
      for (int msk = 16; msk > 0; msk >>= 1) {
        c0 += __shfl_xor_sync(FULL_MASK, c0, msk);
        if (sizeof(T) == 8) c1 += __shfl_xor_sync(FULL_MASK, c1, msk);
        c2 += __shfl_xor_sync(FULL_MASK, c2, msk);
        if (sizeof(T) == 8) c3 += __shfl_xor_sync(FULL_MASK, c3, msk);
        ovf |= __shfl_xor_sync(FULL_MASK, ovf, msk);
      }
      if ((tid & 31) == 0) {
        s_acc[warp][0] = c0;
        s_acc[warp][1] = c1;
        s_acc[warp][2] = c2;
        s_acc[warp][3] = c3;
        s_ovf[warp] = ovf;
      }
    }
    cf_sync();
    if (tid < 7) {  // line l: 0 = the tile, 1-2 = its halves, 3-6 = its quarters
      const int l = tid;
      const int q0 = l == 0 ? 0 : (l < 3 ? (l - 1) * 2 : l - 3);
      const int q1 = l == 0 ? 4 : (l < 3 ? q0 + 2 : q0 + 1);
      i128 sy = 0, sxy = 0;
      int ovf = 0;
      for (int qq = q0; qq < q1; qq++) {
        HalfSums<T> hs;
        for (int w = 2 * qq; w < 2 * qq + 2; w++) {
          hs.s_lo += s_acc[w][0];
          hs.s_hi += s_acc[w][1];
          hs.x_lo += s_acc[w][2];
          hs.x_hi += s_acc[w][3];
          ovf |= s_ovf[w];
        }
        const i128 qy = hs.sy();
        sy += qy;
        sxy += hs.sxy() + (i128)(1024 * (qq - q0)) * qy;  // quarter index -> line index
      }
      int len = cnt - 1024 * q0;
      len = len < 0 ? 0 : (len < 1024 * (q1 - q0) ? len : 1024 * (q1 - q0));
      double t0 = 0.0, t1 = 0.0;
      if (len > 0 && !ovf) solve_line(len, sy, sxy, t0, t1);
      s_t0[l] = t0;
      s_t1[l] = t1;
      s_dir[l] = ovf;
      s_len[l] = len;
      s_safe[l] = len > 0 && !ovf && line_fp64_safe<T>(t0, t1, 0, len - 1);
    }
    cf_sync();
    {  // max |residual| of each value against its quarter's, its half's and the tile's line
      const int ls[3] = {3 + q, 1 + (q >> 1), 0};
      const int off[3] = {0, 1024 * (q & 1), 1024 * q};
      unsigned long long mx[3] = {0, 0, 0};
      if (qlen > 0) {
        bool fast = s_safe[ls[0]] && s_safe[ls[1]] && s_safe[ls[2]];
        if (fast) {  // predict_small and exact integer residuals (see fixed_compress_kernel)
          long long dmax[3] = {0, 0, 0}, dmin[3] = {0, 0, 0};
          double t0[3], t1[3], xd[3];
#pragma unroll
          for (int c = 0; c < 3; c++) {
            t0[c] = s_t0[ls[c]];
            t1[c] = s_t1[ls[c]];
            xd[c] = (double)(r + off[c]);
          }
#pragma unroll 2
          for (int m = 0; m < kCfPerThread; m++) {
            const int i = r + 64 * m;
            if (i < qlen) {
              const T y = xq[i];
              fast &= value_fp64_safe<T>(y);
#pragma unroll
              for (int c = 0; c < 3; c++) {
                const long long d = (long long)y - predict_small(__fma_rn(t1[c], xd[c], t0[c]));
                dmax[c] = d > dmax[c] ? d : dmax[c];
                dmin[c] = d < dmin[c] ? d : dmin[c];
              }
            }
#pragma unroll
            for (int c = 0; c < 3; c++) xd[c] += 64.0;
          }
#pragma unroll
          for (int c = 0; c < 3; c++) mx[c] = (unsigned long long)(dmax[c] > -dmin[c] ? dmax[c] : -dmin[c]);
        }
        if (!fast) {  // exact integer residuals (saturating for uint64)
          for (int c = 0; c < 3; c++) mx[c] = 0;
          for (int m = 0; m < kCfPerThread; m++) {
            const int i = r + 64 * m;
            if (i >= qlen) continue;
            const T y = xq[i];
            for (int c = 0; c < 3; c++) {
              if (s_dir[ls[c]]) continue;
              const long long d =
                  calc_delta<T>(y, predict_from<T>(__fma_rn(s_t1[ls[c]], (double)(i + off[c]), s_t0[ls[c]])));
              const unsigned long long ad = (unsigned long long)abs_ref(d);
              mx[c] = ad > mx[c] ? ad : mx[c];
            }
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 3; c++) {
#pragma unroll
        for (int msk = 16; msk > 0; msk >>= 1) {
          const unsigned long long o = __shfl_xor_sync(FULL_MASK, mx[c], msk);
          mx[c] = o > mx[c] ? o : mx[c];
        }
      }
      if ((tid & 31) == 0) {
        s_m[warp][0] = mx[0];
        s_m[warp][1] = mx[1];
        s_m[warp][2] = mx[2];
      }
    }
    cf_sync();
    if (tid == 0) {
      unsigned long long add[3] = {0, 0, 0};
      for (int l = 0; l < 7; l++) {
        if (s_len[l] <= 0) continue;
        const int c = l == 0 ? 2 : (l < 3 ? 1 : 0);                      // index into s_m's lines
        const int w0 = l == 0 ? 0 : (l < 3 ? 4 * (l - 1) : 2 * (l - 3));  // the line's warps
        const int w1 = l == 0 ? 8 : (l < 3 ? w0 + 4 : w0 + 2);
        unsigned long long m = 0;
        for (int w = w0; w < w1; w++) m = s_m[w][c] > m ? s_m[w][c] : m;
        const int b = s_dir[l] ? (int)sizeof(T) * 8 : bits_for((long long)m);
        add[l == 0 ? 2 : (l < 3 ? 1 : 0)] += (unsigned long long)s_len[l] * (unsigned long long)b;
      }
      for (int c = 0; c < 3; c++)
        if (add[c]) atomicAdd(col.choice_bits + c, add[c]);
    }
    cf_sync();  // every compute thread is done with stage st
    if (tid == 0) mbar_arrive(&empty[st]);
  }
}

// Places every tile of the launch in its column, one CTA per tile: the tile's first bit F (the
// scan of the tiles' bits, relative to the column's first tile) is added to its partitions'
// offsets and descriptors and to its decode-table entry, and the words whose first bit lies in the
// tile are written -- from the tile's slot with a funnel shift, ORed with the first bits of every
// later tile of the column that starts inside the same word (tiles without bits are skipped).  The
// column's last tile writes the final decode-table entry and the total, and zeroes the padding.
__global__ void __launch_bounds__(256) fixed_place_kernel(FixedCompressArgs a) {
  // one warp per tile (many tiles in flight per SM: the copy is bound by the memory latency of
  // each tile's few words)
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t item = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); item < a.nitems; item += nwarps) {
    const CfColumn& col = a.cols ? a.cols[a.owner ? a.owner[item] : 0] : a.single;
    const int64_t t = item - col.item_base;
    const int64_t base = a.tile_first[col.item_base];
    const int64_t first = a.tile_first[item] - base;
    const int64_t bits = a.tile_bits[item];
    const int64_t col_end = col.item_base + col.ntiles;  // the column's items are [item_base, col_end)
    const int64_t e0 = t * kDecodeTile;
    const int cnt = (int)((col.n - e0) < kDecodeTile ? (col.n - e0) : kDecodeTile);
    const int np = (cnt + col.L - 1) / col.L;
    if (lane < np) {
      const int64_t gp = t * col.parts_per_tile + lane;
      col.offs[gp] += first;
      col.desc[gp].bit_off += first;
    }
    const int64_t total = a.tile_first[col_end - 1] - base + a.tile_bits[col_end - 1];
    if (lane == 0) {
      col.tiles[t].bit_lo = first;
      if (t == col.ntiles - 1) {
        TileInfo te;
        te.bit_lo = total;
        te.p_first = te.p_last = (int32_t)(col.P - 1);
        col.tiles[col.ntiles] = te;
        col.stats[0] = (unsigned long long)total;
      }
    }
    const int64_t w_begin = (first + 31) >> 5, w_end = (first + bits + 31) >> 5;
    if (w_end > col.words_cap) {  // the caller sized the array from another count: report, write nothing
      if (lane == 0) atomicExch(a.status, (unsigned long long)DEVERR_BOUNDS);
      continue;
    }
    const uint32_t* slot = a.slots + item * a.slot_words;
    const int r = (int)((32 * w_begin - first) & 31);  // the same shift for every word of the tile
    const int64_t k0 = (32 * w_begin - first) >> 5;
#pragma unroll 4
    for (int64_t w = w_begin + lane; w < w_end; w += 32) {
      const int64_t lb = 32 * w - first;  // tile bit of the word's bit 0 (0 <= lb < bits)
      const int64_t k = k0 + (w - w_begin);
      uint32_t v = r ? __funnelshift_r(slot[k], slot[k + 1], r) : slot[k];
      const int64_t avail = bits - lb;
      if (avail < 32) {  // the tile ends inside the word: the next tiles' first bits follow
        v &= (1u << avail) - 1u;
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
      }
      col.words[w] = v;
    }
    if (t == col.ntiles - 1 && col.nwords_alloc > 0) {  // the decoders' zeroed read-ahead after the bitstream
      const int64_t wt = (total + 31) >> 5;
      int64_t pad_end = ((wt + 3) & ~3ll) + 8;
      pad_end = pad_end < col.nwords_alloc ? pad_end : col.nwords_alloc;
      for (int64_t w = wt + lane; w < pad_end && w < col.words_cap; w += 32) col.words[w] = 0u;
    }
  }
}

template <typename T> static cudaError_t launch_fixed_compress_t(const FixedCompressArgs& a, int num_sms, cudaStream_t s) {
  constexpr int smem = cf_smem_bytes<T>();
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
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fixed_compress_kernel<T>, kCfCTA, smem)) !=
      cudaSuccess)
    return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * num_sms;
  if (grid > a.nitems) grid = a.nitems;
  if (grid < 1) grid = 1;
  fixed_compress_kernel<T><<<(unsigned)grid, kCfCTA, smem, s>>>(a);
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

template <typename T> static cudaError_t launch_choose_t(const FixedCompressArgs& a, int num_sms, cudaStream_t s) {
  constexpr int smem = kCfStages * cf_stage_bytes<T>();
  static PerDeviceFlag attr_set;
  const int dev = current_device();
  cudaError_t e;
  if (!attr_set.test(dev)) {
    if ((e = cudaFuncSetAttribute(choose_lengths_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) !=
        cudaSuccess)
      return e;
    attr_set.set(dev);
  }
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, choose_lengths_kernel<T>, kCfCTA, smem)) !=
      cudaSuccess)
    return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * num_sms;
  if (grid > a.nitems) grid = a.nitems;
  if (grid < 1) grid = 1;
  choose_lengths_kernel<T><<<(unsigned)grid, kCfCTA, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_choose_lengths(glc_dtype dt, const CfColumn* cols, const int32_t* owner, int64_t nitems,
                                  unsigned long long* status, int num_sms, cudaStream_t s) {
  if (nitems <= 0) return cudaSuccess;
  FixedCompressArgs a{};
  a.cols = cols;
  a.owner = owner;
  a.nitems = nitems;
  a.status = status;
  switch (dt) {
    case GLC_I32: return launch_choose_t<int32_t>(a, num_sms, s);
    case GLC_I64: return launch_choose_t<int64_t>(a, num_sms, s);
    case GLC_U64: return launch_choose_t<uint64_t>(a, num_sms, s);
    case GLC_U32: return launch_choose_t<uint32_t>(a, num_sms, s);
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
  const int64_t need = (a.nitems + 7) / 8;  // eight tiles (warps) per CTA
  int64_t grid = need < (int64_t)num_sms * 16 ? need : (int64_t)num_sms * 16;
  if (grid < 1) grid = 1;
  fixed_place_kernel<<<(unsigned)grid, 256, 0, s>>>(a);
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
