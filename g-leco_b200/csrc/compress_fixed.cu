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
//     -  the tile's first bit: a decoupled look-back over per-tile status words (each tile posts
//        its bit count, then its inclusive prefix once known; Merrill & Garland, "Single-pass
//        parallel prefix scan with decoupled look-back", 2016);
//     C  the tile's words from the residual fields, one thread per word; a word the tile shares
//        with a neighbouring tile goes to a side table (edge_head / edge_tail) and
//        fixed_edges_kernel merges it afterwards, so no word is written twice and nothing needs
//        zeroing first;
//     -  the partitions' metadata (the reference's SoA), their 32-byte descriptors and the
//        tile's decode-table entry.
//
// The words go to a buffer of the worst-case size (64 bits per value for 8-byte types, 33 for
// 4-byte types); the caller copies the used words into the column's exact-size array.
#include <type_traits>
#include "glc_internal.h"
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

// Look-back status of a tile: top two bits 1 = its own bit count posted, 2 = its inclusive prefix
// posted; the low 62 bits hold the count.  Zero at launch.
constexpr unsigned long long kLbAgg = 1ull << 62, kLbInc = 2ull << 62, kLbVal = (1ull << 62) - 1;

// A launch: work item i = one 4096-value tile of column owner[i] (every column of one element
// type, tiles in order), or of `single` when cols is null.
struct FixedCompressArgs {
  const CfColumn* cols;
  const int32_t* owner;
  CfColumn single;
  int64_t nitems;
  uint32_t* edge_head;        // per item: its bits of a first word it shares with an earlier tile
  uint32_t* edge_tail;        // per item: its bits of a last word it shares with a later tile
  unsigned long long* state;  // per item look-back status, zero at launch
  unsigned long long* status; // DEVERR_* when a bounded wait gave up
};

__device__ __forceinline__ void cf_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kCfThreads) : "memory"); }

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.volatile.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Sum of the bits of all tiles before t (thread 0 of the compute warps).  Posts t's own count
// first, so later tiles can look past t before t knows its prefix.  false when a wait gave up.
// Sum of the bits of all tiles before t in its column (`state` = the status of the column's tile
// 0), by one warp: every lane reads one predecessor's status, 32 at a time (the warp-wide window of
// the decoupled look-back), until the window holds an inclusive prefix; the aggregates between it
// and t are added.  The warp waits (bounded) while a predecessor in the window has posted nothing.
// Lane 0 posts t's own count first and its inclusive prefix at the end.  false when a wait gave up.
__device__ __forceinline__ bool cf_look_back(unsigned long long* state, int64_t t, unsigned long long agg,
                                             unsigned long long* prefix) {
  const int lane = threadIdx.x & 31;
  if (t == 0) {
    if (lane == 0) atomicExch(state, kLbInc | agg);
    *prefix = 0;
    return true;
  }
  if (lane == 0) atomicExch(state + t, kLbAgg | agg);
  unsigned long long acc = 0;
  int64_t hi = t - 1;
  const uint64_t t0 = global_ns();
  long long it = 0;
  bool ok = true;
  while (true) {
    const int64_t k = hi - lane;
    // below tile 0 nothing is added (tile 0 posts its inclusive prefix, so the window stops there)
    const unsigned long long sv = k >= 0 ? ld_volatile_u64(state + k) : kLbInc;
    if (__any_sync(FULL_MASK, (sv & (kLbAgg | kLbInc)) == 0)) {
      if (++it > kSpinLimit || ((it & 255) == 0 && global_ns() - t0 > 2000000000ull)) { ok = false; break; }
      continue;
    }
    const unsigned inc = __ballot_sync(FULL_MASK, (sv & kLbInc) != 0);
    const int stop = inc ? __ffs(inc) - 1 : 32;  // the nearest inclusive prefix in the window
    unsigned long long v = lane <= stop ? (sv & kLbVal) : 0ull;
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(FULL_MASK, v, m);
    acc += v;
    if (inc) break;
    hi -= 32;
  }
  if (lane == 0) atomicExch(state + t, kLbInc | (acc + agg));
  *prefix = acc;
  return ok;
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
  __shared__ unsigned long long s_bit0;
  __shared__ int s_ok, s_bmax;

  if (threadIdx.x == 0) {
    for (int st = 0; st < kCfStages; st++) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (threadIdx.x >= kCfThreads) {  // ---- producer ----
    if (threadIdx.x != kCfThreads) return;
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
          double md = 0.0;
          if (exact_fp64) {
            // |y| < 2^51 and the predictions inside pred_fp64_safe's bounds: y - pred is below 2^52,
            // so the integer difference is calculateDelta and its double is exact
#pragma unroll 4
            for (int m = 0; m < kCfPerThread; m++) {
              const int i = r_me + g * m;
              if (i < my_len) {
                const T y = xp[i];
                exact_fp64 &= value_fp64_safe<T>(y);
                const T pr = predict_from<T>(__fma_rn(t1, (double)i, t0));
                const long long d = (long long)y - (long long)pr;
                rp[i] = d;
                md = fmax(md, fabs(__ll2double_rn(d)));
              }
            }
            mx = (unsigned long long)md;
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
    if (tid == 0) {  // tile-relative bit ranges
      int acc = 0, bmax = 0;
      for (int p = 0; p < np; p++) {
        s_bl[p] = acc;
        acc += s_len[p] * s_b[p];
        bmax = s_b[p] > bmax ? s_b[p] : bmax;
      }
      s_bl[np] = acc;
      s_bmax = bmax;
    }
    cf_sync();
    if (tid < 32) {  // the look-back (warp 0), the tile's table entry
      const int acc = s_bl[np], bmax = s_bmax;
      unsigned long long prefix = 0;
      const bool lb_ok = cf_look_back(a.state + col.item_base, t, (unsigned long long)acc, &prefix);
      if (tid == 0) {
      if (!lb_ok) atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
      s_bit0 = prefix;
      TileInfo ti;
      ti.bit_lo = (int64_t)prefix;
      ti.p_first = (int32_t)(t * col.parts_per_tile);
      ti.p_last = (int32_t)(t * col.parts_per_tile + np - 1);
      col.tiles[t] = ti;
      if (t == col.ntiles - 1) {
        TileInfo te;
        te.bit_lo = (int64_t)(prefix + acc);
        te.p_first = te.p_last = (int32_t)(col.P - 1);
        col.tiles[col.ntiles] = te;
        col.stats[0] = prefix + acc;
      }
      if (bmax > 0) atomicMax(col.stats + 1, (unsigned long long)bmax);
      }
    }
    cf_sync();
    const unsigned long long bit0 = s_bit0;
    if (tid < np) {  // the partitions' metadata and descriptors
      const int p = tid;
      const int64_t gp = t * col.parts_per_tile + p;
      const int32_t start = (int32_t)(e0 + (int64_t)p * L);
      const int type = s_direct[p] ? MODEL_DIRECT_COPY : MODEL_LINEAR;
      const int64_t off = (int64_t)bit0 + s_bl[p];
      col.starts[gp] = start;
      col.ends[gp] = start + s_len[p];
      col.types[gp] = type;
      col.params[4 * gp] = s_t0[p];
      col.params[4 * gp + 1] = s_t1[p];
      col.params[4 * gp + 2] = 0.0;
      col.params[4 * gp + 3] = 0.0;
      col.bits[gp] = s_b[p];
      col.offs[gp] = off;
      col.err[gp] = s_err[p];
      PartDesc d;
      d.theta0 = s_t0[p];
      d.theta1 = s_t1[p];
      d.bit_off = off;
      d.start = start;
      d.bits_type = (s_b[p] & 0xff) | (type << 8);
      col.desc[gp] = d;
    }

    // ---- C: words.  Word w covers tile-relative bits [32 w - sh0, 32 w - sh0 + 32). ----
    {
      const int sh0 = (int)(bit0 & 31);
      const int tb = s_bl[np];
      const int nw = tb > 0 ? (sh0 + tb + 31) >> 5 : 0;
      const bool first_partial = sh0 != 0;
      const bool last_partial = ((bit0 + (unsigned long long)tb) & 31) != 0;
      const uint32_t* f32 = reinterpret_cast<const uint32_t*>(res);  // low half of residual j at 2 j
      uint32_t* out = col.words + (bit0 >> 5);
      // never past the word array (the caller sized it; a disagreement is reported, not written)
      const bool fits = (int64_t)((bit0 + (unsigned long long)tb + 31) >> 5) <= col.words_cap;
      if (!fits && tid == 0) atomicExch(a.status, (unsigned long long)DEVERR_BOUNDS);
      int qi = 0;
      for (int w = fits ? tid : nw; w < nw; w += kCfThreads) {
        const int wb = 32 * w - sh0;
        int pos = wb > 0 ? wb : 0;
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
        if (w == 0 && first_partial) a.edge_head[item] = word;
        else if (w == nw - 1 && last_partial) a.edge_tail[item] = word;
        else out[w] = word;
      }
    }
    cf_sync();  // every compute thread is done with stage st and the residual array
    if (tid == 0) mbar_arrive(&empty[st]);
  }
}

// The words shared by neighbouring tiles.  Word W holding a tile's last bit, when that tile also
// holds W's first bit, is written here by that tile's thread: its own bits (edge_tail) OR the
// first bits of every later tile of the column that starts inside W (edge_head; tiles without
// bits are skipped).  The column's last tile also zeroes the padding words after its bitstream.
__global__ void fixed_edges_kernel(FixedCompressArgs a) {
  const int64_t item = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= a.nitems) return;
  const CfColumn& col = a.cols ? a.cols[a.owner ? a.owner[item] : 0] : a.single;
  const int64_t t = item - col.item_base;
  const TileInfo* tiles = col.tiles;
  const int64_t b0 = tiles[t].bit_lo, b1 = tiles[t + 1].bit_lo;
  if (t == col.ntiles - 1 && col.nwords_alloc > 0)
    for (int64_t w = (b1 + 31) >> 5; w < col.nwords_alloc && w < col.words_cap; w++) col.words[w] = 0u;
  if (b1 == b0 || (b1 & 31) == 0) return;     // no bits, or a complete last word (already written)
  const int64_t wi = b1 >> 5;
  if (wi >= col.words_cap) return;            // reported by the compress kernel
  if (b0 > (wi << 5)) return;                 // the tile starts inside W: an earlier tile owns it
  uint32_t word = a.edge_tail[item];
  for (int64_t u = t + 1; u < col.ntiles; u++) {
    const int64_t c0 = tiles[u].bit_lo, c1 = tiles[u + 1].bit_lo;
    if (c1 == c0) continue;
    if ((c0 >> 5) != wi) break;
    word |= a.edge_head[col.item_base + u];
    if (c1 > ((wi + 1) << 5) || (c1 & 31) == 0) break;  // u goes past W
  }
  col.words[wi] = word;
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
  // every CTA resident at once: a tile's look-back waits only on tiles that resident CTAs own
  int64_t grid = (int64_t)per_sm * num_sms;
  if (grid > a.nitems) grid = a.nitems;
  if (grid < 1) grid = 1;
  fixed_compress_kernel<T><<<(unsigned)grid, kCfCTA, smem, s>>>(a);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  fixed_edges_kernel<<<(unsigned)((a.nitems + 255) / 256), 256, 0, s>>>(a);
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

bool fixed_compress_supported(int64_t n, int32_t L) {
  return n > 0 && L >= kCfMinLen && L <= kDecodeTile && (kDecodeTile % L) == 0;
}

int64_t fixed_compress_worst_words(glc_dtype dt, int64_t n) {
  const int64_t per_value = (dt == GLC_I64 || dt == GLC_U64) ? 64 : 33;  // widest field of the type
  return (n * per_value + 31) / 32 + 8;
}

size_t fixed_compress_scratch_bytes(int64_t nitems) { return (size_t)nitems * 16 + 64; }

// One column: values (n of dt, fixed partitions of L) into c's metadata arrays and tables
// (allocated by the caller for P = ceil(n / L) partitions) and into `words`
// (fixed_compress_worst_words words; its padding is left to the caller); `scratch` holds
// fixed_compress_scratch_bytes(ntiles) bytes; stats[0] receives the total bits, stats[1] the
// widest field, stats[2] a DEVERR_* code (stats[0..3] zeroed here).
cudaError_t launch_fixed_compress(glc_dtype dt, const void* values, glc_column* c, int32_t L, uint32_t* words,
                                  void* scratch, unsigned long long* stats, cudaStream_t s) {
  FixedCompressArgs a{};
  CfColumn& col = a.single;
  col.values = values;
  col.n = c->n;
  col.L = L;
  col.parts_per_tile = kDecodeTile / L;
  col.P = c->P;
  col.ntiles = c->ntiles;
  col.item_base = 0;
  col.nwords_alloc = 0;
  col.starts = c->d_start;
  col.ends = c->d_end;
  col.types = c->d_types;
  col.params = c->d_params;
  col.bits = c->d_bits;
  col.offs = c->d_offs;
  col.err = c->d_err;
  col.desc = c->d_desc;
  col.tiles = c->d_tiles;
  col.words = words;
  col.words_cap = fixed_compress_worst_words(dt, c->n);
  col.stats = stats;
  a.nitems = c->ntiles;
  uint8_t* sp = reinterpret_cast<uint8_t*>(scratch);
  a.state = reinterpret_cast<unsigned long long*>(sp);
  a.edge_head = reinterpret_cast<uint32_t*>(sp + (size_t)a.nitems * 8);
  a.edge_tail = a.edge_head + a.nitems;
  a.status = stats + 2;
  cudaError_t e;
  if ((e = cudaMemsetAsync(a.state, 0, (size_t)a.nitems * 8, s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned long long), s)) != cudaSuccess) return e;
  return launch_fixed_compress_dt(dt, a, c->ctx ? c->ctx->num_sms : 148, s);
}

// Many columns of one element type in one launch: cols (device, ncols entries, each with its own
// arrays, stats zeroed and nwords_alloc set) and owner (device, nitems entries: the column of each
// item, items in column order).  scratch: fixed_compress_scratch_bytes(nitems) bytes; status: a
// DEVERR_* word.
cudaError_t launch_fixed_compress_batch(glc_dtype dt, const CfColumn* cols, const int32_t* owner, int64_t nitems,
                                        void* scratch, unsigned long long* status, int num_sms, cudaStream_t s) {
  if (nitems <= 0) return cudaSuccess;
  FixedCompressArgs a{};
  a.cols = cols;
  a.owner = owner;
  a.nitems = nitems;
  uint8_t* sp = reinterpret_cast<uint8_t*>(scratch);
  a.state = reinterpret_cast<unsigned long long*>(sp);
  a.edge_head = reinterpret_cast<uint32_t*>(sp + (size_t)nitems * 8);
  a.edge_tail = a.edge_head + nitems;
  a.status = status;
  cudaError_t e;
  if ((e = cudaMemsetAsync(a.state, 0, (size_t)nitems * 8, s)) != cudaSuccess) return e;
  return launch_fixed_compress_dt(dt, a, num_sms, s);
}

}  // namespace glc
