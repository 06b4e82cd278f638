// fit.cu -- per-partition model fit, residual bit width, bit offsets and lookup tables.
//
// Replaces compression/CompressionKernels.cuh:45-218 (wprocessPartitionsKernel: overflow
// check -> MODEL_DIRECT_COPY, linear fit, max |delta|, delta_bits) and :222-238
// (setBitOffsetsKernel, an O(P) loop per partition).
//
// Layout of the work: a partition of any length is cut into chunks of 4096 values; one CTA
// per chunk accumulates exact 128-bit sums (sum y, sum i*y) and the overflow flag, a thread per
// partition combines its chunks and solves the line, one CTA per chunk takes the max |delta|
// (64-bit atomicMax per partition), and a thread per partition sets the bit width.  The
// bit offsets are an exclusive scan of len * bits.  All passes read the values once or twice
// with coalesced loads; nothing here is a contraction, so the bound is HBM bandwidth.
#include <type_traits>
#include "glc_internal.h"
#include "glc_scan.cuh"
#include "glc_tma.cuh"

namespace glc {

constexpr int kFitChunk = 4096;
constexpr int kFitThreads = 256;

__global__ void fixed_partitions_kernel(int32_t* starts, int32_t* ends, int64_t n, int32_t len, int64_t P) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  int64_t s = p * len;
  starts[p] = (int32_t)s;
  ends[p] = (int32_t)(s + len < n ? s + len : n);
}

cudaError_t launch_fixed_partitions(int32_t* starts, int32_t* ends, int64_t n, int32_t len, int64_t P, cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  fixed_partitions_kernel<<<(unsigned)((P + 255) / 256), 256, 0, s>>>(starts, ends, n, len, P);
  return cudaGetLastError();
}

__global__ void chunk_count_kernel(const int32_t* __restrict__ starts, const int32_t* __restrict__ ends, int64_t P,
                                   int64_t* __restrict__ nch) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  int64_t len = (int64_t)ends[p] - starts[p];
  nch[p] = len > 0 ? (len + kFitChunk - 1) / kFitChunk : 0;
}

// owner[c] = the partition of chunk c (one thread per partition writes its chunks), so a fit CTA
// finds its partition with one load instead of a dependent binary search.
__global__ void chunk_owner_kernel(const int64_t* __restrict__ base, const int64_t* __restrict__ nch, int64_t P,
                                   int32_t* __restrict__ owner) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  for (int64_t c = base[p], e = base[p] + nch[p]; c < e; c++) owner[c] = (int32_t)p;
}

struct FitChunkArgs {
  const int32_t* starts;
  const int32_t* ends;
  const int64_t* chunk_base;
  const int64_t* num_chunks;  // device scalar: total chunks
  const int32_t* owner;       // chunk -> partition
  int64_t P;
  i128* sy;
  i128* sxy;
  int* ovf;
};

// Barrier of the kFitThreads compute threads only (named barrier 1; a producer warp may run beside
// them in the same CTA).
__device__ __forceinline__ void fit_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kFitThreads) : "memory"); }

// Sum over the kFitThreads compute threads of two 128-bit values and an OR; valid in thread 0.
__device__ __forceinline__ void block_sums(i128& sy, i128& sxy, int& ovf) {
  sy = warp_sum_i128(sy);
  sxy = warp_sum_i128(sxy);
  ovf = __any_sync(FULL_MASK, ovf);
  __shared__ i128 s_sy[kFitThreads / 32], s_sxy[kFitThreads / 32];
  __shared__ int s_ovf[kFitThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { s_sy[warp] = sy; s_sxy[warp] = sxy; s_ovf[warp] = ovf; }
  fit_sync();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kFitThreads / 32; w++) { sy += s_sy[w]; sxy += s_sxy[w]; ovf |= s_ovf[w]; }
  }
}

// Max over the kFitThreads compute threads; valid in thread 0.
__device__ __forceinline__ long long block_max(long long m) {
  m = warp_max_ll(m);
  __shared__ long long s_m[kFitThreads / 32];
  if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5] = m;
  fit_sync();
  if (threadIdx.x == 0)
    for (int w = 1; w < kFitThreads / 32; w++) m = s_m[w] > m ? s_m[w] : m;
  return m;
}

// Persistent fit passes over a dense list of chunks (chunk j -> partition owner[j], chunk index
// j - base[owner[j]] within it).  CTA = 8 compute warps + 1 producer warp.  The producer (one
// lane) looks up each chunk's partition and stages its values in shared memory with one bulk
// copy (source rounded down and length up to 16 bytes: the extra bytes lie in the same 16-byte
// blocks as the chunk, never in another page), kFitStages chunks ahead, on full/empty mbarriers;
// the compute warps work from shared memory while the next copies land.  Their ring wait is
// done by thread 0 (bounded) and broadcast, so a timeout takes them out of the loop together.
//   PASS 0 (every chunk): overflow flag and exact sums; a partition of at most one chunk is
//     fitted completely -- line, max |delta| -- from the staged values (one HBM read).
//   PASS 1 (chunks of partitions longer than one chunk): max |delta| against the line that
//     fit_solve_kernel derived from the chunk sums, one atomicMax per chunk.
constexpr int kFitStages = 2;

struct FitStreamArgs {
  const int32_t* starts;
  const int32_t* ends;
  const int64_t* count;   // device scalar: chunks in the list
  const int32_t* owner;   // list entry -> partition
  const int64_t* base;    // partition -> its first list entry
  int64_t P;
  i128* sy;               // PASS 0: sums of chunks of long partitions, by chunk number
  i128* sxy;
  int* ovf;
  const int64_t* chunk_base;  // partition -> its first chunk number (PASS 0 list == chunk numbers)
  int32_t* types;
  double* params;
  int64_t* err;
  unsigned long long* status;  // DEVERR_* on a timed-out wait
};

struct FitStage {
  int64_t j;       // list entry, -1 = no more work
  int64_t p, i0;   // partition, first value of the chunk within it
  int64_t len;     // partition length
  double t0, t1;   // PASS 1: the partition's line
  int32_t cnt;     // values in the chunk
  int32_t head;    // byte offset of the first value in the stage
  int32_t skip;    // PASS 1: direct-copy partition, nothing to measure
};

template <typename T> __host__ __device__ constexpr int fit_stage_bytes() { return kFitChunk * (int)sizeof(T) + 32; }

// max over this thread's values x[jj] (jj = tid, tid + 256, ...) of abs_ref(calc_delta(x, pred))
// with pred = predict(t0, t1, i0 + jj): the index advances as an exact double (no conversion per
// value), and the saturating |delta| is formed once from the extreme differences.
template <typename T>
__device__ __forceinline__ long long chunk_max_abs_delta(const T* x, int cnt, double t0, double t1, int64_t i0) {
  if (cnt > 0 && line_fp64_safe<T>(t0, t1, i0, i0 + cnt - 1)) {
    // exact in FP64 (values checked as they are read; a thread with a larger value redoes its own)
    double md = 0.0, xd = (double)(i0 + (int64_t)threadIdx.x);
    bool ok = true;
#pragma unroll 4
    for (int jj = threadIdx.x; jj < cnt; jj += kFitThreads, xd += (double)kFitThreads) {
      const T y = x[jj];
      ok &= value_fp64_safe<T>(y);
      md = fmax(md, abs_resid_fp64((double)(long long)y, __fma_rn(t1, xd, t0)));
    }
    if (ok) return (long long)md;
  }
  double xd = (double)(i0 + (int64_t)threadIdx.x);
  if (TypeTraits<T>::is_signed || sizeof(T) == 4) {
    // calc_delta is the plain (wrapping for 64-bit) signed difference
    long long dmax = 0, dmin = 0;
#pragma unroll 4
    for (int jj = threadIdx.x; jj < cnt; jj += kFitThreads, xd += (double)kFitThreads) {
      const long long d = calc_delta<T>(x[jj], predict_from<T>(__fma_rn(t1, xd, t0)));
      dmax = d > dmax ? d : dmax;
      dmin = d < dmin ? d : dmin;
    }
    const long long a1 = abs_ref(dmax), a2 = abs_ref(dmin);
    return a1 > a2 ? a1 : a2;
  } else {
    // unsigned 64-bit: |a - p| saturated at 2^63 - 1 (calc_delta's saturation, then abs_ref)
    uint64_t um = 0;
#pragma unroll 4
    for (int jj = threadIdx.x; jj < cnt; jj += kFitThreads, xd += (double)kFitThreads) {
      const uint64_t a = (uint64_t)x[jj], p = (uint64_t)predict_from<T>(__fma_rn(t1, xd, t0));
      const uint64_t d = a >= p ? a - p : p - a;
      um = d > um ? d : um;
    }
    return um > 0x7fffffffffffffffull ? 0x7fffffffffffffffll : (long long)um;
  }
}

constexpr int kFitCTA = kFitThreads + 32;  // compute warps + producer warp

template <typename T, int PASS>
__device__ __forceinline__ FitStage fit_stage_for(const T* __restrict__ v, const FitStreamArgs& a, int64_t j) {
  FitStage m;
  m.j = j;
  m.p = a.owner[j];
  const int64_t start = a.starts[m.p];
  m.len = (int64_t)a.ends[m.p] - start;
  m.i0 = (j - a.base[m.p]) * kFitChunk;
  m.cnt = (int)((m.len - m.i0) < kFitChunk ? (m.len - m.i0) : kFitChunk);
  m.skip = 0;
  m.t0 = m.t1 = 0.0;
  if (PASS == 1) {
    m.skip = a.types[m.p] == MODEL_DIRECT_COPY;
    m.t0 = a.params[4 * m.p];
    m.t1 = a.params[4 * m.p + 1];
  }
  const uintptr_t addr = reinterpret_cast<uintptr_t>(v + start + m.i0);
  m.head = (int)(addr & 15);
  return m;
}

template <typename T, int PASS> __global__ void __launch_bounds__(kFitCTA)
fit_stream_kernel(const T* __restrict__ v, FitStreamArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t full[kFitStages], empty[kFitStages];
  __shared__ FitStage s_meta[kFitStages];
  __shared__ int s_ok, s_direct;
  __shared__ double s_t[2];
  if (threadIdx.x == 0) {
    for (int st = 0; st < kFitStages; st++) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (threadIdx.x >= kFitThreads) {  // ---- producer ----
    if (threadIdx.x != kFitThreads) return;
    const int64_t total = *a.count;
    int64_t j = blockIdx.x;
    for (int k = 0;; k++, j += gridDim.x) {
      const int st = k % kFitStages;
      if (k >= kFitStages && !mbar_wait_bounded(&empty[st], (uint32_t)((k / kFitStages) - 1) & 1u)) {
        atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
        s_meta[st].j = -1;  // the compute warps stop at this stage (or time out on it)
        mbar_arrive(&full[st]);
        return;
      }
      if (j >= total) {
        s_meta[st].j = -1;
        mbar_arrive(&full[st]);  // no copy: completes the phase, the compute warps see the end
        return;
      }
      const FitStage m = fit_stage_for<T, PASS>(v, a, j);
      s_meta[st] = m;
      if (m.skip) {
        mbar_arrive(&full[st]);
      } else {
        const uint32_t bytes = (uint32_t)((m.head + (int64_t)m.cnt * (int64_t)sizeof(T) + 15) & ~15ll);
        const void* src = reinterpret_cast<const uint8_t*>(v + a.starts[m.p] + m.i0) - m.head;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive_expect_tx(&full[st], bytes);
        tma_bulk_load(smem + (size_t)st * fit_stage_bytes<T>(), src, bytes, &full[st]);
      }
    }
  }

  // ---- compute warps ----
  for (int k = 0;; k++) {
    const int st = k % kFitStages;
    const uint32_t par = (uint32_t)(k / kFitStages) & 1u;
    if (threadIdx.x == 0) {
      s_ok = mbar_wait_bounded(&full[st], par);
      if (!s_ok) {
        atomicExch(a.status, (unsigned long long)DEVERR_TIMEOUT);
        mbar_wait_bounded(&full[st], par);  // a copy in flight lands before the CTA exits
      }
    }
    fit_sync();
    if (!s_ok) return;
    mbar_try_wait(&full[st], par);  // the phase is complete: orders this thread's reads after the copy
    const FitStage m = s_meta[st];
    if (m.j < 0) return;
    const T* x = reinterpret_cast<const T*>(smem + (size_t)st * fit_stage_bytes<T>() + m.head);
    if (PASS == 0) {
      // Exact sums from 64-bit partials: y = yh * 2^32 + yl, so sum(y) and sum(jj * y) (jj < 4096,
      // the index within the chunk) split into four sums that cannot overflow 64 bits over the
      // 16 values of a thread; sum((i0 + jj) * y) = sum(jj * y) + i0 * sum(y) is added once.
      typedef typename std::conditional<TypeTraits<T>::is_signed, int64_t, uint64_t>::type Acc;
      Acc s_lo = 0, s_hi = 0, x_lo = 0, x_hi = 0;
      int ovf = 0;
#pragma unroll 4
      for (int jj = threadIdx.x; jj < m.cnt; jj += kFitThreads) {
        const T xv = x[jj];
        ovf |= overflows_double<T>(xv) ? 1 : 0;
        if (sizeof(T) == 8) {
          const uint32_t yl = (uint32_t)(uint64_t)xv;
          const Acc yh = TypeTraits<T>::is_signed ? (Acc)(int32_t)((int64_t)xv >> 32) : (Acc)(uint32_t)((uint64_t)xv >> 32);
          s_lo += (Acc)yl;
          s_hi += yh;
          x_lo += (Acc)((uint64_t)(uint32_t)jj * yl);
          x_hi += (Acc)jj * yh;
        } else {
          s_lo += (Acc)xv;
          x_lo += (Acc)jj * (Acc)xv;
        }
      }
      i128 sy = (i128)s_lo + (i128)s_hi * ((i128)1 << 32);
      i128 sxy = (i128)x_lo + (i128)x_hi * ((i128)1 << 32);
      block_sums(sy, sxy, ovf);
      if (threadIdx.x == 0) sxy += (i128)m.i0 * sy;
      if (m.len > kFitChunk) {  // a chunk of a longer partition: its sums, by chunk number
        if (threadIdx.x == 0) { a.sy[m.j] = sy; a.sxy[m.j] = sxy; a.ovf[m.j] = ovf; }
      } else {
        if (threadIdx.x == 0) {
          double t0 = 0.0, t1 = 0.0;
          if (ovf) {
            a.types[m.p] = MODEL_DIRECT_COPY;  // CompressionKernels.cuh:95-105
          } else {
            solve_line(m.len, sy, sxy, t0, t1);
            a.types[m.p] = MODEL_LINEAR;
          }
          a.params[4 * m.p] = t0;
          a.params[4 * m.p + 1] = t1;
          a.params[4 * m.p + 2] = 0.0;
          a.params[4 * m.p + 3] = 0.0;
          s_t[0] = t0;
          s_t[1] = t1;
          s_direct = ovf;
        }
        fit_sync();
        long long mx = 0;
        if (!s_direct) mx = chunk_max_abs_delta<T>(x, m.cnt, s_t[0], s_t[1], 0);
        mx = block_max(mx);
        if (threadIdx.x == 0) a.err[m.p] = mx;
      }
    } else if (!m.skip) {
      long long mx = chunk_max_abs_delta<T>(x, m.cnt, m.t0, m.t1, m.i0);
      mx = block_max(mx);
      if (threadIdx.x == 0 && mx > 0) atomicMax((long long*)a.err + m.p, mx);
    }
    fit_sync();  // every compute thread is done with stage st (and with s_t / s_direct)
    if (threadIdx.x == 0) mbar_arrive(&empty[st]);
  }
}

// Line of every partition longer than one chunk, from its chunks' sums.
template <typename T> __global__ void fit_solve_kernel(FitChunkArgs a, const int64_t* __restrict__ nch,
                                                      int32_t* __restrict__ types, double* __restrict__ params,
                                                      int64_t* __restrict__ err) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.P) return;
  const int64_t len = (int64_t)a.ends[p] - a.starts[p];
  if (len > 0 && len <= kFitChunk) return;  // fitted by PASS 0 of fit_stream_kernel
  const int64_t c0 = a.chunk_base[p], c1 = c0 + nch[p];
  i128 sy = 0, sxy = 0;
  int ovf = 0;
  for (int64_t c = c0; c < c1; c++) { sy += a.sy[c]; sxy += a.sxy[c]; ovf |= a.ovf[c]; }
  double t0 = 0.0, t1 = 0.0;
  if (ovf) {
    types[p] = MODEL_DIRECT_COPY;  // CompressionKernels.cuh:95-105
  } else {
    solve_line(len, sy, sxy, t0, t1);
    types[p] = MODEL_LINEAR;
  }
  params[4 * p] = t0;
  params[4 * p + 1] = t1;
  params[4 * p + 2] = 0.0;
  params[4 * p + 3] = 0.0;
  err[p] = 0;
}

// bits and len*bits; stats[1] = max bits; stats[3] = max over all partitions but the last of
// ceil(4096 / len) (bounds the partitions a 4096-value tile can span); one atomic per warp each.
template <typename T> __global__ void fit_bits_kernel(const int32_t* __restrict__ starts, const int32_t* __restrict__ ends,
                                                     const int32_t* __restrict__ types, const int64_t* __restrict__ err,
                                                     int32_t* __restrict__ bits, int64_t* __restrict__ widths, int64_t P,
                                                     unsigned long long* __restrict__ max_bits,
                                                     unsigned long long* __restrict__ per_tile) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int b = 0;
  unsigned k = 0;
  if (p < P) {
    b = (types[p] == MODEL_DIRECT_COPY) ? (int)sizeof(T) * 8 : bits_for(err[p]);
    bits[p] = b;
    const int64_t len = (int64_t)ends[p] - starts[p];
    widths[p] = len * b;
    if (p < P - 1 && len > 0) k = (unsigned)((kDecodeTile + len - 1) / len);
  }
  b = (int)__reduce_max_sync(FULL_MASK, (unsigned)b);
  k = __reduce_max_sync(FULL_MASK, k);
  if ((threadIdx.x & 31) == 0) {
    if (b > 0) atomicMax(max_bits, (unsigned long long)b);
    if (k > 0) atomicMax(per_tile, (unsigned long long)k);
  }
}

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// nm[p] = chunks of p when p is longer than one chunk (their maximum error takes a second pass).
__global__ void multi_count_kernel(const int32_t* __restrict__ starts, const int32_t* __restrict__ ends,
                                   const int64_t* __restrict__ nch, int64_t P, int64_t* __restrict__ nm) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  nm[p] = ((int64_t)ends[p] - starts[p]) > kFitChunk ? nch[p] : 0;
}

// Fixed partitions of length L (the last one n - (P - 1) L): the chunk tables in closed form, in
// one launch -- chunks per partition, each partition's first chunk, chunk -> partition, and the
// chunk counts of the two fit passes.  Partitions longer than one chunk are all the full ones
// (when L > 4096) and perhaps the last, so the second pass's list is a prefix of the first's
// and shares its tables.
__global__ void fixed_chunk_setup_kernel(int64_t n, int64_t L, int64_t P, int64_t* __restrict__ nch,
                                         int64_t* __restrict__ base, int32_t* __restrict__ owner,
                                         int64_t* __restrict__ nchunks, int64_t* __restrict__ nmulti) {
  const int64_t nch_full = (L + kFitChunk - 1) / kFitChunk;
  const int64_t len_last = n - (P - 1) * L;
  const int64_t nch_last = (len_last + kFitChunk - 1) / kFitChunk;
  const int64_t total = (P - 1) * nch_full + nch_last;
  const int64_t span = P > total ? P : total;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < span; i += (int64_t)gridDim.x * blockDim.x) {
    if (i < P) {
      nch[i] = i < P - 1 ? nch_full : nch_last;
      base[i] = i * nch_full;
    }
    if (i < total) {
      const int64_t o = i / nch_full;
      owner[i] = (int32_t)(o < P - 1 ? o : P - 1);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *nchunks = total;
    *nmulti = (L > kFitChunk ? (P - 1) * nch_full : 0) + (len_last > kFitChunk ? nch_last : 0);
  }
}

size_t fit_scratch_bytes(const int32_t*, int64_t n, int64_t P) {
  int64_t ncmax = n / kFitChunk + P + 1;
  size_t b = 0;
  b += align_up(sizeof(int64_t) * (P + 1), 256) * 4;                  // nch, chunk_base, nm, mbase
  b += align_up(sizeof(int64_t) * (scan_num_tiles(P) + 1), 256);      // scan tiles
  b += align_up(sizeof(int64_t) * 2, 256) * 2;                        // chunk count, long-partition chunk count
  b += align_up(sizeof(i128) * ncmax, 256) * 2;                       // sy, sxy
  b += align_up(sizeof(int) * ncmax, 256);                            // ovf
  b += align_up(sizeof(int32_t) * ncmax, 256) * 2;                    // owner, owner of the long-partition list
  b += align_up(sizeof(int64_t) * (P + 1), 256);                      // widths
  return b;
}

template <typename T, int PASS>
static cudaError_t launch_fit_stream(const T* v, const FitStreamArgs& a, int num_sms, cudaStream_t s) {
  const int smem = kFitStages * fit_stage_bytes<T>();
  static PerDeviceFlag attr_set;  // per instantiation and device
  const int dev = current_device();
  cudaError_t e;
  if (!attr_set.test(dev)) {
    if ((e = cudaFuncSetAttribute(fit_stream_kernel<T, PASS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) !=
        cudaSuccess)
      return e;
    attr_set.set(dev);
  }
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fit_stream_kernel<T, PASS>, kFitCTA, smem)) !=
      cudaSuccess)
    return e;
  if (per_sm < 1) per_sm = 1;
  fit_stream_kernel<T, PASS><<<(unsigned)(per_sm * num_sms), kFitCTA, smem, s>>>(v, a);
  return cudaGetLastError();
}

// A partition longer than one chunk whose max |delta| the variable partitioner measured against
// the same exact least-squares line takes it from there (direct-copy partitions keep 0).
__global__ void fit_known_err_kernel(const int32_t* __restrict__ starts, const int32_t* __restrict__ ends,
                                     const int32_t* __restrict__ types, const long long* __restrict__ known, int64_t P,
                                     int64_t* __restrict__ err) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  if ((int64_t)ends[p] - starts[p] <= kFitChunk || types[p] == MODEL_DIRECT_COPY) return;
  err[p] = known[p];
}

template <typename T>
static cudaError_t fit_typed(const T* v, glc_column* c, void* scratch, int64_t* d_stats, cudaStream_t s,
                             const long long* known_err) {
  const int64_t P = c->P, n = c->n;
  const int64_t ncmax = n / kFitChunk + P + 1;
  char* sp = (char*)scratch;
  auto take = [&](size_t bytes) { void* r = sp; sp += align_up(bytes, 256); return r; };
  int64_t* nch = (int64_t*)take(sizeof(int64_t) * (P + 1));
  int64_t* base = (int64_t*)take(sizeof(int64_t) * (P + 1));
  int64_t* nm = (int64_t*)take(sizeof(int64_t) * (P + 1));
  int64_t* mbase = (int64_t*)take(sizeof(int64_t) * (P + 1));
  int64_t* tiles = (int64_t*)take(sizeof(int64_t) * (scan_num_tiles(P) + 1));
  int64_t* nchunks = (int64_t*)take(sizeof(int64_t) * 2);
  int64_t* nmulti = (int64_t*)take(sizeof(int64_t) * 2);
  i128* sy = (i128*)take(sizeof(i128) * ncmax);
  i128* sxy = (i128*)take(sizeof(i128) * ncmax);
  int* ovf = (int*)take(sizeof(int) * ncmax);
  int32_t* owner = (int32_t*)take(sizeof(int32_t) * ncmax);
  int32_t* owner_m = (int32_t*)take(sizeof(int32_t) * ncmax);
  int64_t* widths = (int64_t*)take(sizeof(int64_t) * (P + 1));
  const unsigned pg = (unsigned)((P + 255) / 256);
  const int num_sms = c->ctx->num_sms;
  cudaError_t e;
  // stats: [0] total bits, [1] max bits, [2] device status of the fit passes, [3] the bound on
  // partitions per 4096-value tile (without the last partition)
  if ((e = cudaMemsetAsync(d_stats, 0, 4 * sizeof(int64_t), s)) != cudaSuccess) return e;

  if (c->fixed_len > 0) {  // fixed partitions: closed-form tables, one launch
    const int64_t span = n / kFitChunk + P + 1;
    int64_t grid = (span + 255) / 256;
    if (grid > 4ll * num_sms) grid = 4ll * num_sms;
    fixed_chunk_setup_kernel<<<(unsigned)grid, 256, 0, s>>>(n, c->fixed_len, P, nch, base, owner, nchunks, nmulti);
    owner_m = owner;  // the second pass's chunks are a prefix of the first's
    mbase = base;
  } else {
    chunk_count_kernel<<<pg, 256, 0, s>>>(c->d_start, c->d_end, P, nch);
    if ((e = exclusive_scan<int64_t>(nch, base, P, nchunks, tiles, s)) != cudaSuccess) return e;
    chunk_owner_kernel<<<pg, 256, 0, s>>>(base, nch, P, owner);
    if (!known_err) {  // the chunks of the second pass (partitions longer than one chunk)
      multi_count_kernel<<<pg, 256, 0, s>>>(c->d_start, c->d_end, nch, P, nm);
      if ((e = exclusive_scan<int64_t>(nm, mbase, P, nmulti, tiles, s)) != cudaSuccess) return e;
      chunk_owner_kernel<<<pg, 256, 0, s>>>(mbase, nm, P, owner_m);
    }
  }

  FitStreamArgs a{c->d_start, c->d_end, nchunks, owner, base, P, sy, sxy, ovf, base,
                  c->d_types, c->d_params, c->d_err, (unsigned long long*)(d_stats + 2)};
  if ((e = launch_fit_stream<T, 0>(v, a, num_sms, s)) != cudaSuccess) return e;
  FitChunkArgs fa{c->d_start, c->d_end, base, nchunks, owner, P, sy, sxy, ovf};
  fit_solve_kernel<T><<<pg, 256, 0, s>>>(fa, nch, c->d_types, c->d_params, c->d_err);
  if (known_err && c->fixed_len == 0) {
    fit_known_err_kernel<<<pg, 256, 0, s>>>(c->d_start, c->d_end, c->d_types, known_err, P, c->d_err);
  } else {
    FitStreamArgs am = a;
    am.count = nmulti;
    am.owner = owner_m;
    am.base = mbase;
    if ((e = launch_fit_stream<T, 1>(v, am, num_sms, s)) != cudaSuccess) return e;
  }
  fit_bits_kernel<T><<<pg, 256, 0, s>>>(c->d_start, c->d_end, c->d_types, c->d_err, c->d_bits, widths, P,
                                         (unsigned long long*)(d_stats + 1), (unsigned long long*)(d_stats + 3));
  // bit offsets = exclusive scan of len*bits; stats[0] = total bits
  e = exclusive_scan<int64_t>(widths, c->d_offs, P, d_stats, tiles, s);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t launch_fit(glc_dtype dt, const void* values, glc_column* c, void* scratch, size_t, int64_t* d_stats,
                       cudaStream_t s, const long long* known_err) {
  switch (dt) {
    case GLC_I32: return fit_typed<int32_t>((const int32_t*)values, c, scratch, d_stats, s, known_err);
    case GLC_I64: return fit_typed<int64_t>((const int64_t*)values, c, scratch, d_stats, s, known_err);
    case GLC_U64: return fit_typed<uint64_t>((const uint64_t*)values, c, scratch, d_stats, s, known_err);
    case GLC_U32: return fit_typed<uint32_t>((const uint32_t*)values, c, scratch, d_stats, s, known_err);
  }
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------------------
// Derived tables: 32-byte partition descriptors and the decode tile table.
// ---------------------------------------------------------------------------------------
// bit_shift: bits between the kernels' word base and the bitstream's first bit (attached blobs)
__global__ void build_desc_kernel(const int32_t* __restrict__ starts, const int32_t* __restrict__ types,
                                  const double* __restrict__ params, const int32_t* __restrict__ bits,
                                  const int64_t* __restrict__ offs, int64_t P, int64_t bit_shift,
                                  PartDesc* __restrict__ desc) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  PartDesc d;
  d.theta0 = params[4 * p];
  d.theta1 = params[4 * p + 1];
  d.bit_off = offs[p] + bit_shift;
  d.start = starts[p];
  d.bits_type = (bits[p] & 0xff) | (types[p] << 8);
  desc[p] = d;
}

// Partition containing position e: the last p with start[p] <= e.
__device__ __forceinline__ int64_t owner_of(const int32_t* __restrict__ starts, int64_t P, int64_t e) {
  int64_t lo = 0, hi = P - 1;
  while (lo < hi) {
    int64_t mid = (lo + hi + 1) >> 1;
    if ((int64_t)starts[mid] <= e) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void build_tiles_kernel(const int32_t* __restrict__ starts, const int32_t* __restrict__ bits,
                                   const int64_t* __restrict__ offs, int64_t P, int64_t n, int64_t ntiles,
                                   int64_t total_bits, int64_t bit_shift, TileInfo* __restrict__ tiles) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t > ntiles) return;
  TileInfo ti;
  if (t == ntiles) {
    ti.bit_lo = total_bits + bit_shift;
    ti.p_first = (int32_t)(P - 1);
    ti.p_last = (int32_t)(P - 1);
  } else {
    int64_t e0 = t * kDecodeTile;
    int64_t e1 = e0 + kDecodeTile < n ? e0 + kDecodeTile : n;
    int64_t pf = owner_of(starts, P, e0);
    int64_t pl = owner_of(starts, P, e1 - 1);
    ti.bit_lo = offs[pf] + (e0 - starts[pf]) * (int64_t)bits[pf] + bit_shift;
    ti.p_first = (int32_t)pf;
    ti.p_last = (int32_t)pl;
  }
  tiles[t] = ti;
}

// Column structure check (contiguous cover of [0, n), widths <= 64, offsets == prefix of
// len*bits, bit ranges inside total_bits).  out[0] = 1 on any violation; out[1] = 1 when the
// partitions are not all of one length (the last may be shorter).
__global__ void validate_kernel(const int32_t* __restrict__ starts, const int32_t* __restrict__ ends,
                                const int32_t* __restrict__ types, const int32_t* __restrict__ bits,
                                const int64_t* __restrict__ offs, int64_t P, int64_t n, int64_t total_bits,
                                int* __restrict__ out) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  int64_t s = starts[p], e = ends[p];
  int b = bits[p], ty = types[p];
  bool ok = (s < e) && (b >= 0) && (b <= 64) && (ty >= 0) && (ty <= MODEL_DIRECT_COPY);
  ok = ok && (p == 0 ? s == 0 : (int64_t)ends[p - 1] == s);
  ok = ok && (p == P - 1 ? e == n : true);
  ok = ok && offs[p] >= 0 && offs[p] + (e - s) * (int64_t)b <= total_bits;
  if (p + 1 < P) ok = ok && (offs[p + 1] == offs[p] + (e - s) * (int64_t)b);
  if (!ok) atomicExch(out, 1);
  const int64_t L = (int64_t)ends[0] - starts[0];
  const bool fixed = (p < P - 1) ? (e - s == L) : (e - s <= L);
  if (!fixed) atomicExch(out + 1, 1);
}

cudaError_t launch_desc_and_tiles(glc_column* c, cudaStream_t s) {
  if (c->P > 0) {
    const int64_t shift = 32 * (int64_t)c->word_shift;
    build_desc_kernel<<<(unsigned)((c->P + 255) / 256), 256, 0, s>>>(c->d_start, c->d_types, c->d_params, c->d_bits,
                                                                       c->d_offs, c->P, shift, c->d_desc);
    build_tiles_kernel<<<(unsigned)((c->ntiles + 1 + 255) / 256), 256, 0, s>>>(
        c->d_start, c->d_bits, c->d_offs, c->P, c->n, c->ntiles, c->total_bits, shift, c->d_tiles);
  }
  return cudaGetLastError();
}

cudaError_t launch_validate(const glc_column* c, int* d_bad, cudaStream_t s) {
  if (c->P <= 0) return cudaSuccess;
  validate_kernel<<<(unsigned)((c->P + 255) / 256), 256, 0, s>>>(c->d_start, c->d_end, c->d_types, c->d_bits, c->d_offs,
                                                                   c->P, c->n, c->total_bits, d_bad);
  return cudaGetLastError();
}

// max over partitions of delta_bits (for deserialized columns).
__global__ void max_bits_kernel(const int32_t* __restrict__ bits, int64_t P, unsigned long long* out) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  int b = bits[p];
  atomicMax(out, (unsigned long long)(b < 0 ? 0 : (b > 64 ? 64 : b)));
}

cudaError_t launch_max_bits(const glc_column* c, int64_t* d_out, cudaStream_t s) {
  if (c->P <= 0) return cudaSuccess;
  max_bits_kernel<<<(unsigned)((c->P + 255) / 256), 256, 0, s>>>(c->d_bits, c->P, (unsigned long long*)d_out);
  return cudaGetLastError();
}

}  // namespace glc
