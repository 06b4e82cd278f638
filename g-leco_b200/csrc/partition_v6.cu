// partition_v6.cu -- the reference's GPU partitioner (compress with use_gpu_partitioning = true,
// GPUVariableLengthPartitionerV6, compression/GpuPartitioner.cuh:34-214), kept as a fast mode
// whose partition boundaries match the reference's.
//
// The reference's algorithm (compression/PartitioningKernels.cuh:647-727):
//  1. cut the column into variance blocks of 8 x base values (base = 2048 in compress,
//     api/G-LeCo.cuh:384-387);
//  2. per block, a "variance" from 128 threads: thread t Kahan-sums v and v^2 over positions
//     start + t + 128k in double, each warp reduces its 32 pairs with a shuffle-down tree, and
//     every warp adds float(S2/n - (S1/n)^2) (n = the block's length) into the block's value;
//  3. thresholds = the values of rank nb/4, nb/2 and 3nb/4 of the sorted block values;
//  4. block i gets partitions of 4 x base values when the i-th SMALLEST block value is below the
//     first threshold, 2 x base below the second, base below the third, otherwise base / 2: the
//     reference sorts the value array in place (GpuPartitioner.cuh:60-61) before the partition
//     kernel reads it by block index, so with distinct values the sizes follow block position
//     and the values only matter through ties; the last partition of a block is cut at the
//     block's (or the column's) end.
// The boundaries are all that the compressor keeps of the partitioner: compress refits every
// partition afterwards (api/G-LeCo.cuh:512-530), exactly as for the other modes.
//
// Here the same arithmetic runs with explicit IEEE operations (Kahan adds, v*v - c as one fma
// and S2/n - m*m as one fma, as the reference's compiler contracts them) so the oracle can
// restate it bit for bit; the four warp values are added in warp order (the reference adds them
// with float atomics in whatever order the warps finish).  The thresholds come from a radix
// select instead of a sort, and partitions are emitted in order from a prefix sum of per-block
// counts instead of atomics followed by a sort.  "The i-th smallest value is below threshold k"
// is "i < the number of values below threshold k", so only those three counts are needed.
#include "glc_internal.h"
#include "glc_scan.cuh"

namespace glc {
namespace {

constexpr int kV6Threads = 128;  // compression/GpuPartitioner.cuh:52

__device__ __forceinline__ double as_double(int32_t v) { return (double)v; }
__device__ __forceinline__ double as_double(uint32_t v) { return (double)v; }
__device__ __forceinline__ double as_double(int64_t v) { return __ll2double_rn(v); }
__device__ __forceinline__ double as_double(uint64_t v) { return __ull2double_rn(v); }

template <typename T>
__global__ void __launch_bounds__(kV6Threads)
v6_variance_kernel(const T* __restrict__ data, int64_t n, int64_t block_len, float* __restrict__ var) {
  const int64_t start = (int64_t)blockIdx.x * block_len;
  const int64_t end = start + block_len < n ? start + block_len : n;
  double s1 = 0.0, s2 = 0.0, c1 = 0.0, c2 = 0.0;
#pragma unroll 4
  for (int64_t i = start + threadIdx.x; i < end; i += kV6Threads) {
    const double v = as_double(__ldg(data + i));
    const double y1 = __dsub_rn(v, c1);
    const double t1 = __dadd_rn(s1, y1);
    c1 = __dsub_rn(__dsub_rn(t1, s1), y1);
    s1 = t1;
    const double y2 = __fma_rn(v, v, -c2);
    const double t2 = __dadd_rn(s2, y2);
    c2 = __dsub_rn(__dsub_rn(t2, s2), y2);
    s2 = t2;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    s1 = __dadd_rn(s1, __shfl_down_sync(FULL_MASK, s1, off));
    s2 = __dadd_rn(s2, __shfl_down_sync(FULL_MASK, s2, off));
  }
  __shared__ float warp_val[kV6Threads / 32];
  if ((threadIdx.x & 31) == 0) {
    const double dn = (double)(end - start);
    const double m = __ddiv_rn(s1, dn);
    warp_val[threadIdx.x >> 5] = __double2float_rn(__fma_rn(-m, m, __ddiv_rn(s2, dn)));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float acc = 0.f;
#pragma unroll
    for (int w = 0; w < kV6Threads / 32; w++) acc = __fadd_rn(acc, warp_val[w]);
    var[blockIdx.x] = acc;
  }
}

// Total order of floats as unsigned keys (negative values reversed below the positive ones).
__device__ __forceinline__ uint32_t float_key(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// The values of rank nb/4, nb/2, 3nb/4 (0-based, ascending): a most-significant-digit radix
// select, 8 bits per pass, one CTA.
__global__ void __launch_bounds__(1024) v6_threshold_kernel(const float* __restrict__ var, int64_t nb,
                                                            float* __restrict__ thr) {
  __shared__ unsigned int hist[256];
  __shared__ uint32_t s_prefix;
  __shared__ long long s_rank;
  for (int q = 0; q < 3; q++) {
    long long rank = q == 0 ? nb / 4 : (q == 1 ? nb / 2 : 3 * nb / 4);
    uint32_t prefix = 0, mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
      for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
      __syncthreads();
      for (int64_t i = threadIdx.x; i < nb; i += blockDim.x) {
        const uint32_t k = float_key(var[i]);
        if ((k & mask) == prefix) atomicAdd(&hist[(k >> shift) & 255u], 1u);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        long long r = rank;
        uint32_t b = 0;
        for (; b < 255u; b++) {
          if (r < (long long)hist[b]) break;
          r -= hist[b];
        }
        s_prefix = prefix | (b << shift);
        s_rank = r;
      }
      __syncthreads();
      prefix = s_prefix;
      rank = s_rank;
      mask |= 0xffu << shift;
      __syncthreads();
    }
    if (threadIdx.x == 0) thr[q] = key_float(prefix);
    __syncthreads();
  }
}

// below[k] = number of block values below threshold k (float comparison, as the reference's).
__global__ void v6_below_kernel(const float* __restrict__ var, int64_t nb, const float* __restrict__ thr,
                                unsigned long long* __restrict__ below) {
  const float t0 = thr[0], t1 = thr[1], t2 = thr[2];
  unsigned long long c0 = 0, c1 = 0, c2 = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += (int64_t)gridDim.x * blockDim.x) {
    const float x = var[i];
    c0 += x < t0;
    c1 += x < t1;
    c2 += x < t2;
  }
  if (c0) atomicAdd(below, c0);
  if (c1) atomicAdd(below + 1, c1);
  if (c2) atomicAdd(below + 2, c2);
}

// Partition size of block i: its rank among the sorted values against the three counts.
__device__ __forceinline__ int64_t v6_size(int64_t i, const unsigned long long* below, int64_t base) {
  return i < (int64_t)below[0] ? 4 * base : (i < (int64_t)below[1] ? 2 * base : (i < (int64_t)below[2] ? base : base / 2));
}

__global__ void v6_count_kernel(int64_t nb, const unsigned long long* __restrict__ below, int64_t n, int64_t base,
                                int64_t* __restrict__ counts) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const int64_t start = i * 8 * base;
  const int64_t end = start + 8 * base < n ? start + 8 * base : n;
  const int64_t size = v6_size(i, below, base);
  counts[i] = (end - start + size - 1) / size;
}

__global__ void v6_emit_kernel(int64_t nb, const unsigned long long* __restrict__ below, int64_t n, int64_t base,
                               const int64_t* __restrict__ offs, int32_t* __restrict__ starts,
                               int32_t* __restrict__ ends) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const int64_t start = i * 8 * base;
  const int64_t end = start + 8 * base < n ? start + 8 * base : n;
  const int64_t size = v6_size(i, below, base);
  int64_t o = offs[i];
  for (int64_t j = start; j < end; j += size, o++) {
    starts[o] = (int32_t)j;
    ends[o] = (int32_t)(j + size < end ? j + size : end);
  }
}

template <typename T>
cudaError_t v6_typed(glc_ctx* ctx, const T* values, int64_t n, int64_t base, int32_t** d_starts, int32_t** d_ends,
                     int64_t* P, cudaStream_t s) {
  const int64_t block_len = 8 * base;
  const int64_t nb = (n + block_len - 1) / block_len;
  float* var = nullptr;
  float* thr = nullptr;  // 3 thresholds, then (8-byte aligned) 3 counts of values below them
  int64_t* counts = nullptr;
  int64_t* scratch = nullptr;
  int64_t* total = nullptr;
  const int64_t ntiles = scan_num_tiles(nb);
  cudaError_t e;
  auto cleanup = [&]() {
    if (var) cudaFreeAsync(var, s);
    if (thr) cudaFreeAsync(thr, s);
    if (counts) cudaFreeAsync(counts, s);
    if (scratch) cudaFreeAsync(scratch, s);
    if (total) cudaFreeAsync(total, s);
  };
  if ((e = pool_alloc(ctx, &var, 4 * nb, s)) != cudaSuccess || (e = pool_alloc(ctx, &thr, 64, s)) != cudaSuccess ||
      (e = pool_alloc(ctx, &counts, 8 * nb, s)) != cudaSuccess ||
      (e = pool_alloc(ctx, &scratch, 8 * (ntiles + 1), s)) != cudaSuccess ||
      (e = pool_alloc(ctx, &total, 8, s)) != cudaSuccess) {
    cleanup();
    return e;
  }
  v6_variance_kernel<T><<<(unsigned)nb, kV6Threads, 0, s>>>(values, n, block_len, var);
  v6_threshold_kernel<<<1, 1024, 0, s>>>(var, nb, thr);
  unsigned long long* below = (unsigned long long*)(thr + 4);
  if ((e = cudaMemsetAsync(below, 0, 3 * sizeof(unsigned long long), s)) != cudaSuccess) {
    cleanup();
    return e;
  }
  const unsigned g = (unsigned)((nb + 255) / 256);
  v6_below_kernel<<<g < 64 ? g : 64, 256, 0, s>>>(var, nb, thr, below);
  v6_count_kernel<<<g, 256, 0, s>>>(nb, below, n, base, counts);
  if ((e = cudaGetLastError()) != cudaSuccess || (e = exclusive_scan<int64_t>(counts, counts, nb, total, scratch, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(ctx->h_stats, total, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess) {
    cleanup();
    return e;
  }
  *P = ctx->h_stats[0];
  if ((e = pool_alloc(ctx, d_starts, 4 * *P, s)) != cudaSuccess || (e = pool_alloc(ctx, d_ends, 4 * *P, s)) != cudaSuccess) {
    cleanup();
    return e;
  }
  v6_emit_kernel<<<g, 256, 0, s>>>(nb, below, n, base, counts, *d_starts, *d_ends);
  e = cudaGetLastError();
  cleanup();
  return e;
}

}  // namespace

cudaError_t launch_partition_v6(glc_ctx* ctx, glc_dtype dt, const void* values, int64_t n, int32_t base,
                                int32_t** d_starts, int32_t** d_ends, int64_t* P, cudaStream_t s) {
  *d_starts = *d_ends = nullptr;
  *P = 0;
  if (n <= 0) return cudaSuccess;
  switch (dt) {
    case GLC_I32: return v6_typed<int32_t>(ctx, (const int32_t*)values, n, base, d_starts, d_ends, P, s);
    case GLC_I64: return v6_typed<int64_t>(ctx, (const int64_t*)values, n, base, d_starts, d_ends, P, s);
    case GLC_U64: return v6_typed<uint64_t>(ctx, (const uint64_t*)values, n, base, d_starts, d_ends, P, s);
    case GLC_U32: return v6_typed<uint32_t>(ctx, (const uint32_t*)values, n, base, d_starts, d_ends, P, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace glc
