// glc_scan.cuh -- device-wide exclusive prefix sum (reduce-then-scan) for any trivially
// copyable value type with operator+ (int64, 128-bit integers, pairs of them).
//
// Three launches: each 1024-thread CTA scans a tile of 4096 items and writes the tile total;
// one CTA scans the tile totals (looping with a carry, so any count works); each CTA then adds
// its tile's base.  The bit offsets of the bitstream are this scan over len * bits
// (the reference computes each offset with an O(P) loop per partition,
// compression/CompressionKernels.cuh:222-238).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "glc_device.cuh"

namespace glc {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename V> __device__ __forceinline__ V shfl_up_any(V v, int d) {
  static_assert(sizeof(V) % 4 == 0, "scan values are multiples of 4 bytes");
  int w[sizeof(V) / 4];
  memcpy(w, &v, sizeof(V));
#pragma unroll
  for (int k = 0; k < (int)(sizeof(V) / 4); k++) w[k] = __shfl_up_sync(FULL_MASK, w[k], d);
  V r;
  memcpy(&r, w, sizeof(V));
  return r;
}

// Exclusive scan of one value per thread across the CTA; returns the CTA total in *total.
template <typename V> __device__ V block_exclusive_scan(V x, V* total, V* s_warp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  V inc = x;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    V y = shfl_up_any(inc, d);
    if (lane >= d) inc = inc + y;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    V w = (lane < nwarps) ? s_warp[lane] : V();
    V winc = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      V y = shfl_up_any(winc, d);
      if (lane >= d) winc = winc + y;
    }
    if (lane < nwarps) s_warp[lane] = winc;  // inclusive warp totals
  }
  __syncthreads();
  V base = (warp > 0) ? s_warp[warp - 1] : V();
  *total = s_warp[nwarps - 1];
  V excl = shfl_up_any(inc, 1);
  if (lane == 0) excl = V();
  __syncthreads();
  return base + excl;
}

template <typename V> __global__ void __launch_bounds__(kScanThreads)
scan_tiles_kernel(const V* __restrict__ in, V* __restrict__ out, int64_t count, V* __restrict__ tile_totals) {
  __shared__ V s_warp[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  V items[kScanItems];
  V sum = V();
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    items[k] = (base + k < count) ? in[base + k] : V();
    sum = sum + items[k];
  }
  V total;
  V ex = block_exclusive_scan(sum, &total, s_warp);
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    if (base + k < count) out[base + k] = ex;
    ex = ex + items[k];
  }
  if (threadIdx.x == 0) tile_totals[blockIdx.x] = total;
}

template <typename V> __global__ void __launch_bounds__(kScanThreads)
scan_totals_kernel(V* __restrict__ totals, int64_t ntiles, V* __restrict__ grand_total) {
  __shared__ V s_warp[32];
  __shared__ V s_carry;
  if (threadIdx.x == 0) s_carry = V();
  __syncthreads();
  for (int64_t off = 0; off < ntiles; off += kScanTile) {
    const int64_t base = off + (int64_t)threadIdx.x * kScanItems;
    V items[kScanItems];
    V sum = V();
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      items[k] = (base + k < ntiles) ? totals[base + k] : V();
      sum = sum + items[k];
    }
    V total;
    V ex = block_exclusive_scan(sum, &total, s_warp);
    V carry = s_carry;
    ex = ex + carry;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      if (base + k < ntiles) totals[base + k] = ex;
      ex = ex + items[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) s_carry = carry + total;
    __syncthreads();
  }
  if (threadIdx.x == 0 && grand_total) *grand_total = s_carry;
}

template <typename V> __global__ void __launch_bounds__(kScanThreads)
scan_add_kernel(V* __restrict__ out, int64_t count, const V* __restrict__ tile_bases) {
  const V b = tile_bases[blockIdx.x];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
#pragma unroll
  for (int k = 0; k < kScanItems; k++)
    if (base + k < count) out[base + k] = out[base + k] + b;
}

inline int64_t scan_num_tiles(int64_t count) { return (count + kScanTile - 1) / kScanTile; }

// Scratch: one V per tile.  in and out may alias.  *grand_total (device) may be null.
template <typename V>
cudaError_t exclusive_scan(const V* in, V* out, int64_t count, V* grand_total, V* tile_scratch, cudaStream_t s) {
  if (count <= 0) {
    if (grand_total) return cudaMemsetAsync(grand_total, 0, sizeof(V), s);
    return cudaSuccess;
  }
  int64_t nt = scan_num_tiles(count);
  scan_tiles_kernel<V><<<(unsigned)nt, kScanThreads, 0, s>>>(in, out, count, tile_scratch);
  scan_totals_kernel<V><<<1, kScanThreads, 0, s>>>(tile_scratch, nt, grand_total);
  scan_add_kernel<V><<<(unsigned)nt, kScanThreads, 0, s>>>(out, count, tile_scratch);
  return cudaGetLastError();
}

}  // namespace glc
