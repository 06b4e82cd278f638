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
#include "glc_internal.h"
#include "glc_scan.cuh"

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

// Partition owning chunk c: the last p with base[p] <= c.
__device__ __forceinline__ int64_t chunk_owner(const int64_t* __restrict__ base, int64_t P, int64_t c) {
  int64_t lo = 0, hi = P - 1;
  while (lo < hi) {
    int64_t mid = (lo + hi + 1) >> 1;
    if (base[mid] <= c) lo = mid; else hi = mid - 1;
  }
  return lo;
}

struct FitChunkArgs {
  const int32_t* starts;
  const int32_t* ends;
  const int64_t* chunk_base;
  const int64_t* num_chunks;  // device scalar: total chunks
  int64_t P;
  i128* sy;
  i128* sxy;
  int* ovf;
};

template <typename T> __global__ void __launch_bounds__(kFitThreads)
fit_sums_kernel(const T* __restrict__ v, FitChunkArgs a) {
  const int64_t c = blockIdx.x;
  if (c >= *a.num_chunks) return;
  const int64_t p = chunk_owner(a.chunk_base, a.P, c);
  const int64_t k = c - a.chunk_base[p];
  const int64_t start = a.starts[p];
  const int64_t len = (int64_t)a.ends[p] - start;
  const int64_t i0 = k * kFitChunk;
  const int64_t i1 = (i0 + kFitChunk < len) ? i0 + kFitChunk : len;
  i128 sy = 0, sxy = 0;
  int ovf = 0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += kFitThreads) {
    T x = __ldg(v + start + i);
    ovf |= overflows_double<T>(x) ? 1 : 0;
    i128 y = (i128)x;
    sy += y;
    sxy += (i128)i * y;
  }
  sy = warp_sum_i128(sy);
  sxy = warp_sum_i128(sxy);
  ovf = __any_sync(FULL_MASK, ovf);
  __shared__ i128 s_sy[kFitThreads / 32], s_sxy[kFitThreads / 32];
  __shared__ int s_ovf[kFitThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { s_sy[warp] = sy; s_sxy[warp] = sxy; s_ovf[warp] = ovf; }
  __syncthreads();
  if (threadIdx.x == 0) {
    i128 ty = 0, txy = 0;
    int to = 0;
    for (int w = 0; w < kFitThreads / 32; w++) { ty += s_sy[w]; txy += s_sxy[w]; to |= s_ovf[w]; }
    a.sy[c] = ty;
    a.sxy[c] = txy;
    a.ovf[c] = to;
  }
}

template <typename T> __global__ void fit_solve_kernel(FitChunkArgs a, const int64_t* __restrict__ nch,
                                                      int32_t* __restrict__ types, double* __restrict__ params,
                                                      int64_t* __restrict__ err) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.P) return;
  const int64_t len = (int64_t)a.ends[p] - a.starts[p];
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

template <typename T> __global__ void __launch_bounds__(kFitThreads)
fit_maxerr_kernel(const T* __restrict__ v, FitChunkArgs a, const int32_t* __restrict__ types,
                  const double* __restrict__ params, long long* __restrict__ err) {
  const int64_t c = blockIdx.x;
  if (c >= *a.num_chunks) return;
  const int64_t p = chunk_owner(a.chunk_base, a.P, c);
  if (types[p] == MODEL_DIRECT_COPY) return;
  const int64_t k = c - a.chunk_base[p];
  const int64_t start = a.starts[p];
  const int64_t len = (int64_t)a.ends[p] - start;
  const int64_t i0 = k * kFitChunk;
  const int64_t i1 = (i0 + kFitChunk < len) ? i0 + kFitChunk : len;
  const double t0 = params[4 * p], t1 = params[4 * p + 1];
  long long m = 0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += kFitThreads) {
    long long d = abs_ref(calc_delta<T>(__ldg(v + start + i), predict<T>(t0, t1, i)));
    m = d > m ? d : m;
  }
  m = warp_max_ll(m);
  __shared__ long long s_m[kFitThreads / 32];
  if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < kFitThreads / 32; w++) t = s_m[w] > t ? s_m[w] : t;
    if (t > 0) atomicMax(err + p, t);
  }
}

// bits and len*bits; stats[1] = max bits.
template <typename T> __global__ void fit_bits_kernel(const int32_t* __restrict__ starts, const int32_t* __restrict__ ends,
                                                     const int32_t* __restrict__ types, const int64_t* __restrict__ err,
                                                     int32_t* __restrict__ bits, int64_t* __restrict__ widths, int64_t P,
                                                     unsigned long long* __restrict__ max_bits) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  int b = (types[p] == MODEL_DIRECT_COPY) ? (int)sizeof(T) * 8 : bits_for(err[p]);
  bits[p] = b;
  widths[p] = ((int64_t)ends[p] - starts[p]) * b;
  atomicMax(max_bits, (unsigned long long)b);
}

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

size_t fit_scratch_bytes(const int32_t*, int64_t n, int64_t P) {
  int64_t ncmax = n / kFitChunk + P + 1;
  size_t b = 0;
  b += align_up(sizeof(int64_t) * (P + 1), 256) * 2;                  // nch, chunk_base
  b += align_up(sizeof(int64_t) * (scan_num_tiles(P) + 1), 256);      // scan tiles
  b += align_up(sizeof(int64_t) * 2, 256);                            // num chunks
  b += align_up(sizeof(i128) * ncmax, 256) * 2;                       // sy, sxy
  b += align_up(sizeof(int) * ncmax, 256);                            // ovf
  b += align_up(sizeof(int64_t) * (P + 1), 256);                      // widths
  return b;
}

template <typename T>
static cudaError_t fit_typed(const T* v, glc_column* c, void* scratch, int64_t* d_stats, cudaStream_t s) {
  const int64_t P = c->P, n = c->n;
  const int64_t ncmax = n / kFitChunk + P + 1;
  char* sp = (char*)scratch;
  auto take = [&](size_t bytes) { void* r = sp; sp += align_up(bytes, 256); return r; };
  int64_t* nch = (int64_t*)take(sizeof(int64_t) * (P + 1));
  int64_t* base = (int64_t*)take(sizeof(int64_t) * (P + 1));
  int64_t* tiles = (int64_t*)take(sizeof(int64_t) * (scan_num_tiles(P) + 1));
  int64_t* nchunks = (int64_t*)take(sizeof(int64_t) * 2);
  i128* sy = (i128*)take(sizeof(i128) * ncmax);
  i128* sxy = (i128*)take(sizeof(i128) * ncmax);
  int* ovf = (int*)take(sizeof(int) * ncmax);
  int64_t* widths = (int64_t*)take(sizeof(int64_t) * (P + 1));
  const unsigned pg = (unsigned)((P + 255) / 256);

  chunk_count_kernel<<<pg, 256, 0, s>>>(c->d_start, c->d_end, P, nch);
  cudaError_t e = exclusive_scan<int64_t>(nch, base, P, nchunks, tiles, s);
  if (e != cudaSuccess) return e;
  FitChunkArgs a{c->d_start, c->d_end, base, nchunks, P, sy, sxy, ovf};
  fit_sums_kernel<T><<<(unsigned)ncmax, kFitThreads, 0, s>>>(v, a);
  fit_solve_kernel<T><<<pg, 256, 0, s>>>(a, nch, c->d_types, c->d_params, c->d_err);
  fit_maxerr_kernel<T><<<(unsigned)ncmax, kFitThreads, 0, s>>>(v, a, c->d_types, c->d_params, (long long*)c->d_err);
  if ((e = cudaMemsetAsync(d_stats, 0, 2 * sizeof(int64_t), s)) != cudaSuccess) return e;
  fit_bits_kernel<T><<<pg, 256, 0, s>>>(c->d_start, c->d_end, c->d_types, c->d_err, c->d_bits, widths, P,
                                         (unsigned long long*)(d_stats + 1));
  // bit offsets = exclusive scan of len*bits; stats[0] = total bits
  e = exclusive_scan<int64_t>(widths, c->d_offs, P, d_stats, tiles, s);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t launch_fit(glc_dtype dt, const void* values, glc_column* c, void* scratch, size_t, int64_t* d_stats,
                       cudaStream_t s) {
  switch (dt) {
    case GLC_I32: return fit_typed<int32_t>((const int32_t*)values, c, scratch, d_stats, s);
    case GLC_I64: return fit_typed<int64_t>((const int64_t*)values, c, scratch, d_stats, s);
    case GLC_U64: return fit_typed<uint64_t>((const uint64_t*)values, c, scratch, d_stats, s);
    case GLC_U32: return fit_typed<uint32_t>((const uint32_t*)values, c, scratch, d_stats, s);
  }
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------------------
// Derived tables: 32-byte partition descriptors and the decode tile table.
// ---------------------------------------------------------------------------------------
__global__ void build_desc_kernel(const int32_t* __restrict__ starts, const int32_t* __restrict__ types,
                                  const double* __restrict__ params, const int32_t* __restrict__ bits,
                                  const int64_t* __restrict__ offs, int64_t P, PartDesc* __restrict__ desc) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  PartDesc d;
  d.theta0 = params[4 * p];
  d.theta1 = params[4 * p + 1];
  d.bit_off = offs[p];
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
                                   int64_t total_bits, TileInfo* __restrict__ tiles) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t > ntiles) return;
  TileInfo ti;
  if (t == ntiles) {
    ti.bit_lo = total_bits;
    ti.p_first = (int32_t)(P - 1);
    ti.p_last = (int32_t)(P - 1);
  } else {
    int64_t e0 = t * kDecodeTile;
    int64_t e1 = e0 + kDecodeTile < n ? e0 + kDecodeTile : n;
    int64_t pf = owner_of(starts, P, e0);
    int64_t pl = owner_of(starts, P, e1 - 1);
    ti.bit_lo = offs[pf] + (e0 - starts[pf]) * (int64_t)bits[pf];
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
    build_desc_kernel<<<(unsigned)((c->P + 255) / 256), 256, 0, s>>>(c->d_start, c->d_types, c->d_params, c->d_bits,
                                                                       c->d_offs, c->P, c->d_desc);
    build_tiles_kernel<<<(unsigned)((c->ntiles + 1 + 255) / 256), 256, 0, s>>>(c->d_start, c->d_bits, c->d_offs, c->P,
                                                                                 c->n, c->ntiles, c->total_bits, c->d_tiles);
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
