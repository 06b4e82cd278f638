// random_access.cu -- one lookup per thread slot, branch-free field extraction.
//
// Replaces decompressOptimizedKernel (decompression/RandomAccessKernels.cuh:55-169, binary search
// over start/end for every query), randomAccessPreUnpackedKernel (:338-448),
// randomAccessFixedPartitionKernel (decompression/FixedPartitionKernels.cuh:50-130) and
// randomAccessFixedPreUnpackedKernel (:134-222).
//
// Per lookup: the position, one 32-byte partition descriptor (theta0, theta1, bit offset,
// start, bits|type -- a single DRAM sector instead of the reference's four arrays), and the
// words that hold the field (or the 8-byte pre-unpacked residual).  Partition lookup is
// pos / L for fixed partitions; for variable partitions a sample of every k-th start lives in
// shared memory, a binary search there narrows the range to k partitions, and a short search
// over the (L2-resident) start array finishes it.  Each thread carries several independent
// lookups through the load stages so their DRAM latencies overlap.
// Positions outside [0, n) yield 0, as the reference's variable-partition kernels do; the
// fixed variants use the same rule here instead of reading past the metadata.
// Cache hints: positions are read and values written exactly once, so they go through L2 as
// streaming (evict-first) accesses and leave L2 to the partition descriptors and hot fields.
#include <cstdlib>
#include "glc_internal.h"

namespace glc {

constexpr int kRAThreads = 256;
constexpr int kRASample = 4096;

struct RAArgs {
  const PartDesc* desc;
  const int32_t* starts;
  const uint32_t* words;
  const int64_t* plain;
  int64_t P, n;
  const int32_t* pos;
  int64_t q;
  void* out;
  int32_t fixed_len;
  int32_t fixed_shift;   // >= 0 when fixed_len is a power of two
  int32_t sample_stride;
  int32_t nsample;
};

// The words holding a field come from one aligned 16-byte load (one sector, one request); a
// second load is needed only when the field continues past that granule.  The word array is
// 16-byte aligned and padded, so the granule never leaves the allocation.
__device__ __forceinline__ uint64_t read_field_global(const uint32_t* __restrict__ w, int64_t pos, int bits) {
  const int64_t wi = pos >> 5;
  const int sh = (int)(pos & 31);
  const int k = (int)(wi & 3);
  const uint4 g = __ldg(reinterpret_cast<const uint4*>(w + (wi - k)));
  const uint32_t a = k == 0 ? g.x : k == 1 ? g.y : k == 2 ? g.z : g.w;
  const int need = (sh + bits + 31) >> 5;  // words the field touches: 1..3
  uint32_t b = k == 0 ? g.y : k == 1 ? g.z : g.w;
  if (k == 3 && need > 1) b = __ldg(w + wi + 1);
  uint64_t f = (((uint64_t)b << 32) | a) >> sh;
  if (need > 2) f |= (uint64_t)__ldg(w + wi + 2) << (64 - sh);
  return low_bits(f, bits);
}

__device__ __forceinline__ PartDesc load_desc(const PartDesc* __restrict__ d) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(d));
  const longlong2 b = __ldg(reinterpret_cast<const longlong2*>(d) + 1);
  PartDesc r;
  r.theta0 = a.x;
  r.theta1 = a.y;
  r.bit_off = b.x;
  r.start = (int32_t)(b.y & 0xffffffffll);
  r.bits_type = (int32_t)(b.y >> 32);
  return r;
}

// MODE 0: fixed, power-of-two length; 1: fixed, any length; 2: variable.
// QPT lookups per thread are carried through the load stages together; MINB is the residency
// the register budget is sized for.
template <typename T, bool PLAIN, int MODE, int kRAQueries, int MINB>
__global__ void __launch_bounds__(kRAThreads, MINB) random_access_kernel(RAArgs a) {
  __shared__ int32_t s_sample[MODE == 2 ? kRASample : 1];  // fixed modes leave L1 to descriptors
  if (MODE == 2) {
    for (int k = threadIdx.x; k < a.nsample; k += kRAThreads) s_sample[k] = a.starts[(int64_t)k * a.sample_stride];
    __syncthreads();
  }
  T* out = reinterpret_cast<T*>(a.out);
  const int64_t chunk = (int64_t)kRAThreads * kRAQueries;
  const int64_t stride = (int64_t)gridDim.x * chunk;
  // The positions of the next chunk are loaded while this chunk's lookups are in flight, so the
  // streaming read of the positions overlaps the random reads instead of preceding them.
  int32_t next_pos[kRAQueries];
#pragma unroll
  for (int k = 0; k < kRAQueries; k++) {
    const int64_t qn = (int64_t)blockIdx.x * chunk + (int64_t)k * kRAThreads + threadIdx.x;
    next_pos[k] = (qn < a.q) ? __ldcs(a.pos + qn) : -1;
  }
  const int32_t last_p = (int32_t)(a.P - 1);
  for (int64_t base = (int64_t)blockIdx.x * chunk; base < a.q; base += stride) {
    // 32-bit positions and partition numbers (positions are int32 by the API), one bit of
    // `valid` per lookup: fewer registers per lookup, more lookups resident per SM.
    int32_t pos[kRAQueries], p[kRAQueries];
    uint32_t valid = 0;
#pragma unroll
    for (int k = 0; k < kRAQueries; k++) {
      const int64_t qi = base + (int64_t)k * kRAThreads + threadIdx.x;
      pos[k] = next_pos[k];
      if (qi < a.q && pos[k] >= 0 && pos[k] < a.n) valid |= 1u << k; else pos[k] = 0;
    }
#pragma unroll
    for (int k = 0; k < kRAQueries; k++) {
      const int64_t qn = base + stride + (int64_t)k * kRAThreads + threadIdx.x;
      next_pos[k] = (qn < a.q) ? __ldcs(a.pos + qn) : -1;
    }
    long long r[kRAQueries];
    if (PLAIN) {  // the residual depends on the position only: issue it before the descriptor
#pragma unroll
      for (int k = 0; k < kRAQueries; k++) r[k] = __ldg(a.plain + pos[k]);
    }
#pragma unroll
    for (int k = 0; k < kRAQueries; k++) {
      if (MODE == 0) {
        p[k] = pos[k] >> a.fixed_shift;
        p[k] = p[k] < last_p ? p[k] : last_p;
      } else if (MODE == 1) {
        p[k] = pos[k] / a.fixed_len;
        p[k] = p[k] < last_p ? p[k] : last_p;
      } else {
        int lo = 0, hi = a.nsample - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (s_sample[mid] <= pos[k]) lo = mid; else hi = mid - 1;
        }
        int32_t plo = lo * a.sample_stride;
        int32_t phi = plo + a.sample_stride - 1;
        if (phi > last_p) phi = last_p;
        while (plo < phi) {
          const int32_t mid = (plo + phi + 1) >> 1;
          if (__ldg(a.starts + mid) <= pos[k]) plo = mid; else phi = mid - 1;
        }
        p[k] = plo;
      }
    }
    double2 th[kRAQueries];  // theta0, theta1
    int2 sb[kRAQueries];     // start, bits | type << 8
    if (PLAIN) {  // the bit offset is not needed: read the 24 bytes that are
#pragma unroll
      for (int k = 0; k < kRAQueries; k++) {
        th[k] = __ldg(reinterpret_cast<const double2*>(a.desc + p[k]));
        sb[k] = __ldg(reinterpret_cast<const int2*>(a.desc + p[k]) + 3);
      }
    } else {
#pragma unroll
      for (int k = 0; k < kRAQueries; k++) {
        const PartDesc d = load_desc(a.desc + p[k]);
        th[k] = make_double2(d.theta0, d.theta1);
        sb[k] = make_int2(d.start, d.bits_type);
        const int bits = d.bits_type & 0xff;
        const int64_t local = pos[k] - d.start;
        const uint64_t f = bits > 0 ? read_field_global(a.words, d.bit_off + local * bits, bits) : 0ull;
        r[k] = ((d.bits_type >> 8) == MODEL_DIRECT_COPY) ? (long long)f : sign_extend(f, bits);
      }
    }
#pragma unroll
    for (int k = 0; k < kRAQueries; k++) {
      const int64_t qi = base + (int64_t)k * kRAThreads + threadIdx.x;
      if (qi >= a.q) continue;
      T v;
      if ((sb[k].y >> 8) == MODEL_DIRECT_COPY) v = (T)r[k];
      else v = apply_delta<T>(predict<T>(th[k].x, th[k].y, (int64_t)(pos[k] - sb[k].x)), r[k]);
      __stcs(out + qi, ((valid >> k) & 1u) ? v : (T)0);
    }
  }
}

template <typename T, bool PLAIN, int QPT, int MINB>
static cudaError_t ra_shape(glc_ctx* ctx, const RAArgs& a, int mode, cudaStream_t s) {
  void (*k)(RAArgs) = mode == 0 ? random_access_kernel<T, PLAIN, 0, QPT, MINB>
                    : mode == 1 ? random_access_kernel<T, PLAIN, 1, QPT, MINB>
                                : random_access_kernel<T, PLAIN, 2, QPT, MINB>;
  int per_sm = 0;
  cudaError_t e;
  if (mode != 2) {  // no shared memory in the fixed modes: prefer the largest L1 for descriptors
    static PerDeviceFlag carveout_set;  // per instantiation and device
    const int dev = current_device();
    if (!carveout_set.test(dev)) {
      cudaFuncSetAttribute(random_access_kernel<T, PLAIN, 0, QPT, MINB>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
      cudaFuncSetAttribute(random_access_kernel<T, PLAIN, 1, QPT, MINB>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
      carveout_set.set(dev);
    }
  }
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kRAThreads, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  const int64_t chunk = (int64_t)kRAThreads * QPT;
  int64_t grid = (a.q + chunk - 1) / chunk;
  const int64_t cap = (int64_t)per_sm * ctx->num_sms;
  if (grid > cap) grid = cap;
  if (grid < 1) grid = 1;
  k<<<(unsigned)grid, kRAThreads, 0, s>>>(a);
  return cudaGetLastError();
}

// Launch shapes (lookups per thread, CTAs per SM): 0 = (4, 1), 1 = (4, 5), 2 = (2, 8), 3 = (8, 2),
// 4 = (2, 6).  The untuned defaults were measured on 100M lookups into a 64M int64 column: packed
// fields -> shape 4 (40 registers, more warps resident); pre-unpacked residuals (every lookup a
// DRAM sector) -> shape 3.  The context's tuning table picks per element type and field width;
// GLC_RA_SHAPE overrides it for sweeps.
template <typename T, bool PLAIN>
static cudaError_t ra_typed(glc_ctx* ctx, const RAArgs& a, int mode, int shape, cudaStream_t s) {
  switch (shape) {
    case 1: return ra_shape<T, PLAIN, 4, 5>(ctx, a, mode, s);
    case 2: return ra_shape<T, PLAIN, 2, 8>(ctx, a, mode, s);
    case 3: return ra_shape<T, PLAIN, 8, 2>(ctx, a, mode, s);
    case 4: return ra_shape<T, PLAIN, 2, 6>(ctx, a, mode, s);
    default: return ra_shape<T, PLAIN, 4, 1>(ctx, a, mode, s);
  }
}

cudaError_t launch_random_access(glc_ctx* ctx, const glc_column* c, int plain_src, const int32_t* pos, int64_t q,
                                 void* out, int32_t fixed_len, cudaStream_t s) {
  const char* v = getenv("GLC_RA_SHAPE");
  const int shape = (v && *v) ? atoi(v) : tune_entry(ctx, c->dtype, c->max_bits, plain_src).ra_shape;
  return launch_random_access_shape(ctx, c, plain_src, pos, q, out, fixed_len, shape, s);
}

cudaError_t launch_random_access_shape(glc_ctx* ctx, const glc_column* c, int plain_src, const int32_t* pos, int64_t q,
                                       void* out, int32_t fixed_len, int shape, cudaStream_t s) {
  if (q <= 0) return cudaSuccess;
  RAArgs a;
  a.desc = c->d_desc;
  a.starts = c->d_start;
  a.words = c->d_words;
  a.plain = c->d_plain;
  a.P = c->P;
  a.n = c->n;
  a.pos = pos;
  a.q = q;
  a.out = out;
  a.fixed_len = fixed_len;
  a.fixed_shift = -1;
  int mode = 2;
  if (c->P <= 0 || c->n <= 0) {
    // empty column: every position is outside
    return cudaMemsetAsync(out, 0, (size_t)q * dtype_size(c->dtype), s);
  }
  if (fixed_len > 0) {
    mode = 1;
    if ((fixed_len & (fixed_len - 1)) == 0) {
      mode = 0;
      a.fixed_shift = __builtin_ctz((unsigned)fixed_len);
    }
  }
  a.sample_stride = (int32_t)((c->P + kRASample - 1) / kRASample);
  if (a.sample_stride < 1) a.sample_stride = 1;
  a.nsample = (int32_t)((c->P + a.sample_stride - 1) / a.sample_stride);
  switch (c->dtype) {
    case GLC_I32: return plain_src ? ra_typed<int32_t, true>(ctx, a, mode, shape, s) : ra_typed<int32_t, false>(ctx, a, mode, shape, s);
    case GLC_I64: return plain_src ? ra_typed<int64_t, true>(ctx, a, mode, shape, s) : ra_typed<int64_t, false>(ctx, a, mode, shape, s);
    case GLC_U64: return plain_src ? ra_typed<uint64_t, true>(ctx, a, mode, shape, s) : ra_typed<uint64_t, false>(ctx, a, mode, shape, s);
    case GLC_U32: return plain_src ? ra_typed<uint32_t, true>(ctx, a, mode, shape, s) : ra_typed<uint32_t, false>(ctx, a, mode, shape, s);
  }
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------------------
// Lookups of many requests into many columns in one launch (the serving path).  Lookup i
// belongs to the request whose [base, base + count) holds i; the request names the column and
// where its values go (device or staging memory, byte offset).
// ---------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void lookup_one(const RAColumn& c, int64_t pos, uint8_t* out) {
  T v = (T)0;
  if (pos >= 0 && pos < c.n) {
    int64_t p;
    if (c.fixed_len > 0) {
      p = pos / c.fixed_len;
      p = p < c.P ? p : c.P - 1;
    } else {
      int64_t lo = 0, hi = c.P - 1;
      while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if ((int64_t)__ldg(c.starts + mid) <= pos) lo = mid; else hi = mid - 1;
      }
      p = lo;
    }
    const PartDesc d = load_desc(c.desc + p);
    const int bits = d.bits_type & 0xff, type = d.bits_type >> 8;
    const int64_t local = pos - d.start;
    const uint64_t f = bits > 0 ? read_field_global(c.words, d.bit_off + local * bits, bits) : 0ull;
    if (type == MODEL_DIRECT_COPY) v = (T)f;
    else v = apply_delta<T>(predict<T>(d.theta0, d.theta1, local), sign_extend(f, bits));
  }
  *reinterpret_cast<T*>(out) = v;
}

__global__ void __launch_bounds__(256)
multi_lookup_kernel(const RAColumn* __restrict__ cols, const RARequest* __restrict__ reqs, int nreq,
                    int64_t total) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = nreq - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (reqs[mid].base <= i) lo = mid; else hi = mid - 1;
    }
    const RARequest r = reqs[lo];
    const RAColumn c = cols[r.col];
    const int64_t k = i - r.base;
    const int64_t pos = __ldg(r.pos + k);
    switch (c.dtype) {
      case GLC_I32: lookup_one<int32_t>(c, pos, r.out + 4 * k); break;
      case GLC_U32: lookup_one<uint32_t>(c, pos, r.out + 4 * k); break;
      case GLC_I64: lookup_one<int64_t>(c, pos, r.out + 8 * k); break;
      default: lookup_one<uint64_t>(c, pos, r.out + 8 * k); break;
    }
  }
}

cudaError_t launch_multi_lookup(const RAColumn* cols, const RARequest* reqs, int nreq, int64_t total, int num_sms,
                                cudaStream_t s) {
  if (total <= 0) return cudaSuccess;
  int64_t grid = (total + 255) / 256;
  const int64_t cap = (int64_t)num_sms * 8;
  if (grid > cap) grid = cap;
  multi_lookup_kernel<<<(unsigned)grid, 256, 0, s>>>(cols, reqs, nreq, total);
  return cudaGetLastError();
}

}  // namespace glc
