// noalloc.cu -- range decode into host memory that allocates nothing (glc_decompress_range_noalloc).
//
// For callers that cannot allocate device memory while they run: request handlers under a fixed
// device-memory budget (every byte accounted for up front), code that must not block on the
// allocator or trigger its device-wide synchronisation, and code paths where allocation is not
// permitted.  The regular glc_decompress_range(..., GLC_HOST_OUT) takes a device staging buffer
// from the context's pool on every call; this entry point instead uses one file-scope device
// array for the decode kernel's scratch (its work-stealing tile counter and error word) and for
// the staging of the decoded values, so a call issues only a memset, the kernel, and two copies.
//
// The array is GLC_NOALLOC_MAX_OUTPUT_BYTES plus 272 bytes and lives on every GPU that loads the
// library until the process exits.  Every call shares it: overlapping calls on the GPU race
// (serialise them, e.g. on one stream).  Each call clears the counter and error word first; the
// staging area keeps the previous call's bytes, and only the bytes a call writes are read back.
#include <atomic>
#include "glc_internal.h"

namespace {

constexpr size_t kHeadBytes = 256;  // [0] work counter, [1] error word, rest unused
constexpr size_t kScratchBytes = kHeadBytes + GLC_NOALLOC_MAX_OUTPUT_BYTES + 16;
constexpr int kMaxDevices = 64;

}  // namespace

// The decode kernel's scratch and the staging of decoded values for glc_decompress_range_noalloc.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

std::atomic<unsigned char*> g_scratch_addr[kMaxDevices];
std::atomic<int> g_num_sms[kMaxDevices];

// Device address of the array on the current device.  In host code the array's name is only a
// host-side stand-in, so the address comes from cudaGetSymbolAddress, once per device, with that
// device current.  The first call on a device does this set-up.
cudaError_t scratch_for_device(int dev, unsigned char** ptr, int* num_sms) {
  unsigned char* p = g_scratch_addr[dev].load(std::memory_order_acquire);
  int sms = g_num_sms[dev].load(std::memory_order_acquire);
  if (!p || sms <= 0) {
    void* addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    p = static_cast<unsigned char*>(addr);
    g_num_sms[dev].store(sms, std::memory_order_release);
    g_scratch_addr[dev].store(p, std::memory_order_release);
  }
  *ptr = p;
  *num_sms = sms;
  return cudaSuccess;
}

}  // namespace

extern "C" glc_status glc_decompress_range_noalloc(const glc_column* col, int64_t first, int64_t count,
                                                     void* host_out, glc_stream stream) {
  if (!col) return GLC_ERR_INVALID_ARG;
  const size_t es = (size_t)glc::dtype_size(col->dtype);
  // the size limit first: then count * es cannot overflow, nor can the range test below
  if (count < 0 || (uint64_t)count > (uint64_t)GLC_NOALLOC_MAX_OUTPUT_BYTES / es) return GLC_ERR_INVALID_ARG;
  if (first < 0 || first > col->n || count > col->n - first) return GLC_ERR_INVALID_ARG;
  if (count == 0) return GLC_OK;
  if (!host_out) return GLC_ERR_INVALID_ARG;
  if (!col->d_words) return GLC_ERR_UNSUPPORTED;
  int dev = col->ctx ? col->ctx->device : 0;
  if (dev < 0 || dev >= kMaxDevices) return GLC_ERR_INVALID_ARG;
  glc::DeviceScope device_scope(dev);  // the caller's current device is given back on return
  if (!device_scope.ok()) return GLC_ERR_CUDA;
  cudaStream_t s = stream ? (cudaStream_t)stream : (col->ctx ? col->ctx->own_stream : nullptr);
  unsigned char* scratch = nullptr;
  int num_sms = 0;
  if (scratch_for_device(dev, &scratch, &num_sms) != cudaSuccess) return GLC_ERR_CUDA;
  int* counter = reinterpret_cast<int*>(scratch);
  // the counter and the error word must start at zero; the previous call left them set
  if (cudaMemsetAsync(scratch, 0, 2 * sizeof(int), s) != cudaSuccess) return GLC_ERR_CUDA;
  // value e is written at base + e with 16-byte stores, so base must be 16-byte aligned
  const size_t shift = (size_t)(first * (int64_t)es) & 15;
  unsigned char* staged = scratch + kHeadBytes + shift;
  unsigned char* base = staged - first * (int64_t)es;
  if (glc::launch_decode_scratch(col, first, first + count, base, counter, counter + 1, num_sms, s) != cudaSuccess)
    return GLC_ERR_CUDA;
  int err_word = 0;
  if (cudaMemcpyAsync(host_out, staged, (size_t)count * es, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(&err_word, counter + 1, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return GLC_ERR_CUDA;
  return err_word == glc::DEVERR_NONE ? GLC_OK : GLC_ERR_TIMEOUT;
}
