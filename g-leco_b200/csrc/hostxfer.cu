// hostxfer.cu -- copies between host memory and device memory for the calls that take host
// buffers (GLC_HOST_IN / GLC_HOST_OUT, and so every LeCoGPU<T> method of the drop-in header,
// whose std::vector arguments are ordinary pageable memory).
//
// Pinned host memory goes straight to the DMA engine.  A pageable buffer is copied by the driver
// through its own staging at 11 GB/s (host to device) and 21 GB/s (device to host) on this
// machine, against 55-57 GB/s from pinned memory; so pageable transfers of at least kStageMin
// bytes go through two pinned chunks of the context instead: host threads fill one chunk (upload)
// or empty it (download) while the DMA engine moves the other.  Eight threads copy pageable to
// pinned memory at ~72 GB/s, which keeps the DMA engine busy.
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "glc_internal.h"

namespace glc {
namespace {

constexpr size_t kStageChunk = 32u << 20;  // bytes per pinned chunk (two per context)
constexpr size_t kStageMin = 4u << 20;     // smaller pageable transfers go to the driver directly

// memcpy split over the calling thread and a few helper threads.
class CopyPool {
 public:
  explicit CopyPool(int helpers) {
    for (int i = 0; i < helpers; i++) th_.emplace_back([this, i] { run(i + 1); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  void copy(void* dst, const void* src, size_t bytes) {
    const int parts = (int)th_.size() + 1;
    if (bytes < ((size_t)1 << 20) || parts == 1) {
      std::memcpy(dst, src, bytes);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      dst_ = (uint8_t*)dst;
      src_ = (const uint8_t*)src;
      bytes_ = bytes;
      pending_ = parts - 1;
      gen_++;
    }
    cv_.notify_all();
    part(0);
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [&] { return pending_ == 0; });
  }

 private:
  void part(int i) {
    const int parts = (int)th_.size() + 1;
    const size_t step = ((bytes_ / parts) + 63) & ~(size_t)63;
    const size_t lo = std::min(bytes_, step * i), hi = (i == parts - 1) ? bytes_ : std::min(bytes_, lo + step);
    if (hi > lo) std::memcpy(dst_ + lo, src_ + lo, hi - lo);
  }
  void run(int i) {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      part(i);
      std::lock_guard<std::mutex> lk(mu_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  uint64_t gen_ = 0;
  int pending_ = 0;
  bool stop_ = false;
  uint8_t* dst_ = nullptr;
  const uint8_t* src_ = nullptr;
  size_t bytes_ = 0;
};

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // clear the error of an unknown pointer
    return false;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}

}  // namespace

struct HostStager {
  std::mutex mu;  // one staged transfer at a time per context
  uint8_t* pin[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool used[2] = {false, false};
  CopyPool* pool = nullptr;
};

static cudaError_t stager_get(glc_ctx* ctx, HostStager** out) {
  std::lock_guard<std::mutex> lk(ctx->stage_mu);
  if (!ctx->stager) {
    HostStager* st = new (std::nothrow) HostStager();
    if (!st) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && e == cudaSuccess; i++) {
      e = cudaHostAlloc((void**)&st->pin[i], kStageChunk, cudaHostAllocDefault);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st->ev[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
      for (int i = 0; i < 2; i++) {
        if (st->pin[i]) cudaFreeHost(st->pin[i]);
        if (st->ev[i]) cudaEventDestroy(st->ev[i]);
      }
      delete st;
      return e;
    }
    const unsigned hw = std::thread::hardware_concurrency();
    const int helpers = (int)std::min(7u, hw > 2 ? hw / 2 - 1 : 0u);
    st->pool = new CopyPool(helpers);
    ctx->stager = st;
  }
  *out = ctx->stager;
  return cudaSuccess;
}

void stager_free(glc_ctx* ctx) {
  HostStager* st = ctx->stager;
  if (!st) return;
  for (int i = 0; i < 2; i++) {
    if (st->used[i]) cudaEventSynchronize(st->ev[i]);
    cudaEventDestroy(st->ev[i]);
    cudaFreeHost(st->pin[i]);
  }
  delete st->pool;
  delete st;
  ctx->stager = nullptr;
}

cudaError_t host_upload(glc_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return cudaSuccess;
  if (bytes < kStageMin || is_pinned(src)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  HostStager* st = nullptr;
  cudaError_t e = stager_get(ctx, &st);
  if (e != cudaSuccess) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  std::lock_guard<std::mutex> lk(st->mu);
  for (size_t off = 0, k = 0; off < bytes && e == cudaSuccess; off += kStageChunk, k++) {
    const int b = (int)(k & 1);
    const size_t len = std::min(kStageChunk, bytes - off);
    if (st->used[b] && (e = cudaEventSynchronize(st->ev[b])) != cudaSuccess) break;  // its last DMA is done
    st->pool->copy(st->pin[b], (const uint8_t*)src + off, len);
    e = cudaMemcpyAsync((uint8_t*)dst + off, st->pin[b], len, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(st->ev[b], s);
    st->used[b] = e == cudaSuccess;
  }
  return e;
}

cudaError_t host_download(glc_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return cudaSuccess;
  if (bytes < kStageMin || is_pinned(dst)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
  HostStager* st = nullptr;
  cudaError_t e = stager_get(ctx, &st);
  if (e != cudaSuccess) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
  std::lock_guard<std::mutex> lk(st->mu);
  for (int b = 0; b < 2; b++)  // an upload's DMA may still read a chunk
    if (st->used[b] && (e = cudaEventSynchronize(st->ev[b])) != cudaSuccess) return e;
  const size_t nchunks = (bytes + kStageChunk - 1) / kStageChunk;
  // chunk k lands in pin[k % 2]; while it is in flight the host empties chunk k - 1
  for (size_t k = 0; k <= nchunks && e == cudaSuccess; k++) {
    if (k < nchunks) {
      const size_t off = k * kStageChunk, len = std::min(kStageChunk, bytes - off);
      e = cudaMemcpyAsync(st->pin[k & 1], (const uint8_t*)src + off, len, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaEventRecord(st->ev[k & 1], s);
      st->used[k & 1] = e == cudaSuccess;
    }
    if (k > 0 && e == cudaSuccess) {
      const size_t j = k - 1, off = j * kStageChunk, len = std::min(kStageChunk, bytes - off);
      if ((e = cudaEventSynchronize(st->ev[j & 1])) == cudaSuccess)
        st->pool->copy((uint8_t*)dst + off, st->pin[j & 1], len);
    }
  }
  return e;
}

}  // namespace glc
