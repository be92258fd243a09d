// Shared infrastructure: status plumbing, device/pinned buffers, the per-device
// library stream, launch accounting and small device reductions.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>
#include <atomic>
#include <cmath>
#include <limits>
#include "../../include/fagra_b200.h"

namespace fg {

void set_error(const std::string& text);
fg_status cuda_status(cudaError_t e, const char* what);
extern std::atomic<uint64_t> g_launches;

#define FG_CUDA(call)                                         \
  do {                                                        \
    cudaError_t e__ = (call);                                 \
    if (e__ != cudaSuccess) return ::fg::cuda_status(e__, #call); \
  } while (0)
#define FG_TRY(expr)                  \
  do {                                \
    fg_status s__ = (expr);           \
    if (s__ != FG_OK) return s__;     \
  } while (0)
// Launch bookkeeping: every kernel launch goes through FG_LAUNCH so the library
// can report how many of its kernels ran.
#define FG_LAUNCH(kernel, grid, block, smem, stream, ...)                      \
  do {                                                                         \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                \
    ::fg::g_launches.fetch_add(1, std::memory_order_relaxed);                  \
    cudaError_t e__ = cudaGetLastError();                                      \
    if (e__ != cudaSuccess) return ::fg::cuda_status(e__, #kernel);            \
  } while (0)
// Programmatic dependent launch for the kernels of a PCG iteration: the
// kernel may be scheduled while the kernel before it on the stream is still
// running (once every CTA of that one has called pdl_trigger or exited), so
// its launch latency hides behind the previous kernel's tail. Every kernel
// launched this way calls pdl_wait() before its first global memory access
// (including early-exit tests): the wait returns when the previous grid has
// completed and its writes are visible, and because each such kernel waits
// before it can complete, completion is transitive along the stream.
#define FG_LAUNCH_PDL(kernel, grid_, block_, smem_, stream_, ...)      \
  do {                                                                 \
    cudaLaunchConfig_t cfg__ = {};                                     \
    cfg__.gridDim = dim3(grid_);                                       \
    cfg__.blockDim = dim3(block_);                                     \
    cfg__.dynamicSmemBytes = (smem_);                                  \
    cfg__.stream = (stream_);                                          \
    cudaLaunchAttribute at__[1];                                       \
    at__[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;   \
    at__[0].val.programmaticStreamSerializationAllowed = 1;            \
    cfg__.attrs = at__;                                                \
    cfg__.numAttrs = 1;                                                \
    cudaError_t e__ = cudaLaunchKernelEx(&cfg__, kernel, __VA_ARGS__); \
    ::fg::g_launches.fetch_add(1, std::memory_order_relaxed);          \
    if (e__ != cudaSuccess) return ::fg::cuda_status(e__, #kernel);    \
  } while (0)

fg_status device_stream(int device, cudaStream_t* out);
fg_status select_device(int device);
int sm_count(int device);
// The library's stream-ordered memory pool on a device (keeps up to 4 GiB of
// freed memory mapped for reuse); nullptr if the device has none.
cudaMemPool_t library_pool(int device);

// Grow-only device buffer: a warm workspace never reallocates. A buffer given
// a stream with use_pool() allocates from the library pool in that stream's
// order and frees without a device synchronization (for objects whose memory
// only that stream touches, e.g. per-problem storage).
template <class T>
struct DBuf {
  T* ptr = nullptr;
  size_t n = 0, cap = 0;
  cudaStream_t pool_stream = nullptr;
  cudaMemPool_t pool = nullptr;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void use_pool(int device, cudaStream_t s) {
    if (ptr) return;  // only before the first allocation
    pool = library_pool(device);
    pool_stream = pool ? s : nullptr;
  }
  void release() {
    if (ptr) {
      if (pool_stream) cudaFreeAsync(ptr, pool_stream);
      else cudaFree(ptr);
    }
    ptr = nullptr;
  }
  fg_status resize(size_t count) {
    if (count > cap) {
      release();
      cap = 0;
      size_t want = count + count / 8 + 16;
      cudaError_t e = pool_stream ? cudaMallocFromPoolAsync(reinterpret_cast<void**>(&ptr), want * sizeof(T), pool,
                                                            pool_stream)
                                  : cudaMalloc(&ptr, want * sizeof(T));
      if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation failed");
        return FG_OUT_OF_MEMORY;
      }
      cap = want;
    }
    n = count;
    return FG_OK;
  }
  // Grow to `count` elements keeping the first `keep` (device copy on `s`).
  fg_status grow_keep(size_t count, size_t keep, cudaStream_t s) {
    if (count <= cap) {
      n = count;
      return FG_OK;
    }
    T* old = ptr;
    const size_t oldcap = cap;
    ptr = nullptr;
    cap = 0;
    fg_status st = resize(count);
    if (st != FG_OK) {
      ptr = old;
      cap = oldcap;
      return st;
    }
    if (old && keep) {
      cudaError_t e = cudaMemcpyAsync(ptr, old, keep * sizeof(T), cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return cuda_status(e, "grow_keep copy");
    }
    if (old) {
      if (pool_stream) cudaFreeAsync(old, pool_stream);
      else {
        cudaStreamSynchronize(s);
        cudaFree(old);
      }
    }
    return FG_OK;
  }
  T* get() const { return ptr; }
  size_t size() const { return n; }
  size_t bytes() const { return n * sizeof(T); }
};

// Grow-only pinned host buffer.
template <class T>
struct HBuf {
  T* ptr = nullptr;
  size_t n = 0, cap = 0;
  HBuf() = default;
  HBuf(const HBuf&) = delete;
  HBuf& operator=(const HBuf&) = delete;
  ~HBuf() { if (ptr) cudaFreeHost(ptr); }
  fg_status resize(size_t count) {
    if (count > cap) {
      T* fresh = nullptr;
      size_t want = count + count / 8 + 16;
      cudaError_t e = cudaMallocHost(&fresh, want * sizeof(T));
      if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("pinned allocation failed");
        return FG_OUT_OF_MEMORY;
      }
      if (ptr) {
        std::memcpy(fresh, ptr, n * sizeof(T));
        cudaFreeHost(ptr);
      }
      ptr = fresh;
      cap = want;
    }
    n = count;
    return FG_OK;
  }
  T* get() const { return ptr; }
  size_t size() const { return n; }
};

template <class T>
fg_status upload(DBuf<T>& d, const T* h, size_t count, cudaStream_t s) {
  FG_TRY(d.resize(count));
  if (count) FG_CUDA(cudaMemcpyAsync(d.ptr, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  return FG_OK;
}

// Event-pair timer on the library stream (used for SchurTimings).
struct EventTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  bool armed = false;
  ~EventTimer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
  void start(cudaStream_t s) {
    if (!a) { cudaEventCreate(&a); cudaEventCreate(&b); }
    cudaEventRecord(a, s);
    armed = true;
  }
  double stop(cudaStream_t s) {  // seconds; synchronizes on the end event
    if (!armed) return 0;
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    armed = false;
    return ms * 1e-3;
  }
};

inline unsigned grid_for(size_t n, unsigned block) {
  size_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 0x7fffffffu) g = 0x7fffffffu;
  return (unsigned)g;
}

// The device side of FG_LAUNCH_PDL (griddepcontrol, sm_90 and later; both are
// no-ops in a grid launched without the attribute).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

}  // namespace fg
