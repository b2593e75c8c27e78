// Shared device/host utilities of the invDFT B200 library.
#pragma once
#include <utility>

#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

namespace invdft {

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string &m) : std::runtime_error(m) {}
};
struct StatusError : std::runtime_error {
  int status;
  StatusError(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};

#define INVDFT_CUDA(call)                                                        \
  do {                                                                           \
    cudaError_t _e = (call);                                                     \
    if (_e != cudaSuccess)                                                       \
      throw ::invdft::CudaError(std::string(#call) + ": " + cudaGetErrorString(_e) + \
                                " (" __FILE__ ":" + std::to_string(__LINE__) + ")"); \
  } while (0)

#define INVDFT_LAUNCH_CHECK() INVDFT_CUDA(cudaGetLastError())

// Bytes currently held by all DevBuf allocations of this process.
inline std::atomic<long long> &device_bytes() {
  static std::atomic<long long> b{0};
  return b;
}
inline std::atomic<long long> &device_bytes_peak() {
  static std::atomic<long long> b{0};
  return b;
}

// Owning device buffer.
template <typename T> struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) {
      cudaError_t e = cudaMalloc(&p, count * sizeof(T));
      if (e != cudaSuccess) {
        p = nullptr; n = 0;
        (void)cudaGetLastError();
        throw StatusError(4, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
      }
      const long long now = device_bytes() += (long long)(count * sizeof(T));
      long long pk = device_bytes_peak().load();
      while (now > pk && !device_bytes_peak().compare_exchange_weak(pk, now)) {
      }
    }
  }
  void ensure(size_t count) { if (count > n) alloc(count); }
  // exchange the allocations of two buffers (pointer and size)
  void swap(DevBuf &o) noexcept {
    std::swap(p, o.p);
    std::swap(n, o.n);
  }
  void release() {
    if (p) {
      cudaFree(p);
      device_bytes() -= (long long)(n * sizeof(T));
    }
    p = nullptr; n = 0;
  }
  void upload(const T *h, size_t count, cudaStream_t s = 0) {
    ensure(count);
    if (count) INVDFT_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T> &h, cudaStream_t s = 0) { upload(h.data(), h.size(), s); }
  void download(T *h, size_t count, cudaStream_t s = 0) const {
    if (count) INVDFT_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  void zero(cudaStream_t s = 0) { if (n) INVDFT_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
  T *get() const { return p; }
};

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block reduction: every thread passes its value; thread 0 gets the sum.
template <int NT> __device__ __forceinline__ double block_sum(double v, double *red) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = (threadIdx.x < NT / 32) ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
  }
  return t;
}

}  // namespace invdft
