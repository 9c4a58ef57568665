// Shared helpers for the TEMF3DT B200 library (host + device).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace temf {

struct CudaError : public std::runtime_error {
  explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};
struct ArgError : public std::runtime_error {
  explicit ArgError(const std::string& s) : std::runtime_error(s) {}
};
struct StateError : public std::runtime_error {
  explicit StateError(const std::string& s) : std::runtime_error(s) {}
};

#define TEMF_CUDA(call)                                                                   \
  do {                                                                                    \
    cudaError_t _e = (call);                                                              \
    if (_e != cudaSuccess)                                                                \
      throw ::temf::CudaError(std::string(#call) + ": " + cudaGetErrorString(_e) + " (" + \
                              __FILE__ + ":" + std::to_string(__LINE__) + ")");           \
  } while (0)

#define TEMF_CHECK_LAUNCH() TEMF_CUDA(cudaGetLastError())

// Device buffer with RAII ownership.
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    reset();
    if (count == 0) count = 1;
    TEMF_CUDA(cudaMalloc((void**)&p, count * sizeof(T)));
    n = count;
  }
  void upload(const T* h, size_t count, cudaStream_t s) {
    alloc(count);
    if (count) TEMF_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  size_t bytes() const { return n * sizeof(T); }
};

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

}  // namespace temf
