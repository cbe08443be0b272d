// Owning, move-only device buffer (the reference's CudaBuffer<T>,
// src/cuda/cuda_buffer.h:8-76): allocate() throws std::runtime_error when
// cudaMalloc fails, zero() is a no-op on an empty buffer.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <stdexcept>
#include <string>

#include "cuda_check.h"

template <typename T>
struct CudaBuffer {
  T* ptr = nullptr;
  size_t size = 0;

  CudaBuffer() = default;
  explicit CudaBuffer(size_t n) { allocate(n); }
  ~CudaBuffer() { free(); }
  CudaBuffer(const CudaBuffer&) = delete;
  CudaBuffer& operator=(const CudaBuffer&) = delete;
  CudaBuffer(CudaBuffer&& o) noexcept : ptr(o.ptr), size(o.size) {
    o.ptr = nullptr;
    o.size = 0;
  }
  CudaBuffer& operator=(CudaBuffer&& o) noexcept {
    if (this != &o) {
      free();
      ptr = o.ptr;
      size = o.size;
      o.ptr = nullptr;
      o.size = 0;
    }
    return *this;
  }

  void allocate(size_t n) {
    free();
    cudaError_t e = cudaMalloc(&ptr, (n ? n : 1) * sizeof(T));
    if (e != cudaSuccess) {
      ptr = nullptr;
      size = 0;
      throw std::runtime_error("[CUDA] cudaMalloc failed (" +
                               std::to_string(n * sizeof(T) / (1024 * 1024)) +
                               " MB): " + cudaGetErrorString(e));
    }
    size = n;
  }

  void free() {
    if (ptr) {
      CUDA_WARN(cudaFree(ptr));
      ptr = nullptr;
      size = 0;
    }
  }

  void zero() {
    if (ptr) CUDA_CHECK(cudaMemset(ptr, 0, size * sizeof(T)));
  }

  operator T*() { return ptr; }
  operator const T*() const { return ptr; }
};
