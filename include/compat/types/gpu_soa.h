// Base of the GPU struct-of-arrays types (src/types/gpu_soa.h:21-35): a
// subclass lists its buffers in fields(); allocate(n) and zero() follow.
#pragma once
#include <vector>

#include "../cuda/cuda_buffer.h"

struct GpuSoA {
  int count = 0;
  virtual std::vector<CudaBuffer<float>*> fields() = 0;
  virtual void allocate(int n) {
    for (auto* f : fields()) f->allocate(n);
    count = n;
  }
  void zero() {
    for (auto* f : fields()) f->zero();
  }
  virtual ~GpuSoA() = default;
};
