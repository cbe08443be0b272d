// Pinned staging ring for small host -> device uploads (HostStage).
#include <string.h>

#include "ds_internal.h"

namespace ds {

HostStage::~HostStage() { release(); }

void HostStage::release() {
  for (auto& e : ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  if (host) cudaFreeHost(host);
  host = nullptr;
  next = 0;
}

int HostStage::upload(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes > kSlotBytes) return DS_ERR_ARG;
  if (!host) {
    int st = cuda_status(cudaHostAlloc((void**)&host, kSlots * kSlotBytes, cudaHostAllocDefault));
    for (int k = 0; k < kSlots && st == DS_OK; ++k)
      st = cuda_status(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
    if (st != DS_OK) {
      release();
      return st;
    }
  }
  const int k = next;
  next = (next + 1) % kSlots;
  DS_CUDA(cudaEventSynchronize(ev[k]));  // the copy that last read slot k
  unsigned char* slot = host + (size_t)k * kSlotBytes;
  memcpy(slot, src, bytes);
  DS_CUDA(cudaMemcpyAsync(dst, slot, bytes, cudaMemcpyHostToDevice, s));
  DS_CUDA(cudaEventRecord(ev[k], s));
  return DS_OK;
}

}  // namespace ds
