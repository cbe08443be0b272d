// Error macros of the drop-in API (same behaviour as the reference's
// src/cuda/cuda_check.h: print and continue in release builds, print and exit
// when DEBUG is defined).
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

#ifdef DEBUG
#define DS_COMPAT_FAIL() exit(EXIT_FAILURE)
#else
#define DS_COMPAT_FAIL() ((void)0)
#endif

#define CUDA_WARN(err)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (err);                                                               \
    if (e_ != cudaSuccess)                                                                \
      fprintf(stderr, "[CUDA] Error at %s:%d: %s\n", __FILE__, __LINE__,                  \
              cudaGetErrorString(e_));                                                    \
  } while (0)

#define CUDA_CHECK(err)                                                                   \
  do {                                                                                    \
    cudaError_t e_ = (err);                                                               \
    if (e_ != cudaSuccess) {                                                              \
      fprintf(stderr, "[CUDA] Error at %s:%d: %s\n", __FILE__, __LINE__,                  \
              cudaGetErrorString(e_));                                                    \
      DS_COMPAT_FAIL();                                                                   \
    }                                                                                     \
  } while (0)

#ifdef DEBUG
#define CUDA_SYNC_CHECK()               \
  do {                                  \
    cudaDeviceSynchronize();            \
    CUDA_CHECK(cudaGetLastError());     \
  } while (0)
#else
#define CUDA_SYNC_CHECK() CUDA_CHECK(cudaGetLastError())
#endif

// Status of a libdiffsplat_b200 call: print like CUDA_CHECK.
#define DS_COMPAT_CHECK(st)                                                               \
  do {                                                                                    \
    int s_ = (st);                                                                        \
    if (s_ != 0) {                                                                        \
      fprintf(stderr, "[diffsplat_b200] Error at %s:%d: %s\n", __FILE__, __LINE__,        \
              ds_status_string(s_));                                                      \
      DS_COMPAT_FAIL();                                                                   \
    }                                                                                     \
  } while (0)
