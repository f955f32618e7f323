// Shared definitions for the lynx_b200 CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/lynx_b200.h"

namespace lynxb {

// Largest finite-difference half-width (FD order / 2) the kernels are built for.
constexpr int kMaxRadius = 8;

// Per-thread error string, returned by lynx_last_error().
void set_error(const char* fmt, ...);

// Raises a kernel's dynamic shared-memory cap (cudaFuncAttributeMaxDynamicSharedMemorySize) to at
// least `bytes`.  The cap is one value per function and device for the whole process, and host
// threads solving different grids launch the same kernel with different sizes at once: a thread
// that lowered it would make another thread's larger launch fail.  So the cap only grows, under
// a lock.
cudaError_t raise_smem_cap(const void* func, size_t bytes);
template <typename K>
cudaError_t smem_cap(K* kern, size_t bytes) {
    return raise_smem_cap(reinterpret_cast<const void*>(kern), bytes);
}

}  // namespace lynxb

#define LYNX_CUDA_TRY(...)                                                                      \
    do {                                                                                        \
        cudaError_t _e = (__VA_ARGS__);                                                         \
        if (_e != cudaSuccess) {                                                                \
            ::lynxb::set_error("%s failed: %s (%s:%d)", #__VA_ARGS__, cudaGetErrorString(_e), __FILE__, \
                               __LINE__);                                                       \
            return _e == cudaErrorMemoryAllocation ? LYNX_ERR_OOM : LYNX_ERR_CUDA;              \
        }                                                                                       \
    } while (0)

#define LYNX_TRY(...)                  \
    do {                               \
        int _s = (__VA_ARGS__);        \
        if (_s != LYNX_OK) return _s;  \
    } while (0)

#define LYNX_CHECK_ARG(cond, msg)                                   \
    do {                                                            \
        if (!(cond)) {                                              \
            ::lynxb::set_error("bad argument: %s", msg);            \
            return LYNX_ERR_BAD_ARG;                                \
        }                                                           \
    } while (0)
