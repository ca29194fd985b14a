// capi_util.cuh -- status codes and thread-local error text for the C ABI.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#include "slm_b200.h"

namespace slm {

void set_error(const char* fmt, ...);
void clear_error();
int num_sms();

inline bool aligned(const void* p, size_t a) { return ((uintptr_t)p % a) == 0; }

}  // namespace slm

#define SLM_REQUIRE(cond, ...)                       \
    do {                                             \
        if (!(cond)) {                               \
            ::slm::set_error(__VA_ARGS__);           \
            return SLM_ERR_ARGS;                     \
        }                                            \
    } while (0)

#define SLM_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            ::slm::set_error("%s failed: %s", #call, cudaGetErrorString(e_));       \
            return SLM_ERR_CUDA;                                                    \
        }                                                                           \
    } while (0)

#define SLM_LAUNCHED(what)                                                          \
    do {                                                                            \
        cudaError_t e_ = cudaGetLastError();                                        \
        if (e_ != cudaSuccess) {                                                    \
            ::slm::set_error("%s launch failed: %s", what, cudaGetErrorString(e_)); \
            return SLM_ERR_CUDA;                                                    \
        }                                                                           \
    } while (0)
