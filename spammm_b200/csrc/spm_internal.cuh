// spm_internal.cuh -- shared host-side plumbing of libspmb200.so: argument
// checks, thread-local error text, launch-error translation.
#pragma once
#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include "spm_b200.h"

namespace spm {

// Records a printf-style message as this thread's last error and returns code.
int set_error(int code, const char* fmt, ...);
// Clears this thread's last error.
void clear_error();

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Translates the pending launch error (if any) into SPM_ERR_CUDA.
inline int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(SPM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return SPM_OK;
}

// n*m overflow-safe product for element counts.
inline bool mul_ok(long long a, long long b, long long* out) {
    if (a < 0 || b < 0) return false;
    if (a != 0 && b > (long long)INT64_MAX / a) return false;
    *out = a * b;
    return true;
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace spm

#define SPM_REQUIRE(cond, ...)                                   \
    do {                                                         \
        if (!(cond)) return spm::set_error(SPM_ERR_ARG, __VA_ARGS__); \
    } while (0)
