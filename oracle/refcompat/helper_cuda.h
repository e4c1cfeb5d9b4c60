// Stand-in for the CUDA Samples' helper_cuda.h, which the reference includes
// (stereotgv/stereotgv.h:9) but which is not part of the CUDA toolkit.
// TEST INFRASTRUCTURE ONLY (see vfs_ref_compat.h).
//
// checkCudaErrors(call) keeps the reference's meaning (stop on a failed CUDA call) but throws
// std::runtime_error instead of calling exit(), so the C wrapper can return an error code.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <stdexcept>
#include <string>

inline void vfs_ref_check(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        char buf[512];
        std::snprintf(buf, sizeof(buf), "%s:%d: %s failed: %s", file, line, what, cudaGetErrorString(e));
        throw std::runtime_error(buf);
    }
}

#define checkCudaErrors(val) vfs_ref_check((val), #val, __FILE__, __LINE__)
#define getLastCudaError(msg) vfs_ref_check(cudaGetLastError(), (msg), __FILE__, __LINE__)
