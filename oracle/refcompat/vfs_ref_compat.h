// Compatibility layer that lets the reference's own CUDA sources (stereotgv/*.cu of
// menandro/vfs) compile UNMODIFIED with CUDA 12.9 on Linux, for use as a test oracle.
//
// TEST INFRASTRUCTURE ONLY.  It is force-included (nvcc -include) ahead of every reference
// translation unit by oracle/Makefile.ref; nothing in the vfs_b200 library includes it.
//
// What it replaces, and why:
//  * Legacy texture references.  The reference declares file-scope
//    `texture<T, cudaTextureType2D, cudaReadModeElementType> NAME;` objects
//    (calcTensor.cu:3-4, computeDerivatives.cu:3-4, downscale.cu:4-5, upscale.cu:4-5,
//    warpImage.cu:4-7), sets addressMode / filterMode / normalized on the host, binds them with
//    cudaBindTexture2D and samples them with tex2D(NAME, x, y).  CUDA 12 removed that API.
//    Here `texture` names a plain struct that lives in managed memory (so host code can set its
//    fields and device code can read it), cudaBindTexture2D builds a texture object with the
//    same pitch-2D resource, address, filter, read and normalisation modes, and tex2D(NAME, x, y)
//    samples that object.  Legacy bindings were snapshotted at launch; a texture object stored in
//    memory is not, so a rebind first waits for the device (every kernel that may still read the
//    previous binding has finished) before it replaces the object.  Sampling therefore goes
//    through the same texture unit with the same configuration as the reference.
//  * cudaMalloc.  The reference leaves its buffers uninitialised, and masked-out pixels carry
//    whatever a buffer held (stale-value behaviour).  Every allocation is zero-filled here so
//    that runs are deterministic and comparable with implementations that start from zero.
//    Each allocation also gets a zero-filled guard zone of kVfsRefGuard bytes before and after
//    it: where the mask reaches the first image row, the masked kernels form neighbour indices
//    up to one row before the buffer start (e.g. the `up` index of row 0 in
//    thresholdingL1.cu:139-177), which on the reference's own build reads whatever memory lies
//    there.  Here such reads land in the guard and read 0.  Release with vfs_ref_cuda_free.
//  * helper_cuda.h (CUDA Samples) and OpenCV: see helper_cuda.h and opencv2/opencv.hpp beside
//    this file.  checkCudaErrors throws instead of calling exit(), so that a failure surfaces
//    as an error code at the C wrapper (oracle/ref_capi.cu) rather than ending the process.
// Kernel arithmetic is untouched: the .cu files are compiled exactly as written.
#pragma once

#include <cuda_runtime.h>
#include <texture_types.h>
#include <texture_indirect_functions.h>
#include <device_launch_parameters.h>

#include <cstdio>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

// ---------------------------------------------------------------- texture references
template <class T, int Dim, enum cudaTextureReadMode Mode>
struct vfs_ref_texture {
    // Field names of the removed `struct textureReference` that the reference sets.
    enum cudaTextureAddressMode addressMode[3];
    enum cudaTextureFilterMode filterMode;
    int normalized;
    struct cudaChannelFormatDesc channelDesc;
    cudaTextureObject_t obj;  // current binding (0 = unbound)
};

template <class T, int Dim, enum cudaTextureReadMode Mode>
__device__ __forceinline__ T tex2D(const vfs_ref_texture<T, Dim, Mode>& t, float x, float y) {
    return tex2D<T>(t.obj, x, y);
}

template <class T, int Dim, enum cudaTextureReadMode Mode>
inline cudaError_t cudaBindTexture2D(size_t* offset, vfs_ref_texture<T, Dim, Mode>& tex,
                                     const void* devPtr, size_t width, size_t height, size_t pitch) {
    if (offset) *offset = 0;
    // The previous binding may still be read by kernels in flight on any stream.
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return e;
    if (tex.obj) {
        cudaDestroyTextureObject(tex.obj);
        tex.obj = 0;
    }
    cudaResourceDesc res;
    std::memset(&res, 0, sizeof(res));
    res.resType = cudaResourceTypePitch2D;
    res.res.pitch2D.devPtr = const_cast<void*>(devPtr);
    res.res.pitch2D.desc = cudaCreateChannelDesc<T>();
    res.res.pitch2D.width = width;
    res.res.pitch2D.height = height;
    res.res.pitch2D.pitchInBytes = pitch;
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof(td));
    td.addressMode[0] = tex.addressMode[0];
    td.addressMode[1] = tex.addressMode[1];
    td.addressMode[2] = tex.addressMode[2];
    td.filterMode = tex.filterMode;
    td.readMode = Mode;
    td.normalizedCoords = tex.normalized;
    cudaTextureObject_t obj = 0;
    e = cudaCreateTextureObject(&obj, &res, &td, nullptr);
    if (e != cudaSuccess) return e;
    tex.obj = obj;
    return cudaSuccess;
}

// `texture<T, dim, mode> NAME;` at file scope becomes a managed struct of the type above.
#define texture __managed__ vfs_ref_texture

// ---------------------------------------------------------------- zero-filled allocations
constexpr size_t kVfsRefGuard = 64 * 1024;  // > one row of float4 at any supported width

inline cudaError_t vfs_ref_cuda_malloc_zero(void** p, size_t n) {
    void* base = nullptr;
    cudaError_t e = cudaMalloc(&base, n + 2 * kVfsRefGuard);
    if (e != cudaSuccess) return e;
    e = cudaMemset(base, 0, n + 2 * kVfsRefGuard);
    if (e != cudaSuccess) {
        cudaFree(base);
        return e;
    }
    *p = static_cast<char*>(base) + kVfsRefGuard;
    return cudaSuccess;
}

inline cudaError_t vfs_ref_cuda_free(void* p) {
    return p ? cudaFree(static_cast<char*>(p) - kVfsRefGuard) : cudaSuccess;
}
#define cudaMalloc(p, n) vfs_ref_cuda_malloc_zero(reinterpret_cast<void**>(p), (n))
