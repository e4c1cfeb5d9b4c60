// C wrapper over the reference's own StereoTgv class (stereotgv/stereotgv.h:14-124 of
// menandro/vfs), compiled from the reference's unmodified CUDA sources by oracle/Makefile.ref
// into oracle/_ref/.  Used by the GPU tests as the reference-build oracle: the vfs_b200 drop-in
// path is compared with what the reference itself computes on the same inputs.
//
// TEST INFRASTRUCTURE ONLY: nothing in the vfs_b200 library links or loads it.
//
// Every entry point returns 0 on success and -1 on failure; vref_last_error() gives the
// message (the reference's checkCudaErrors throws in this build, see refcompat/helper_cuda.h).
// Host arrays are tightly packed (row length = width), as the reference's uchar* overload of
// copyImagesToDevice expects; padding to the stride happens inside the reference's methods.
#include "stereotgv.h"

#include <cstdint>
#include <cstring>
#include <set>
#include <string>

namespace {

thread_local std::string g_err;

// The reference's constructor leaves the pointer members unset; `initialized` records whether
// initialize() has filled them, so that vref_destroy frees only real allocations.
struct Ref {
    StereoTgv s;
    bool initialized = false;
    // Set by vref_copy_mask when some pyramid level of the mask has an on pixel in its first or
    // last row or column.  The reference's masked kernels then form neighbour indices before
    // their buffers' start (thresholdingL1.cu:139-177: the `up` index of row 0 is negative);
    // in this build those reads land in the zero guard of every allocation
    // (refcompat/vfs_ref_compat.h) and read 0.
    bool mask_touches_border = false;
    int border_level = -1;
};

StereoTgv* get(void* h) { return &static_cast<Ref*>(h)->s; }

template <class F>
int guarded(F&& f) {
    try {
        f();
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            g_err = std::string("CUDA error: ") + cudaGetErrorString(e);
            return -1;
        }
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

// Copies a width x height ROI view (row step = Mat::step) into a packed host array.
void copy_roi(const cv::Mat& m, void* out) {
    const size_t row = size_t(m.cols) * m.elemSize();
    for (int y = 0; y < m.rows; ++y)
        std::memcpy(static_cast<char*>(out) + size_t(y) * row, m.ptr(y), row);
}

}  // namespace

extern "C" {

const char* vref_last_error() { return g_err.c_str(); }

void* vref_create() {
    try {
        return new Ref();
    } catch (...) {
        return nullptr;
    }
}

// Frees every device buffer the instance still points at (the reference itself never frees).
void vref_destroy(void* h) {
    if (!h) return;
    Ref* r = static_cast<Ref*>(h);
    if (!r->initialized) {
        delete r;
        return;
    }
    StereoTgv* s = &r->s;
    std::set<void*> ptrs;
    auto add = [&](void* p) { if (p) ptrs.insert(p); };
    for (auto* p : s->pI0) add(p);
    for (auto* p : s->pI1) add(p);
    for (auto* p : s->pTvForward) add(p);
    for (auto* p : s->pTvBackward) add(p);
    for (auto* p : s->pFisheyeMask) add(p);
    void* fields[] = {s->d_i0, s->d_i1, s->d_i1warp, s->d_i08uc3, s->d_i18uc3, s->d_i08u, s->d_i18u,
                      s->d_i0smooth, s->d_i1smooth, s->d_Iu, s->d_Iz, s->d_u, s->d_du, s->d_us,
                      s->d_depth, s->d_warpUV, s->d_warpUVs, s->d_dwarpUV, s->d_uvrgb,
                      s->d_fisheyeMask, s->d_a, s->d_b, s->d_c, s->d_etau, s->d_etav1, s->d_etav2,
                      s->d_p, s->d_q, s->d_u_, s->d_u_s, s->d_u_last, s->d_v, s->d_vs, s->d_v_,
                      s->d_v_s, s->d_gradv, s->d_Tp, s->d_tvForward, s->d_tvBackward, s->d_tv2,
                      s->d_cv, s->d_i1calibrated, s->d_X, s->debug_depth};
    cudaDeviceSynchronize();
    for (void* p : fields) add(p);
    for (void* p : ptrs) vfs_ref_cuda_free(p);
    delete r;
}

int vref_initialize(void* h, int w, int hgt, float beta, float gamma, float alpha0, float alpha1,
                    float tsl, float lambda, int n_levels, float f_scale, int n_warp, int n_iter) {
    Ref* r = static_cast<Ref*>(h);
    if (r->initialized) {
        g_err = "initialize called twice on one instance";
        return -1;
    }
    if (hgt > w) {
        // The tensor kernels size their x grid from the height (calcTensor.cu:81,227); with
        // height > width their threads index past the last row.
        g_err = "height > width is not supported by the reference build";
        return -1;
    }
    if ((size_t((w + 31) / 32 * 32) + 1) * 16 > kVfsRefGuard) {
        // reads before a buffer's start reach back one row of float4 at most
        g_err = "width too large for the allocation guard of the reference build";
        return -1;
    }
    StereoTgv* s = &r->s;
    s->d_fisheyeMask = nullptr;  // declared by the reference but never allocated
    r->initialized = true;
    return guarded([&] {
        s->initialize(w, hgt, beta, gamma, alpha0, alpha1, tsl, lambda, n_levels, f_scale, n_warp, n_iter);
    });
}

int vref_set_limit_range(void* h, float v) {
    get(h)->limitRange = v;
    return 0;
}

int vref_stride(void* h) { return get(h)->stride; }

// tv, cv: height x width x 2 float32 (the CV_32FC2 maps of loadVectorFields).
int vref_load_vector_fields(void* h, const float* tv, const float* cv) {
    StereoTgv* s = get(h);
    return guarded([&] {
        cv::Mat t(cv::Size(s->width, s->height), CV_32FC2, const_cast<float*>(tv));
        cv::Mat c(cv::Size(s->width, s->height), CV_32FC2, const_cast<float*>(cv));
        s->loadVectorFields(t, c);
    });
}

// mask: height x width float32 in {0, 1}.
int vref_copy_mask(void* h, const float* mask) {
    Ref* r = static_cast<Ref*>(h);
    StereoTgv* s = &r->s;
    return guarded([&] {
        cv::Mat m(cv::Size(s->width, s->height), CV_32F, const_cast<float*>(mask));
        s->copyMaskToDevice(m);
        r->mask_touches_border = false;
        r->border_level = -1;
        for (int l = 0; l < s->nLevels && !r->mask_touches_border; ++l) {
            const int w = s->pW[l], hh = s->pH[l], st = s->pS[l];
            std::vector<float> lv(size_t(st) * hh);
            checkCudaErrors(cudaMemcpy(lv.data(), s->pFisheyeMask[l], lv.size() * sizeof(float),
                                       cudaMemcpyDeviceToHost));
            for (int y = 0; y < hh; ++y)
                for (int x = 0; x < w; ++x)
                    if ((y == 0 || y == hh - 1 || x == 0 || x == w - 1) && lv[size_t(y) * st + x] != 0.0f) {
                        r->mask_touches_border = true;
                        r->border_level = l;
                    }
        }
    });
}

// 1 when the current mask reaches an image border at some pyramid level.
int vref_mask_touches_border(void* h) { return static_cast<Ref*>(h)->mask_touches_border ? 1 : 0; }

int vref_copy_images_u8(void* h, const uint8_t* i0, const uint8_t* i1) {
    StereoTgv* s = get(h);
    return guarded([&] { s->copyImagesToDevice(const_cast<uint8_t*>(i0), const_cast<uint8_t*>(i1)); });
}

// kind: 0 = CV_8U, 1 = CV_32F, 2 = CV_8UC3 (the cv::Mat overload of copyImagesToDevice).
int vref_copy_images_mat(void* h, const void* i0, const void* i1, int kind) {
    StereoTgv* s = get(h);
    const int type = kind == 0 ? CV_8U : kind == 1 ? CV_32F : CV_8UC3;
    return guarded([&] {
        cv::Mat a(cv::Size(s->width, s->height), type, const_cast<void*>(i0));
        cv::Mat b(cv::Size(s->width, s->height), type, const_cast<void*>(i1));
        s->copyImagesToDevice(a, b);
    });
}

int vref_solve(void* h, int masked) {
    Ref* r = static_cast<Ref*>(h);
    StereoTgv* s = &r->s;
    if (s->width < 2 || s->height < 2) {
        g_err = "images must be at least 2 x 2";
        return -1;
    }
    return guarded([&] {
        if (masked)
            s->solveStereoForwardMasked();
        else
            s->solveStereoForward();
    });
}

// out: height x width float32 (copy1DDisparityToHost).
int vref_copy_disparity_1d(void* h, float* out) {
    StereoTgv* s = get(h);
    return guarded([&] {
        cv::Mat m;
        s->copy1DDisparityToHost(m);
        copy_roi(m, out);
    });
}

// out: height x width x 2 float32 (copyDisparityToHost, the 2-D warp vector).
int vref_copy_disparity_2d(void* h, float* out) {
    StereoTgv* s = get(h);
    return guarded([&] {
        cv::Mat m;
        s->copyDisparityToHost(m);
        copy_roi(m, out);
    });
}

// out: height x width x 3 float32 (copyDisparityVisToHost, the flow colour map).
int vref_copy_disparity_vis(void* h, float* out, float flow_scale) {
    StereoTgv* s = get(h);
    return guarded([&] {
        cv::Mat m;
        s->copyDisparityVisToHost(m, flow_scale);
        copy_roi(m, out);
    });
}

// out: height x width float32 (copyWarpedImageToHost).
int vref_copy_warped_image(void* h, float* out) {
    StereoTgv* s = get(h);
    return guarded([&] {
        cv::Mat m;
        s->copyWarpedImageToHost(m);
        copy_roi(m, out);
    });
}

// depth: height x width float32; X: height x width x 3 float32 (copyStereoToHost).
int vref_copy_stereo(void* h, float* depth, float* X, float fx, float fy, float cx, float cy, float d1,
                     float d2, float d3, float d4, float t1, float t2, float t3) {
    StereoTgv* s = get(h);
    return guarded([&] {
        cv::Mat d, x;
        s->copyStereoToHost(d, x, fx, fy, cx, cy, d1, d2, d3, d4, t1, t2, t3);
        copy_roi(d, depth);
        copy_roi(x, X);
    });
}

// Overwrites the first width x height elements of a device plane with a packed host array of
// `comps` floats per pixel (padding columns are left as they are); "warpUV" and "u" only.
// Used to give the reference's output kernels (FlowToHSV, ConvertKB) the exact flow the
// drop-in path produced, so that those kernels are compared on identical inputs.
int vref_set_plane(void* h, const char* name, const float* in, int comps) {
    StereoTgv* s = get(h);
    const std::string n(name);
    void* p = nullptr;
    if (n == "warpUV" && comps == 2) p = s->d_warpUV;
    else if (n == "u" && comps == 1) p = s->d_u;
    if (!p) {
        g_err = "plane " + n + " cannot be set with " + std::to_string(comps) + " components";
        return -1;
    }
    return guarded([&] {
        const size_t row = size_t(s->width) * comps * sizeof(float);
        checkCudaErrors(cudaMemcpy2D(p, size_t(s->stride) * comps * sizeof(float), in, row, row, s->height,
                                     cudaMemcpyHostToDevice));
    });
}

// Raw copy of one of the instance's device planes (stride x height elements of `comps` floats),
// by member name, for intermediate comparisons.
int vref_get_plane(void* h, const char* name, float* out, int comps) {
    StereoTgv* s = get(h);
    const std::string n(name);
    const void* p = nullptr;
    if (n == "u") p = s->d_u;
    else if (n == "u_") p = s->d_u_;
    else if (n == "warpUV") p = s->d_warpUV;
    else if (n == "i1warp") p = s->d_i1warp;
    else if (n == "Iu") p = s->d_Iu;
    else if (n == "Iz") p = s->d_Iz;
    else if (n == "a") p = s->d_a;
    else if (n == "b") p = s->d_b;
    else if (n == "c") p = s->d_c;
    else if (n == "etau") p = s->d_etau;
    else if (n == "p") p = s->d_p;
    else if (n == "q") p = s->d_q;
    else if (n == "v_") p = s->d_v_;
    else if (n == "tv2") p = s->d_tv2;
    else if (n == "Tp") p = s->d_Tp;
    else if (n == "i0smooth") p = s->d_i0smooth;
    else if (n == "I0") p = s->pI0.empty() ? nullptr : s->pI0[0];
    else if (n == "I1") p = s->pI1.empty() ? nullptr : s->pI1[0];
    if (!p) {
        g_err = "unknown plane " + n;
        return -1;
    }
    return guarded([&] {
        checkCudaErrors(cudaMemcpy(out, p, size_t(s->stride) * s->height * comps * sizeof(float),
                                   cudaMemcpyDeviceToHost));
    });
}

}  // extern "C"
