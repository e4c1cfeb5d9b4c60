// Minimal stand-in for the parts of OpenCV's core API that the reference's StereoTgv host code
// uses (stereotgv/stereotgv.cu: cv::Mat headers over host buffers, ROI views, copyMakeBorder
// for row padding, split, and the imshow / waitKey debug windows).  OpenCV's C++ headers and
// libraries are not installed here, and no graphics stack exists, so imshow and waitKey do
// nothing.
// TEST INFRASTRUCTURE ONLY (see ../vfs_ref_compat.h).
//
// Semantics kept from OpenCV where the reference depends on them:
//  * a Mat is a reference-counted header: copies and ROIs share the pixels;
//  * Mat(Size, type, data) wraps caller memory without owning it;
//  * create() reallocates only when the size or type changes;
//  * copyMakeBorder(..., BORDER_CONSTANT, 0) pads with zeros on every channel.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

typedef unsigned char uchar;

#define CV_CN_SHIFT 3
#define CV_DEPTH_MAX (1 << CV_CN_SHIFT)
#define CV_MAT_DEPTH(flags) ((flags) & (CV_DEPTH_MAX - 1))
#define CV_MAT_CN(flags) ((((flags) >> CV_CN_SHIFT) & 63) + 1)
#define CV_MAKETYPE(depth, cn) (CV_MAT_DEPTH(depth) + (((cn) - 1) << CV_CN_SHIFT))
#define CV_8U 0
#define CV_32F 5
#define CV_8UC1 CV_MAKETYPE(CV_8U, 1)
#define CV_8UC3 CV_MAKETYPE(CV_8U, 3)
#define CV_32FC1 CV_MAKETYPE(CV_32F, 1)
#define CV_32FC2 CV_MAKETYPE(CV_32F, 2)
#define CV_32FC3 CV_MAKETYPE(CV_32F, 3)
#define CV_32FC4 CV_MAKETYPE(CV_32F, 4)

// Only used by lib_link.h inside MSVC `#pragma comment(lib, ...)`, which gcc ignores.
#define CV_MAJOR_VERSION 4
#define CV_MINOR_VERSION 5
#define CV_SUBMINOR_VERSION 1
#define CVAUX_STR_EXP(x) #x
#define CVAUX_STR(x) CVAUX_STR_EXP(x)

namespace cv {

enum BorderTypes { BORDER_CONSTANT = 0 };

struct Size {
    int width = 0, height = 0;
    Size() = default;
    Size(int w, int h) : width(w), height(h) {}
};

struct Rect {
    int x = 0, y = 0, width = 0, height = 0;
    Rect() = default;
    Rect(int x_, int y_, int w_, int h_) : x(x_), y(y_), width(w_), height(h_) {}
};

inline size_t depth_size(int depth) {
    switch (depth) {
        case CV_8U: return 1;
        case CV_32F: return 4;
        default: throw std::runtime_error("cv shim: unsupported depth");
    }
}

class Mat {
public:
    int rows = 0, cols = 0;
    uchar* data = nullptr;
    size_t step = 0;  // bytes per row

    Mat() = default;
    Mat(int r, int c, int type) { create(r, c, type); }
    Mat(Size sz, int type) { create(sz.height, sz.width, type); }
    Mat(Size sz, int type, void* ext) : rows(sz.height), cols(sz.width), type_(type) {
        data = static_cast<uchar*>(ext);
        step = size_t(cols) * elemSize();
    }

    void create(int r, int c, int type) {
        if (holder_ && rows == r && cols == c && type_ == type) return;
        rows = r;
        cols = c;
        type_ = type;
        step = size_t(c) * elemSize();
        holder_ = std::make_shared<std::vector<uchar>>(step * size_t(r));
        data = holder_->data();
    }

    int type() const { return type_; }
    int depth() const { return CV_MAT_DEPTH(type_); }
    int channels() const { return CV_MAT_CN(type_); }
    size_t elemSize() const { return depth_size(depth()) * size_t(channels()); }
    bool empty() const { return data == nullptr || rows == 0 || cols == 0; }

    uchar* ptr(int r = 0) { return data + size_t(r) * step; }
    const uchar* ptr(int r = 0) const { return data + size_t(r) * step; }

    template <class T>
    T& at(int r, int c) { return *reinterpret_cast<T*>(ptr(r) + size_t(c) * elemSize()); }

    Mat operator()(const Rect& roi) const {
        Mat m(*this);
        m.rows = roi.height;
        m.cols = roi.width;
        m.data = data + size_t(roi.y) * step + size_t(roi.x) * elemSize();
        return m;
    }

private:
    int type_ = CV_8UC1;
    std::shared_ptr<std::vector<uchar>> holder_;
};

inline void copyMakeBorder(const Mat& src, Mat& dst, int top, int bottom, int left, int right,
                           int borderType, double value = 0.0) {
    if (borderType != BORDER_CONSTANT || value != 0.0)
        throw std::runtime_error("cv shim: only BORDER_CONSTANT with 0 is supported");
    Mat s = src;  // keeps src alive if dst aliases it
    const int r = s.rows + top + bottom, c = s.cols + left + right;
    dst.create(r, c, s.type());
    const size_t es = s.elemSize();
    for (int y = 0; y < r; ++y) std::memset(dst.ptr(y), 0, size_t(c) * es);
    for (int y = 0; y < s.rows; ++y)
        std::memcpy(dst.ptr(y + top) + size_t(left) * es, s.ptr(y), size_t(s.cols) * es);
}

inline void split(const Mat& src, Mat* out) {
    const int cn = src.channels();
    const size_t ds = depth_size(src.depth());
    for (int k = 0; k < cn; ++k) {
        out[k].create(src.rows, src.cols, CV_MAKETYPE(src.depth(), 1));
        for (int y = 0; y < src.rows; ++y)
            for (int x = 0; x < src.cols; ++x)
                std::memcpy(out[k].ptr(y) + size_t(x) * ds, src.ptr(y) + (size_t(x) * cn + k) * ds, ds);
    }
}

inline void imshow(const std::string&, const Mat&) {}
inline int waitKey(int = 0) { return -1; }

}  // namespace cv
