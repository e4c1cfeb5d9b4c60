// File readers used by the reference-shaped Init() entry point: Middlebury .flo
// vector fields (read by cv::readOpticalFlow in dllhook/vfs.cpp:26-27) and 8-bit
// grayscale images (PNG or binary PGM; cv::imread(..., IMREAD_GRAYSCALE) in
// dllhook/vfs.cpp:19).
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

namespace vfs {

// Reads a .flo file: float tag 202021.25, int32 width, int32 height, then
// width*height*2 float32.  Returns false with a message on failure.
bool read_flo(const std::string& path, int& w, int& h, std::vector<float>& data, std::string& err);
bool write_flo(const std::string& path, int w, int h, const float* data, std::string& err);

// Reads an 8-bit image as grayscale (PNG colour types 0, 2, 4, 6 at bit depth 8,
// non-interlaced; or binary PGM P5 with maxval 255).  Colour is converted with
// the ITU-R BT.601 weights that cv::imread uses for IMREAD_GRAYSCALE.
bool read_gray8(const std::string& path, int& w, int& h, std::vector<uint8_t>& data, std::string& err);

}  // namespace vfs
