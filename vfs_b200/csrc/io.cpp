#include "io.hpp"

#include <zlib.h>

#include <cmath>
#include <cstdio>
#include <cstring>

namespace vfs {

static bool read_file(const std::string& path, std::vector<uint8_t>& buf, std::string& err) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  std::fseek(f, 0, SEEK_END);
  long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (n < 0) {
    std::fclose(f);
    err = "cannot size " + path;
    return false;
  }
  buf.resize((size_t)n);
  size_t got = n ? std::fread(buf.data(), 1, (size_t)n, f) : 0;
  std::fclose(f);
  if (got != (size_t)n) {
    err = "short read " + path;
    return false;
  }
  return true;
}

bool read_flo(const std::string& path, int& w, int& h, std::vector<float>& data, std::string& err) {
  std::vector<uint8_t> b;
  if (!read_file(path, b, err)) return false;
  if (b.size() < 12) {
    err = path + ": too short for a .flo header";
    return false;
  }
  float tag;
  int32_t ww, hh;
  std::memcpy(&tag, b.data(), 4);
  std::memcpy(&ww, b.data() + 4, 4);
  std::memcpy(&hh, b.data() + 8, 4);
  if (tag != 202021.25f || ww <= 0 || hh <= 0 || ww > (1 << 16) || hh > (1 << 16)) {
    err = path + ": not a .flo file";
    return false;
  }
  size_t n = (size_t)ww * hh * 2;
  if (b.size() < 12 + n * 4) {
    err = path + ": truncated .flo data";
    return false;
  }
  data.resize(n);
  std::memcpy(data.data(), b.data() + 12, n * 4);
  w = ww;
  h = hh;
  return true;
}

bool write_flo(const std::string& path, int w, int h, const float* data, std::string& err) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot create " + path;
    return false;
  }
  float tag = 202021.25f;
  int32_t ww = w, hh = h;
  bool ok = std::fwrite(&tag, 4, 1, f) == 1 && std::fwrite(&ww, 4, 1, f) == 1 && std::fwrite(&hh, 4, 1, f) == 1 &&
            std::fwrite(data, 4, (size_t)w * h * 2, f) == (size_t)w * h * 2;
  std::fclose(f);
  if (!ok) err = "short write " + path;
  return ok;
}

static uint32_t be32(const uint8_t* p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

static uint8_t to_gray(int r, int g, int b) {
  // BT.601 luma, rounded to nearest
  double y = 0.299 * r + 0.587 * g + 0.114 * b;
  int v = (int)std::floor(y + 0.5);
  return (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
}

static bool read_png_gray(const std::vector<uint8_t>& b, int& w, int& h, std::vector<uint8_t>& out,
                          std::string& err) {
  static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  if (b.size() < 8 || std::memcmp(b.data(), sig, 8)) {
    err = "not a PNG";
    return false;
  }
  size_t off = 8;
  int depth = 0, ctype = -1, interlace = 0;
  std::vector<uint8_t> idat;
  while (off + 8 <= b.size()) {
    uint32_t len = be32(&b[off]);
    const uint8_t* type = &b[off + 4];
    if (off + 12 + (size_t)len > b.size()) break;
    const uint8_t* d = &b[off + 8];
    if (!std::memcmp(type, "IHDR", 4) && len >= 13) {
      w = (int)be32(d);
      h = (int)be32(d + 4);
      depth = d[8];
      ctype = d[9];
      interlace = d[12];
    } else if (!std::memcmp(type, "IDAT", 4)) {
      idat.insert(idat.end(), d, d + len);
    } else if (!std::memcmp(type, "IEND", 4)) {
      break;
    }
    off += 12 + len;
  }
  int ch = ctype == 0 ? 1 : ctype == 2 ? 3 : ctype == 4 ? 2 : ctype == 6 ? 4 : 0;
  if (depth != 8 || ch == 0 || interlace != 0 || w <= 0 || h <= 0) {
    err = "unsupported PNG (need 8-bit gray/RGB/GA/RGBA, non-interlaced)";
    return false;
  }
  size_t rowb = (size_t)w * ch;
  std::vector<uint8_t> raw((rowb + 1) * h);
  uLongf rawlen = (uLongf)raw.size();
  if (uncompress(raw.data(), &rawlen, idat.data(), (uLong)idat.size()) != Z_OK || rawlen != raw.size()) {
    err = "PNG image data does not inflate";
    return false;
  }
  std::vector<uint8_t> img(rowb * h), prev(rowb, 0);
  for (int y = 0; y < h; y++) {
    uint8_t ft = raw[y * (rowb + 1)];
    const uint8_t* src = &raw[y * (rowb + 1) + 1];
    uint8_t* dst = &img[y * rowb];
    for (size_t x = 0; x < rowb; x++) {
      int a = x >= (size_t)ch ? dst[x - ch] : 0, up = prev[x], c = x >= (size_t)ch ? prev[x - ch] : 0;
      int v = src[x];
      switch (ft) {
        case 0: break;
        case 1: v += a; break;
        case 2: v += up; break;
        case 3: v += (a + up) / 2; break;
        case 4: {
          int p = a + up - c, pa = std::abs(p - a), pb = std::abs(p - up), pc = std::abs(p - c);
          v += (pa <= pb && pa <= pc) ? a : (pb <= pc ? up : c);
          break;
        }
        default: err = "bad PNG filter"; return false;
      }
      dst[x] = (uint8_t)v;
    }
    std::memcpy(prev.data(), dst, rowb);
  }
  out.resize((size_t)w * h);
  for (size_t i = 0; i < (size_t)w * h; i++) {
    const uint8_t* p = &img[i * ch];
    out[i] = (ch == 1 || ch == 2) ? p[0] : to_gray(p[0], p[1], p[2]);
  }
  return true;
}

static bool read_pgm(const std::vector<uint8_t>& b, int& w, int& h, std::vector<uint8_t>& out, std::string& err) {
  size_t i = 2;
  int vals[3];
  for (int k = 0; k < 3; k++) {
    while (i < b.size() && (isspace(b[i]) || b[i] == '#')) {
      if (b[i] == '#')
        while (i < b.size() && b[i] != '\n') i++;
      else
        i++;
    }
    int v = 0;
    bool any = false;
    while (i < b.size() && isdigit(b[i])) {
      v = v * 10 + (b[i++] - '0');
      any = true;
    }
    if (!any) {
      err = "bad PGM header";
      return false;
    }
    vals[k] = v;
  }
  i++;  // single whitespace
  w = vals[0];
  h = vals[1];
  if (vals[2] != 255 || w <= 0 || h <= 0 || b.size() < i + (size_t)w * h) {
    err = "unsupported PGM";
    return false;
  }
  out.assign(b.begin() + i, b.begin() + i + (size_t)w * h);
  return true;
}

bool read_gray8(const std::string& path, int& w, int& h, std::vector<uint8_t>& data, std::string& err) {
  std::vector<uint8_t> b;
  if (!read_file(path, b, err)) return false;
  bool ok;
  if (b.size() >= 2 && b[0] == 'P' && b[1] == '5') ok = read_pgm(b, w, h, data, err);
  else ok = read_png_gray(b, w, h, data, err);
  if (!ok) err = path + ": " + err;
  return ok;
}

}  // namespace vfs
