// Texture-unit probe: samples pitch-2D float/float2 textures (normalized coords,
// mirror addressing, linear and point filtering) at many coordinates and dumps
// (coords, results) so the CPU emulation can be fitted/verified.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <cmath>
#include <random>
#include <cuda_runtime.h>

#define CK(x) do { cudaError_t e = (x); if (e != cudaSuccess) { fprintf(stderr, "CUDA %s at %s:%d\n", cudaGetErrorString(e), __FILE__, __LINE__); exit(1);} } while (0)

__global__ void sample1(cudaTextureObject_t t, const float2* xy, float* out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = tex2D<float>(t, xy[i].x, xy[i].y);
}
__global__ void sample2(cudaTextureObject_t t, const float2* xy, float2* out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = tex2D<float2>(t, xy[i].x, xy[i].y);
}

static int alignUp(int n) { return (n + 31) / 32 * 32; }

static cudaTextureObject_t mk(void* dptr, int w, int h, size_t pitchBytes, bool f2, bool linear) {
  cudaResourceDesc rd; memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypePitch2D;
  rd.res.pitch2D.devPtr = dptr;
  rd.res.pitch2D.desc = f2 ? cudaCreateChannelDesc<float2>() : cudaCreateChannelDesc<float>();
  rd.res.pitch2D.width = w; rd.res.pitch2D.height = h; rd.res.pitch2D.pitchInBytes = pitchBytes;
  cudaTextureDesc td; memset(&td, 0, sizeof(td));
  td.addressMode[0] = cudaAddressModeMirror; td.addressMode[1] = cudaAddressModeMirror;
  td.filterMode = linear ? cudaFilterModeLinear : cudaFilterModePoint;
  td.readMode = cudaReadModeElementType; td.normalizedCoords = 1;
  cudaTextureObject_t t; CK(cudaCreateTextureObject(&t, &rd, &td, nullptr));
  return t;
}

struct Case { const char* name; int w, h; bool f2, linear; std::vector<float> tex; std::vector<float2> xy; };

static void run(Case& c, FILE* f) {
  int s = alignUp(c.w); int comps = c.f2 ? 2 : 1;
  size_t bytes = (size_t)s * c.h * comps * sizeof(float);
  void* d; CK(cudaMalloc(&d, bytes)); CK(cudaMemset(d, 0, bytes));
  // tex vector holds w*h*comps tightly; copy with pitch
  CK(cudaMemcpy2D(d, s * comps * sizeof(float), c.tex.data(), c.w * comps * sizeof(float), c.w * comps * sizeof(float), c.h, cudaMemcpyHostToDevice));
  cudaTextureObject_t t = mk(d, c.w, c.h, s * comps * sizeof(float), c.f2, c.linear);
  int n = (int)c.xy.size();
  float2* dxy; CK(cudaMalloc(&dxy, n * sizeof(float2)));
  CK(cudaMemcpy(dxy, c.xy.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
  void* dout; CK(cudaMalloc(&dout, (size_t)n * comps * sizeof(float)));
  if (c.f2) sample2<<<(n + 255) / 256, 256>>>(t, dxy, (float2*)dout, n);
  else sample1<<<(n + 255) / 256, 256>>>(t, dxy, (float*)dout, n);
  CK(cudaGetLastError()); CK(cudaDeviceSynchronize());
  std::vector<float> out((size_t)n * comps);
  CK(cudaMemcpy(out.data(), dout, out.size() * sizeof(float), cudaMemcpyDeviceToHost));
  // record: name(32) w h f2 linear n ; tex ; xy ; out
  char nm[32] = {0}; strncpy(nm, c.name, 31);
  fwrite(nm, 1, 32, f);
  int hdr[5] = {c.w, c.h, (int)c.f2, (int)c.linear, n};
  fwrite(hdr, sizeof(int), 5, f);
  fwrite(c.tex.data(), sizeof(float), c.tex.size(), f);
  fwrite(c.xy.data(), sizeof(float2), c.xy.size(), f);
  fwrite(out.data(), sizeof(float), out.size(), f);
  CK(cudaDestroyTextureObject(t)); CK(cudaFree(d)); CK(cudaFree(dxy)); CK(cudaFree(dout));
  printf("case %s w=%d h=%d f2=%d lin=%d n=%d ok\n", c.name, c.w, c.h, (int)c.f2, (int)c.linear, n);
}

int main(int argc, char** argv) {
  const char* path = argc > 1 ? argv[1] : "texprobe.bin";
  FILE* f = fopen(path, "wb"); if (!f) { perror("open"); return 1; }
  std::mt19937 rng(1234);
  std::uniform_real_distribution<float> U01(0.f, 1.f);
  std::vector<Case> cases;
  // 1) step in x: columns >= k0 are 1, else 0. Fine sweep around k0.
  for (int lin = 0; lin < 2; ++lin) {
    Case c; c.name = lin ? "stepx_lin" : "stepx_pt"; c.w = 53; c.h = 50; c.f2 = false; c.linear = lin;
    int k0 = 20;
    c.tex.resize(c.w * c.h);
    for (int y = 0; y < c.h; ++y) for (int x = 0; x < c.w; ++x) c.tex[y * c.w + x] = x >= k0 ? 1.f : 0.f;
    for (int i = -16384; i <= 16384; ++i) {
      float ft = (float)(k0 - 0.5) + (float)i / 8192.0f;  // texel-space coordinate of sample centre
      float xn = (ft + 0.5f) / (float)c.w;
      c.xy.push_back(make_float2(xn, (10.5f) / (float)c.h));
    }
    cases.push_back(c);
  }
  // 2) step in y
  for (int lin = 0; lin < 2; ++lin) {
    Case c; c.name = lin ? "stepy_lin" : "stepy_pt"; c.w = 53; c.h = 50; c.f2 = false; c.linear = lin;
    int k0 = 17;
    c.tex.resize(c.w * c.h);
    for (int y = 0; y < c.h; ++y) for (int x = 0; x < c.w; ++x) c.tex[y * c.w + x] = y >= k0 ? 1.f : 0.f;
    for (int i = -16384; i <= 16384; ++i) {
      float ft = (float)(k0 - 0.5) + (float)i / 8192.0f;
      float yn = (ft + 0.5f) / (float)c.h;
      c.xy.push_back(make_float2(20.5f / (float)c.w, yn));
    }
    cases.push_back(c);
  }
  // 3) random texture, random coords in [-2.5, 3.5] normalized (mirror behaviour), several sizes
  int sizes[3][2] = {{53, 50}, {13, 7}, {106, 100}};
  for (int si = 0; si < 3; ++si) for (int lin = 0; lin < 2; ++lin) for (int f2 = 0; f2 < 2; ++f2) {
    Case c; c.name = "rand"; c.w = sizes[si][0]; c.h = sizes[si][1]; c.f2 = f2; c.linear = lin;
    int comps = f2 ? 2 : 1;
    c.tex.resize((size_t)c.w * c.h * comps);
    for (auto& v : c.tex) v = U01(rng) * 2.f - 0.5f;
    int n = 100000;
    std::uniform_real_distribution<float> Uc(-2.5f, 3.5f);
    for (int i = 0; i < n; ++i) {
      float xn, yn;
      if (i % 4 == 0) { xn = Uc(rng); yn = Uc(rng); }
      else { xn = U01(rng) * 1.2f - 0.1f; yn = U01(rng) * 1.2f - 0.1f; }
      c.xy.push_back(make_float2(xn, yn));
    }
    cases.push_back(c);
  }
  // 4) structured coordinates as used by a downscale / gaussian / upscale / tensor pass
  int lv[6][2] = {{848, 800}, {424, 400}, {212, 200}, {106, 100}, {53, 50}, {640, 480}};
  for (int li = 0; li < 6; ++li) for (int lin = 0; lin < 2; ++lin) {
    int W = lv[li][0], H = lv[li][1];
    Case c; c.name = "struct"; c.w = W; c.h = H; c.f2 = false; c.linear = lin;
    c.tex.resize((size_t)W * H);
    for (auto& v : c.tex) v = U01(rng);
    // downscale-style (coarse grid W/2,H/2 sampling a fine texture W,H)
    int nw = W / 2, nh = H / 2;
    float dx = 1.0f / (float)nw, dy = 1.0f / (float)nh;
    int st1 = nh * nw * 5 / 40000 + 1;
    for (int iy = 0; iy < nh; iy += st1) for (int ix = 0; ix < nw; ++ix) {
      float x = ((float)ix + 0.5f) * dx, y = ((float)iy + 0.5f) * dy;
      c.xy.push_back(make_float2(x - dx * 0.25f, y));
      c.xy.push_back(make_float2(x + dx * 0.25f, y));
      c.xy.push_back(make_float2(x, y - dy * 0.25f));
      c.xy.push_back(make_float2(x, y + dy * 0.25f));
      c.xy.push_back(make_float2(x, y));
    }
    // same-grid stencil (gaussian / tensor style)
    float ex = 1.0f / (float)W, ey = 1.0f / (float)H;
    int st2 = H * W * 5 / 40000 + 1;
    for (int iy = 0; iy < H; iy += st2) for (int ix = 0; ix < W; ++ix) {
      float x = ((float)ix + 0.5f) * ex, y = ((float)iy + 0.5f) * ey;
      c.xy.push_back(make_float2(x, y));
      c.xy.push_back(make_float2(x + 1.0f * ex, y + 1.0f * ey));
      c.xy.push_back(make_float2(x - 1.0f * ex, y - 1.0f * ey));
      c.xy.push_back(make_float2(x + 1.0f * ex, y));
      c.xy.push_back(make_float2(x, y + 1.0f * ey));
    }
    // upscale style: fine grid 2W,2H sampling this texture
    int uw = 2 * W, uh = 2 * H;
    int st3 = uh * uw / 40000 + 1;
    for (int iy = 0; iy < uh; iy += st3) for (int ix = 0; ix < uw; ++ix) {
      float x = ((float)ix + 0.5f) / (float)uw, y = ((float)iy + 0.5f) / (float)uh;
      c.xy.push_back(make_float2(x, y));
    }
    cases.push_back(c);
  }
  for (auto& c : cases) run(c, f);
  fclose(f);
  printf("done\n");
  return 0;
}
