// Probe 2: measure the four bilinear weights directly with one-hot parity textures.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <random>
#include <cuda_runtime.h>
#define CK(x) do { cudaError_t e = (x); if (e != cudaSuccess) { fprintf(stderr, "CUDA %s at %s:%d\n", cudaGetErrorString(e), __FILE__, __LINE__); exit(1);} } while (0)
__global__ void sample1(cudaTextureObject_t t, const float2* xy, float* out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = tex2D<float>(t, xy[i].x, xy[i].y);
}
static cudaTextureObject_t mk(void* dptr, int w, int h, size_t pitch) {
  cudaResourceDesc rd; memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypePitch2D; rd.res.pitch2D.devPtr = dptr;
  rd.res.pitch2D.desc = cudaCreateChannelDesc<float>();
  rd.res.pitch2D.width = w; rd.res.pitch2D.height = h; rd.res.pitch2D.pitchInBytes = pitch;
  cudaTextureDesc td; memset(&td, 0, sizeof(td));
  td.addressMode[0] = cudaAddressModeMirror; td.addressMode[1] = cudaAddressModeMirror;
  td.filterMode = cudaFilterModeLinear; td.readMode = cudaReadModeElementType; td.normalizedCoords = 1;
  cudaTextureObject_t t; CK(cudaCreateTextureObject(&t, &rd, &td, nullptr)); return t;
}
int main(int argc, char** argv) {
  FILE* f = fopen(argc > 1 ? argv[1] : "texprobe_weights.bin", "wb");
  const int W = 53, H = 50, S = 64;
  std::mt19937 rng(77); std::uniform_real_distribution<float> U(0.f, 1.f);
  int n = 200000;
  std::vector<float2> xy(n);
  for (int i = 0; i < n; ++i) {
    if (i < 66049) { int ia = i % 257, ib = i / 257;  // grid of sub-texel positions between texels 20/21 and 17/18
      float tx = 20.0f + ia / 256.0f + 1.0f / 1024.0f * ((i * 7) % 3 - 1) * 0.0f;
      float ty = 17.0f + ib / 256.0f;
      xy[i] = make_float2((tx + 0.5f) / W, (ty + 0.5f) / H);
    } else { xy[i] = make_float2(U(rng) * 0.9f + 0.05f, U(rng) * 0.9f + 0.05f); }
  }
  float2* dxy; CK(cudaMalloc(&dxy, n * sizeof(float2)));
  CK(cudaMemcpy(dxy, xy.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
  float* dout; CK(cudaMalloc(&dout, n * sizeof(float)));
  float* dtex; CK(cudaMalloc(&dtex, S * H * sizeof(float)));
  std::vector<float> out(n), tex(S * H);
  fwrite(&n, 4, 1, f); fwrite(xy.data(), 8, n, f);
  // 4 parity one-hot textures + 3 random textures
  for (int k = 0; k < 7; ++k) {
    for (int y = 0; y < H; ++y) for (int x = 0; x < S; ++x) {
      float v;
      if (k < 4) v = (((x & 1) | ((y & 1) << 1)) == k) ? 1.f : 0.f;
      else if (k == 4) v = U(rng);
      else if (k == 5) v = U(rng) * 2.f - 0.5f;
      else v = (float)((int)(U(rng) * 256)) / 256.0f;
      tex[y * S + x] = v;
    }
    CK(cudaMemcpy(dtex, tex.data(), S * H * 4, cudaMemcpyHostToDevice));
    cudaTextureObject_t t = mk(dtex, W, H, S * 4);
    sample1<<<(n + 255) / 256, 256>>>(t, dxy, dout, n);
    CK(cudaGetLastError()); CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(out.data(), dout, n * 4, cudaMemcpyDeviceToHost));
    fwrite(tex.data(), 4, S * H, f); fwrite(out.data(), 4, n, f);
    CK(cudaDestroyTextureObject(t));
  }
  fclose(f); printf("done\n"); return 0;
}
