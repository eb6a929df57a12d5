// Headless colour-map export: the reference's fragment shader (src/shaders.h:57-123) restated as
// a CUDA kernel for an orthographic top-down view, writing an RGBA8 image instead of a GL
// framebuffer (the reference's OpenGL viewer, src/vis.cpp, has no headless path).
//
// Per cell (image row 0 = the northern edge, like a map):
//   * terrain == no_data: transparent black (the shader's Valid < 0.9999 branch);
//   * water deeper than 1 cm: MATLAB "jet" of min(1, value / vmax), where value is the depth
//     (mode 0), the speed sqrt(ux^2 + uy^2) with ux = qx / max(0.01, (h + h_east) / 2) and
//     uy = qy / max(0.01, (h + h_north) / 2) (mode 1), or the maximum depth (mode 2);
//   * otherwise the shaded terrain: normal = normalize(h_W - h_E, 2, h_S - h_N), light from
//     normalize(1, -5, 1), ambient 0.15 + 0.55 diffuse + 0.3 specular^4 with the eye straight
//     above (view direction (0, 1, 0) in the shader's y-up frame), white base colour.
// Neighbour reads clamp at the domain edge like the reference's GL_CLAMP_TO_EDGE textures.
// Colour channels are clamped to [0, 1] and rounded to 8 bits.
#include <cuda_runtime.h>
#include <stdint.h>

#include "render.h"

namespace fip {

namespace {

__device__ __forceinline__ float jet_red(float x) { return x < 0.7f ? 4.0f * x - 1.5f : -4.0f * x + 4.5f; }
__device__ __forceinline__ float jet_green(float x) { return x < 0.5f ? 4.0f * x - 0.5f : -4.0f * x + 3.5f; }
__device__ __forceinline__ float jet_blue(float x) { return x < 0.3f ? 4.0f * x + 0.5f : -4.0f * x + 2.5f; }
__device__ __forceinline__ float clamp01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }
__device__ __forceinline__ unsigned char to8(float v) { return (unsigned char)__float2int_rn(clamp01(v) * 255.0f); }

__global__ void render_kernel(const float* __restrict__ h, const float* __restrict__ qx, const float* __restrict__ qy,
                              const float* __restrict__ sohle, int W, int H, int pitch, float no_value, int mode,
                              float vmax, uchar4* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (c >= W || r >= H) return;
  const size_t o = (size_t)r * pitch + c;
  const int cw = c > 0 ? c - 1 : 0, ce = c < W - 1 ? c + 1 : W - 1;
  const int rs = r > 0 ? r - 1 : 0, rn = r < H - 1 ? r + 1 : H - 1;
  uchar4 px;
  const float s = sohle[o];
  const float ah = h[o];
  if (s == no_value) {
    px = make_uchar4(0, 0, 0, 0);
  } else if (ah > 0.01f) {
    float v = ah;
    if (mode == FIP_RENDER_VELOCITY) {
      const float ah_east = h[(size_t)r * pitch + ce];
      const float ah_north = h[(size_t)rn * pitch + c];
      const float ux = qx[o] / fmaxf(0.01f, (ah + ah_east) * 0.5f);
      const float uy = qy[o] / fmaxf(0.01f, (ah + ah_north) * 0.5f);
      v = sqrtf(ux * ux + uy * uy);
    }
    const float x = fminf(1.0f, v / vmax);
    px = make_uchar4(to8(jet_red(x)), to8(jet_green(x)), to8(jet_blue(x)), 255);
  } else {
    const float hL = sohle[(size_t)r * pitch + cw], hR = sohle[(size_t)r * pitch + ce];
    const float hD = sohle[(size_t)rs * pitch + c], hU = sohle[(size_t)rn * pitch + c];
    float nx = hL - hR, ny = 2.0f, nz = hD - hU;
    const float nl = rsqrtf(nx * nx + ny * ny + nz * nz);
    nx *= nl;
    ny *= nl;
    nz *= nl;
    const float ll = rsqrtf(1.0f + 25.0f + 1.0f);
    const float lx = 1.0f * ll, ly = -5.0f * ll, lz = 1.0f * ll;
    // reflect(I, N) = I - 2 dot(N, I) N; specular uses its y component (eye straight above)
    const float d = nx * lx + ny * ly + nz * lz;
    const float ry = ly - 2.0f * d * ny;
    const float diffuse = fmaxf(0.0f, -d);
    const float sp = fmaxf(0.0f, ry);
    const float specular = (sp * sp) * (sp * sp);
    const float g = 0.15f + 0.55f * diffuse + 0.3f * specular;
    const unsigned char b = to8(g);
    px = make_uchar4(b, b, b, 255);
  }
  out[(size_t)(H - 1 - r) * W + c] = px;
}

}  // namespace

cudaError_t launch_render(const float* h, const float* qx, const float* qy, const float* sohle, int W, int H, int pitch,
                          float no_value, int mode, float vmax, unsigned char* rgba, cudaStream_t stream) {
  dim3 grid((W + 255) / 256, H);
  render_kernel<<<grid, 256, 0, stream>>>(h, qx, qy, sohle, W, H, pitch, no_value, mode, vmax,
                                          reinterpret_cast<uchar4*>(rgba));
  return cudaGetLastError();
}

}  // namespace fip
