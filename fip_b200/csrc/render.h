// Headless colour-map export (render.cu) and PNG writing (png.cpp), internal to libfip_b200.
#pragma once
#include <cuda_runtime.h>

#include <string>

#define FIP_RENDER_DEPTH 0     // water depth, jet scale 0 .. vmax metres
#define FIP_RENDER_VELOCITY 1  // flow speed, jet scale 0 .. vmax m/s
#define FIP_RENDER_HMAX 2      // flood-plain (maximum depth) map

namespace fip {

// RGBA8 image of W x H pixels (row 0 = northern edge) into device memory `rgba`.
cudaError_t launch_render(const float* h, const float* qx, const float* qy, const float* sohle, int W, int H, int pitch,
                          float no_value, int mode, float vmax, unsigned char* rgba, cudaStream_t stream);

// 8-bit RGBA PNG (zlib-compressed). Returns an empty string or an error message.
std::string write_png_rgba(const std::string& path, const unsigned char* rgba, int W, int H);

}  // namespace fip
