// 2D three-channel (RGB) NLM filter and the Anscombe transforms of the
// reference's colour path (Color/color_denoising.h, Color/colorspace.h,
// Denoiser/iternlm_cpu.cpp:272-400, 932-1075).
#pragma once

#include <cuda_runtime.h>

namespace inlm {

struct RgbArgs {
    const float* raw[3];   // unpadded channel planes, nx * ny
    const float* prev[3];  // previous iterate (raw at iteration 1)
    float* out[3];
    const int2* search;    // S offsets (dx, dy), reference order
    const int2* taps;      // P taps, tap 0 = centre
    const float* w;        // P setup_distweight values
    float mult[3];         // -1 / (sigma_c^2 beta) per channel
    int nx, ny, S, P;
    int hx, hy;            // staged halo of prev: search + patch radius per axis
    int sx, sy;            // staged halo of raw: search radius per axis
    int independent;       // params.color.independent_channels
    int tap_radius;        // r > 0: the unrolled kernel for patch radius (r, r) (tap order
                           // checked by the host against the table); 0: the generic kernel
};

constexpr int kRgbTX = 32, kRgbTY = 8;

size_t rgb_smem_bytes(const RgbArgs& a);
// Tap order (dx, dy pairs) of the unrolled kernel for patch radius (r, r);
// returns the tap count, or -1 when no such kernel exists.
int rgb_tap_order(int r, int* dxdy, int max_taps);
cudaError_t launch_rgb_filter(const RgbArgs& a, cudaStream_t st);
// forward (2 sqrt(v + 3/8)) or inverse ((v/2)^2 - 3/8) Anscombe transform of n
// values in place, colorspace.h:83-125
cudaError_t launch_anscombe(float* v, long long n, bool inverse, cudaStream_t st);

}  // namespace inlm
