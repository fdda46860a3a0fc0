#pragma once

#include <cuda_runtime.h>

namespace inlm {

// stack holds slices z_base.. of the volume (a z-slab; 0 = the whole volume).
cudaError_t launch_noise_patchstd(const float* stack, long long pitch_y, long long pitch_z, int nx,
                                  long long nslice, const long long* samples, long long n,
                                  int patchsize, float* out, cudaStream_t st, int z_base = 0);
// windows[w] = inclusive sample range; scratch_off[w] = byte offset of the
// window's assignment array inside scratch.
// mean_window: average samples per window; from kEmWideWindow on, each window
// gets a 1024-thread CTA (else 256).
constexpr long long kEmWideWindow = 32768;
cudaError_t launch_noise_em(const float* values, const int2* windows, int n_windows,
                            const long long* scratch_off, signed char* scratch, float* out_mean,
                            float* out_sd, cudaStream_t st, long long mean_window = 0);
// Allocation-free EM (static device scratch): limits of the file-scope arrays.
constexpr long long kNoAllocAssignBytes = 16ll << 20;  // sum of window lengths, samples
constexpr int kNoAllocMaxWindows = 16384;
constexpr int kNoAllocMaxDevices = 64;
// windows_host: 2 values (first, last inclusive) per window, host memory.
cudaError_t launch_noise_em_noalloc(int device, const float* values, const long long* windows_host,
                                    int n_windows, float* out_mean, float* out_sd,
                                    cudaStream_t st);
cudaError_t launch_noise_finalize(float* mean, float* sd, int nz, int zadaptive, float shift,
                                  float* sigma, cudaStream_t st);

}  // namespace inlm
