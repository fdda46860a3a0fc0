// FP16-storage filter (fast form) declarations.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "filter_kernels.cuh"

namespace inlm {

struct FastArgs {
    int nx, ny, nz;
    int tiles_x, tiles_y;
    int px, py, pz;
    int sxr, syr, szc;
    int S;                                  // full-search offset count
    const int2* __restrict__ search_delta;  // (prev-box delta, raw shared delta) per offset
    const int* __restrict__ plan_offsets;   // per-CTA lists of search-offset indices
    const int* __restrict__ plan_start;     // CTA c uses plan_offsets[start[c] .. start[c]+count[c])
    const int* __restrict__ plan_count;
    int pbx, pby, pbz;                      // FP16 prev box extents (x in halves)
    int rbx, rby, rbz;                      // raw box extents
    const __half* __restrict__ raw_pad;     // padded FP16 raw
    long long gpitch_y, gpitch_z;           // padded pitches (elements)
    float* __restrict__ out;
    const float* __restrict__ mult;
    int* err;
    float* aux;                             // non-NULL: write 1/weight sum here (no result);
                                            // MASS launches read it
    float* map;                             // MASS: per-8^3-tile weight mass [tile][S]
    int t8x, t8y;                           // 8^3 tile grid (x, y)
    float w[kMaxTaps];
    __half2 wh[kMaxTaps];                   // the same weights in FP16, both halves
    int scale_tz;                           // column form: the tile depth of the squared
                                            // differences' scale (the tile kernel's CTA depth)
};

struct FastConfig {
    int rx, ry, rz;
    int tz;
    int tx;       // CTA width: 32 (full search) or 8 (one 8^3 tile per CTA, per-tile plans)
    bool d_half;  // squared-difference planes in FP16 (else FP32)
    size_t smem_bytes;
    bool column = false;  // the column form (filter_column.cu): tz = its CTA depth, tx = 32
};

size_t fast_smem_bytes(const FastConfig& c, const FastArgs& a);
// mass = true: the weight-mass instantiation (training targets).
cudaError_t launch_fast_kernel(const FastConfig& c, const CUtensorMap* tm_prev, const FastArgs& a,
                               int tiles_z, cudaStream_t st, bool mass = false);
// The FP16 column form (filter_column.cu), patch radius 1.
cudaError_t launch_column_fast_kernel(const FastConfig& c, const CUtensorMap* tm_prev, const FastArgs& a,
                                      int tiles_z, cudaStream_t st);
cudaError_t launch_pad_reflective_half(const float* in, int nx, int ny, int nz, void* out, int px,
                                       int py, int pz, long long pitch_y, long long pitch_z,
                                       cudaStream_t st);

}  // namespace inlm
