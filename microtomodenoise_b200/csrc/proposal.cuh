// Learned search-offset proposal: network layout, kernels and launchers.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace inlm {

constexpr int kNetC = 16;  // channels of every hidden layer

// Flat parameter vector: conv weights [27 taps][Cin][Cout] (tap = (dz+1)*9 +
// (dy+1)*3 + (dx+1)), biases [Cout], head weights [S][16], head bias [S].
struct NetLayout {
    int S = 0;
    long long w1 = 0, b1 = 0, w2 = 0, b2 = 0, w3 = 0, b3 = 0, w4 = 0, b4 = 0, wh = 0, bh = 0;
    long long total = 0;
};
NetLayout net_layout(int S);

struct Dim3i {
    int x, y, z;
};

// Level sizes: 0 = voxels, 1..3 after each stride-2 layer (level 3 = 8^3 tiles).
void net_levels(int nx, int ny, int nz, Dim3i lv[4]);

// Network input: a volume with a reflective halo of at least one voxel, and a
// per-slice scale (1/(sigma sqrt(beta)) of the slice's filter multiplier).
struct NetIn {
    const void* base;  // element (0,0,0) inside the padded buffer
    bool half;         // __half elements (else float)
    long long py, pz;  // pitches in elements
    int nx, ny, nz;
    const float* scale;
};

struct NetActs {
    float* a1;  // level 1 x 16
    float* a2;  // level 2 x 16
    float* a3;  // level 3 x 16
    float* a4;  // level 3 x 16 (tile features)
};

// Tensor-core switch of the forward pass: layers 2-4 as tcgen05 implicit
// GEMMs (proposal_tc.cu) instead of the CUDA-core kernels; err (nullable)
// receives DEV_TMA_TIMEOUT if a bounded wait of those kernels runs out.
struct NetTc {
    bool on = false;
    int* err = nullptr;
};
cudaError_t net_forward(const NetLayout& L, const __nv_bfloat16* wb, const float* wf, const NetIn& in,
                        const NetActs& act, cudaStream_t st, const NetTc& tc = NetTc());
// One 3^3 conv layer (16 -> 16, stride 1 or 2, bias, ReLU) on the tensor cores.
cudaError_t net_conv_fwd_tc(const float* in, Dim3i li, float* out, Dim3i lo, int stride,
                            const __nv_bfloat16* W, const float* b, int* err, cudaStream_t st);
cudaError_t net_logits(const NetLayout& L, const __nv_bfloat16* wb, const float* wf, const float* a4,
                       int n_tiles, float* logits, cudaStream_t st);

// Backward of the loss sum_tiles inv_n * sum_k t_k (log Z - l_k) (soft-target
// cross entropy, targets normalised per tile); accumulates into grad.
// g_logit (n_tiles x S) and d1..d4 (level-sized x 16) are scratch.
struct NetGradScratch {
    float* g_logit;
    float* d1;
    float* d2;
    float* d3;
    float* d4;
};
cudaError_t net_backward(const NetLayout& L, const __nv_bfloat16* wb, const float* wf, const NetIn& in,
                         const NetActs& act, const float* target, float inv_n,
                         const NetGradScratch& s, float* grad, double* loss, cudaStream_t st,
                         const NetTc& tc = NetTc());
// Input gradient of one 3^3 conv layer on the tensor cores: din = [ain > 0] *
// the transposed conv of G (level lo) with W, over level li.
cudaError_t net_conv_dgrad_tc(const float* G, Dim3i lo, const __nv_bfloat16* W, const float* ain, Dim3i li,
                              float* din, int stride, int* err, cudaStream_t st);

cudaError_t net_adam(float* w, float* m, float* v, const float* g, __nv_bfloat16* wb, long long n,
                     float lr, float beta1, float beta2, float eps, float bc1, float bc2,
                     cudaStream_t st);
cudaError_t net_round_bf16(const float* w, __nv_bfloat16* wb, long long n, cudaStream_t st);

// Per tile: top-K offsets by logit, predicted kept mass, fallback to every
// offset when it is below min_mass. bitmap: n_tiles x nwords (bit k%32 of
// word k/32 = offset k kept); counters[0] += fallback tiles.
cudaError_t net_select(const NetLayout& L, const __nv_bfloat16* wb, const float* wf, const float* a4,
                       int n_tiles, int K, float min_mass, unsigned* bitmap, int nwords,
                       float* pred_mass, int* counters, cudaStream_t st);

// Per 8^3 tile: its kept offsets in ascending order at plan_off[tile * S],
// their number in plan_count[tile]; counters[1] += entries written.
// Selection per group of G 8^3 tiles along x (t8: the 8^3 tile grid); bitmap
// and pred_mass have one entry per group, groups ordered (z, y, x).
cudaError_t net_select_group(const NetLayout& L, const __nv_bfloat16* wb, const float* wf, const float* a4,
                             Dim3i t8, int G, int K, float min_mass, unsigned* bitmap, int nwords,
                             float* pred_mass, int* counters, cudaStream_t st);
// rel > 0: lists whose pred_mass is below rel x its mean take every offset
// (mass_sum: one double of device scratch).
cudaError_t net_plan_tiles(const unsigned* bitmap, int nwords, long long n_tiles, int S,
                           int* plan_off, int* plan_count, int* counters, cudaStream_t st,
                           const float* pred_mass = nullptr, double* mass_sum = nullptr, float rel = 0.f);

// Per-slice input scale from the filter multiplier m = -1/(sigma^2 beta).
cudaError_t net_scale_from_mult(const float* mult, int nz, float* scale, cudaStream_t st);
// Unpadded FP32 copy of the interior of a padded FP16 volume.
cudaError_t unpad_half_to_float(const void* padded, long long py, long long pz, int px, int pyy,
                                int pz0, int nx, int ny, int nz, float* out, cudaStream_t st);
// Per-tile normalisation of weight-mass maps (rows of S sum to 1, or stay 0).
cudaError_t normalise_rows(float* map, long long rows, int S, cudaStream_t st);

}  // namespace inlm
