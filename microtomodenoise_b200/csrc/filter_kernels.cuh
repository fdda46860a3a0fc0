// Declarations shared by the filter kernels and the host orchestration.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

namespace inlm {

constexpr int kMaxTaps = 128;

// Tiled FP32 kernel geometry: a CTA owns TX x TY x TZ output voxels; a warp
// owns one z-plane of 32 x 8 voxels with 4 lanes along x (8 consecutive
// voxels each) and 8 lanes along y.
constexpr int kTX = 32;
constexpr int kTY = 8;
constexpr int kVoxPerThread = 8;
// Offsets per barrier step of the exact kernel (D buffers in shared memory).
// Two measured 3.4% faster than one (eight independent chains per thread);
// three gave 0.3% more for 21 KB more shared memory at patch radius 2.
constexpr int kOffGroup = 2;

struct TileArgs {
    int nx, ny, nz;               // unpadded volume
    int tiles_x, tiles_y;         // grid decomposition (z from blockIdx)
    int px, py, pz;               // padding per side
    int sxr, syr, szc;            // search radius x, y and clipped z
    int S;                        // number of search offsets
    const int2* __restrict__ search_delta;  // (prev-box delta, raw delta) per offset
    int pbx, pby, pbz;            // prev box (shared memory) extents
    int rbx, rby, rbz;            // raw box extents (raw staged in shared memory)
    int rplane;                   // raw box plane pitch (floats): rows of rbx + 1, padded so a
                                  // warp's 8 rows x 4 planes hit distinct banks
    int raw_slab;                 // raw staged as a slab of rbz = TZ + 1 planes of the raw box
    const int* __restrict__ group_zb;  // slab: per offset group, the z offset of its first plane
    const float* __restrict__ raw_pad;   // padded raw (global) for the raw-global form
    long long gpitch_y, gpitch_z;        // padded global pitches (elements)
    float* __restrict__ out;      // unpadded result
    const float* __restrict__ mult;      // per-slice -1/(sigma^2 beta)
    int* err;
    float w[kMaxTaps];            // patch weights in reference tap order
};

struct GenericArgs {
    int nx, ny, nz;
    int px, py, pz;
    long long gpitch_y, gpitch_z;
    int S, P;
    const long long* __restrict__ search_off;  // padded-linear offsets
    const long long* __restrict__ patch_off;
    const float* __restrict__ weights;
    const float* __restrict__ raw_pad;
    const float* __restrict__ prev_pad;
    float* __restrict__ out;
    const float* __restrict__ mult;
};

// Host-side launch descriptors.
struct TileConfig {
    int rx, ry, rz;   // patch radii of the instantiation
    int tz;           // CTA depth: z-planes = warps (4, 8), or 16 with two planes per thread
    bool raw_smem;    // raw box staged in shared memory
    size_t smem_bytes;
    bool fused = false;  // the fused FP32 form (FFMA taps, Horner Pade, fast division): the
                         // 8-deep tile kernel or the column form
    bool raw_slab = false;  // raw staged as TZ + 1 planes per z offset pair (raw_smem, tz 8 or 16)
    bool column = false;    // the column form (filter_column.cu): patch radius 1, raw from global
    bool ws = false;        // warp-specialised 8-deep kernel (raw from global, a ring of D buffers)
};

// Returns false when no tiled instantiation exists for the patch shape.
bool tile_kernel_available(int rx, int ry, int rz);
// Column form (filter_column.cu): its CTA depth for a patch shape (0: none),
// shared-memory bytes (the prev box) and launch.
int column_kernel_depth(int rx, int ry, int rz);
size_t column_smem_bytes(const TileArgs& a);
cudaError_t launch_column_kernel(const TileConfig& c, const CUtensorMap* tm_prev, const TileArgs& a,
                                 int tiles_z, cudaStream_t st);
// Shared-memory bytes for a configuration (0 if it cannot fit).
size_t tile_smem_bytes(const TileConfig& c, const TileArgs& a);
// Shared-memory bytes of the warp-specialised kernel (prev box and 4 D buffers).
size_t tile_ws_smem_bytes(const TileConfig& c, const TileArgs& a);
cudaError_t launch_tile_kernel(const TileConfig& c, const CUtensorMap* tm_prev,
                               const CUtensorMap* tm_raw, const TileArgs& a, int tiles_z,
                               cudaStream_t st);
cudaError_t launch_generic_kernel(const GenericArgs& a, cudaStream_t st);
cudaError_t launch_pad_reflective(const float* in, int nx, int ny, int nz, float* out, int px,
                                  int py, int pz, long long pitch_y, long long pitch_z,
                                  cudaStream_t st);
cudaError_t launch_sigma_to_mult(const float* sigma, float beta, float* mult, int nz,
                                 cudaStream_t st);
cudaError_t launch_sigma_blend(const float* sigma0, float* sigma1, float alpha, int nz,
                               cudaStream_t st);
// ---- persistent batch kernel (exact FP32 tiles of many volumes) ----
constexpr int kBatchMax = 24;  // volumes per launch (the kernel parameter block holds them all)
enum BatchKind : int {
    kBatchP111Smem = 0,
    kBatchP111Glob = 1,
    kBatchP222Smem = 2,
    kBatchP222Glob = 3,
    kBatchP333Smem = 4,
    kBatchP333Glob = 5,
    kBatchP111Slab = 6,  // raw staged as a z-offset slab
    kBatchP222Slab = 7,
    kBatchP333Slab = 8,
    kBatchKinds = 9,
};
struct BatchParams {
    CUtensorMap maps[kBatchMax];     // prev-box maps (64-byte aligned, first)
    TileArgs args[kBatchMax];
    int kind[kBatchMax];
    int item_begin[kBatchMax + 1];   // tile items of volume v: [item_begin[v], item_begin[v+1])
    int n;
    unsigned* counter;               // zeroed before each launch
};
// Batch body of a tile configuration (tz 8, patch (1,1,1) (2,2,2) (3,3,3)), or
// -1: one persistent kernel per kind (patch shape kind / 2, raw placement
// kind % 2: 0 shared memory, 1 global).
int batch_kind(const TileConfig& c);
cudaError_t batch_kernel_setup(int kind, size_t smem, int* ctas_per_sm);
cudaError_t launch_batch_kernel(int kind, const BatchParams& bp, int ctas, size_t smem,
                                cudaStream_t st);

// Compile-time tap rows of an instantiation, flattened as (x,y,z) triples in
// the order the kernel accumulates them; used to check host/device agreement.
int tile_kernel_tap_order(int rx, int ry, int rz, int* xyz, int max_taps);

// Failure-path self-test: a bounded mbarrier wait that nothing satisfies,
// with a budget of `cycles`; records DEV_TMA_TIMEOUT in *err.
cudaError_t launch_selftest_wait(int* err, long long cycles, cudaStream_t st);

}  // namespace inlm
