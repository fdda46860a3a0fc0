// Tensor-core forward of the proposal network's 3^3 convolutions (layers 2-4:
// 16 -> 16 channels, stride 2 or 1, zero padding, bias, ReLU) on sm_100a's
// fifth-generation tensor cores.
//
// Each conv is an implicit GEMM: out[o][co] = sum over (tap t, ci) of
// in[s*o + d_t][ci] * W[t][ci][co], M = output voxels, N = 16, K = 27 x 16.
// A CTA takes tiles of 128 output voxels (M = 128) in turn:
//   * every thread gathers one voxel's 16 input channels for 9 taps at a
//     time into shared memory in the no-swizzle K-major layout the tensor
//     core reads (8-row x 16-byte core matrices), two stages double-buffered;
//   * one thread issues tcgen05.mma kind::tf32 (A: the gathered activations,
//     B: the BF16 weights widened once per CTA, both from shared memory
//     through matrix descriptors), 2 per tap, accumulating the 128 x 16 FP32
//     tile in tensor memory (32 columns allocated per CTA), and
//     tcgen05.commit signals an mbarrier when a stage's products are done;
//   * the four warps read their 32 rows back with tcgen05.ld, add the bias,
//     apply the ReLU and store the FP32 activations.
// TF32 keeps the BF16 weights exact; the tensor core reads each FP32
// activation (or output gradient) as TF32, dropping its low 13 mantissa bits
// (the CUDA-core kernels keep FP32 operands); products accumulate in FP32. Every mbarrier wait is bounded: on expiry the CTA
// records DEV_TMA_TIMEOUT, releases its tensor memory and returns.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "proposal.cuh"

namespace inlm {

namespace {

constexpr int kTcM = 128;                                    // output voxels per tile
constexpr int kTapsPerStage = 9;
constexpr int kCore = 128;                                   // bytes per core matrix (8 rows x 16 B)
constexpr int kAChunks = kTapsPerStage * 4;                  // 16-byte K chunks of an A stage
constexpr int kAStage = (kTcM / 8) * kAChunks * kCore;       // 73728 B
constexpr int kBChunks = 27 * 4;                             // K chunks of B (27 taps x 16 ci)
constexpr int kBBytes = (kNetC / 8) * kBChunks * kCore;      // 27648 B
constexpr int kTmemCols = 32;                                // >= N, a power of two
constexpr size_t kTcSmem = 1024 + kBBytes + 2 * (size_t)kAStage;

// kind::tf32, D F32, A and B TF32, both K-major, N = 16, M = 128 (dense).
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kNetC >> 3) << 17) |
                            ((uint32_t)(kTcM >> 4) << 24);

// Shared-memory matrix descriptor: no swizzle, K-major; lbo = byte distance
// of the two 16-byte K chunks an MMA reads, sbo = byte distance of adjacent
// 8-row groups; version 1 (bit 46).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive FP32 columns of the warp's 32 TMEM lanes (one row per thread).
__device__ __forceinline__ void tc_load16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
        "%13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// DGRAD = false: the forward conv, out[o] over the output level lo from in
// at level li. DGRAD = true: its input gradient, out[i] over the input level
// li from the output gradient in = G at level lo: out[i][ci] = [act[i][ci] >
// 0] * sum over taps t with STRIDE*o + d_t = i of sum_co G[o][co] W[t][ci][co]
// (B row ci, K index (t, co)); no bias.
template <int STRIDE, bool DGRAD>
__global__ void __launch_bounds__(kTcM, 1)
    net_conv_tc_kernel(const float* __restrict__ in, Dim3i li, float* __restrict__ out, Dim3i lo,
                       const __nv_bfloat16* __restrict__ W, const float* __restrict__ bias,
                       const float* __restrict__ act, int* err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem);           // 2 mbarriers
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + 64);
    unsigned char* Bs = smem + 1024;
    unsigned char* As[2] = {Bs + kBBytes, Bs + kBBytes + kAStage};
    const int tid = threadIdx.x, warp = tid >> 5;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    // B: W[t][ci][co] as row co, K index t*16 + ci (forward) or row ci, K
    // index t*16 + co (input gradient), widened to FP32 (exact)
    for (int i = tid; i < 27 * kNetC * kNetC; i += kTcM) {
        const int t = i / (kNetC * kNetC), ci = (i / kNetC) % kNetC, co = i % kNetC;
        const int row = DGRAD ? ci : co, kk = DGRAD ? co : ci;
        const int kc = t * 4 + kk / 4;
        float* dst = reinterpret_cast<float*>(Bs + ((row >> 3) * kBChunks + kc) * kCore + (row & 7) * 16);
        dst[kk & 3] = __bfloat162float(W[i]);
    }
    float bs[kNetC];
#pragma unroll
    for (int c = 0; c < kNetC; c++) bs[c] = DGRAD ? 0.f : bias[c];
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t b_base = smem_u32(Bs);
    const uint32_t a_base[2] = {smem_u32(As[0]), smem_u32(As[1])};

    uint32_t phase[2] = {0u, 0u};
    bool ok = true;
    // rows of the GEMM: output voxels (forward) or input voxels (gradient)
    const Dim3i lr = DGRAD ? li : lo;  // the level of the rows
    const Dim3i lg = DGRAD ? lo : li;  // the level gathered from
    const long long n = (long long)lr.x * lr.y * lr.z;
    const long long tiles = (n + kTcM - 1) / kTcM;
    for (long long tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const long long o = tile * kTcM + tid;
        int ox = 0, oy = 0, oz = 0;
        const bool live = o < n;
        if (live) {
            ox = (int)(o % lr.x);
            const long long r = o / lr.x;
            oy = (int)(r % lr.y);
            oz = (int)(r / lr.y);
        }
        // stage s gathers taps 9s .. 9s + 8 into buffer s % 2
        for (int s = 0; s < 3 && ok; s++) {
            const int buf = s & 1;
            if (s == 2) {
                // buffer 0 is free once stage 0's products are done
                const bool got = mbar_wait_bounded(&bars[0], phase[0]);
                ok = __syncthreads_and(got);
                phase[0] ^= 1u;
                if (!ok) break;
            }
            unsigned char* A = As[buf];
#pragma unroll 1
            for (int lt = 0; lt < kTapsPerStage; lt++) {
                const int t = s * kTapsPerStage + lt;
                const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
                int ix, iy, iz;
                bool inside;
                if (!DGRAD) {
                    ix = STRIDE * ox + dx;
                    iy = STRIDE * oy + dy;
                    iz = STRIDE * oz + dz;
                    inside = true;
                } else {
                    // the output voxel whose tap t reads this input voxel
                    const int qx = ox - dx, qy = oy - dy, qz = oz - dz;
                    inside = (STRIDE == 1) || (((qx | qy | qz) & 1) == 0);
                    ix = qx / STRIDE;
                    iy = qy / STRIDE;
                    iz = qz / STRIDE;
                }
                float4 v[4];
                if (live && inside && ix >= 0 && ix < lg.x && iy >= 0 && iy < lg.y && iz >= 0 && iz < lg.z) {
                    const float4* src = reinterpret_cast<const float4*>(
                        in + (((long long)iz * lg.y + iy) * lg.x + ix) * kNetC);
#pragma unroll
                    for (int q = 0; q < 4; q++) v[q] = __ldg(src + q);
                } else {
#pragma unroll
                    for (int q = 0; q < 4; q++) v[q] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (int q = 0; q < 4; q++)
                    *reinterpret_cast<float4*>(A + ((tid >> 3) * kAChunks + lt * 4 + q) * kCore + (tid & 7) * 16) =
                        v[q];
            }
            fence_proxy_async_smem();
            tc_fence_before();
            __syncthreads();
            if (tid == 0) {
                tc_fence_after();
#pragma unroll 1
                for (int lt = 0; lt < kTapsPerStage; lt++) {
                    const int t = s * kTapsPerStage + lt;
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        const uint64_t ad = smem_desc(a_base[buf] + (lt * 4 + 2 * j) * kCore, kCore, kAChunks * kCore);
                        const uint64_t bd = smem_desc(b_base + (t * 4 + 2 * j) * kCore, kCore, kBChunks * kCore);
                        tc_mma(tmem, ad, bd, (t | j) ? 1u : 0u);
                    }
                }
                tc_commit(&bars[buf]);
            }
        }
        if (!ok) break;
        // stage 2 (buffer 0) done implies every earlier product; stage 1's
        // barrier completes too and is consumed here to keep its phase
        {
            const bool g0 = mbar_wait_bounded(&bars[0], phase[0]);
            const bool g1 = mbar_wait_bounded(&bars[1], phase[1]);
            ok = __syncthreads_and(g0 && g1);
            phase[0] ^= 1u;
            phase[1] ^= 1u;
            if (!ok) break;
        }
        tc_fence_after();
        float acc[16];
        tc_load16(tmem + ((uint32_t)(warp * 32) << 16), acc);
        if (live) {
            float4* dst = reinterpret_cast<float4*>(out + o * kNetC);
            if (!DGRAD) {
#pragma unroll
                for (int q = 0; q < 4; q++)
                    dst[q] = make_float4(fmaxf(acc[4 * q] + bs[4 * q], 0.f), fmaxf(acc[4 * q + 1] + bs[4 * q + 1], 0.f),
                                         fmaxf(acc[4 * q + 2] + bs[4 * q + 2], 0.f),
                                         fmaxf(acc[4 * q + 3] + bs[4 * q + 3], 0.f));
            } else {
                // the ReLU of the layer that produced this input
                const float4* am = reinterpret_cast<const float4*>(act + o * kNetC);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float4 a = __ldg(am + q);
                    dst[q] = make_float4(a.x > 0.f ? acc[4 * q] : 0.f, a.y > 0.f ? acc[4 * q + 1] : 0.f,
                                         a.z > 0.f ? acc[4 * q + 2] : 0.f, a.w > 0.f ? acc[4 * q + 3] : 0.f);
                }
            }
        }
        // the next tile's first product overwrites the accumulator
        tc_fence_before();
        __syncthreads();
    }
    if (!ok && tid == 0) set_error(err, DEV_TMA_TIMEOUT);
    // products still in flight after a timeout would write tensor memory we
    // are about to release: give them a bounded chance to finish
    if (!ok) {
        mbar_wait_bounded(&bars[0], phase[0]);
        mbar_wait_bounded(&bars[1], phase[1]);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                     : "memory");
    }
}

}  // namespace

template <int STRIDE, bool DGRAD>
static cudaError_t launch_tc(const float* in, Dim3i li, float* out, Dim3i lo, const __nv_bfloat16* W,
                             const float* b, const float* act, int* err, cudaStream_t st) {
    const Dim3i lr = DGRAD ? li : lo;
    const long long n = (long long)lr.x * lr.y * lr.z;
    if (n <= 0) return cudaSuccess;
    const long long tiles = (n + kTcM - 1) / kTcM;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)std::min<long long>(tiles, sms);
    cudaError_t e = cudaFuncSetAttribute(net_conv_tc_kernel<STRIDE, DGRAD>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
    if (e != cudaSuccess) return e;
    net_conv_tc_kernel<STRIDE, DGRAD><<<grid, kTcM, kTcSmem, st>>>(in, li, out, lo, W, b, act, err);
    return cudaGetLastError();
}

cudaError_t net_conv_fwd_tc(const float* in, Dim3i li, float* out, Dim3i lo, int stride,
                            const __nv_bfloat16* W, const float* b, int* err, cudaStream_t st) {
    return stride == 2 ? launch_tc<2, false>(in, li, out, lo, W, b, nullptr, err, st)
                       : launch_tc<1, false>(in, li, out, lo, W, b, nullptr, err, st);
}

cudaError_t net_conv_dgrad_tc(const float* G, Dim3i lo, const __nv_bfloat16* W, const float* ain, Dim3i li,
                              float* din, int stride, int* err, cudaStream_t st) {
    return stride == 2 ? launch_tc<2, true>(G, li, din, lo, W, nullptr, ain, err, st)
                       : launch_tc<1, true>(G, li, din, lo, W, nullptr, ain, err, st);
}

}  // namespace inlm
