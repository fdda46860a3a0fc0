// Learned search-offset proposal (sm_100a).
//
// Network (no counterpart in the reference; the filter it prunes is
// Denoiser/iternlm_cpu.cpp:758-843):
//   L1  3^3 difference stencil, stride 2, 1 -> 16 channels, ReLU. Its inputs
//       are scale(z) * (v(c + tap) - v(c)) around the centre voxel c = 2o, so
//       the features do not depend on the grey-value offset of the volume and
//       are in units of the filter's sigma.
//   L2  3^3 conv, stride 2, 16 -> 16, ReLU
//   L3  3^3 conv, stride 2, 16 -> 16, ReLU   (one output per 8^3 tile)
//   L4  3^3 conv, stride 1, 16 -> 16, ReLU
//   head  linear 16 -> S logits per tile, softmax over the search offsets.
// Weights are BF16 (rounded from FP32 masters after every optimiser step);
// biases, activations and all accumulation are FP32. Zero padding between
// layers; the input's reflective halo serves L1.
//
// The layers are tiny next to the filter (about 0.1% of its FLOPs at search
// radius 5), so they run on the FP32 pipe: one thread per output voxel with
// the 27x16x16 weight block broadcast from shared memory.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "proposal.cuh"

namespace inlm {

NetLayout net_layout(int S) {
    NetLayout L;
    long long o = 0;
    L.S = S;
    L.w1 = o;
    o += 27 * kNetC;
    L.b1 = o;
    o += kNetC;
    L.w2 = o;
    o += 27 * kNetC * kNetC;
    L.b2 = o;
    o += kNetC;
    L.w3 = o;
    o += 27 * kNetC * kNetC;
    L.b3 = o;
    o += kNetC;
    L.w4 = o;
    o += 27 * kNetC * kNetC;
    L.b4 = o;
    o += kNetC;
    L.wh = o;
    o += (long long)S * kNetC;
    L.bh = o;
    o += S;
    L.total = o;
    return L;
}

void net_levels(int nx, int ny, int nz, Dim3i lv[4]) {
    lv[0] = {nx, ny, nz};
    for (int l = 1; l < 4; l++)
        lv[l] = {(lv[l - 1].x + 1) / 2, (lv[l - 1].y + 1) / 2, (lv[l - 1].z + 1) / 2};
}

__host__ __device__ static inline long long nvox(Dim3i d) { return (long long)d.x * d.y * d.z; }

static inline int grid_for(long long n, int block) {
    long long g = (n + block - 1) / block;
    if (g > 148 * 32) g = 148 * 32;
    return (int)(g < 1 ? 1 : g);
}

__device__ __forceinline__ float ldv(const float* p, long long i) { return __ldg(p + i); }
__device__ __forceinline__ float ldv(const __half* p, long long i) {
    return __half2float(__ushort_as_half(__ldg(reinterpret_cast<const unsigned short*>(p) + i)));
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum / max (every thread gets the result); red: >= 32 floats.
template <bool MAX>
__device__ float block_reduce(float v, float* red) {
    v = MAX ? warp_max(v) : warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    float r = red[0];
    for (int i = 1; i < nw; i++) r = MAX ? fmaxf(r, red[i]) : r + red[i];
    return r;
}

// ---------------- forward ----------------

template <typename T>
__global__ void __launch_bounds__(256)
    net_l1_fwd_kernel(NetIn in, Dim3i lo, const __nv_bfloat16* __restrict__ W,
                      const float* __restrict__ b, float* __restrict__ out) {
    __shared__ float ws[27 * kNetC];
    __shared__ float bs[kNetC];
    for (int i = threadIdx.x; i < 27 * kNetC; i += blockDim.x) ws[i] = __bfloat162float(W[i]);
    if (threadIdx.x < kNetC) bs[threadIdx.x] = b[threadIdx.x];
    __syncthreads();
    const T* base = static_cast<const T*>(in.base);
    const long long n = nvox(lo);
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n;
         o += (long long)gridDim.x * blockDim.x) {
        const int ox = (int)(o % lo.x);
        const long long r = o / lo.x;
        const int oy = (int)(r % lo.y);
        const int oz = (int)(r / lo.y);
        const long long c = 2LL * oz * in.pz + 2LL * oy * in.py + 2 * ox;
        const float s = in.scale[2 * oz];
        const float xc = ldv(base, c);
        float acc[kNetC];
#pragma unroll
        for (int co = 0; co < kNetC; co++) acc[co] = bs[co];
#pragma unroll
        for (int t = 0; t < 27; t++) {
            const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
            const float d = s * (ldv(base, c + dz * in.pz + dy * in.py + dx) - xc);
#pragma unroll
            for (int co = 0; co < kNetC; co++) acc[co] = fmaf(ws[t * kNetC + co], d, acc[co]);
        }
        float4* dst = reinterpret_cast<float4*>(out + o * kNetC);
#pragma unroll
        for (int q = 0; q < 4; q++)
            dst[q] = make_float4(fmaxf(acc[4 * q], 0.f), fmaxf(acc[4 * q + 1], 0.f),
                                 fmaxf(acc[4 * q + 2], 0.f), fmaxf(acc[4 * q + 3], 0.f));
    }
}

__device__ __forceinline__ void load16(const float* p, float (&a)[kNetC]) {
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        float4 v = __ldg(q + i);
        a[4 * i] = v.x;
        a[4 * i + 1] = v.y;
        a[4 * i + 2] = v.z;
        a[4 * i + 3] = v.w;
    }
}

__device__ __forceinline__ void load_wblock(float* ws, const __nv_bfloat16* __restrict__ W) {
    for (int i = threadIdx.x; i < 27 * kNetC * kNetC; i += blockDim.x) ws[i] = __bfloat162float(W[i]);
}

template <int STRIDE>
__global__ void __launch_bounds__(128)
    net_conv_fwd_kernel(const float* __restrict__ in, Dim3i li, float* __restrict__ out, Dim3i lo,
                        const __nv_bfloat16* __restrict__ W, const float* __restrict__ b) {
    __shared__ __align__(16) float ws[27 * kNetC * kNetC];
    __shared__ float bs[kNetC];
    load_wblock(ws, W);
    if (threadIdx.x < kNetC) bs[threadIdx.x] = b[threadIdx.x];
    __syncthreads();
    const long long n = nvox(lo);
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n;
         o += (long long)gridDim.x * blockDim.x) {
        const int ox = (int)(o % lo.x);
        const long long r = o / lo.x;
        const int oy = (int)(r % lo.y);
        const int oz = (int)(r / lo.y);
        float acc[kNetC];
#pragma unroll
        for (int co = 0; co < kNetC; co++) acc[co] = bs[co];
        for (int dz = -1; dz <= 1; dz++) {
            const int iz = STRIDE * oz + dz;
            if (iz < 0 || iz >= li.z) continue;
            for (int dy = -1; dy <= 1; dy++) {
                const int iy = STRIDE * oy + dy;
                if (iy < 0 || iy >= li.y) continue;
#pragma unroll
                for (int dx = -1; dx <= 1; dx++) {
                    const int ix = STRIDE * ox + dx;
                    if (ix < 0 || ix >= li.x) continue;
                    const int t = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                    float a[kNetC];
                    load16(in + (((long long)iz * li.y + iy) * li.x + ix) * kNetC, a);
                    const float4* wr = reinterpret_cast<const float4*>(ws + t * kNetC * kNetC);
#pragma unroll
                    for (int ci = 0; ci < kNetC; ci++) {
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const float4 w = wr[ci * 4 + q];
                            acc[4 * q] = fmaf(w.x, a[ci], acc[4 * q]);
                            acc[4 * q + 1] = fmaf(w.y, a[ci], acc[4 * q + 1]);
                            acc[4 * q + 2] = fmaf(w.z, a[ci], acc[4 * q + 2]);
                            acc[4 * q + 3] = fmaf(w.w, a[ci], acc[4 * q + 3]);
                        }
                    }
                }
            }
        }
        float4* dst = reinterpret_cast<float4*>(out + o * kNetC);
#pragma unroll
        for (int q = 0; q < 4; q++)
            dst[q] = make_float4(fmaxf(acc[4 * q], 0.f), fmaxf(acc[4 * q + 1], 0.f),
                                 fmaxf(acc[4 * q + 2], 0.f), fmaxf(acc[4 * q + 3], 0.f));
    }
}

__device__ __forceinline__ float head_logit(const __nv_bfloat16* __restrict__ Wh, const float* bh,
                                            const float* h, int k) {
    const __nv_bfloat162* wr = reinterpret_cast<const __nv_bfloat162*>(Wh + (long long)k * kNetC);
    float l = bh[k];
#pragma unroll
    for (int c = 0; c < kNetC / 2; c++) {
        float2 w = __bfloat1622float2(wr[c]);
        l = fmaf(w.x, h[2 * c], l);
        l = fmaf(w.y, h[2 * c + 1], l);
    }
    return l;
}

__global__ void __launch_bounds__(256)
    net_logits_kernel(const float* __restrict__ a4, int S, const __nv_bfloat16* __restrict__ Wh,
                      const float* __restrict__ bh, float* __restrict__ logits) {
    __shared__ float h[kNetC];
    const long long tile = blockIdx.x;
    if (threadIdx.x < kNetC) h[threadIdx.x] = a4[tile * kNetC + threadIdx.x];
    __syncthreads();
    for (int k = threadIdx.x; k < S; k += blockDim.x) logits[tile * S + k] = head_logit(Wh, bh, h, k);
}

// ---------------- backward ----------------

// Per tile: softmax, soft-target cross entropy, dL/dlogit, and dL/d(pre-ReLU
// L4 output).
__global__ void __launch_bounds__(256)
    net_head_train_kernel(const float* __restrict__ a4, int S, const __nv_bfloat16* __restrict__ Wh,
                          const float* __restrict__ bh, const float* __restrict__ target,
                          float inv_n, float* __restrict__ G, float* __restrict__ d4,
                          double* loss) {
    extern __shared__ float sl[];  // S logits
    __shared__ float h[kNetC];
    __shared__ float red[32];
    __shared__ float dh[8][kNetC];
    const long long tile = blockIdx.x;
    if (threadIdx.x < kNetC) h[threadIdx.x] = a4[tile * kNetC + threadIdx.x];
    __syncthreads();
    float m = -INFINITY;
    for (int k = threadIdx.x; k < S; k += blockDim.x) {
        const float l = head_logit(Wh, bh, h, k);
        sl[k] = l;
        m = fmaxf(m, l);
    }
    const float M = block_reduce<true>(m, red);
    float z = 0.f, T = 0.f, TL = 0.f;
    const float* tr = target + tile * S;
    for (int k = threadIdx.x; k < S; k += blockDim.x) {
        z += expf(sl[k] - M);
        const float t = tr[k];
        T += t;
        TL = fmaf(t, sl[k] - M, TL);
    }
    const float Z = block_reduce<false>(z, red);
    const float Tt = block_reduce<false>(T, red);
    const float TLt = block_reduce<false>(TL, red);
    if (threadIdx.x == 0) atomicAdd(loss, (double)(Tt * logf(Z) - TLt) * (double)inv_n);
    float dhl[kNetC];
#pragma unroll
    for (int c = 0; c < kNetC; c++) dhl[c] = 0.f;
    const float invZ = 1.f / Z;
    for (int k = threadIdx.x; k < S; k += blockDim.x) {
        const float p = expf(sl[k] - M) * invZ;
        const float g = (p * Tt - tr[k]) * inv_n;
        G[tile * S + k] = g;
        const __nv_bfloat162* wr = reinterpret_cast<const __nv_bfloat162*>(Wh + (long long)k * kNetC);
#pragma unroll
        for (int c = 0; c < kNetC / 2; c++) {
            float2 w = __bfloat1622float2(wr[c]);
            dhl[2 * c] = fmaf(g, w.x, dhl[2 * c]);
            dhl[2 * c + 1] = fmaf(g, w.y, dhl[2 * c + 1]);
        }
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int c = 0; c < kNetC; c++) {
        float v = warp_sum(dhl[c]);
        if (l == 0) dh[w][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < kNetC) {
        float v = 0.f;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) v += dh[i][threadIdx.x];
        d4[tile * kNetC + threadIdx.x] = h[threadIdx.x] > 0.f ? v : 0.f;
    }
}

// dWh[k][c] += sum_tiles G[tile][k] h[tile][c]; dbh[k] += sum_tiles G[tile][k].
__global__ void __launch_bounds__(128)
    net_head_wgrad_kernel(const float* __restrict__ G, const float* __restrict__ a4, int n_tiles,
                          int S, int tiles_per_block, float* dWh, float* dbh) {
    __shared__ float hs[64][kNetC];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int t0 = blockIdx.y * tiles_per_block;
    const int t1 = min(n_tiles, t0 + tiles_per_block);
    float acc[kNetC], gb = 0.f;
#pragma unroll
    for (int c = 0; c < kNetC; c++) acc[c] = 0.f;
    for (int tb = t0; tb < t1; tb += 64) {
        const int nt = min(64, t1 - tb);
        __syncthreads();
        for (int i = threadIdx.x; i < nt * kNetC; i += blockDim.x)
            hs[i / kNetC][i % kNetC] = a4[(long long)tb * kNetC + i];
        __syncthreads();
        if (k < S) {
            for (int tt = 0; tt < nt; tt++) {
                const float g = G[(long long)(tb + tt) * S + k];
                gb += g;
#pragma unroll
                for (int c = 0; c < kNetC; c++) acc[c] = fmaf(g, hs[tt][c], acc[c]);
            }
        }
    }
    if (k < S) {
#pragma unroll
        for (int c = 0; c < kNetC; c++) atomicAdd(&dWh[(long long)k * kNetC + c], acc[c]);
        atomicAdd(&dbh[k], gb);
    }
}

// dW[t][ci][co] += sum_o G[o][co] in[STRIDE*o + t][ci]; db[co] += sum_o G[o][co].
// Thread (ci, co); the block walks a run of output voxels.
template <int STRIDE>
__global__ void __launch_bounds__(256)
    net_conv_wgrad_kernel(const float* __restrict__ in, Dim3i li, const float* __restrict__ G,
                          Dim3i lo, int per_block, float* dW, float* db) {
    const int ci = threadIdx.x >> 4, co = threadIdx.x & 15;
    float acc[27], bacc = 0.f;
#pragma unroll
    for (int t = 0; t < 27; t++) acc[t] = 0.f;
    const long long n = nvox(lo);
    const long long o0 = (long long)blockIdx.x * per_block;
    const long long o1 = min(n, o0 + per_block);
    for (long long o = o0; o < o1; o++) {
        const int ox = (int)(o % lo.x);
        const long long r = o / lo.x;
        const int oy = (int)(r % lo.y);
        const int oz = (int)(r / lo.y);
        const float g = G[o * kNetC + co];
        bacc += g;
#pragma unroll
        for (int t = 0; t < 27; t++) {
            const int iz = STRIDE * oz + t / 9 - 1, iy = STRIDE * oy + (t / 3) % 3 - 1,
                      ix = STRIDE * ox + t % 3 - 1;
            if (iz >= 0 && iz < li.z && iy >= 0 && iy < li.y && ix >= 0 && ix < li.x)
                acc[t] = fmaf(g, __ldg(in + (((long long)iz * li.y + iy) * li.x + ix) * kNetC + ci),
                              acc[t]);
        }
    }
#pragma unroll
    for (int t = 0; t < 27; t++) atomicAdd(&dW[(t * kNetC + ci) * kNetC + co], acc[t]);
    if (ci == 0) atomicAdd(&db[co], bacc);
}

// dL1 weights: thread (tap, co), 27 x 16 threads.
template <typename T>
__global__ void __launch_bounds__(432)
    net_l1_wgrad_kernel(NetIn in, Dim3i lo, const float* __restrict__ G, int per_block, float* dW,
                        float* db) {
    const int t = threadIdx.x >> 4, co = threadIdx.x & 15;
    const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
    const long long off = dz * in.pz + dy * in.py + dx;
    const T* base = static_cast<const T*>(in.base);
    float acc = 0.f, bacc = 0.f;
    const long long n = nvox(lo);
    const long long o0 = (long long)blockIdx.x * per_block;
    const long long o1 = min(n, o0 + per_block);
    for (long long o = o0; o < o1; o++) {
        const int ox = (int)(o % lo.x);
        const long long r = o / lo.x;
        const int oy = (int)(r % lo.y);
        const int oz = (int)(r / lo.y);
        const long long c = 2LL * oz * in.pz + 2LL * oy * in.py + 2 * ox;
        const float s = in.scale[2 * oz];
        const float d = s * (ldv(base, c + off) - ldv(base, c));
        const float g = G[o * kNetC + co];
        acc = fmaf(g, d, acc);
        bacc += g;
    }
    atomicAdd(&dW[t * kNetC + co], acc);
    if (t == 0) atomicAdd(&db[co], bacc);
}

// dIn[i][ci] = [a_in[i][ci] > 0] * sum over (o, t) with STRIDE*o + t = i of
// sum_co W[t][ci][co] G[o][co]   (gather form, one thread per input voxel).
template <int STRIDE>
__global__ void __launch_bounds__(128)
    net_conv_dgrad_kernel(const float* __restrict__ G, Dim3i lo, const __nv_bfloat16* __restrict__ W,
                          const float* __restrict__ ain, Dim3i li, float* __restrict__ din) {
    __shared__ __align__(16) float ws[27 * kNetC * kNetC];
    load_wblock(ws, W);
    __syncthreads();
    const long long n = nvox(li);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i % li.x);
        const long long r = i / li.x;
        const int iy = (int)(r % li.y);
        const int iz = (int)(r / li.y);
        float acc[kNetC];
#pragma unroll
        for (int c = 0; c < kNetC; c++) acc[c] = 0.f;
        for (int dz = -1; dz <= 1; dz++) {
            int oz = iz - dz;
            if (STRIDE == 2) {
                if (oz & 1) continue;
                oz >>= 1;
            }
            if (oz < 0 || oz >= lo.z) continue;
            for (int dy = -1; dy <= 1; dy++) {
                int oy = iy - dy;
                if (STRIDE == 2) {
                    if (oy & 1) continue;
                    oy >>= 1;
                }
                if (oy < 0 || oy >= lo.y) continue;
                for (int dx = -1; dx <= 1; dx++) {
                    int ox = ix - dx;
                    if (STRIDE == 2) {
                        if (ox & 1) continue;
                        ox >>= 1;
                    }
                    if (ox < 0 || ox >= lo.x) continue;
                    const int t = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                    float g[kNetC];
                    load16(G + (((long long)oz * lo.y + oy) * lo.x + ox) * kNetC, g);
                    const float4* wr = reinterpret_cast<const float4*>(ws + t * kNetC * kNetC);
#pragma unroll
                    for (int ci = 0; ci < kNetC; ci++) {
                        float s = acc[ci];
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const float4 w = wr[ci * 4 + q];
                            s = fmaf(w.x, g[4 * q], s);
                            s = fmaf(w.y, g[4 * q + 1], s);
                            s = fmaf(w.z, g[4 * q + 2], s);
                            s = fmaf(w.w, g[4 * q + 3], s);
                        }
                        acc[ci] = s;
                    }
                }
            }
        }
        float a[kNetC];
        load16(ain + i * kNetC, a);
        float4* dst = reinterpret_cast<float4*>(din + i * kNetC);
#pragma unroll
        for (int q = 0; q < 4; q++)
            dst[q] = make_float4(a[4 * q] > 0.f ? acc[4 * q] : 0.f,
                                 a[4 * q + 1] > 0.f ? acc[4 * q + 1] : 0.f,
                                 a[4 * q + 2] > 0.f ? acc[4 * q + 2] : 0.f,
                                 a[4 * q + 3] > 0.f ? acc[4 * q + 3] : 0.f);
    }
}

__global__ void net_adam_kernel(float* w, float* m, float* v, const float* g, __nv_bfloat16* wb,
                                long long n, float lr, float b1, float b2, float eps, float bc1,
                                float bc2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        w[i] = wi;
        wb[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void net_round_kernel(const float* w, __nv_bfloat16* wb, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        wb[i] = __float2bfloat16_rn(w[i]);
}

// ---------------- inference: top-K and plans ----------------

__device__ __forceinline__ unsigned order_key(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Radix select over the values sl[0..S) of one warp: on return the kept set is
// every key above *prefix plus the first *remaining keys equal to it in
// offset order (the Ke largest values, ties towards lower offsets); 8 bits
// per pass over a warp-private 256-bin histogram.
__device__ __forceinline__ void warp_topk_threshold(const float* sl, int S, int Ke, unsigned* hist,
                                                    int lane, unsigned* prefix_out, int* remaining_out) {
    unsigned prefix = 0, pmask = 0;
    int remaining = Ke;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = lane; b < 256; b += 32) hist[b] = 0;
        __syncwarp();
        for (int k = lane; k < S; k += 32) {
            const unsigned key = order_key(sl[k]);
            if ((key & pmask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
        }
        __syncwarp();
        // lane L owns bins 255-8L .. 248-8L (from the top); counts above them
        // by an exclusive scan over the lanes
        int own[8], tot = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            own[q] = (int)hist[255 - 8 * lane - q];
            tot += own[q];
        }
        int incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int above = incl - tot;  // keys in higher bins than this lane's
        int found_bin = -1, found_above = 0;
        if (above < remaining && incl >= remaining) {
            int cum = above;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                if (found_bin < 0 && cum + own[q] >= remaining) {
                    found_bin = 255 - 8 * lane - q;
                    found_above = cum;
                }
                cum += own[q];
            }
        }
        const unsigned ball = __ballot_sync(0xffffffffu, found_bin >= 0);
        const int src = __ffs(ball) - 1;  // exactly one lane holds the bin
        found_bin = __shfl_sync(0xffffffffu, found_bin, src < 0 ? 0 : src);
        found_above = __shfl_sync(0xffffffffu, found_above, src < 0 ? 0 : src);
        if (src < 0) found_bin = 0;  // unreachable for consistent counts
        prefix |= (unsigned)found_bin << shift;
        pmask |= 255u << shift;
        remaining -= found_above;
        __syncwarp();
    }
    *prefix_out = prefix;
    *remaining_out = remaining;
}

// Sum over the kept offsets of val(k), warp-reduced.
template <class F>
__device__ __forceinline__ float warp_kept_sum(const float* sl, int S, unsigned prefix, int remaining,
                                               int lane, F val) {
    float kept = 0.f;
    int ties_before = 0;
    const int rounds = (S + 31) / 32;
    for (int i = 0; i < rounds; i++) {
        const int k = 32 * i + lane;
        const unsigned key = k < S ? order_key(sl[k]) : 0u;
        const bool tie = k < S && key == prefix;
        const unsigned tb = __ballot_sync(0xffffffffu, tie);
        const int rank = ties_before + __popc(tb & ((1u << lane) - 1u));
        const bool s = k < S && (key > prefix || (tie && rank < remaining));
        ties_before += __popc(tb);
        if (s) kept += val(k);
    }
    return warp_sum(kept);
}

// Kept flags as bitmap words (word i = offsets 32i .. 32i+31); every offset
// under fallback.
__device__ __forceinline__ void warp_write_bitmap(const float* sl, int S, unsigned prefix, int remaining,
                                                  bool fallback, unsigned* out, int nwords, int lane) {
    int ties_before = 0;
    const int rounds = (S + 31) / 32;
    for (int i = 0; i < rounds; i++) {
        const int k = 32 * i + lane;
        const unsigned key = k < S ? order_key(sl[k]) : 0u;
        const bool tie = k < S && key == prefix;
        const unsigned tb = __ballot_sync(0xffffffffu, tie);
        const int rank = ties_before + __popc(tb & ((1u << lane) - 1u));
        ties_before += __popc(tb);
        const bool s = k < S && (fallback || key > prefix || (tie && rank < remaining));
        const unsigned word = __ballot_sync(0xffffffffu, s);
        if (lane == 0 && i < nwords) out[i] = word;
    }
}

// One warp per tile: logits in the warp's shared-memory row, softmax
// normaliser by shuffles, radix select of the K-th largest logit (8 bits per
// pass, a warp-private 256-bin histogram), ties broken towards lower offsets;
// offsets k = 32 i + lane are handled in rounds i, so a ballot of the kept
// flags in round i is bitmap word i.
constexpr int kSelWarps = 4;

__global__ void __launch_bounds__(32 * kSelWarps)
    net_select_kernel(const float* __restrict__ a4, long long n_tiles, int S,
                      const __nv_bfloat16* __restrict__ Wh, const float* __restrict__ bh, int K,
                      float min_mass, unsigned* __restrict__ bitmap, int nwords,
                      float* __restrict__ pred_mass, int* counters) {
    extern __shared__ unsigned sel_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rowlen = (S + 3) / 4 * 4;
    float* sl = reinterpret_cast<float*>(sel_smem) + warp * rowlen;
    unsigned* hist = sel_smem + kSelWarps * rowlen + warp * 256;
    const long long tile = blockIdx.x * (long long)kSelWarps + warp;
    if (tile >= n_tiles) return;
    float h[kNetC];
    load16(a4 + tile * kNetC, h);
    float m = -INFINITY;
    for (int k = lane; k < S; k += 32) {
        const float l = head_logit(Wh, bh, h, k);
        sl[k] = l;
        m = fmaxf(m, l);
    }
    const float M = warp_max(m);
    float z = 0.f;
    for (int k = lane; k < S; k += 32) z += expf(sl[k] - M);
    const float Z = warp_sum(z);
    __syncwarp();

    const int Ke = min(max(K, 1), S);
    unsigned prefix;
    int remaining;
    warp_topk_threshold(sl, S, Ke, hist, lane, &prefix, &remaining);
    float kept = warp_kept_sum(sl, S, prefix, remaining, lane, [&](int k) { return expf(sl[k] - M); });
    kept = kept / Z;
    const bool fallback = !(kept >= min_mass);
    warp_write_bitmap(sl, S, prefix, remaining, fallback, bitmap + tile * nwords, nwords, lane);
    if (lane == 0) {
        pred_mass[tile] = kept;
        if (fallback) atomicAdd(&counters[0], 1);
    }
}

// One warp per group of up to G consecutive 8^3 tiles along x (the 32 x 8 x 8
// CTA of the full-width filter kernel for G = 4): each tile's softmax over the
// offsets, summed over the group's tiles, ranked and cut at the top K (ties
// towards lower offsets). The predicted kept mass is the mean over the tiles
// of each tile's kept probability; below min_mass the group keeps everything.
__global__ void __launch_bounds__(32 * kSelWarps)
    net_select_group_kernel(const float* __restrict__ a4, int t8x, long long n_groups, int gx, int G,
                            int S, const __nv_bfloat16* __restrict__ Wh, const float* __restrict__ bh,
                            int K, float min_mass, unsigned* __restrict__ bitmap, int nwords,
                            float* __restrict__ pred_mass, int* counters) {
    extern __shared__ unsigned sel_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rowlen = (S + 3) / 4 * 4;
    float* sc = reinterpret_cast<float*>(sel_smem) + warp * 2 * rowlen;
    float* sl = sc + rowlen;
    unsigned* hist = sel_smem + kSelWarps * 2 * rowlen + warp * 256;
    const long long g = blockIdx.x * (long long)kSelWarps + warp;
    if (g >= n_groups) return;
    const long long row = g / gx;  // (z, y) tile row
    const int gxi = (int)(g - row * gx);
    for (int k = lane; k < S; k += 32) sc[k] = 0.f;
    int ng = 0;
    for (int j = 0; j < G; j++) {
        const int tx = gxi * G + j;
        if (tx >= t8x) break;
        const long long tile = row * t8x + tx;
        float h[kNetC];
        load16(a4 + tile * kNetC, h);
        float m = -INFINITY;
        for (int k = lane; k < S; k += 32) {
            const float l = head_logit(Wh, bh, h, k);
            sl[k] = l;
            m = fmaxf(m, l);
        }
        const float M = warp_max(m);
        float z = 0.f;
        for (int k = lane; k < S; k += 32) z += expf(sl[k] - M);
        const float Z = warp_sum(z);
        for (int k = lane; k < S; k += 32) sc[k] += expf(sl[k] - M) / Z;  // lane-owned entries
        ng++;
        __syncwarp();
    }
    const int Ke = min(max(K, 1), S);
    unsigned prefix;
    int remaining;
    warp_topk_threshold(sc, S, Ke, hist, lane, &prefix, &remaining);
    const float kept = warp_kept_sum(sc, S, prefix, remaining, lane, [&](int k) { return sc[k]; }) / ng;
    const bool fallback = !(kept >= min_mass);
    warp_write_bitmap(sc, S, prefix, remaining, fallback, bitmap + g * nwords, nwords, lane);
    if (lane == 0) {
        pred_mass[g] = kept;
        if (fallback) atomicAdd(&counters[0], 1);
    }
}

// Sum of the n predicted kept masses in a fixed order (one CTA: strided
// per-thread sums, then a tree), so the mean, and the relative fallback
// threshold taken from it, are the same on every run.
__global__ void __launch_bounds__(1024) net_mass_sum_kernel(const float* __restrict__ mass, long long n,
                                                            double* __restrict__ out) {
    __shared__ double red[1024];
    double s = 0.0;
    for (long long i = threadIdx.x; i < n; i += 1024) s += (double)mass[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0];
}

// Per plan list (one warp): the kept offsets in ascending order, compacted
// from the list's bitmap into plan_off[t * S ...]; plan_count[t]. With
// rel > 0 a list whose predicted kept mass is below rel x the mean over all
// lists (mass_sum / n_tiles) takes every offset instead (counters[0] counts
// it).
__global__ void net_plan_tiles_kernel(const unsigned* __restrict__ bitmap, int nwords,
                                      long long n_tiles, int S, int* __restrict__ plan_off,
                                      int* __restrict__ plan_count, int* counters,
                                      const float* __restrict__ pred_mass, const double* __restrict__ mass_sum,
                                      float rel) {
    const int lane = threadIdx.x & 31;
    const long long t = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    if (t >= n_tiles) return;
    const unsigned* row = bitmap + t * nwords;
    int* out = plan_off + t * (long long)S;
    if (rel > 0.f && pred_mass[t] < (float)((double)rel * (mass_sum[0] / (double)n_tiles))) {
        for (int k = lane; k < S; k += 32) out[k] = k;
        if (lane == 0) {
            plan_count[t] = S;
            atomicAdd(&counters[0], 1);
            atomicAdd(&counters[1], S);
        }
        return;
    }
    int n = 0;
    for (int w0 = 0; w0 < nwords; w0 += 32) {
        const int wd = w0 + lane;
        unsigned u = wd < nwords ? row[wd] : 0u;
        const int cnt = __popc(u);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        int pos = n + incl - cnt;
        while (u) {
            const int bit = __ffs(u) - 1;
            u &= u - 1;
            const int k = wd * 32 + bit;
            if (pos < S && k < S) out[pos] = k;
            pos++;
        }
        n += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) {
        plan_count[t] = min(n, S);
        atomicAdd(&counters[1], min(n, S));
    }
}

__global__ void net_scale_kernel(const float* mult, int nz, float* scale) {
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < nz; z += gridDim.x * blockDim.x) {
        const float m = -mult[z];
        // sigma = 0 (m = inf) or a non-positive multiplier: no usable scale
        scale[z] = (m > 0.f && m < 1e8f) ? sqrtf(m) : 0.f;
    }
}

__global__ void unpad_half_kernel(const __half* __restrict__ in, long long py, long long pz, int nx,
                                  int ny, int nz, float* __restrict__ out) {
    const long long n = (long long)nx * ny * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const long long r = i / nx;
        const int y = (int)(r % ny);
        const int z = (int)(r / ny);
        out[i] = __half2float(in[z * pz + y * py + x]);
    }
}

__global__ void __launch_bounds__(256) normalise_rows_kernel(float* map, int S) {
    __shared__ float red[32];
    float* row = map + (long long)blockIdx.x * S;
    float s = 0.f;
    for (int k = threadIdx.x; k < S; k += blockDim.x) s += row[k];
    s = block_reduce<false>(s, red);
    if (s > 0.f) {
        const float inv = 1.f / s;
        for (int k = threadIdx.x; k < S; k += blockDim.x) row[k] *= inv;
    }
}

// ---------------- launchers ----------------

#define INLM_LAUNCH_CHECK() \
    do {                    \
        cudaError_t e_ = cudaGetLastError(); \
        if (e_ != cudaSuccess) return e_;    \
    } while (0)

cudaError_t net_forward(const NetLayout& L, const __nv_bfloat16* wb, const float* wf, const NetIn& in,
                        const NetActs& act, cudaStream_t st, const NetTc& tc) {
    Dim3i lv[4];
    net_levels(in.nx, in.ny, in.nz, lv);
    if (in.half)
        net_l1_fwd_kernel<__half><<<grid_for(nvox(lv[1]), 256), 256, 0, st>>>(in, lv[1], wb + L.w1,
                                                                              wf + L.b1, act.a1);
    else
        net_l1_fwd_kernel<float><<<grid_for(nvox(lv[1]), 256), 256, 0, st>>>(in, lv[1], wb + L.w1,
                                                                             wf + L.b1, act.a1);
    INLM_LAUNCH_CHECK();
    if (tc.on) {
        cudaError_t e = net_conv_fwd_tc(act.a1, lv[1], act.a2, lv[2], 2, wb + L.w2, wf + L.b2, tc.err, st);
        if (e != cudaSuccess) return e;
        e = net_conv_fwd_tc(act.a2, lv[2], act.a3, lv[3], 2, wb + L.w3, wf + L.b3, tc.err, st);
        if (e != cudaSuccess) return e;
        return net_conv_fwd_tc(act.a3, lv[3], act.a4, lv[3], 1, wb + L.w4, wf + L.b4, tc.err, st);
    }
    net_conv_fwd_kernel<2><<<grid_for(nvox(lv[2]), 128), 128, 0, st>>>(act.a1, lv[1], act.a2, lv[2],
                                                                       wb + L.w2, wf + L.b2);
    INLM_LAUNCH_CHECK();
    net_conv_fwd_kernel<2><<<grid_for(nvox(lv[3]), 128), 128, 0, st>>>(act.a2, lv[2], act.a3, lv[3],
                                                                       wb + L.w3, wf + L.b3);
    INLM_LAUNCH_CHECK();
    net_conv_fwd_kernel<1><<<grid_for(nvox(lv[3]), 128), 128, 0, st>>>(act.a3, lv[3], act.a4, lv[3],
                                                                       wb + L.w4, wf + L.b4);
    return cudaGetLastError();
}

cudaError_t net_logits(const NetLayout& L, const __nv_bfloat16* wb, const float* wf, const float* a4,
                       int n_tiles, float* logits, cudaStream_t st) {
    if (n_tiles <= 0) return cudaSuccess;
    net_logits_kernel<<<n_tiles, 256, 0, st>>>(a4, L.S, wb + L.wh, wf + L.bh, logits);
    return cudaGetLastError();
}

static int per_block_for(long long n, int target_blocks) {
    long long p = (n + target_blocks - 1) / target_blocks;
    return (int)(p < 16 ? 16 : p);
}

cudaError_t net_backward(const NetLayout& L, const __nv_bfloat16* wb, const float* wf, const NetIn& in,
                         const NetActs& act, const float* target, float inv_n,
                         const NetGradScratch& s, float* grad, double* loss, cudaStream_t st,
                         const NetTc& tc) {
    Dim3i lv[4];
    net_levels(in.nx, in.ny, in.nz, lv);
    const int n_tiles = (int)nvox(lv[3]);
    const size_t hsm = (size_t)L.S * 4;
    if (hsm > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(net_head_train_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsm);
        if (e != cudaSuccess) return e;
    }
    net_head_train_kernel<<<n_tiles, 256, hsm, st>>>(act.a4, L.S, wb + L.wh, wf + L.bh, target, inv_n,
                                                     s.g_logit, s.d4, loss);
    INLM_LAUNCH_CHECK();
    {
        const int tpb = 256;
        dim3 g((L.S + 127) / 128, (n_tiles + tpb - 1) / tpb);
        net_head_wgrad_kernel<<<g, 128, 0, st>>>(s.g_logit, act.a4, n_tiles, L.S, tpb, grad + L.wh,
                                                 grad + L.bh);
        INLM_LAUNCH_CHECK();
    }
    const int nb = 148 * 4;
    // L4 (stride 1, level 3 -> level 3)
    {
        int pb = per_block_for(nvox(lv[3]), nb);
        net_conv_wgrad_kernel<1><<<(int)((nvox(lv[3]) + pb - 1) / pb), 256, 0, st>>>(
            act.a3, lv[3], s.d4, lv[3], pb, grad + L.w4, grad + L.b4);
        INLM_LAUNCH_CHECK();
        if (tc.on) {
            cudaError_t e = net_conv_dgrad_tc(s.d4, lv[3], wb + L.w4, act.a3, lv[3], s.d3, 1, tc.err, st);
            if (e != cudaSuccess) return e;
        } else {
            net_conv_dgrad_kernel<1><<<grid_for(nvox(lv[3]), 128), 128, 0, st>>>(s.d4, lv[3], wb + L.w4,
                                                                                 act.a3, lv[3], s.d3);
            INLM_LAUNCH_CHECK();
        }
    }
    // L3 (stride 2, level 2 -> level 3)
    {
        int pb = per_block_for(nvox(lv[3]), nb);
        net_conv_wgrad_kernel<2><<<(int)((nvox(lv[3]) + pb - 1) / pb), 256, 0, st>>>(
            act.a2, lv[2], s.d3, lv[3], pb, grad + L.w3, grad + L.b3);
        INLM_LAUNCH_CHECK();
        if (tc.on) {
            cudaError_t e = net_conv_dgrad_tc(s.d3, lv[3], wb + L.w3, act.a2, lv[2], s.d2, 2, tc.err, st);
            if (e != cudaSuccess) return e;
        } else {
            net_conv_dgrad_kernel<2><<<grid_for(nvox(lv[2]), 128), 128, 0, st>>>(s.d3, lv[3], wb + L.w3,
                                                                                 act.a2, lv[2], s.d2);
            INLM_LAUNCH_CHECK();
        }
    }
    // L2 (stride 2, level 1 -> level 2)
    {
        int pb = per_block_for(nvox(lv[2]), nb);
        net_conv_wgrad_kernel<2><<<(int)((nvox(lv[2]) + pb - 1) / pb), 256, 0, st>>>(
            act.a1, lv[1], s.d2, lv[2], pb, grad + L.w2, grad + L.b2);
        INLM_LAUNCH_CHECK();
        if (tc.on) {
            cudaError_t e = net_conv_dgrad_tc(s.d2, lv[2], wb + L.w2, act.a1, lv[1], s.d1, 2, tc.err, st);
            if (e != cudaSuccess) return e;
        } else {
            net_conv_dgrad_kernel<2><<<grid_for(nvox(lv[1]), 128), 128, 0, st>>>(s.d2, lv[2], wb + L.w2,
                                                                                 act.a1, lv[1], s.d1);
            INLM_LAUNCH_CHECK();
        }
    }
    // L1
    {
        int pb = per_block_for(nvox(lv[1]), nb);
        const int blocks = (int)((nvox(lv[1]) + pb - 1) / pb);
        if (in.half)
            net_l1_wgrad_kernel<__half><<<blocks, 432, 0, st>>>(in, lv[1], s.d1, pb, grad + L.w1,
                                                                grad + L.b1);
        else
            net_l1_wgrad_kernel<float><<<blocks, 432, 0, st>>>(in, lv[1], s.d1, pb, grad + L.w1,
                                                               grad + L.b1);
    }
    return cudaGetLastError();
}

cudaError_t net_adam(float* w, float* m, float* v, const float* g, __nv_bfloat16* wb, long long n,
                     float lr, float beta1, float beta2, float eps, float bc1, float bc2,
                     cudaStream_t st) {
    net_adam_kernel<<<grid_for(n, 256), 256, 0, st>>>(w, m, v, g, wb, n, lr, beta1, beta2, eps, bc1,
                                                      bc2);
    return cudaGetLastError();
}

cudaError_t net_round_bf16(const float* w, __nv_bfloat16* wb, long long n, cudaStream_t st) {
    net_round_kernel<<<grid_for(n, 256), 256, 0, st>>>(w, wb, n);
    return cudaGetLastError();
}

cudaError_t net_select(const NetLayout& L, const __nv_bfloat16* wb, const float* wf, const float* a4,
                       int n_tiles, int K, float min_mass, unsigned* bitmap, int nwords,
                       float* pred_mass, int* counters, cudaStream_t st) {
    if (n_tiles <= 0) return cudaSuccess;
    const size_t sm = (size_t)kSelWarps * ((L.S + 3) / 4 * 4 + 256) * 4;
    if (sm > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(net_select_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
    }
    const long long blocks = ((long long)n_tiles + kSelWarps - 1) / kSelWarps;
    net_select_kernel<<<(unsigned)blocks, 32 * kSelWarps, sm, st>>>(
        a4, n_tiles, L.S, wb + L.wh, wf + L.bh, K, min_mass, bitmap, nwords, pred_mass, counters);
    return cudaGetLastError();
}

cudaError_t net_select_group(const NetLayout& L, const __nv_bfloat16* wb, const float* wf, const float* a4,
                             Dim3i t8, int G, int K, float min_mass, unsigned* bitmap, int nwords,
                             float* pred_mass, int* counters, cudaStream_t st) {
    const int gx = (t8.x + G - 1) / G;
    const long long n_groups = (long long)gx * t8.y * t8.z;
    if (n_groups <= 0) return cudaSuccess;
    const size_t sm = (size_t)kSelWarps * (2 * ((L.S + 3) / 4 * 4) + 256) * 4;
    cudaError_t e = cudaFuncSetAttribute(net_select_group_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    const long long blocks = (n_groups + kSelWarps - 1) / kSelWarps;
    net_select_group_kernel<<<(unsigned)blocks, 32 * kSelWarps, sm, st>>>(
        a4, t8.x, n_groups, gx, G, L.S, wb + L.wh, wf + L.bh, K, min_mass, bitmap, nwords, pred_mass,
        counters);
    return cudaGetLastError();
}

cudaError_t net_plan_tiles(const unsigned* bitmap, int nwords, long long n_tiles, int S,
                           int* plan_off, int* plan_count, int* counters, cudaStream_t st,
                           const float* pred_mass, double* mass_sum, float rel) {
    if (n_tiles <= 0) return cudaSuccess;
    if (rel > 0.f) {
        net_mass_sum_kernel<<<1, 1024, 0, st>>>(pred_mass, n_tiles, mass_sum);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    const long long blocks = (n_tiles * 32 + 127) / 128;
    net_plan_tiles_kernel<<<(unsigned)blocks, 128, 0, st>>>(bitmap, nwords, n_tiles, S, plan_off,
                                                            plan_count, counters, pred_mass, mass_sum, rel);
    return cudaGetLastError();
}

cudaError_t net_scale_from_mult(const float* mult, int nz, float* scale, cudaStream_t st) {
    net_scale_kernel<<<(nz + 255) / 256, 256, 0, st>>>(mult, nz, scale);
    return cudaGetLastError();
}

cudaError_t unpad_half_to_float(const void* padded, long long py, long long pz, int px, int pyy,
                                int pz0, int nx, int ny, int nz, float* out, cudaStream_t st) {
    const __half* base = static_cast<const __half*>(padded) + pz0 * pz + pyy * py + px;
    unpad_half_kernel<<<grid_for((long long)nx * ny * nz, 256), 256, 0, st>>>(base, py, pz, nx, ny, nz,
                                                                             out);
    return cudaGetLastError();
}

cudaError_t normalise_rows(float* map, long long rows, int S, cudaStream_t st) {
    if (rows <= 0) return cudaSuccess;
    normalise_rows_kernel<<<(unsigned)rows, 256, 0, st>>>(map, S);
    return cudaGetLastError();
}

}  // namespace inlm
