// RGB filter kernel: one CTA per 32 x 8 pixel tile, the three channels of the
// previous iterate staged in shared memory over the tile plus search and
// patch halo, the raw channels over the tile plus search halo, reflective
// padding applied while staging (no padded copies). One thread per pixel
// evaluates every search offset in reference order with the reference's
// rounding: per tap and channel a separately rounded square, weight product
// and sum; the joint distance (d0 + d1 + d2) / 3; the Pade[3/3] weight under
// the cutoff; sums of w * raw per channel, the weight sum and the maximum
// weight (IterativeNLM_CPU::filterslice_3channels, iternlm_cpu.cpp:932-1075).
#include "color_kernels.cuh"

namespace inlm {

namespace {

// mirror without edge repeat, repeated while out of range
// (pad_reflective, iternlm_prepare.cpp:28-37)
__device__ __forceinline__ int reflect(int i, int n) {
    while (i < 0 || i >= n) {
        if (i < 0) i = -i;
        if (i >= n) i = 2 * n - i - 2;
    }
    return i;
}

// expapproximation (iternlm_cpu.h:125) with the reference's association:
// ((120 + 60x) + (12x)x + (xx)x) / ((120 - 60x) + (12x)x - (xx)x)
__device__ __forceinline__ float pade(float x) {
    const float t60 = __fmul_rn(60.f, x);
    const float t12 = __fmul_rn(__fmul_rn(12.f, x), x);
    const float t3 = __fmul_rn(__fmul_rn(x, x), x);
    const float num = __fadd_rn(__fadd_rn(__fadd_rn(120.f, t60), t12), t3);
    const float den = __fsub_rn(__fadd_rn(__fsub_rn(120.f, t60), t12), t3);
    return __fdiv_rn(num, den);
}

constexpr float kCutoff = -3.56648f;  // iternlm_cpu.h:126

__global__ void __launch_bounds__(kRgbTX * kRgbTY) nlm_rgb_kernel(const RgbArgs a) {
    extern __shared__ float sm[];
    const int X0 = blockIdx.x * kRgbTX, Y0 = blockIdx.y * kRgbTY;
    const int pw = kRgbTX + 2 * a.hx, ph = kRgbTY + 2 * a.hy;  // prev tile
    const int rw = kRgbTX + 2 * a.sx, rh = kRgbTY + 2 * a.sy;  // raw tile
    float* sp = sm;                  // 3 x ph x pw
    float* sr = sm + 3 * pw * ph;    // 3 x rh x rw
    const int tid = threadIdx.y * kRgbTX + threadIdx.x;
    const int nt = kRgbTX * kRgbTY;
    for (int i = tid; i < pw * ph; i += nt) {
        const int yy = i / pw, xx = i - yy * pw;
        const int gx = reflect(X0 - a.hx + xx, a.nx), gy = reflect(Y0 - a.hy + yy, a.ny);
        const long long g = (long long)gy * a.nx + gx;
#pragma unroll
        for (int c = 0; c < 3; c++) sp[c * pw * ph + i] = a.prev[c][g];
    }
    for (int i = tid; i < rw * rh; i += nt) {
        const int yy = i / rw, xx = i - yy * rw;
        const int gx = reflect(X0 - a.sx + xx, a.nx), gy = reflect(Y0 - a.sy + yy, a.ny);
        const long long g = (long long)gy * a.nx + gx;
#pragma unroll
        for (int c = 0; c < 3; c++) sr[c * rw * rh + i] = a.raw[c][g];
    }
    __syncthreads();
    const int x = X0 + threadIdx.x, y = Y0 + threadIdx.y;
    if (x >= a.nx || y >= a.ny) return;

    const int po = (threadIdx.y + a.hy) * pw + threadIdx.x + a.hx;  // origin in the prev tile
    const int ro = (threadIdx.y + a.sy) * rw + threadIdx.x + a.sx;  // origin in the raw tile
    const int pch = pw * ph, rch = rw * rh;
    float fv[3] = {0.f, 0.f, 0.f}, fw[3] = {0.f, 0.f, 0.f}, mw[3] = {0.f, 0.f, 0.f};
    for (int s = 0; s < a.S; s++) {
        const int2 o = __ldg(&a.search[s]);
        const int pq = po + o.y * pw + o.x;
        float d[3] = {0.f, 0.f, 0.f};
        for (int q = 0; q < a.P; q++) {
            const int2 t = __ldg(&a.taps[q]);
            const float dw = __ldg(&a.w[q]);
            const int tt = t.y * pw + t.x;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float tmp = __fsub_rn(sp[c * pch + pq + tt], sp[c * pch + po + tt]);
                d[c] = __fadd_rn(d[c], __fmul_rn(__fmul_rn(tmp, tmp), dw));
            }
        }
#pragma unroll
        for (int c = 0; c < 3; c++) d[c] = __fmul_rn(d[c], a.mult[c]);
        const int rq = ro + o.y * rw + o.x;
        if (!a.independent) {
            const float ds = __fdiv_rn(__fadd_rn(__fadd_rn(d[0], d[1]), d[2]), 3.f);
            const float wt = (ds > kCutoff) ? pade(ds) : 0.0f;
#pragma unroll
            for (int c = 0; c < 3; c++) fv[c] = __fadd_rn(fv[c], __fmul_rn(wt, sr[c * rch + rq]));
            fw[0] = __fadd_rn(fw[0], wt);
            if (wt > mw[0]) mw[0] = wt;
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float wt = (d[c] > kCutoff) ? pade(d[c]) : 0.0f;
                fv[c] = __fadd_rn(fv[c], __fmul_rn(wt, sr[c * rch + rq]));
                fw[c] = __fadd_rn(fw[c], wt);
                if (wt > mw[c]) mw[c] = wt;
            }
        }
    }
    const long long g = (long long)y * a.nx + x;
    if (!a.independent) {
        if (mw[0] > 0.0f) {
            const float wsum = __fadd_rn(fw[0], mw[0]);
#pragma unroll
            for (int c = 0; c < 3; c++)
                a.out[c][g] = __fdiv_rn(__fadd_rn(fv[c], __fmul_rn(mw[0], sr[c * rch + ro])), wsum);
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++) a.out[c][g] = sr[c * rch + ro];
        }
    } else {
        // independent channels: no centre term (iternlm_cpu.cpp:1055-1060)
#pragma unroll
        for (int c = 0; c < 3; c++) a.out[c][g] = (mw[c] > 0.0f) ? __fdiv_rn(fv[c], fw[c]) : sr[c * rch + ro];
    }
}

__global__ void anscombe_kernel(float* v, long long n, bool inverse) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float r = v[i];
        if (inverse) {
            const float h = __fdiv_rn(r, 2.f);
            v[i] = __fsub_rn(__fmul_rn(h, h), 0.375f);  // (r/2)(r/2) - 3/8
        } else {
            v[i] = __fmul_rn(2.f, __fsqrt_rn(__fadd_rn(r, 0.375f)));  // 2 sqrt(r + 3/8)
        }
    }
}

}  // namespace

size_t rgb_smem_bytes(const RgbArgs& a) {
    const size_t pw = kRgbTX + 2 * a.hx, ph = kRgbTY + 2 * a.hy;
    const size_t rw = kRgbTX + 2 * a.sx, rh = kRgbTY + 2 * a.sy;
    return 3 * 4 * (pw * ph + rw * rh);
}

cudaError_t launch_rgb_filter(const RgbArgs& a, cudaStream_t st) {
    const size_t smem = rgb_smem_bytes(a);
    cudaError_t e = cudaFuncSetAttribute(nlm_rgb_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((a.nx + kRgbTX - 1) / kRgbTX, (a.ny + kRgbTY - 1) / kRgbTY);
    nlm_rgb_kernel<<<grid, dim3(kRgbTX, kRgbTY), smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_anscombe(float* v, long long n, bool inverse, cudaStream_t st) {
    anscombe_kernel<<<148 * 4, 256, 0, st>>>(v, n, inverse);
    return cudaGetLastError();
}

}  // namespace inlm
