// RGB filter kernel: one CTA per 32 x 8 pixel tile, the three channels of the
// previous iterate staged in shared memory over the tile plus search and
// patch halo, the raw channels over the tile plus search halo, reflective
// padding applied while staging (no padded copies). One thread per pixel
// evaluates every search offset in reference order with the reference's
// rounding: per tap and channel a separately rounded square, weight product
// and sum; the joint distance (d0 + d1 + d2) / 3; the Pade[3/3] weight under
// the cutoff; sums of w * raw per channel, the weight sum and the maximum
// weight (IterativeNLM_CPU::filterslice_3channels, iternlm_cpu.cpp:932-1075).
#include <utility>

#include "color_kernels.cuh"
#include "geometry.hpp"

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

// Compile-time 2D tap table of patch radius (R, R) in reference order: the
// centre, then y ascending, x ascending inside the ellipse.
template <int R>
struct RgbTaps {
    static constexpr PatchRows rows = make_patch_rows(R, R, 0);
    static constexpr int P = rows.ntaps;
    struct Table {
        int dx[64], dy[64];
    };
    static constexpr Table make() {
        Table t{};
        int n = 1;
        for (int ri = 0; ri < rows.n; ri++)
            for (int xp = -rows.e[ri]; xp <= rows.e[ri]; xp++)
                if (!(rows.yp[ri] == 0 && xp == 0)) {
                    t.dx[n] = xp;
                    t.dy[n] = rows.yp[ri];
                    n++;
                }
        return t;
    }
};

// Tap Q of patch radius R (compile-time offsets from the table).
template <int R, int Q>
__device__ __forceinline__ void load_origin_tap(float (&vo)[3][RgbTaps<R>::P], float (&w)[RgbTaps<R>::P],
                                                const float* sp, int pch, int po, int pw, const float* wt) {
    constexpr auto t = RgbTaps<R>::make();
    w[Q] = __ldg(&wt[Q]);
#pragma unroll
    for (int c = 0; c < 3; c++) vo[c][Q] = sp[c * pch + po + t.dy[Q] * pw + t.dx[Q]];
}
template <int R, int Q>
__device__ __forceinline__ void dist_tap(float (&d)[3], const float (&vo)[3][RgbTaps<R>::P],
                                         const float (&w)[RgbTaps<R>::P], const float* sp, int pch, int pq,
                                         int pw) {
    constexpr auto t = RgbTaps<R>::make();
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float tmp = __fsub_rn(sp[c * pch + pq + t.dy[Q] * pw + t.dx[Q]], vo[c][Q]);
        d[c] = __fadd_rn(d[c], __fmul_rn(__fmul_rn(tmp, tmp), w[Q]));
    }
}
template <int R, int... Q>
__device__ __forceinline__ void load_origin(std::integer_sequence<int, Q...>, float (&vo)[3][RgbTaps<R>::P],
                                            float (&w)[RgbTaps<R>::P], const float* sp, int pch, int po,
                                            int pw, const float* wt) {
    (load_origin_tap<R, Q>(vo, w, sp, pch, po, pw, wt), ...);
}
// taps in reference order (the comma fold runs left to right)
template <int R, int... Q>
__device__ __forceinline__ void dist_all(std::integer_sequence<int, Q...>, float (&d)[3],
                                         const float (&vo)[3][RgbTaps<R>::P], const float (&w)[RgbTaps<R>::P],
                                         const float* sp, int pch, int pq, int pw) {
    (dist_tap<R, Q>(d, vo, w, sp, pch, pq, pw), ...);
}

// The same filter with the patch unrolled: the origin's patch values and the
// weights stay in registers across all offsets, one row base per (channel,
// patch row) per offset and the taps of a row as immediate offsets. Same
// operations in the same order as nlm_rgb_kernel.
template <int R>
__global__ void __launch_bounds__(kRgbTX * kRgbTY) nlm_rgb_tap_kernel(const RgbArgs a) {
    using T = RgbTaps<R>;
    constexpr int P = T::P;
    extern __shared__ float sm[];
    const int X0 = blockIdx.x * kRgbTX, Y0 = blockIdx.y * kRgbTY;
    const int pw = kRgbTX + 2 * a.hx, ph = kRgbTY + 2 * a.hy;
    const int rw = kRgbTX + 2 * a.sx, rh = kRgbTY + 2 * a.sy;
    float* sp = sm;
    float* sr = sm + 3 * pw * ph;
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

    const int pch = pw * ph, rch = rw * rh;
    const int po = (threadIdx.y + a.hy) * pw + threadIdx.x + a.hx;
    const int ro = (threadIdx.y + a.sy) * rw + threadIdx.x + a.sx;
    float w[P], vo[3][P];
    load_origin<R>(std::make_integer_sequence<int, P>{}, vo, w, sp, pch, po, pw, a.w);
    float fv[3] = {0.f, 0.f, 0.f}, fw[3] = {0.f, 0.f, 0.f}, mw[3] = {0.f, 0.f, 0.f};
    for (int s = 0; s < a.S; s++) {
        const int2 o = __ldg(&a.search[s]);
        const int pq = po + o.y * pw + o.x;
        float d[3] = {0.f, 0.f, 0.f};
        dist_all<R>(std::make_integer_sequence<int, P>{}, d, vo, w, sp, pch, pq, pw);
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

template <int R>
static int tap_order_impl(int* dxdy, int max_taps) {
    using T = RgbTaps<R>;
    constexpr auto t = T::make();
    for (int q = 0; q < T::P && q < max_taps; q++) {
        dxdy[2 * q] = t.dx[q];
        dxdy[2 * q + 1] = t.dy[q];
    }
    return T::P;
}

int rgb_tap_order(int r, int* dxdy, int max_taps) {
    switch (r) {
        case 1: return tap_order_impl<1>(dxdy, max_taps);
        case 2: return tap_order_impl<2>(dxdy, max_taps);
        case 3: return tap_order_impl<3>(dxdy, max_taps);
        default: return -1;
    }
}

template <typename K>
static cudaError_t launch_with(K kern, const RgbArgs& a, cudaStream_t st) {
    const size_t smem = rgb_smem_bytes(a);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((a.nx + kRgbTX - 1) / kRgbTX, (a.ny + kRgbTY - 1) / kRgbTY);
    kern<<<grid, dim3(kRgbTX, kRgbTY), smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_rgb_filter(const RgbArgs& a, cudaStream_t st) {
    switch (a.tap_radius) {
        case 1: return launch_with(nlm_rgb_tap_kernel<1>, a, st);
        case 2: return launch_with(nlm_rgb_tap_kernel<2>, a, st);
        case 3: return launch_with(nlm_rgb_tap_kernel<3>, a, st);
        default: return launch_with(nlm_rgb_kernel, a, st);
    }
}

cudaError_t launch_anscombe(float* v, long long n, bool inverse, cudaStream_t st) {
    anscombe_kernel<<<148 * 4, 256, 0, st>>>(v, n, inverse);
    return cudaGetLastError();
}

}  // namespace inlm
