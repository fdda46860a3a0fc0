// Column form of the plain FP32 iterNLM filter for small patches (sm_100a),
// bit-identical to the reference CPU filter like the tile kernel
// (Denoiser/iternlm_cpu_kernels.cpp:7-160 for patch radius 1,
// iternlm_cpu.cpp:758-843).
//
// At patch radius 1 (7 taps, the reference's default) the tile kernel's
// squared-difference planes save little: each D value serves 7 voxels, but
// forming the planes, the two barriers around them and the prev box with the
// whole search halo (one 8-warp CTA per SM) cost more than the taps. Here a
// CTA stages the same prev box by one TMA load and then runs without
// barriers: a warp owns 32 consecutive x voxels on 8 rows of one z plane,
// each thread its 8 voxels along y. The patch splits into columns of constant
// (zp, xp) with yp in [-e, e]; per search offset a thread reads each column of
// the shifted previous iterate at y in [-e, 7 + e] (a warp load is 32
// consecutive floats: no bank conflict), forms the squared differences
// against the origin values it keeps in registers (the same D values the
// tile kernel stores), and adds w * D in the reference's tap order for every
// voxel. Raw comes from global memory, one offset ahead. FUSED = true is the
// fused FP32 form: each tap one fused multiply-add, the Horner Pade with a
// fast division (not bit-identical; within 1e-4 relative of the reference
// except where a weight crosses the cutoff).
#include <cuda_fp16.h>

#include "common.cuh"
#include "filter_fast.cuh"
#include "filter_kernels.cuh"
#include "geometry.hpp"
#include "pair_math.cuh"
#include "tile_common.cuh"

namespace inlm {

namespace {

// Patch columns: constant (zp, xp), yp in [-e, e] (the ellipsoid is convex
// and symmetric, so each column is one symmetric run). first[c]: register
// offset of the column's 8 + 2e values in the per-thread arrays.
struct PatchCols {
    int n;
    int zp[64], xp[64], e[64], first[64];
    int nvals;
};

constexpr PatchCols make_patch_cols(int rx, int ry, int rz) {
    PatchCols c{};
    const float fx = float(rx < 1 ? 1 : rx), fy = float(ry < 1 ? 1 : ry), fz = float(rz < 1 ? 1 : rz);
    for (int zp = -rz; zp <= rz; zp++)
        for (int xp = -rx; xp <= rx; xp++) {
            if (!ell_member(xp, 0, zp, fx, fy, fz)) continue;
            int e = 0;
            while (e + 1 <= ry && ell_member(xp, e + 1, zp, fx, fy, fz)) e++;
            c.zp[c.n] = zp;
            c.xp[c.n] = xp;
            c.e[c.n] = e;
            c.first[c.n] = c.nvals;
            c.nvals += kVoxPerThread + 2 * e;
            c.n++;
        }
    return c;
}

constexpr int col_of(const PatchCols& c, int zp, int xp) {
    for (int i = 0; i < c.n; i++)
        if (c.zp[i] == zp && c.xp[i] == xp) return i;
    return -1;
}

// Reference tap order (centre first, then rows (zp, yp) ascending, xp
// ascending), each tap as (column, yp).
struct TapSeq {
    int n;
    int col[128], yp[128];
};

constexpr TapSeq make_tap_seq(int rx, int ry, int rz) {
    const PatchRows rows = make_patch_rows(rx, ry, rz);
    const PatchCols cols = make_patch_cols(rx, ry, rz);
    TapSeq t{};
    t.col[0] = col_of(cols, 0, 0);
    t.yp[0] = 0;
    t.n = 1;
    for (int r = 0; r < rows.n; r++)
        for (int xp = -rows.e[r]; xp <= rows.e[r]; xp++) {
            if (rows.zp[r] == 0 && rows.yp[r] == 0 && xp == 0) continue;
            t.col[t.n] = col_of(cols, rows.zp[r], xp);
            t.yp[t.n] = rows.yp[r];
            t.n++;
        }
    return t;
}

template <int RX, int RY, int RZ>
struct ColGeom {
    static constexpr PatchCols cols = make_patch_cols(RX, RY, RZ);
    static constexpr TapSeq taps = make_tap_seq(RX, RY, RZ);
    static constexpr int NV = cols.nvals;  // values per thread over all columns
};

static_assert(ColGeom<1, 1, 1>::taps.n == 7 && ColGeom<1, 1, 1>::NV == 42, "p111 columns");
static_assert(ColGeom<1, 1, 2>::taps.n == 9, "p112 columns");
static_assert(ColGeom<1, 1, 3>::taps.n == 11, "p113 columns");

// First tap (in reference order) that reads column C: the column's squared
// differences are formed there, so each lives only from its first to its last
// use.
template <int RX, int RY, int RZ, int C>
constexpr int first_use() {
    using CG = ColGeom<RX, RY, RZ>;
    for (int t = 0; t < CG::taps.n; t++)
        if (CG::taps.col[t] == C) return t;
    return -1;
}

// Squared differences of column C for offset delta dlx: D[first + i] for y in
// [-e, 7 + e], as register pairs (the column length 8 + 2e is even).
template <int RX, int RY, int RZ, int C>
__device__ __forceinline__ void column_d(const float* __restrict__ prevb, int pb, int dlx, int pbx,
                                         int pplane, const f32x2 (&og)[ColGeom<RX, RY, RZ>::NV / 2],
                                         f32x2 (&D)[ColGeom<RX, RY, RZ>::NV / 2]) {
    using CG = ColGeom<RX, RY, RZ>;
    constexpr int e = CG::cols.e[C];
    constexpr int f = CG::cols.first[C];
    const float* src = prevb + pb + dlx + CG::cols.zp[C] * pplane + CG::cols.xp[C] - e * pbx;
#pragma unroll
    for (int i = 0; i < kVoxPerThread + 2 * e; i += 2) {
        const f32x2 v = pack2(src[i * pbx], src[(i + 1) * pbx]);
        const f32x2 t = sub2(v, og[(f + i) / 2]);
        D[(f + i) / 2] = mul2_to_mul(t, t);  // feeds only products
    }
}

// Taps T.. of the reference order: form each column at its first use, then
// add w_t * D to the 8 voxels' distances (pairs of y voxels).
template <int RX, int RY, int RZ, int T, bool FUSED>
__device__ __forceinline__ void column_taps(const float* __restrict__ prevb, int pb, int dlx, int pbx,
                                            int pplane, const f32x2 (&og)[ColGeom<RX, RY, RZ>::NV / 2],
                                            f32x2 (&D)[ColGeom<RX, RY, RZ>::NV / 2],
                                            f32x2 (&d)[kVoxPerThread / 2], const TileArgs& a) {
    using CG = ColGeom<RX, RY, RZ>;
    if constexpr (T < CG::taps.n) {
        constexpr int C = CG::taps.col[T];
        constexpr int yp = CG::taps.yp[T];
        constexpr int e = CG::cols.e[C];
        constexpr int f = CG::cols.first[C];
        if constexpr (first_use<RX, RY, RZ, C>() == T) column_d<RX, RY, RZ, C>(prevb, pb, dlx, pbx, pplane, og, D);
        const float w = a.w[T];
#pragma unroll
        for (int p = 0; p < kVoxPerThread / 2; p++) {
            // voxels 2p, 2p + 1 read the column at y = 2p + yp, 2p + 1 + yp
            // (value index y + e; every column starts on a pair)
            const int i = f + e + 2 * p + yp;
            const float2 lo = unpack2(D[i / 2]);
            float v0, v1;
            if ((i & 1) == 0) {
                v0 = lo.x;
                v1 = lo.y;
            } else {
                const float2 hi = unpack2(D[i / 2 + 1]);
                v0 = lo.y;
                v1 = hi.x;
            }
            if (T == 0)
                d[p] = mul_pair(v0, v1, w);
            else if (FUSED)
                d[p] = fma2(pack2(v0, v1), splat2(w), d[p]);
            else
                d[p] = add2(d[p], mul_pair(v0, v1, w));
        }
        column_taps<RX, RY, RZ, T + 1, FUSED>(prevb, pb, dlx, pbx, pplane, og, D, d, a);
    }
}

// Origin values of columns C.. (the unshifted previous iterate), as pairs.
template <int RX, int RY, int RZ, int C>
__device__ __forceinline__ void load_origins(const float* __restrict__ prevb, int pb, int pbx, int pplane,
                                             f32x2 (&og)[ColGeom<RX, RY, RZ>::NV / 2]) {
    using CG = ColGeom<RX, RY, RZ>;
    if constexpr (C < CG::cols.n) {
        constexpr int e = CG::cols.e[C];
        constexpr int f = CG::cols.first[C];
        const float* src = prevb + pb + CG::cols.zp[C] * pplane + CG::cols.xp[C] - e * pbx;
#pragma unroll
        for (int i = 0; i < kVoxPerThread + 2 * e; i += 2) og[(f + i) / 2] = pack2(src[i * pbx], src[(i + 1) * pbx]);
        load_origins<RX, RY, RZ, C + 1>(prevb, pb, pbx, pplane, og);
    }
}

template <int RX, int RY, int RZ, int TZ, bool FUSED>
__global__ void __launch_bounds__(32 * TZ, 1)
    nlm_column_f32_kernel(const __grid_constant__ CUtensorMap tm_prev, const __grid_constant__ TileArgs a) {
    using CG = ColGeom<RX, RY, RZ>;
    constexpr int NP = kVoxPerThread / 2;
    constexpr int NV2 = CG::NV / 2;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    float* prevb = reinterpret_cast<float*>(smem + 128);
    const int tid = threadIdx.x;
    const int X0 = blockIdx.x * kTX;
    const int Y0 = blockIdx.y * kTY;
    const int Z0 = blockIdx.z * TZ;
    const int pplane = a.pbx * a.pby;
    if (tid == 0) {
        prefetch_tmap(&tm_prev);
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        mbar_arrive_expect_tx(bar, (uint32_t)(pplane * a.pbz) * 4u);
        tma_load_3d(prevb, &tm_prev, X0, Y0, Z0, bar);
    }
    // lane = x within the CTA's 32 columns, warp = z plane; voxels y = 0..7
    const int lane = tid & 31, k = tid >> 5;
    const int pb = (k + a.pz) * pplane + a.py * a.pbx + lane + a.px;  // voxel (lane, 0, k)
    const long long gbase = (long long)(Z0 + k + a.pz) * a.gpitch_z + (long long)(Y0 + a.py) * a.gpitch_y +
                            (X0 + lane + a.px);
    const f32x2 m2 = splat2(a.mult[min(Z0 + k, a.nz - 1)]);

    // raw of the first offset, loaded while the prev box arrives
    int2 dl = __ldg(&a.search_delta[0]);
    float rn[kVoxPerThread];
#pragma unroll
    for (int r = 0; r < kVoxPerThread; r++) rn[r] = __ldg(&a.raw_pad[gbase + r * a.gpitch_y + dl.y]);

    const bool arrived = mbar_wait_bounded(bar, 0);
    if (!__syncthreads_and(arrived)) {
        if (tid == 0) set_error(a.err, DEV_TMA_TIMEOUT);
        return;
    }
    // origin values of every column, kept for all offsets
    f32x2 og[NV2];
    load_origins<RX, RY, RZ, 0>(prevb, pb, a.pbx, pplane, og);

    f32x2 acc[NP], wsum[NP];
    float wmax[kVoxPerThread];
#pragma unroll
    for (int p = 0; p < NP; p++) acc[p] = wsum[p] = 0ull;  // (+0, +0)
#pragma unroll
    for (int r = 0; r < kVoxPerThread; r++) wmax[r] = 0.0f;

    for (int s = 0; s < a.S; s++) {
        float rc[kVoxPerThread];
#pragma unroll
        for (int r = 0; r < kVoxPerThread; r++) rc[r] = rn[r];
        const int2 dln = __ldg(&a.search_delta[min(s + 1, a.S - 1)]);
        if (s + 1 < a.S) {
#pragma unroll
            for (int r = 0; r < kVoxPerThread; r++) rn[r] = __ldg(&a.raw_pad[gbase + r * a.gpitch_y + dln.y]);
        }
        f32x2 D[NV2];
        f32x2 d[NP];
        column_taps<RX, RY, RZ, 0, FUSED>(prevb, pb, dl.x, a.pbx, pplane, og, D, d, a);
#pragma unroll
        for (int p = 0; p < NP; p++) {
            if (FUSED)
                fused_weight_pair(d[p], m2, make_float2(rc[2 * p], rc[2 * p + 1]), acc[p], wsum[p], wmax[2 * p],
                                  wmax[2 * p + 1]);
            else
                exact_weight_pair(d[p], m2, make_float2(rc[2 * p], rc[2 * p + 1]), acc[p], wsum[p], wmax[2 * p],
                                  wmax[2 * p + 1]);
        }
        dl = dln;
    }

    const int z = Z0 + k, x = X0 + lane;
    if (z >= a.nz || x >= a.nx) return;
#pragma unroll
    for (int r = 0; r < kVoxPerThread; r++) {
        const int y = Y0 + r;
        if (y >= a.ny) break;
        const float raw0 = __ldg(&a.raw_pad[gbase + r * a.gpitch_y]);
        const float2 acp = unpack2(acc[r / 2]), wsp = unpack2(wsum[r / 2]);
        float ac = (r & 1) ? acp.y : acp.x;
        float ws = (r & 1) ? wsp.y : wsp.x;
        float res;
        if (wmax[r] > 0.0f) {
            ac = __fadd_rn(ac, __fmul_rn(wmax[r], raw0));
            ws = __fadd_rn(ws, wmax[r]);
            res = __fdiv_rn(ac, ws);
        } else {
            res = raw0;
        }
        a.out[((long long)z * a.ny + y) * a.nx + x] = res;
    }
}

template <int RX, int RY, int RZ, int TZ>
cudaError_t launch_column(const CUtensorMap* tm, const TileArgs& a, int tiles_z, size_t smem, bool fused,
                          cudaStream_t st) {
    auto kern = fused ? nlm_column_f32_kernel<RX, RY, RZ, TZ, true> : nlm_column_f32_kernel<RX, RY, RZ, TZ, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid(a.tiles_x, a.tiles_y, tiles_z);
    kern<<<grid, 32 * TZ, smem, st>>>(*tm, a);
    return cudaGetLastError();
}

// Origin values of columns C.. read from the FP16 prev box, as floats.
template <int RX, int RY, int RZ, int C>
__device__ __forceinline__ void load_fast_origins(const __half* __restrict__ prevb, int pb, int pbx, int pplane,
                                                  float (&og)[ColGeom<RX, RY, RZ>::NV]) {
    using CG = ColGeom<RX, RY, RZ>;
    if constexpr (C < CG::cols.n) {
        constexpr int e = CG::cols.e[C];
        constexpr int f = CG::cols.first[C];
        const __half* src = prevb + pb + CG::cols.zp[C] * pplane + CG::cols.xp[C] - e * pbx;
#pragma unroll
        for (int i = 0; i < kVoxPerThread + 2 * e; i++) og[f + i] = __half2float(src[i * pbx]);
        load_fast_origins<RX, RY, RZ, C + 1>(prevb, pb, pbx, pplane, og);
    }
}

// ---- FP16-storage column form ----
//
// The FP16 form's arithmetic voxel for voxel, so its result equals the FP16
// tile kernel's (nlm_tile_fast_kernel) bit for bit: prev and raw read as
// halves; each squared difference formed in FP32 as (t * scale) * t, t =
// prev(. + s) - prev(.), with the scale of the voxel's tile of scale_tz
// planes (the tile kernel's CTA scale); with D_HALF rounded to FP16 and
// summed by half2 fused multiply-adds in tap order (half2 weights), else
// summed by FP32 fused multiply-adds; x = dist * (m / scale); the Pade weight
// in Horner form with a fast division; the weighted sums in FP32 and the
// final normalisation in FP64.

template <int RX, int RY, int RZ, int C, bool D_HALF>
__device__ __forceinline__ void fast_column_d(const __half* __restrict__ prevb, int pb, int dlx, int pbx,
                                              int pplane, float scale,
                                              const float (&og)[ColGeom<RX, RY, RZ>::NV],
                                              __half2 (&Dh)[ColGeom<RX, RY, RZ>::NV / 2],
                                              float (&Df)[ColGeom<RX, RY, RZ>::NV]) {
    using CG = ColGeom<RX, RY, RZ>;
    constexpr int e = CG::cols.e[C];
    constexpr int f = CG::cols.first[C];
    const __half* src = prevb + pb + dlx + CG::cols.zp[C] * pplane + CG::cols.xp[C] - e * pbx;
#pragma unroll
    for (int i = 0; i < kVoxPerThread + 2 * e; i += 2) {
        const float t0 = __half2float(src[i * pbx]) - og[f + i];
        const float t1 = __half2float(src[(i + 1) * pbx]) - og[f + i + 1];
        const float d0 = (t0 * scale) * t0, d1 = (t1 * scale) * t1;
        if constexpr (D_HALF) {
            Dh[(f + i) / 2] = __floats2half2_rn(d0, d1);  // the column starts on a pair
        } else {
            Df[f + i] = d0;
            Df[f + i + 1] = d1;
        }
    }
}

template <int RX, int RY, int RZ, int T, bool D_HALF>
__device__ __forceinline__ void fast_column_taps(const __half* __restrict__ prevb, int pb, int dlx, int pbx,
                                                 int pplane, float scale,
                                                 const float (&og)[ColGeom<RX, RY, RZ>::NV],
                                                 __half2 (&Dh)[ColGeom<RX, RY, RZ>::NV / 2],
                                                 float (&Df)[ColGeom<RX, RY, RZ>::NV],
                                                 __half2 (&dh)[kVoxPerThread / 2],
                                                 float (&dist)[kVoxPerThread], const FastArgs& a) {
    using CG = ColGeom<RX, RY, RZ>;
    if constexpr (T < CG::taps.n) {
        constexpr int C = CG::taps.col[T];
        constexpr int yp = CG::taps.yp[T];
        constexpr int e = CG::cols.e[C];
        constexpr int f = CG::cols.first[C];
        if constexpr (first_use<RX, RY, RZ, C>() == T)
            fast_column_d<RX, RY, RZ, C, D_HALF>(prevb, pb, dlx, pbx, pplane, scale, og, Dh, Df);
        if constexpr (D_HALF) {
            const __half2 w = a.wh[T];
#pragma unroll
            for (int p = 0; p < kVoxPerThread / 2; p++) {
                const int i = f + e + 2 * p + yp;  // voxels 2p, 2p + 1
                const __half2 v = (i & 1) == 0 ? Dh[i / 2]
                                               : __halves2half2(__high2half(Dh[i / 2]), __low2half(Dh[i / 2 + 1]));
                dh[p] = (T == 0) ? __hmul2(v, w) : __hfma2(v, w, dh[p]);
            }
        } else {
            const float w = a.w[T];
#pragma unroll
            for (int r = 0; r < kVoxPerThread; r++) {
                const int i = f + e + r + yp;
                dist[r] = (T == 0) ? Df[i] * w : fmaf(Df[i], w, dist[r]);
            }
        }
        fast_column_taps<RX, RY, RZ, T + 1, D_HALF>(prevb, pb, dlx, pbx, pplane, scale, og, Dh, Df, dh, dist, a);
    }
}

template <int RX, int RY, int RZ, int TZ, bool D_HALF>
__global__ void __launch_bounds__(32 * TZ, 1)
    nlm_column_fast_kernel(const __grid_constant__ CUtensorMap tm_prev, const __grid_constant__ FastArgs a) {
    using CG = ColGeom<RX, RY, RZ>;
    constexpr int NV = CG::NV;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    __half* prevb = reinterpret_cast<__half*>(smem + 128);
    const int tid = threadIdx.x;
    const int X0 = blockIdx.x * kTX;
    const int Y0 = blockIdx.y * kTY;
    const int Z0 = blockIdx.z * TZ;
    const int pplane = a.pbx * a.pby;
    if (tid == 0) {
        prefetch_tmap(&tm_prev);
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        mbar_arrive_expect_tx(bar, (uint32_t)(pplane * a.pbz) * 2u);
        tma_load_3d(prevb, &tm_prev, X0, Y0, Z0, bar);
    }
    const int lane = tid & 31, k = tid >> 5;
    const int pb = (k + a.pz) * pplane + a.py * a.pbx + lane + a.px;
    const long long gbase = (long long)(Z0 + k + a.pz) * a.gpitch_z + (long long)(Y0 + a.py) * a.gpitch_y +
                            (X0 + lane + a.px);
    // the tile kernel's scale: the middle slice of the voxel's scale_tz-plane tile
    const int zt = (Z0 + k) / a.scale_tz * a.scale_tz;
    const float scale = -a.mult[min(zt + a.scale_tz / 2, a.nz - 1)];
    const float rel = a.mult[min(Z0 + k, a.nz - 1)] / scale;

    int2 dl = __ldg(&a.search_delta[0]);
    float rn[kVoxPerThread];
#pragma unroll
    for (int r = 0; r < kVoxPerThread; r++) rn[r] = __half2float(a.raw_pad[gbase + r * a.gpitch_y + dl.y]);

    const bool arrived = mbar_wait_bounded(bar, 0);
    if (!__syncthreads_and(arrived)) {
        if (tid == 0) set_error(a.err, DEV_TMA_TIMEOUT);
        return;
    }
    float og[NV];
    load_fast_origins<RX, RY, RZ, 0>(prevb, pb, a.pbx, pplane, og);

    float acc[kVoxPerThread], wsum[kVoxPerThread], wmax[kVoxPerThread];
#pragma unroll
    for (int r = 0; r < kVoxPerThread; r++) acc[r] = wsum[r] = wmax[r] = 0.0f;

    for (int s = 0; s < a.S; s++) {
        float rc[kVoxPerThread];
#pragma unroll
        for (int r = 0; r < kVoxPerThread; r++) rc[r] = rn[r];
        const int2 dln = __ldg(&a.search_delta[min(s + 1, a.S - 1)]);
        if (s + 1 < a.S) {
#pragma unroll
            for (int r = 0; r < kVoxPerThread; r++)
                rn[r] = __half2float(a.raw_pad[gbase + r * a.gpitch_y + dln.y]);
        }
        __half2 Dh[NV / 2];
        float Df[NV];
        __half2 dh[kVoxPerThread / 2];
        float dist[kVoxPerThread];
        fast_column_taps<RX, RY, RZ, 0, D_HALF>(prevb, pb, dl.x, a.pbx, pplane, scale, og, Dh, Df, dh, dist, a);
        if constexpr (D_HALF) {
#pragma unroll
            for (int p = 0; p < kVoxPerThread / 2; p++) {
                const float2 fd = __half22float2(dh[p]);
                dist[2 * p] = fd.x;
                dist[2 * p + 1] = fd.y;
            }
        }
#pragma unroll
        for (int r = 0; r < kVoxPerThread; r++) {
            const float x = dist[r] * rel;
            // Pade[3/3] of exp in Horner form, FMA
            const float num = fmaf(fmaf(x + 12.f, x, 60.f), x, 120.f);
            const float den = fmaf(fmaf(12.f - x, x, -60.f), x, 120.f);
            const float q = __fdividef(num, den);  // formed, then selected
            const float w = (x > -3.56648f) ? q : 0.0f;
            acc[r] = fmaf(w, rc[r], acc[r]);
            wsum[r] += w;
            wmax[r] = fmaxf(wmax[r], w);
        }
        dl = dln;
    }

    const int z = Z0 + k, x = X0 + lane;
    if (z >= a.nz || x >= a.nx) return;
#pragma unroll
    for (int r = 0; r < kVoxPerThread; r++) {
        const int y = Y0 + r;
        if (y >= a.ny) break;
        const float raw0 = __half2float(a.raw_pad[gbase + r * a.gpitch_y]);
        float res = raw0;
        if (wmax[r] > 0.0f) {
            // per-voxel weight-sum normalisation in FP64
            const double num = (double)acc[r] + (double)wmax[r] * (double)raw0;
            const double den = (double)wsum[r] + (double)wmax[r];
            res = (float)(num / den);
        }
        a.out[((long long)z * a.ny + y) * a.nx + x] = res;
    }
}

}  // namespace

template <int RX, int RY, int RZ, int TZ>
cudaError_t launch_column_fast(const CUtensorMap* tm, const FastArgs& a, int tiles_z, size_t smem, bool d_half,
                               cudaStream_t st) {
    auto kern = d_half ? nlm_column_fast_kernel<RX, RY, RZ, TZ, true> : nlm_column_fast_kernel<RX, RY, RZ, TZ, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid(a.tiles_x, a.tiles_y, tiles_z);
    kern<<<grid, 32 * TZ, smem, st>>>(*tm, a);
    return cudaGetLastError();
}

cudaError_t launch_column_fast_kernel(const FastConfig& c, const CUtensorMap* tm_prev, const FastArgs& a,
                                      int tiles_z, cudaStream_t st) {
    if (c.rx == 1 && c.ry == 1 && c.rz == 1 && c.tz == 16)
        return launch_column_fast<1, 1, 1, 16>(tm_prev, a, tiles_z, c.smem_bytes, c.d_half, st);
    if (c.rx == 1 && c.ry == 1 && c.rz == 2 && c.tz == 8)
        return launch_column_fast<1, 1, 2, 8>(tm_prev, a, tiles_z, c.smem_bytes, c.d_half, st);
    if (c.rx == 1 && c.ry == 1 && c.rz == 3 && c.tz == 8)
        return launch_column_fast<1, 1, 3, 8>(tm_prev, a, tiles_z, c.smem_bytes, c.d_half, st);
    return cudaErrorInvalidConfiguration;
}

int column_kernel_depth(int rx, int ry, int rz) {
    if (rx == 1 && ry == 1 && rz == 1) return 16;
    if (rx == 1 && ry == 1 && (rz == 2 || rz == 3)) return 8;
    return 0;
}

size_t column_smem_bytes(const TileArgs& a) { return 128 + (size_t)a.pbx * a.pby * a.pbz * 4; }

cudaError_t launch_column_kernel(const TileConfig& c, const CUtensorMap* tm_prev, const TileArgs& a,
                                 int tiles_z, cudaStream_t st) {
    if (c.rx == 1 && c.ry == 1 && c.rz == 1 && c.tz == 16)
        return launch_column<1, 1, 1, 16>(tm_prev, a, tiles_z, c.smem_bytes, c.fused, st);
    if (c.rx == 1 && c.ry == 1 && c.rz == 2 && c.tz == 8)
        return launch_column<1, 1, 2, 8>(tm_prev, a, tiles_z, c.smem_bytes, c.fused, st);
    if (c.rx == 1 && c.ry == 1 && c.rz == 3 && c.tz == 8)
        return launch_column<1, 1, 3, 8>(tm_prev, a, tiles_z, c.smem_bytes, c.fused, st);
    return cudaErrorInvalidConfiguration;
}

}  // namespace inlm
