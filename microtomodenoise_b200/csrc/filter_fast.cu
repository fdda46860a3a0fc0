// FP16-storage form of the iterNLM filter (sm_100a).
//
// Same algorithm as the FP32 kernel (filter_kernels.cu) with the precision
// split the fast form uses:
//   * the padded raw and previous-iterate volumes are FP16 in HBM and in
//     shared memory (the previous-iterate box arrives by one 3D TMA load), so
//     two CTAs (16 warps) share an SM;
//   * squared differences D = (prev(.+s) - prev(.))^2 are formed in FP32 and
//     kept in shared memory as FP16 (D_HALF) or FP32, scaled by the tile's
//     1/sigma^2 so FP16 holds them in its normal range;
//   * patch distances: with FP16 D planes, half2 fused multiply-adds on pairs
//     of voxels straight from the FP16 rows (two taps per instruction, no
//     conversions; the weight-mass passes keep FP32 sums); with FP32 D planes,
//     FP32 fused multiply-adds;
//   * Pade weights, weighted sums and weight sums accumulate in FP32 with
//     fused multiply-adds;
//   * the final per-voxel normalisation (acc + wmax*raw)/(wsum + wmax) is FP64.
// Offsets: every search offset, or a per-CTA list of offset indices. With
// TX = 8 a CTA is one 8^3 tile, so a list is the learned proposal's top-K for
// that tile and the tile pays for exactly its own offsets.
// MASS instantiations evaluate every offset and add each offset's weight,
// divided by the voxel's weight sum (from a WSUM-only pass), into a per-8^3-
// tile map: the training targets of the proposal network.
#include <cuda_fp16.h>

#include "common.cuh"
#include "filter_fast.cuh"
#include "tile_common.cuh"

namespace inlm {

// D row pitch for FP16 planes: a multiple of 8 halves (16-byte rows) with an
// odd number of 16-byte chunks, so the warp's row reads spread evenly over
// the bank groups.
constexpr int dpitch_h(int w) {
    int p = (w + 7) / 8 * 8;
    return ((p / 8) % 2 == 0) ? p + 8 : p;
}

template <int RX, int RY, int RZ, int TZ, int TX, bool D_HALF>
struct FastGeom {
    using G = TileGeom<RX, RY, RZ, TZ, TX>;
    static constexpr int DP = D_HALF ? dpitch_h(G::DW) : G::DP;  // elements
    static constexpr int DPLANE = DP * G::DH;
    static constexpr int DSZ = D_HALF ? (DPLANE * G::DD + 63) / 64 * 64
                                      : round_up32(DPLANE * G::DD);  // elements
    static constexpr int DBYTES = DSZ * (D_HALF ? 2 : 4);
};

// 16-value window of one D row (columns [x0, x0+16)) as FP32.
template <bool D_HALF, int LO, int HI>
__device__ __forceinline__ void load_row(const void* rowp, float (&win)[16]) {
    if constexpr (D_HALF) {
        // halves: columns [8c, 8c+8) per 16-byte chunk; convert the span used
#pragma unroll
        for (int c = LO / 8; c <= HI / 8; c++) {
            uint4 v = reinterpret_cast<const uint4*>(rowp)[c];
            const __half2* h = reinterpret_cast<const __half2*>(&v);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int i0 = 8 * c + 2 * q;
                if (i0 + 1 >= LO && i0 <= HI) {
                    float2 f = __half22float2(h[q]);
                    win[i0] = f.x;
                    win[i0 + 1] = f.y;
                }
            }
        }
    } else {
#pragma unroll
        for (int c = LO / 4; c <= HI / 4; c++) {
            float4 v = reinterpret_cast<const float4*>(rowp)[c];
            win[4 * c + 0] = v.x;
            win[4 * c + 1] = v.y;
            win[4 * c + 2] = v.z;
            win[4 * c + 3] = v.w;
        }
    }
}

// Patch distances of a thread's VPT consecutive voxels: rows of the D planes
// in the reference tap order. XOFF = the voxels' first column within the
// 16-byte-aligned row start rowoff points at.
template <int RX, int RY, int RZ, int TZ, int TX, bool D_HALF, int VPT, int XOFF, int RI>
__device__ __forceinline__ void fast_rows(const unsigned char* __restrict__ Db, int rowoff,
                                          float (&dist)[VPT], const FastArgs& a) {
    using G = TileGeom<RX, RY, RZ, TZ, TX>;
    using F = FastGeom<RX, RY, RZ, TZ, TX, D_HALF>;
    if constexpr (RI < G::rows.n) {
        constexpr int zp = G::rows.zp[RI];
        constexpr int yp = G::rows.yp[RI];
        constexpr int e = G::rows.e[RI];
        constexpr int first = RowFirst<RX, RY, RZ, RI>::value;
        constexpr int esz = D_HALF ? 2 : 4;
        static_assert(XOFF + RX + VPT - 1 + e < 16, "row window");
        const unsigned char* rowp =
            Db + (size_t)(rowoff + (zp + RZ) * F::DPLANE + (yp + RY) * F::DP) * esz;
        float win[16];
        load_row<D_HALF, XOFF + RX - e, XOFF + RX + VPT - 1 + e>(rowp, win);
#pragma unroll
        for (int xp = -e; xp <= e; xp++) {
            if (zp == 0 && yp == 0 && xp == 0) continue;
            const int t = first + (xp + e) - ((zp == 0 && yp == 0 && xp > 0) ? 1 : 0);
            const float w = a.w[t];
#pragma unroll
            for (int r = 0; r < VPT; r++) dist[r] = fmaf(win[XOFF + RX + r + xp], w, dist[r]);
        }
        fast_rows<RX, RY, RZ, TZ, TX, D_HALF, VPT, XOFF, RI + 1>(Db, rowoff, dist, a);
    }
}

// Patch distances in half2 pairs (voxels 2p, 2p+1): the FP16 D row is read as
// half2 registers; pairs that start on an odd column are assembled from two
// neighbours; taps are HFMA2 with the tap weight in both halves.
template <int RX, int RY, int RZ, int TZ, int TX, int VPT, int XOFF, int RI>
__device__ __forceinline__ void fast_rows_h2(const unsigned char* __restrict__ Db, int rowoff,
                                             __half2 (&dist)[VPT / 2], const FastArgs& a) {
    using G = TileGeom<RX, RY, RZ, TZ, TX>;
    using F = FastGeom<RX, RY, RZ, TZ, TX, true>;
    if constexpr (RI < G::rows.n) {
        constexpr int zp = G::rows.zp[RI];
        constexpr int yp = G::rows.yp[RI];
        constexpr int e = G::rows.e[RI];
        constexpr int first = RowFirst<RX, RY, RZ, RI>::value;
        constexpr int LO = XOFF + RX - e, HI = XOFF + RX + VPT - 1 + e;
        static_assert(HI < 16, "row window");
        const uint4* rowp = reinterpret_cast<const uint4*>(
            Db + (size_t)(rowoff + (zp + RZ) * F::DPLANE + (yp + RY) * F::DP) * 2);
        __half2 hw[8];
#pragma unroll
        for (int c = LO / 8; c <= HI / 8; c++) {
            const uint4 v = rowp[c];
            hw[4 * c + 0] = *reinterpret_cast<const __half2*>(&v.x);
            hw[4 * c + 1] = *reinterpret_cast<const __half2*>(&v.y);
            hw[4 * c + 2] = *reinterpret_cast<const __half2*>(&v.z);
            hw[4 * c + 3] = *reinterpret_cast<const __half2*>(&v.w);
        }
#pragma unroll
        for (int xp = -e; xp <= e; xp++) {
            if (zp == 0 && yp == 0 && xp == 0) continue;
            const int t = first + (xp + e) - ((zp == 0 && yp == 0 && xp > 0) ? 1 : 0);
            const __half2 w = a.wh[t];
#pragma unroll
            for (int p = 0; p < VPT / 2; p++) {
                const int i = XOFF + RX + 2 * p + xp;
                const __half2 v = (i & 1) == 0 ? hw[i / 2]
                                               : __halves2half2(__high2half(hw[i / 2]),
                                                                __low2half(hw[i / 2 + 1]));
                dist[p] = __hfma2(v, w, dist[p]);
            }
        }
        fast_rows_h2<RX, RY, RZ, TZ, TX, VPT, XOFF, RI + 1>(Db, rowoff, dist, a);
    }
}

template <int RX, int RY, int RZ, int TZ, int TX, int VPT, int XOFF>
__device__ __forceinline__ void tile_distances_h2(const unsigned char* __restrict__ Dr, int rowoff,
                                                  float (&dist)[VPT], const FastArgs& a) {
    using F = FastGeom<RX, RY, RZ, TZ, TX, true>;
    constexpr int LO = XOFF + RX, HI = XOFF + RX + VPT - 1;
    const uint4* rowp = reinterpret_cast<const uint4*>(Dr + (size_t)(rowoff + RZ * F::DPLANE + RY * F::DP) * 2);
    __half2 hw[8];
#pragma unroll
    for (int c = LO / 8; c <= (HI + 1) / 8 && c < 2; c++) {
        const uint4 v = rowp[c];
        hw[4 * c + 0] = *reinterpret_cast<const __half2*>(&v.x);
        hw[4 * c + 1] = *reinterpret_cast<const __half2*>(&v.y);
        hw[4 * c + 2] = *reinterpret_cast<const __half2*>(&v.z);
        hw[4 * c + 3] = *reinterpret_cast<const __half2*>(&v.w);
    }
    __half2 dh[VPT / 2];
    const __half2 w0 = a.wh[0];
#pragma unroll
    for (int p = 0; p < VPT / 2; p++) {
        const int i = LO + 2 * p;
        const __half2 v = (i & 1) == 0 ? hw[i / 2]
                                       : __halves2half2(__high2half(hw[i / 2]), __low2half(hw[i / 2 + 1]));
        dh[p] = __hmul2(v, w0);
    }
    fast_rows_h2<RX, RY, RZ, TZ, TX, VPT, XOFF, 0>(Dr, rowoff, dh, a);
#pragma unroll
    for (int p = 0; p < VPT / 2; p++) {
        const float2 f = __half22float2(dh[p]);
        dist[2 * p] = f.x;
        dist[2 * p + 1] = f.y;
    }
}

template <int RX, int RY, int RZ, int TZ, int TX, bool D_HALF, int VPT, int XOFF>
__device__ __forceinline__ void tile_distances(const unsigned char* __restrict__ Dr, int rowoff,
                                               float (&dist)[VPT], const FastArgs& a) {
    using F = FastGeom<RX, RY, RZ, TZ, TX, D_HALF>;
    float win[16];
    constexpr int esz = D_HALF ? 2 : 4;
    load_row<D_HALF, XOFF + RX, XOFF + RX + VPT - 1>(
        Dr + (size_t)(rowoff + RZ * F::DPLANE + RY * F::DP) * esz, win);
    const float w0 = a.w[0];
#pragma unroll
    for (int r = 0; r < VPT; r++) dist[r] = win[XOFF + RX + r] * w0;
    fast_rows<RX, RY, RZ, TZ, TX, D_HALF, VPT, XOFF, 0>(Dr, rowoff, dist, a);
}

// Voxels per thread. 8 for both CTA widths: 4 per thread (a 4-warp one-tile
// CTA, 20 warps per SM) measured 12% slower than 8 (10 warps per SM), the
// extra row-window loads and conversions costing more than the occupancy
// returns.
template <int TX>
struct FastThreads {
    static constexpr int VPT = kVoxPerThread;
};

// TX = 32: CTA of 32 x 8 x TZ voxels (four 8^3 tiles along x when TZ = 8),
// two CTAs per SM; TX = 8: CTA of one 8 x 8 x TZ tile (64 threads), five
// CTAs per SM.
template <int RX, int RY, int RZ, int TZ, int TX, bool D_HALF, bool MASS>
__global__ void __launch_bounds__(TX * TZ * 8 / FastThreads<TX>::VPT, TX == 32 ? 2 : 5)
    nlm_tile_fast_kernel(const __grid_constant__ CUtensorMap tm_prev,
                         const __grid_constant__ FastArgs a) {
    using G = TileGeom<RX, RY, RZ, TZ, TX>;
    using F = FastGeom<RX, RY, RZ, TZ, TX, D_HALF>;
    constexpr int VPT = FastThreads<TX>::VPT;
    constexpr int NT = TX * TZ * 8 / VPT;  // threads
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    __half* prevb = reinterpret_cast<__half*>(smem + 128);
    const int pplane = a.pbx * a.pby;
    const int PB = pplane * a.pbz;  // halves
    // TX = 8 reads raw through L1 from global memory (its CTAs are small, so
    // shared memory bounds how many share an SM); TX = 32 stages the raw box.
    constexpr bool RAW_G = (TX == 8);
    __half* rawb = reinterpret_cast<__half*>(smem + 128 + (size_t)(PB + 63) / 64 * 128);
    const int rpx = a.rbx + 1;
    const int RB = RAW_G ? 0 : rpx * a.rby * a.rbz;  // halves
    unsigned char* D0 = reinterpret_cast<unsigned char*>(rawb) + (size_t)(RB + 63) / 64 * 128;

    const int tid = threadIdx.x;
    const int X0 = blockIdx.x * TX;
    const int Y0 = blockIdx.y * kTY;
    const int Z0 = blockIdx.z * TZ;
    const int cta = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;

    if (tid == 0) {
        prefetch_tmap(&tm_prev);
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        mbar_arrive_expect_tx(bar, (uint32_t)PB * 2u);
        tma_load_3d(prevb, &tm_prev, X0, Y0, Z0, bar);
    }
    if (!RAW_G) {
        // raw over tile + search halo (FP16), odd row pitch
        const int rb_n = a.rbx * a.rby * a.rbz;
        const __half* rsrc = a.raw_pad + (long long)(Z0 + RZ) * a.gpitch_z +
                             (long long)(Y0 + RY) * a.gpitch_y + X0;
        for (int i = tid; i < rb_n; i += NT) {
            int xx = i % a.rbx;
            int rest = i / a.rbx;
            int yy = rest % a.rby;
            int zz = rest / a.rby;
            rawb[(zz * a.rby + yy) * rpx + xx] =
                rsrc[(long long)zz * a.gpitch_z + (long long)yy * a.gpitch_y + xx];
        }
    }

    // offsets of this CTA: all, or its list
    int s_begin = 0, s_count = a.S;
    if (a.plan_start) {
        s_begin = a.plan_start[cta];
        s_count = min(a.plan_count[cta], a.S);
    }

    // the (prev box, raw) deltas of this CTA's offsets, staged once
    int2* sdl = reinterpret_cast<int2*>(D0 + 2 * (size_t)F::DBYTES);
    for (int i = tid; i < s_count; i += NT) {
        const int e = a.plan_offsets ? min(max(a.plan_offsets[s_begin + i], 0), a.S - 1) : i;
        sdl[i] = __ldg(&a.search_delta[e]);
    }
    __syncthreads();

    // scale D by 1/sigma^2 of the tile's middle slice (FP16 normal range)
    const float scale = -a.mult[min(Z0 + TZ / 2, a.nz - 1)];

    constexpr int NPAIR = G::ND / 2;
    constexpr int NQ = (NPAIR + NT - 1) / NT;
    int qpi[NQ], qdi[NQ];
#pragma unroll
    for (int k = 0; k < NQ; k++) {
        int q = min(tid + k * NT, NPAIR - 1);
        int f = 2 * q;
        int c = f % G::DW;
        int rest = f / G::DW;
        int r = rest % G::DH;
        int p = rest / G::DH;
        qpi[k] = (p - RZ + a.pz) * pplane + (r - RY + a.py) * a.pbx + (c - RX + a.px);
        qdi[k] = p * F::DPLANE + r * F::DP + c;
    }
    if (!mbar_wait_bounded(bar, 0)) {
        set_error(a.err, DEV_TMA_TIMEOUT);
        return;
    }
    float og0[NQ], og1[NQ];
#pragma unroll
    for (int k = 0; k < NQ; k++) {
        og0[k] = __half2float(prevb[qpi[k]]);
        og1[k] = __half2float(prevb[qpi[k] + 1]);
    }

    auto phase_a = [&](unsigned char* Dw, int dlx) {
#pragma unroll
        for (int k = 0; k < NQ; k++) {
            float t0 = __half2float(prevb[qpi[k] + dlx]) - og0[k];
            float t1 = __half2float(prevb[qpi[k] + dlx + 1]) - og1[k];
            float d0 = (t0 * scale) * t0, d1 = (t1 * scale) * t1;
            if constexpr (D_HALF) {
                reinterpret_cast<__half2*>(Dw)[qdi[k] / 2] = __floats2half2_rn(d0, d1);
            } else {
                reinterpret_cast<float2*>(Dw)[qdi[k] / 2] = make_float2(d0, d1);
            }
        }
    };

    // Phase B lane map: a warp covers VPT x 8 x 4 voxels of one 8^3 tile, lane
    // = (row j, plane), VPT consecutive x voxels each. TX = 32: warp w takes x
    // sub-block g = w % 4 (columns 8g..8g+7) and planes 4*(w/4)..+3; TX = 8:
    // x half w / 2 (columns 4*(w/2)..+3) and planes 4*(w%2)..+3.
    const int warp = tid >> 5, lane = tid & 31;
    const int g = (TX == 32) ? (warp & 3) : 0;
    const int xh = (TX == 32) ? 0 : (warp >> 1);
    const int j = lane & 7;
    const int zw = (TX == 32) ? 4 * (warp >> 2) : 4 * (warp & 1);  // first plane of the warp
    const int kp = zw + (lane >> 3);                                 // z-plane of the CTA
    const int x0 = (TX == 32) ? g * VPT : xh * VPT;
    const int zk = min(Z0 + kp, a.nz - 1);
    const float rel = a.mult[zk] / scale;  // x = dist' * rel
    // D row start (16-byte aligned): TX = 32 includes x0, TX = 8 passes the
    // x half as a compile-time column offset
    const int rowoff = kp * F::DPLANE + j * F::DP + (TX == 32 ? x0 : 0);
    // raw of the lane's first voxel: shared box index, or padded global index
    // (the offset deltas dl.y index the same space)
    const long long rbase =
        RAW_G ? (long long)(Z0 + kp + a.pz) * a.gpitch_z + (long long)(Y0 + j + a.py) * a.gpitch_y +
                    (X0 + x0 + a.px)
              : (long long)((a.szc + kp) * (rpx * a.rby) + (a.syr + j) * rpx + (RX + a.sxr + x0));
    const __half* rsrc_v = RAW_G ? a.raw_pad : rawb;

    float acc[VPT], wsum[VPT], wmax[VPT];
#pragma unroll
    for (int r = 0; r < VPT; r++) acc[r] = wsum[r] = wmax[r] = 0.0f;
    float inv[VPT];  // MASS: 1 / weight sum of the voxel (0 outside the volume)
    if constexpr (MASS) {
        const int z = Z0 + kp, y = Y0 + j;
#pragma unroll
        for (int r = 0; r < VPT; r++) {
            const int x = X0 + x0 + r;
            inv[r] = (z < a.nz && y < a.ny && x < a.nx)
                         ? a.aux[((long long)z * a.ny + y) * a.nx + x]
                         : 0.0f;
        }
    }

    if (s_count > 0) {
        int ent = 0;
        int2 dl = sdl[0];
        // global raw (TX = 8): the next offset's VPT values are loaded one
        // offset ahead so the loads overlap a whole offset's arithmetic
        float rnext[VPT];
        if constexpr (RAW_G && !MASS) {
#pragma unroll
            for (int r = 0; r < VPT; r++) rnext[r] = __half2float(rsrc_v[rbase + dl.y + r]);
        }
        phase_a(D0, dl.x);
        __syncthreads();
        for (int i = 0; i < s_count; i++) {
            const unsigned char* Dr = D0 + (size_t)(i & 1) * F::DBYTES;
            const int dly = dl.y;
            const int scur = ent;  // offset index (MASS runs without a plan)
            float rcur[VPT];
            if constexpr (RAW_G && !MASS) {
#pragma unroll
                for (int r = 0; r < VPT; r++) rcur[r] = rnext[r];
            }
            if (i + 1 < s_count) {
                ent = i + 1;
                dl = sdl[i + 1];
                if constexpr (RAW_G && !MASS) {
#pragma unroll
                    for (int r = 0; r < VPT; r++)
                        rnext[r] = __half2float(rsrc_v[rbase + dl.y + r]);
                }
                phase_a(D0 + (size_t)((i + 1) & 1) * F::DBYTES, dl.x);
            }
            {
                float dist[VPT];
                if constexpr (TX == 8 && VPT < kVoxPerThread) {
                    if (xh)  // warp-uniform
                        tile_distances<RX, RY, RZ, TZ, TX, D_HALF, VPT, VPT>(Dr, rowoff, dist, a);
                    else
                        tile_distances<RX, RY, RZ, TZ, TX, D_HALF, VPT, 0>(Dr, rowoff, dist, a);
                } else if constexpr (D_HALF && !MASS) {
                    // the weight-sum pass of the mass maps keeps FP32 sums, like
                    // the MASS pass it normalises (a uniform branch)
                    if (a.aux)
                        tile_distances<RX, RY, RZ, TZ, TX, D_HALF, VPT, 0>(Dr, rowoff, dist, a);
                    else
                        tile_distances_h2<RX, RY, RZ, TZ, TX, VPT, 0>(Dr, rowoff, dist, a);
                } else {
                    tile_distances<RX, RY, RZ, TZ, TX, D_HALF, VPT, 0>(Dr, rowoff, dist, a);
                }
                float part = 0.0f;
#pragma unroll
                for (int r = 0; r < VPT; r++) {
                    const float x = dist[r] * rel;
                    // Pade[3/3] of exp in Horner form, FMA
                    const float num = fmaf(fmaf(x + 12.f, x, 60.f), x, 120.f);
                    const float den = fmaf(fmaf(12.f - x, x, -60.f), x, 120.f);
                    const float q = __fdividef(num, den);  // formed, then selected
                    const float w = (x > -3.56648f) ? q : 0.0f;
                    if constexpr (MASS) {
                        part = fmaf(w, inv[r], part);
                    } else {
                        float rs;
                        if constexpr (RAW_G)
                            rs = rcur[r];
                        else
                            rs = __half2float(rsrc_v[rbase + dly + r]);
                        acc[r] = fmaf(w, rs, acc[r]);
                        wsum[r] += w;
                        wmax[r] = fmaxf(wmax[r], w);
                    }
                }
                if constexpr (MASS) {
                    // the warp's voxels all lie in one 8^3 tile
#pragma unroll
                    for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
                    if (lane == 0 && part != 0.0f) {
                        const long long t8 =
                            ((long long)((Z0 + zw) >> 3) * a.t8y + (Y0 >> 3)) * a.t8x + (X0 >> 3) + g;
                        atomicAdd(&a.map[t8 * a.S + scur], part);
                    }
                }
            }
            __syncthreads();
        }
    }
    if constexpr (MASS) return;

    const int z = Z0 + kp, y = Y0 + j;
    if (z < a.nz && y < a.ny) {
        float* orow = a.out + ((long long)z * a.ny + y) * a.nx;
        if (a.aux && !MASS) {
            // weight-sum pass of the mass maps: 1 / (sum of the offsets' weights)
            float* arow = a.aux + ((long long)z * a.ny + y) * a.nx;
#pragma unroll
            for (int r = 0; r < VPT; r++) {
                const int x = X0 + x0 + r;
                if (x < a.nx) arow[x] = wsum[r] > 0.0f ? 1.0f / wsum[r] : 0.0f;
            }
            return;
        }
#pragma unroll
        for (int r = 0; r < VPT; r++) {
            int x = X0 + x0 + r;
            if (x < a.nx) {
                const float raw0 = __half2float(rsrc_v[rbase + r]);
                float res = raw0;
                if (wmax[r] > 0.0f) {
                    // per-voxel weight-sum normalisation in FP64
                    double num = (double)acc[r] + (double)wmax[r] * (double)raw0;
                    double den = (double)wsum[r] + (double)wmax[r];
                    res = (float)(num / den);
                }
                orow[x] = res;
            }
        }
    }
}

// FP32 result -> padded FP16 volume (reflective), for raw and the previous iterate.
__global__ void pad_reflective_half_kernel(const float* __restrict__ in, int nx, int ny, int nz,
                                           __half* __restrict__ out, int px, int py, int pz,
                                           long long pitch_y, long long pitch_z) {
    const int nxp = nx + 2 * px, nyp = ny + 2 * py, nzp = nz + 2 * pz;
    const long long total = (long long)nxp * nyp * nzp;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int x1 = (int)(i % nxp);
        long long r = i / nxp;
        int y1 = (int)(r % nyp);
        int z1 = (int)(r / nyp);
        int x0 = x1 - px, y0 = y1 - py, z0 = z1 - pz;
        for (int guard = 0; guard < 64 && (z0 < 0 || z0 >= nz || y0 < 0 || y0 >= ny || x0 < 0 ||
                                           x0 >= nx);
             guard++) {
            if (z0 < 0) z0 = -z0;
            if (y0 < 0) y0 = -y0;
            if (x0 < 0) x0 = -x0;
            if (z0 >= nz) z0 = 2 * nz - z0 - 2;
            if (y0 >= ny) y0 = 2 * ny - y0 - 2;
            if (x0 >= nx) x0 = 2 * nx - x0 - 2;
        }
        x0 = min(max(x0, 0), nx - 1);
        y0 = min(max(y0, 0), ny - 1);
        z0 = min(max(z0, 0), nz - 1);
        out[z1 * pitch_z + y1 * pitch_y + x1] =
            __float2half_rn(in[((long long)z0 * ny + y0) * nx + x0]);
    }
}

template <int RX, int RY, int RZ, int TZ, int TX, bool D_HALF>
static size_t fast_smem_for(const FastArgs& a) {
    using F = FastGeom<RX, RY, RZ, TZ, TX, D_HALF>;
    size_t pb = (size_t)(a.pbx * a.pby * a.pbz + 63) / 64 * 128;  // bytes
    size_t rb = TX == 8 ? 0 : (size_t)((a.rbx + 1) * a.rby * a.rbz + 63) / 64 * 128;
    const size_t dl = ((size_t)a.S * sizeof(int2) + 127) / 128 * 128;  // staged offset deltas
    return 128 + pb + rb + 2 * (size_t)F::DBYTES + dl;
}

template <int RX, int RY, int RZ, int TZ, int TX, bool D_HALF>
static cudaError_t fast_launch_inst(const CUtensorMap* tmp, const FastArgs& a, int tiles_z,
                                    size_t smem, cudaStream_t st, bool mass) {
    auto kern = nlm_tile_fast_kernel<RX, RY, RZ, TZ, TX, D_HALF, false>;
    if (mass) {
        // weight-mass maps run on the full-search (TX = 32) configuration
        if constexpr (TX == 32)
            kern = nlm_tile_fast_kernel<RX, RY, RZ, TZ, TX, D_HALF, true>;
        else
            return cudaErrorInvalidConfiguration;
    }
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid(a.tiles_x, a.tiles_y, tiles_z);
    kern<<<grid, TX * TZ * 8 / FastThreads<TX>::VPT, smem, st>>>(*tmp, a);
    return cudaGetLastError();
}

#define INLM_FAST_SHAPES(X) \
    X(1, 1, 1) X(1, 1, 2) X(1, 1, 3) X(2, 2, 1) X(2, 2, 2) X(3, 3, 1) X(3, 3, 2) X(3, 3, 3)

size_t fast_smem_bytes(const FastConfig& c, const FastArgs& a) {
#define X(A, B, C)                                                                          \
    if (c.rx == A && c.ry == B && c.rz == C) {                                              \
        if (c.tx == 32 && c.tz == 8 && c.d_half) return fast_smem_for<A, B, C, 8, 32, true>(a);   \
        if (c.tx == 32 && c.tz == 8 && !c.d_half) return fast_smem_for<A, B, C, 8, 32, false>(a); \
        if (c.tx == 32 && c.tz == 4 && c.d_half) return fast_smem_for<A, B, C, 4, 32, true>(a);   \
        if (c.tx == 8 && c.tz == 8 && c.d_half) return fast_smem_for<A, B, C, 8, 8, true>(a);     \
        if (c.tx == 8 && c.tz == 8 && !c.d_half) return fast_smem_for<A, B, C, 8, 8, false>(a);   \
    }
    INLM_FAST_SHAPES(X)
#undef X
    return 0;
}

cudaError_t launch_fast_kernel(const FastConfig& c, const CUtensorMap* tm_prev, const FastArgs& a,
                               int tiles_z, cudaStream_t st, bool mass) {
#define X(A, B, C)                                                                           \
    if (c.rx == A && c.ry == B && c.rz == C) {                                               \
        const size_t sm = c.smem_bytes;                                                      \
        if (c.tx == 32 && c.tz == 8 && c.d_half)                                             \
            return fast_launch_inst<A, B, C, 8, 32, true>(tm_prev, a, tiles_z, sm, st, mass);  \
        if (c.tx == 32 && c.tz == 8 && !c.d_half)                                            \
            return fast_launch_inst<A, B, C, 8, 32, false>(tm_prev, a, tiles_z, sm, st, mass); \
        if (c.tx == 32 && c.tz == 4 && c.d_half)                                             \
            return fast_launch_inst<A, B, C, 4, 32, true>(tm_prev, a, tiles_z, sm, st, mass);  \
        if (c.tx == 8 && c.tz == 8 && c.d_half)                                              \
            return fast_launch_inst<A, B, C, 8, 8, true>(tm_prev, a, tiles_z, sm, st, mass);   \
        if (c.tx == 8 && c.tz == 8 && !c.d_half)                                             \
            return fast_launch_inst<A, B, C, 8, 8, false>(tm_prev, a, tiles_z, sm, st, mass);  \
    }
    INLM_FAST_SHAPES(X)
#undef X
    return cudaErrorInvalidConfiguration;
}

cudaError_t launch_pad_reflective_half(const float* in, int nx, int ny, int nz, void* out, int px,
                                       int py, int pz, long long pitch_y, long long pitch_z,
                                       cudaStream_t st) {
    pad_reflective_half_kernel<<<148 * 8, 256, 0, st>>>(in, nx, ny, nz, (__half*)out, px, py, pz,
                                                        pitch_y, pitch_z);
    return cudaGetLastError();
}

}  // namespace inlm
