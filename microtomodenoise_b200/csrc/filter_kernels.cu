// Plain FP32 iterNLM filter for sm_100a, bit-identical to the reference CPU
// filter (Denoiser/iternlm_cpu_kernels.cpp:7-1108, iternlm_cpu.cpp:758-843).
//
// Per voxel x and search offset s (reference order, iternlm_prepare.cpp:102):
//   dist  = sum_p w_p * (prev[x+s+p] - prev[x+p])^2      (taps in reference order)
//   w     = dist*m > -3.56648 ? Pade33(dist*m) : 0          (m = -1/(sigma_z^2 beta))
//   acc  += w*raw[x+s];  wsum += w;  wmax = max(wmax, w)
// out = wmax > 0 ? (acc + wmax*raw[x]) / (wsum + wmax) : raw[x].
// Every product and sum is rounded separately (__fmul_rn/__fadd_rn) in the
// reference's order, so the result equals the reference's g++ -O3 (SSE, no
// FMA) build bit for bit.
//
// Tiled kernel: a CTA stages the padded previous iterate over its tile plus
// search+patch halo into shared memory with one 3D TMA load and raw over the
// tile plus search halo with coalesced loads (odd row pitch): the whole raw
// box when it fits, else a slab of TZ + 1 planes that follows the z-major
// offsets, else none (raw read from global memory as aligned float4s).
// Offsets go in groups of two: it writes the squared-difference volumes
// D_s = (prev(.+s) - prev(.))^2 of both over the tile plus patch halo to
// shared memory, then each thread applies the patch stencil to both for 8
// consecutive x voxels held as 4 register pairs each: a tap is two scalar
// FMULs (weight as a constant operand) and one paired FADD2 (sm_100 f32x2),
// from a 16-float register window per patch row loaded as float4s from a
// conflict-free row pitch; the two offsets are then weighted and accumulated
// in reference order. Each D value is computed once per offset and read by
// every voxel whose patch covers it.
#include <cstdio>

#include "common.cuh"
#include "filter_kernels.cuh"
#include "geometry.hpp"
#include "pair_math.cuh"
#include "tile_common.cuh"

namespace inlm {

// r[0..8) = p[0..8) through three aligned float4 loads (p is 4-byte aligned;
// the 16-byte block before and after p must be readable). The raw reads of the
// global-raw tile path: a warp's lanes sit on 32 different rows, so each load
// instruction touches 32 cache lines; three vector loads instead of eight
// scalar ones cut those L1 wavefronts by 2.7x (1.35x faster at patch radius 1,
// search radius 10). The misalignment is (padding + offset x) mod 4, the same
// for every lane of the warp, so the switch does not diverge. Reads stay in
// the allocation: every raw position lies at least one padded plane after
// its start, and zeroed slack planes follow its end.
__device__ __forceinline__ void load8_global(const float* __restrict__ p, float (&r)[8]) {
    const int sh = (int)((reinterpret_cast<unsigned long long>(p) >> 2) & 3);
    const float4* q = reinterpret_cast<const float4*>(p - sh);
    const float4 u = __ldg(q), v = __ldg(q + 1), w = __ldg(q + 2);
    const float t[12] = {u.x, u.y, u.z, u.w, v.x, v.y, v.z, v.w, w.x, w.y, w.z, w.w};
    switch (sh) {
        case 0:
#pragma unroll
            for (int i = 0; i < 8; i++) r[i] = t[i];
            break;
        case 1:
#pragma unroll
            for (int i = 0; i < 8; i++) r[i] = t[i + 1];
            break;
        case 2:
#pragma unroll
            for (int i = 0; i < 8; i++) r[i] = t[i + 2];
            break;
        default:
#pragma unroll
            for (int i = 0; i < 8; i++) r[i] = t[i + 3];
            break;
    }
}

// Loads columns [x0 + 4*LO, x0 + 4*HI + 4) of one D row into win (float4s).
template <int LO, int HI>
__device__ __forceinline__ void load_window(const float* __restrict__ rowp, float (&win)[16]) {
#pragma unroll
    for (int c = LO; c <= HI; c++) {
        float4 v = reinterpret_cast<const float4*>(rowp)[c];
        win[4 * c + 0] = v.x;
        win[4 * c + 1] = v.y;
        win[4 * c + 2] = v.z;
        win[4 * c + 3] = v.w;
    }
}

// Patch sums of NO offsets at once (D planes D0 + o*DSZ): the same operations
// as one offset's patch sum on each, interleaved row by row so a thread has 4*NO
// independent chains in flight.
template <int RX, int RY, int RZ, int TZ, int NO, int RI, bool FUSED = false>
__device__ __forceinline__ void accumulate_rows_n(const float* __restrict__ D0, int dsz, int rowoff,
                                                  f32x2 (&d)[NO][kVoxPerThread / 2],
                                                  const TileArgs& a) {
    using G = TileGeom<RX, RY, RZ, TZ>;
    if constexpr (RI < G::rows.n) {
        constexpr int zp = G::rows.zp[RI];
        constexpr int yp = G::rows.yp[RI];
        constexpr int e = G::rows.e[RI];
        constexpr int first = RowFirst<RX, RY, RZ, RI>::value;
        constexpr int lo = (RX - e) / 4;
        constexpr int hi = (RX + kVoxPerThread - 1 + e) / 4;
        const int ro = rowoff + (zp + RZ) * G::DPLANE + (yp + RY) * G::DP;
        float win[NO][16];
#pragma unroll
        for (int o = 0; o < NO; o++) load_window<lo, hi>(D0 + o * dsz + ro, win[o]);
#pragma unroll
        for (int xp = -e; xp <= e; xp++) {
            if (zp == 0 && yp == 0 && xp == 0) continue;
            const int t = first + (xp + e) - ((zp == 0 && yp == 0 && xp > 0) ? 1 : 0);
            const float w = a.w[t];
#pragma unroll
            for (int p = 0; p < kVoxPerThread / 2; p++) {
                const int i = RX + 2 * p + xp;
#pragma unroll
                for (int o = 0; o < NO; o++) {
                    if (!FUSED) {
                        d[o][p] = add2(d[o][p], mul_pair(win[o][i], win[o][i + 1], w));
                    } else if ((i & 1) == 0) {
                        // an even window index is an aligned register pair
                        d[o][p] = fma2(pack2(win[o][i], win[o][i + 1]), splat2(w), d[o][p]);
                    } else {
                        const float2 c = unpack2(d[o][p]);
                        d[o][p] = pack2(__fmaf_rn(win[o][i], w, c.x), __fmaf_rn(win[o][i + 1], w, c.y));
                    }
                }
            }
        }
        accumulate_rows_n<RX, RY, RZ, TZ, NO, RI + 1, FUSED>(D0, dsz, rowoff, d, a);
    }
}


template <int RX, int RY, int RZ, int TZ, bool RAW_SMEM, bool FUSED = false, bool SLAB = false>
// aw supplies the patch weights: a kernel parameter at a fixed offset, so
// every tap's weight is a constant-bank operand (the batch kernel passes its
// group's first volume, whose weights every volume of the group shares; read
// through a runtime volume index they would cost a load per tap).
__device__ __forceinline__ bool tile_f32_body(const CUtensorMap* tm_prev, const TileArgs& a, int bx,
                                              int by, int bz, unsigned char* smem,
                                              uint32_t parity, const TileArgs& aw) {
    using G = TileGeom<RX, RY, RZ, TZ>;
    static_assert(!SLAB || RAW_SMEM, "the raw slab is a shared-memory staging");
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    float* prevb = reinterpret_cast<float*>(smem + 128);
    const int pplane = a.pbx * a.pby;
    const int PB = pplane * a.pbz;
    float* rawb = prevb + round_up32(PB);
    // raw is staged with an odd row pitch (rpx = rbx + 1) so the phase-B reads
    // of a warp's 8 rows fall in distinct banks
    const int rpx = a.rbx + 1;
    const int RB = RAW_SMEM ? a.rplane * a.rbz : 0;
    float* D = rawb + round_up32(RB);
    constexpr int DSZ = round_up32(G::DPLANE * G::DD);
    // kOffGroup D buffers: phase A writes one per offset of the group, a
    // barrier, phase B reads them all, a barrier.
    float* const D0 = D;

    const int tid = threadIdx.x;
    const int X0 = bx * kTX;
    const int Y0 = by * kTY;
    const int Z0 = bz * TZ;

    if (tid == 0) {
        mbar_arrive_expect_tx(bar, (uint32_t)PB * 4u);
        // prev box starts at the tile origin in padded coordinates (x aligned to 32)
        tma_load_3d(prevb, tm_prev, X0, Y0, Z0, bar);
    }
    // raw over tile + search halo, planes [zoff, zoff + rbz) of the raw box,
    // coalesced rows re-pitched; positions past the volume read the zeroed
    // slack planes behind it and are never used
    auto stage_raw = [&](int zoff) {
        const int rb_n = a.rbx * a.rby * a.rbz;
        const float* rsrc = a.raw_pad + (long long)(Z0 + RZ + zoff) * a.gpitch_z +
                            (long long)(Y0 + RY) * a.gpitch_y + X0;
        for (int i = tid; i < rb_n; i += G::NT) {
            int xx = i % a.rbx;
            int rest = i / a.rbx;
            int yy = rest % a.rby;
            int zz = rest / a.rby;
            rawb[zz * a.rplane + yy * rpx + xx] =
                __ldg(rsrc + (long long)zz * a.gpitch_z + (long long)yy * a.gpitch_y + xx);
        }
    };
    // Slab form (the whole raw box does not fit beside the prev box): the
    // offsets run z-major, so a group of offsets reads at most two z offsets;
    // shared memory holds the TZ + 1 planes from z offset slab_zb on and is
    // restaged when a group needs later planes.
    int slab_zb = 0;
    if (RAW_SMEM) {
        // staged while the prev box's TMA load is in flight
        if (SLAB) slab_zb = __ldg(&a.group_zb[0]);
        stage_raw(SLAB ? a.szc + slab_zb : 0);
    }

    // Each thread owns NQ fixed column pairs of the D volume (rows have an
    // even width); their prev-box and D indices, and the origin values, are
    // the same for every search offset and stay in registers.
    constexpr int NPAIR = G::ND / 2;
    constexpr int NQ = (NPAIR + G::NT - 1) / G::NT;
    int qpi[NQ], qdi[NQ];
#pragma unroll
    for (int k = 0; k < NQ; k++) {
        int q = min(tid + k * G::NT, NPAIR - 1);  // the tail repeats the last pair
        int f = 2 * q;
        int c = f % G::DW;
        int rest = f / G::DW;
        int r = rest % G::DH;
        int p = rest / G::DH;
        qpi[k] = (p - RZ + a.pz) * pplane + (r - RY + a.py) * a.pbx + (c - RX + a.px);
        qdi[k] = p * G::DPLANE + r * G::DP + c;
    }

    const bool arrived = mbar_wait_bounded(bar, parity);
    if (!__syncthreads_and(arrived)) {
        if (tid == 0) set_error(a.err, DEV_TMA_TIMEOUT);
        return false;
    }
    f32x2 qog[NQ];
#pragma unroll
    for (int k = 0; k < NQ; k++) qog[k] = pack2(prevb[qpi[k]], prevb[qpi[k] + 1]);

    // Phase B lane map: a warp covers 8 x 8 x 4 voxels (x sub-block w % 4 of
    // the CTA's 32 columns, z-planes 4*(w/4)..+3), lane = (row j, plane), 8
    // consecutive x voxels each; every voxel's arithmetic is the same under
    // any map.
    const int warp = tid >> 5, lane = tid & 31;
    const int k = 4 * (warp >> 2) + (lane >> 3);  // z-plane of the CTA
    const int j = lane & 7;
    const int x0 = (warp & 3) * kVoxPerThread;
    const int zk = min(Z0 + k, a.nz - 1);
    const float m = a.mult[zk];
    const f32x2 m2 = splat2(m);
    const int rowoff = k * G::DPLANE + j * G::DP + x0;

    // raw positions: rbase + delta in raw-box coordinates (shared memory; in
    // the slab form shifted by the slab's first plane), gbase + delta in the
    // padded volume (global)
    const int rbase_box = RAW_SMEM ? (a.szc + k) * a.rplane + (a.syr + j) * rpx + (RX + a.sxr + x0) : 0;
    int rbase = rbase_box - (SLAB ? (a.szc + slab_zb) * a.rplane : 0);
    const long long gbase = (long long)(Z0 + k + a.pz) * a.gpitch_z +
                            (long long)(Y0 + j + a.py) * a.gpitch_y + (X0 + x0 + a.px);

    constexpr int NP = kVoxPerThread / 2;
    f32x2 acc[NP], wsum[NP];
    float wmax[kVoxPerThread];
#pragma unroll
    for (int p = 0; p < NP; p++) acc[p] = wsum[p] = 0ull;  // (+0, +0)
#pragma unroll
    for (int r = 0; r < kVoxPerThread; r++) wmax[r] = 0.0f;

    // phase A for one offset: D = (prev(.+s) - prev(.))^2 over tile + patch halo
    auto phase_a = [&](float* Dw, int dlx) {
#pragma unroll
        for (int k = 0; k < NQ; k++) {
            f32x2 sh = pack2(prevb[qpi[k] + dlx], prevb[qpi[k] + dlx + 1]);
            f32x2 v = sub2(sh, qog[k]);
            *reinterpret_cast<f32x2*>(Dw + qdi[k]) = mul2_to_mul(v, v);  // stored, not added
        }
    };

    // weight and accumulation of one offset for the thread's 8 voxels
    auto accumulate = [&](const f32x2 (&dist)[NP], int dly) {
        float rg[kVoxPerThread];
        if (!RAW_SMEM) load8_global(a.raw_pad + gbase + dly, rg);
#pragma unroll
        for (int p = 0; p < NP; p++) {
            float2 rsv;
            if (RAW_SMEM) {
                rsv = make_float2(rawb[rbase + dly + 2 * p], rawb[rbase + dly + 2 * p + 1]);
            } else {
                rsv = make_float2(rg[2 * p], rg[2 * p + 1]);
            }
            if (FUSED)
                fused_weight_pair(dist[p], m2, rsv, acc[p], wsum[p], wmax[2 * p], wmax[2 * p + 1]);
            else
                exact_weight_pair(dist[p], m2, rsv, acc[p], wsum[p], wmax[2 * p], wmax[2 * p + 1]);
        }
    };

    // Offsets in groups of NO: phase A writes D of offsets s..s+NO-1 into NO
    // buffers, phase B forms their patch sums together (4*NO independent
    // chains per thread) and accumulates them in offset order (the
    // reference's). Two barriers per group. The last group forms the sums of
    // missing offsets on stale buffers and discards them.
    constexpr int NO = kOffGroup;
    // the next group's search deltas load while this group runs
    int2 dl[NO];
#pragma unroll
    for (int o = 0; o < NO; o++) dl[o] = __ldg(&a.search_delta[min(o, a.S - 1)]);
    for (int s = 0; s < a.S; s += NO) {
        if (SLAB) {
            // every thread reads the same entry: a uniform branch; the
            // previous group's raw reads ended at its closing barrier, and
            // the barrier after phase A publishes the new planes
            const int zb = __ldg(&a.group_zb[s / NO]);
            if (zb != slab_zb) {
                slab_zb = zb;
                stage_raw(a.szc + zb);
                rbase = rbase_box - (a.szc + zb) * a.rplane;
            }
        }
        int2 dln[NO];
#pragma unroll
        for (int o = 0; o < NO; o++) dln[o] = __ldg(&a.search_delta[min(s + NO + o, a.S - 1)]);
#pragma unroll
        for (int o = 0; o < NO; o++)
            if (s + o < a.S) phase_a(D0 + o * DSZ, dl[o].x);
        __syncthreads();
        f32x2 d[NO][NP];
        {
            const int ro = rowoff + RZ * G::DPLANE + RY * G::DP;
            const float w0 = aw.w[0];
#pragma unroll
            for (int o = 0; o < NO; o++) {
                float win[16];
                load_window<RX / 4, (RX + kVoxPerThread - 1) / 4>(D0 + o * DSZ + ro, win);
#pragma unroll
                for (int p = 0; p < NP; p++) d[o][p] = mul_pair(win[RX + 2 * p], win[RX + 2 * p + 1], w0);
            }
        }
        accumulate_rows_n<RX, RY, RZ, TZ, NO, 0, FUSED>(D0, DSZ, rowoff, d, aw);
#pragma unroll
        for (int o = 0; o < NO; o++)
            if (s + o < a.S) accumulate(d[o], dl[o].y);
        __syncthreads();
#pragma unroll
        for (int o = 0; o < NO; o++) dl[o] = dln[o];
    }

    const int z = Z0 + k, y = Y0 + j;
    if (z < a.nz && y < a.ny) {
        float* orow = a.out + ((long long)z * a.ny + y) * a.nx;
#pragma unroll
        for (int r = 0; r < kVoxPerThread; r++) {
            int x = X0 + x0 + r;
            if (x < a.nx) {
                float raw0 = (RAW_SMEM && !SLAB) ? rawb[rbase + r] : __ldg(&a.raw_pad[gbase + r]);
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
                orow[x] = res;
            }
        }
    }
    return true;
}

// ---- two z-planes per thread: CTA of 32 x 8 x 16 voxels ----
//
// The per-voxel arithmetic of tile_f32_body, with a thread owning 8 x voxels
// on two adjacent planes k and k + 1. Patch row (zp, yp) of plane k + 1 is D
// row (zp + 1, yp) counted from plane k, so one D row serves plane k's patch
// row (dz, yp) and plane k + 1's patch row (dz - 1, yp): each row window is
// loaded once for both planes (patch radius 2: 18 windows per offset for 16
// voxels instead of 26). Walking the rows in (dz, yp) order keeps each plane's
// patch rows in reference order, so every sum is formed in the same order as
// before. One offset per barrier step: a second D buffer does not fit beside
// the 16-deep prev box.

struct RowPairs {
    int n;
    int dz[64], yp[64];
    int r0[64], r1[64];  // patch row of plane k / of plane k + 1 read from this D row, or -1
};

constexpr RowPairs make_row_pairs(int rx, int ry, int rz) {
    const PatchRows rows = make_patch_rows(rx, ry, rz);
    RowPairs u{};
    for (int dz = -rz; dz <= rz + 1; dz++)
        for (int yp = -ry; yp <= ry; yp++) {
            int r0 = -1, r1 = -1;
            for (int i = 0; i < rows.n; i++) {
                if (rows.zp[i] == dz && rows.yp[i] == yp) r0 = i;
                if (rows.zp[i] == dz - 1 && rows.yp[i] == yp) r1 = i;
            }
            if (r0 < 0 && r1 < 0) continue;
            u.dz[u.n] = dz;
            u.yp[u.n] = yp;
            u.r0[u.n] = r0;
            u.r1[u.n] = r1;
            u.n++;
        }
    return u;
}

template <int RX, int RY, int RZ>
struct RowPairsOf {
    static constexpr RowPairs v = make_row_pairs(RX, RY, RZ);
};

// The taps of patch row RI (reference order) on a loaded row window.
template <int RX, int RY, int RZ, int RI>
__device__ __forceinline__ void row_taps(const float (&win)[16], f32x2 (&d)[kVoxPerThread / 2],
                                         const TileArgs& a) {
    using G = TileGeom<RX, RY, RZ, 16>;
    constexpr int zp = G::rows.zp[RI];
    constexpr int yp = G::rows.yp[RI];
    constexpr int e = G::rows.e[RI];
    constexpr int first = RowFirst<RX, RY, RZ, RI>::value;
#pragma unroll
    for (int xp = -e; xp <= e; xp++) {
        if (zp == 0 && yp == 0 && xp == 0) continue;
        const int t = first + (xp + e) - ((zp == 0 && yp == 0 && xp > 0) ? 1 : 0);
        const float w = a.w[t];
#pragma unroll
        for (int p = 0; p < kVoxPerThread / 2; p++) {
            const int i = RX + 2 * p + xp;
            d[p] = add2(d[p], mul_pair(win[i], win[i + 1], w));
        }
    }
}

template <int RX, int RY, int RZ, int TZ, int UI>
__device__ __forceinline__ void accumulate_row_pairs(const float* __restrict__ D, int rowoff,
                                                     f32x2 (&d0)[kVoxPerThread / 2],
                                                     f32x2 (&d1)[kVoxPerThread / 2],
                                                     const TileArgs& a) {
    using G = TileGeom<RX, RY, RZ, TZ>;
    using U = RowPairsOf<RX, RY, RZ>;
    if constexpr (UI < U::v.n) {
        constexpr int r0 = U::v.r0[UI];
        constexpr int r1 = U::v.r1[UI];
        constexpr int e0 = r0 >= 0 ? G::rows.e[r0 >= 0 ? r0 : 0] : 0;
        constexpr int e1 = r1 >= 0 ? G::rows.e[r1 >= 0 ? r1 : 0] : 0;
        constexpr int em = e0 > e1 ? e0 : e1;
        constexpr int lo = (RX - em) / 4;
        constexpr int hi = (RX + kVoxPerThread - 1 + em) / 4;
        const int ro = rowoff + (U::v.dz[UI] + RZ) * G::DPLANE + (U::v.yp[UI] + RY) * G::DP;
        float win[16];
        load_window<lo, hi>(D + ro, win);
        if constexpr (r0 >= 0) row_taps<RX, RY, RZ, (r0 >= 0 ? r0 : 0)>(win, d0, a);
        if constexpr (r1 >= 0) row_taps<RX, RY, RZ, (r1 >= 0 ? r1 : 0)>(win, d1, a);
        accumulate_row_pairs<RX, RY, RZ, TZ, UI + 1>(D, rowoff, d0, d1, a);
    }
}

// Raw staged in shared memory: the whole box (SLAB = false) or TZ + 1 planes
// following the z-major offsets (SLAB = true), as in tile_f32_body.
template <int RX, int RY, int RZ, bool SLAB>
__device__ __forceinline__ void tile_f32_z2_body(const CUtensorMap* tm_prev, const TileArgs& a,
                                                 unsigned char* smem) {
    constexpr int TZ = 16;
    constexpr int NT = 256;
    using G = TileGeom<RX, RY, RZ, TZ>;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    float* prevb = reinterpret_cast<float*>(smem + 128);
    const int pplane = a.pbx * a.pby;
    const int PB = pplane * a.pbz;
    float* rawb = prevb + round_up32(PB);
    const int rpx = a.rbx + 1;
    float* D = rawb + round_up32(a.rplane * a.rbz);

    const int tid = threadIdx.x;
    const int X0 = blockIdx.x * kTX;
    const int Y0 = blockIdx.y * kTY;
    const int Z0 = blockIdx.z * TZ;

    if (tid == 0) {
        mbar_arrive_expect_tx(bar, (uint32_t)PB * 4u);
        tma_load_3d(prevb, tm_prev, X0, Y0, Z0, bar);
    }
    auto stage_raw = [&](int zoff) {
        const int rb_n = a.rbx * a.rby * a.rbz;
        const float* rsrc = a.raw_pad + (long long)(Z0 + RZ + zoff) * a.gpitch_z +
                            (long long)(Y0 + RY) * a.gpitch_y + X0;
        for (int i = tid; i < rb_n; i += NT) {
            int xx = i % a.rbx;
            int rest = i / a.rbx;
            int yy = rest % a.rby;
            int zz = rest / a.rby;
            rawb[zz * a.rplane + yy * rpx + xx] =
                __ldg(rsrc + (long long)zz * a.gpitch_z + (long long)yy * a.gpitch_y + xx);
        }
    };
    int slab_zb = 0;
    if (SLAB) slab_zb = __ldg(&a.group_zb[0]);
    stage_raw(SLAB ? a.szc + slab_zb : 0);

    constexpr int NPAIR = G::ND / 2;
    constexpr int NQ = (NPAIR + NT - 1) / NT;
    int qpi[NQ], qdi[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        int e = min(tid + q * NT, NPAIR - 1);  // the tail repeats the last pair
        int f = 2 * e;
        int c = f % G::DW;
        int rest = f / G::DW;
        int r = rest % G::DH;
        int p = rest / G::DH;
        qpi[q] = (p - RZ + a.pz) * pplane + (r - RY + a.py) * a.pbx + (c - RX + a.px);
        qdi[q] = p * G::DPLANE + r * G::DP + c;
    }

    const bool arrived = mbar_wait_bounded(bar, 0);
    if (!__syncthreads_and(arrived)) {
        if (tid == 0) set_error(a.err, DEV_TMA_TIMEOUT);
        return;
    }
    f32x2 qog[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) qog[q] = pack2(prevb[qpi[q]], prevb[qpi[q] + 1]);

    // lane map: warp w covers x sub-block w % 4 and planes 8*(w/4)..+7; lane =
    // (row j, plane pair), planes k and k + 1
    const int warp = tid >> 5, lane = tid & 31;
    const int k = 8 * (warp >> 2) + 2 * (lane >> 3);
    const int j = lane & 7;
    const int x0 = (warp & 3) * kVoxPerThread;
    const f32x2 m0 = splat2(a.mult[min(Z0 + k, a.nz - 1)]);
    const f32x2 m1 = splat2(a.mult[min(Z0 + k + 1, a.nz - 1)]);
    const int rowoff = k * G::DPLANE + j * G::DP + x0;
    const int rbase_box = (a.szc + k) * a.rplane + (a.syr + j) * rpx + (RX + a.sxr + x0);
    int rbase = rbase_box - (SLAB ? (a.szc + slab_zb) * a.rplane : 0);

    constexpr int NP = kVoxPerThread / 2;
    f32x2 acc0[NP], wsum0[NP], acc1[NP], wsum1[NP];
    float wmax0[kVoxPerThread], wmax1[kVoxPerThread];
#pragma unroll
    for (int p = 0; p < NP; p++) acc0[p] = wsum0[p] = acc1[p] = wsum1[p] = 0ull;
#pragma unroll
    for (int r = 0; r < kVoxPerThread; r++) wmax0[r] = wmax1[r] = 0.0f;

    auto phase_a = [&](int dlx) {
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            f32x2 sh = pack2(prevb[qpi[q] + dlx], prevb[qpi[q] + dlx + 1]);
            f32x2 v = sub2(sh, qog[q]);
            *reinterpret_cast<f32x2*>(D + qdi[q]) = mul2_to_mul(v, v);  // stored, not added
        }
    };

    // weight and accumulation of one offset for one plane's 8 voxels (the
    // exact Pade form of tile_f32_body)
    auto accumulate = [&](const f32x2 (&dist)[NP], const f32x2 m2, int rb, f32x2 (&acc)[NP],
                          f32x2 (&wsum)[NP], float (&wmax)[kVoxPerThread]) {
#pragma unroll
        for (int p = 0; p < NP; p++) {
            const float2 rsv = make_float2(rawb[rb + 2 * p], rawb[rb + 2 * p + 1]);
            exact_weight_pair(dist[p], m2, rsv, acc[p], wsum[p], wmax[2 * p], wmax[2 * p + 1]);
        }
    };

    int2 dl = __ldg(&a.search_delta[0]);
    for (int s = 0; s < a.S; s++) {
        if (SLAB) {
            // uniform branch; the previous offset's raw reads ended at its
            // closing barrier and the barrier after phase A publishes the planes
            const int zb = __ldg(&a.group_zb[s / kOffGroup]);
            if (zb != slab_zb) {
                slab_zb = zb;
                stage_raw(a.szc + zb);
                rbase = rbase_box - (a.szc + zb) * a.rplane;
            }
        }
        const int2 dln = __ldg(&a.search_delta[min(s + 1, a.S - 1)]);
        phase_a(dl.x);
        __syncthreads();
        f32x2 d0[NP], d1[NP];
        {
            const float w0 = a.w[0];
            float win[16];
            load_window<RX / 4, (RX + kVoxPerThread - 1) / 4>(D + rowoff + RZ * G::DPLANE + RY * G::DP, win);
#pragma unroll
            for (int p = 0; p < NP; p++) d0[p] = mul_pair(win[RX + 2 * p], win[RX + 2 * p + 1], w0);
            load_window<RX / 4, (RX + kVoxPerThread - 1) / 4>(
                D + rowoff + (RZ + 1) * G::DPLANE + RY * G::DP, win);
#pragma unroll
            for (int p = 0; p < NP; p++) d1[p] = mul_pair(win[RX + 2 * p], win[RX + 2 * p + 1], w0);
        }
        accumulate_row_pairs<RX, RY, RZ, TZ, 0>(D, rowoff, d0, d1, a);
        accumulate(d0, m0, rbase + dl.y, acc0, wsum0, wmax0);
        accumulate(d1, m1, rbase + a.rplane + dl.y, acc1, wsum1, wmax1);
        __syncthreads();
        dl = dln;
    }

    const int y = Y0 + j;
#pragma unroll
    for (int pl = 0; pl < 2; pl++) {
        const int z = Z0 + k + pl;
        if (z >= a.nz || y >= a.ny) continue;
        float* orow = a.out + ((long long)z * a.ny + y) * a.nx;
        const long long gb = (long long)(z + a.pz) * a.gpitch_z + (long long)(y + a.py) * a.gpitch_y +
                             (X0 + x0 + a.px);
#pragma unroll
        for (int r = 0; r < kVoxPerThread; r++) {
            const int x = X0 + x0 + r;
            if (x < a.nx) {
                const float raw0 = SLAB ? __ldg(&a.raw_pad[gb + r]) : rawb[rbase + pl * a.rplane + r];
                const float2 acp = unpack2(pl ? acc1[r / 2] : acc0[r / 2]);
                const float2 wsp = unpack2(pl ? wsum1[r / 2] : wsum0[r / 2]);
                const float wm = pl ? wmax1[r] : wmax0[r];
                float ac = (r & 1) ? acp.y : acp.x;
                float ws = (r & 1) ? wsp.y : wsp.x;
                float res;
                if (wm > 0.0f) {
                    ac = __fadd_rn(ac, __fmul_rn(wm, raw0));
                    ws = __fadd_rn(ws, wm);
                    res = __fdiv_rn(ac, ws);
                } else {
                    res = raw0;
                }
                orow[x] = res;
            }
        }
    }
}

template <int RX, int RY, int RZ, bool SLAB>
__global__ void __launch_bounds__(256, 1)
    nlm_tile_f32_z2_kernel(const __grid_constant__ CUtensorMap tm_prev, const __grid_constant__ TileArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    if (threadIdx.x == 0) {
        prefetch_tmap(&tm_prev);
        mbar_init(reinterpret_cast<uint64_t*>(smem), 1);
        fence_mbar_init();
    }
    __syncthreads();
    tile_f32_z2_body<RX, RY, RZ, SLAB>(&tm_prev, a, smem);
}

// ---- warp-specialised tile kernel ----
//
// The 8-deep tile kernel's two phases on different warps, so that the
// squared differences of the next offsets are formed while the patch sums of
// the current ones run: producer warps write the D planes of NO offsets into
// one of NSLOT slots (a ring of D buffers), 8 consumer warps (the lane map and
// per-voxel arithmetic of tile_f32_body's phase B) read a slot, weight and
// accumulate its offsets in reference order and release it. Raw is staged in
// shared memory (RAW_SMEM: the raw box, one offset per slot, three slots) or
// read from global memory as aligned float4s (two offsets per slot, two
// slots). Full / empty mbarriers per slot, every wait bounded (on expiry the
// CTA records DEV_TMA_TIMEOUT and its warps return; the other role's waits then
// expire too). Bit-identical to the reference like tile_f32_body; FUSED: the
// fused FP32 form's taps and weights (as tile_f32_body's FUSED form, whose
// results it equals bit for bit).
//
// Producer warps: 8 at patch radius 1 and 2 (measured 6 % faster than 4 at
// p2 s5 and s7, where the consumers waited on the ring), 4 at radius 3 (8
// would cap the larger consumer bodies at 128 registers: measured 2 % slower).
template <int RX>
struct WsThreads {
    static constexpr int NPR = RX >= 3 ? 128 : 256;  // producer threads
    static constexpr int N = 256 + NPR;
};

template <int RX, int RY, int RZ, bool RAW_SMEM, bool FUSED>
__global__ void __launch_bounds__(WsThreads<RX>::N, 1)
    nlm_tile_f32_ws_kernel(const __grid_constant__ CUtensorMap tm_prev, const __grid_constant__ TileArgs a) {
    constexpr int TZ = 8;
    using G = TileGeom<RX, RY, RZ, TZ>;
    constexpr int NC = 256;  // consumer threads (phase B)
    constexpr int NPR = WsThreads<RX>::NPR;  // producer threads (phase A)
    constexpr int NO = RAW_SMEM ? 1 : 2;     // offsets per slot
    constexpr int NSLOT = RAW_SMEM ? 3 : 2;  // slots in the ring
    constexpr int NP = kVoxPerThread / 2;
    constexpr int DSZ = round_up32(G::DPLANE * G::DD);
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);  // prev box, full[NSLOT], empty[NSLOT]
    uint64_t* full = bar + 1;
    uint64_t* empty = bar + 1 + NSLOT;
    float* prevb = reinterpret_cast<float*>(smem + 128);
    const int pplane = a.pbx * a.pby;
    const int PB = pplane * a.pbz;
    float* rawb = prevb + round_up32(PB);
    const int rpx = a.rbx + 1;
    float* Dring = rawb + (RAW_SMEM ? round_up32(a.rplane * a.rbz) : 0);
    const int tid = threadIdx.x;
    const int X0 = blockIdx.x * kTX;
    const int Y0 = blockIdx.y * kTY;
    const int Z0 = blockIdx.z * TZ;
    if (tid == 0) {
        prefetch_tmap(&tm_prev);
        mbar_init(&bar[0], 1);
        for (int i = 0; i < NSLOT; i++) {
            mbar_init(&full[i], NPR);
            mbar_init(&empty[i], NC);
        }
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0) {
        mbar_arrive_expect_tx(&bar[0], (uint32_t)PB * 4u);
        tma_load_3d(prevb, &tm_prev, X0, Y0, Z0, &bar[0]);
    }
    if (RAW_SMEM) {
        // raw over tile + search halo, odd row pitch (as tile_f32_body), while
        // the prev box arrives; the barrier below publishes it
        const int rb_n = a.rbx * a.rby * a.rbz;
        const float* rsrc = a.raw_pad + (long long)(Z0 + RZ) * a.gpitch_z + (long long)(Y0 + RY) * a.gpitch_y + X0;
        for (int i = tid; i < rb_n; i += NC + NPR) {
            int xx = i % a.rbx;
            int rest = i / a.rbx;
            int yy = rest % a.rby;
            int zz = rest / a.rby;
            rawb[zz * a.rplane + yy * rpx + xx] =
                __ldg(rsrc + (long long)zz * a.gpitch_z + (long long)yy * a.gpitch_y + xx);
        }
    }
    const bool arrived = mbar_wait_bounded(&bar[0], 0);
    if (!__syncthreads_and(arrived)) {
        if (tid == 0) set_error(a.err, DEV_TMA_TIMEOUT);
        return;
    }
    const int npairs = (a.S + NO - 1) / NO;

    if (tid >= NC) {
        // ---- producers: D = (prev(. + s) - prev(.))^2 over tile + patch halo
        const int pt = tid - NC;
        constexpr int NPAIR = G::ND / 2;
        constexpr int NQ = (NPAIR + NPR - 1) / NPR;
        int qpi[NQ], qdi[NQ];
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            int e = min(pt + q * NPR, NPAIR - 1);  // the tail repeats the last pair
            int f = 2 * e;
            int c = f % G::DW;
            int rest = f / G::DW;
            int r = rest % G::DH;
            int pz = rest / G::DH;
            qpi[q] = (pz - RZ + a.pz) * pplane + (r - RY + a.py) * a.pbx + (c - RX + a.px);
            qdi[q] = pz * G::DPLANE + r * G::DP + c;
        }
        f32x2 qog[NQ];
#pragma unroll
        for (int q = 0; q < NQ; q++) qog[q] = pack2(prevb[qpi[q]], prevb[qpi[q] + 1]);
        for (int j = 0; j < npairs; j++) {
            const int slot = j % NSLOT;
            if (j >= NSLOT && !mbar_wait_bounded(&empty[slot], (j / NSLOT - 1) & 1)) {
                set_error(a.err, DEV_TMA_TIMEOUT);
                return;
            }
#pragma unroll
            for (int o = 0; o < NO; o++) {
                const int s = j * NO + o;
                if (s < a.S) {
                    const int dlx = __ldg(&a.search_delta[s]).x;
                    float* Dw = Dring + (slot * NO + o) * DSZ;
                    // every pair index has the parity of px - RX (box pitches
                    // are even): an 8-byte aligned shifted pair is one load
                    if (((a.px - RX + dlx) & 1) == 0) {
#pragma unroll
                        for (int q = 0; q < NQ; q++) {
                            f32x2 sh = *reinterpret_cast<const f32x2*>(prevb + qpi[q] + dlx);
                            f32x2 v = sub2(sh, qog[q]);
                            *reinterpret_cast<f32x2*>(Dw + qdi[q]) = mul2_to_mul(v, v);  // stored, not added
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < NQ; q++) {
                            f32x2 sh = pack2(prevb[qpi[q] + dlx], prevb[qpi[q] + dlx + 1]);
                            f32x2 v = sub2(sh, qog[q]);
                            *reinterpret_cast<f32x2*>(Dw + qdi[q]) = mul2_to_mul(v, v);
                        }
                    }
                }
            }
            mbar_arrive(&full[slot]);
        }
        return;
    }

    // ---- consumers: patch sums, weights and sums (phase B of tile_f32_body)
    const int warp = tid >> 5, lane = tid & 31;
    const int k = 4 * (warp >> 2) + (lane >> 3);
    const int j8 = lane & 7;
    const int x0 = (warp & 3) * kVoxPerThread;
    const int zk = min(Z0 + k, a.nz - 1);
    const f32x2 m2 = splat2(a.mult[zk]);
    const int rowoff = k * G::DPLANE + j8 * G::DP + x0;
    const long long gbase = (long long)(Z0 + k + a.pz) * a.gpitch_z + (long long)(Y0 + j8 + a.py) * a.gpitch_y +
                            (X0 + x0 + a.px);
    const int rbase = RAW_SMEM ? (a.szc + k) * a.rplane + (a.syr + j8) * rpx + (RX + a.sxr + x0) : 0;
    f32x2 acc[NP], wsum[NP];
    float wmax[kVoxPerThread];
#pragma unroll
    for (int p = 0; p < NP; p++) acc[p] = wsum[p] = 0ull;  // (+0, +0)
#pragma unroll
    for (int r = 0; r < kVoxPerThread; r++) wmax[r] = 0.0f;
    bool ok = true;
    for (int j = 0; j < npairs; j++) {
        const int slot = j % NSLOT;
        if (!mbar_wait_bounded(&full[slot], (j / NSLOT) & 1)) {
            set_error(a.err, DEV_TMA_TIMEOUT);
            ok = false;
            break;
        }
        const float* D0 = Dring + slot * NO * DSZ;
        f32x2 d[NO][NP];
        {
            const int ro = rowoff + RZ * G::DPLANE + RY * G::DP;
            const float w0 = a.w[0];
#pragma unroll
            for (int o = 0; o < NO; o++) {
                float win[16];
                load_window<RX / 4, (RX + kVoxPerThread - 1) / 4>(D0 + o * DSZ + ro, win);
#pragma unroll
                for (int p = 0; p < NP; p++) d[o][p] = mul_pair(win[RX + 2 * p], win[RX + 2 * p + 1], w0);
            }
        }
        accumulate_rows_n<RX, RY, RZ, TZ, NO, 0, FUSED>(D0, DSZ, rowoff, d, a);
        // the slot's D planes are no longer read: hand it back before the weights
        mbar_arrive(&empty[slot]);
#pragma unroll
        for (int o = 0; o < NO; o++) {
            const int s = j * NO + o;
            if (s < a.S) {
                const int dly = __ldg(&a.search_delta[s]).y;
                float rg[kVoxPerThread];
                if (RAW_SMEM) {
#pragma unroll
                    for (int r = 0; r < kVoxPerThread; r++) rg[r] = rawb[rbase + dly + r];
                } else {
                    load8_global(a.raw_pad + gbase + dly, rg);
                }
#pragma unroll
                for (int p = 0; p < NP; p++) {
                    if (FUSED)
                        fused_weight_pair(d[o][p], m2, make_float2(rg[2 * p], rg[2 * p + 1]), acc[p], wsum[p],
                                          wmax[2 * p], wmax[2 * p + 1]);
                    else
                        exact_weight_pair(d[o][p], m2, make_float2(rg[2 * p], rg[2 * p + 1]), acc[p], wsum[p],
                                          wmax[2 * p], wmax[2 * p + 1]);
                }
            }
        }
    }
    if (!ok) return;
    const int z = Z0 + k, y = Y0 + j8;
    if (z < a.nz && y < a.ny) {
        float* orow = a.out + ((long long)z * a.ny + y) * a.nx;
#pragma unroll
        for (int r = 0; r < kVoxPerThread; r++) {
            const int x = X0 + x0 + r;
            if (x < a.nx) {
                const float raw0 = RAW_SMEM ? rawb[rbase + r] : __ldg(&a.raw_pad[gbase + r]);
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
                orow[x] = res;
            }
        }
    }
}

template <int RX, int RY, int RZ, int TZ, bool RAW_SMEM, bool FUSED, bool SLAB>
__global__ void __launch_bounds__(32 * TZ, 1)
    nlm_tile_f32_kernel(const __grid_constant__ CUtensorMap tm_prev, const __grid_constant__ TileArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    if (threadIdx.x == 0) {
        prefetch_tmap(&tm_prev);
        mbar_init(reinterpret_cast<uint64_t*>(smem), 1);
        fence_mbar_init();
    }
    __syncthreads();
    tile_f32_body<RX, RY, RZ, TZ, RAW_SMEM, FUSED, SLAB>(&tm_prev, a, blockIdx.x, blockIdx.y, blockIdx.z,
                                                        smem, 0, a);
}

// Persistent batch kernel: CTAs take (volume, tile) items from a counter
// until the batch is done; each volume runs the body of its patch shape and
// tile configuration (kind). Items are numbered volume by volume in the order
// the host gives (heaviest tiles first), tiles x-fastest within a volume.
template <int RX, int RY, int RZ, bool RAW_SMEM, bool SLAB>
__device__ __forceinline__ bool batch_item(const BatchParams& bp, int v, int local,
                                           unsigned char* smem, uint32_t parity) {
    const TileArgs& a = bp.args[v];
    const int bx = local % a.tiles_x;
    const int rest = local / a.tiles_x;
    const int by = rest % a.tiles_y;
    const int bz = rest / a.tiles_y;
    return tile_f32_body<RX, RY, RZ, 8, RAW_SMEM, false, SLAB>(&bp.maps[v], a, bx, by, bz, smem, parity,
                                                              bp.args[0]);
}

static_assert(sizeof(BatchParams) <= 32764, "batch parameter block exceeds the kernel parameter limit");

// One persistent kernel per patch shape R and raw placement (a kernel mixing
// bodies would carry the largest one's registers, shared memory and code for
// every tile); volumes of any size and search radius. Radius 1 keeps to 128
// registers so two CTAs fit an SM, as its per-volume kernel does.
template <int R, bool RAW_SMEM, bool SLAB = false>
__global__ void __launch_bounds__(256, R == 1 ? 2 : 1)
    nlm_batch_f32_kernel(const __grid_constant__ BatchParams bp) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_item;
    if (threadIdx.x == 0) {
        for (int v = 0; v < bp.n; v++) prefetch_tmap(&bp.maps[v]);
        mbar_init(reinterpret_cast<uint64_t*>(smem), 1);
        fence_mbar_init();
    }
    uint32_t parity = 0;
    for (;;) {
        __syncthreads();  // the previous item's shared memory is free
        if (threadIdx.x == 0) s_item = (int)atomicAdd(bp.counter, 1u);
        __syncthreads();
        const int item = s_item;
        if (item >= bp.item_begin[bp.n]) break;
        int v = 0;
        while (v + 1 < bp.n && item >= bp.item_begin[v + 1]) v++;
        const int local = item - bp.item_begin[v];
        const bool ok = batch_item<R, R, R, RAW_SMEM, SLAB>(bp, v, local, smem, parity);
        if (!ok) break;  // uniform over the CTA; the error flag is set
        parity ^= 1u;
    }
}

// ---- generic exact kernel: any patch shape, one thread per voxel ----
__global__ void __launch_bounds__(256) nlm_generic_f32_kernel(const __grid_constant__ GenericArgs a) {
    long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long nvox = (long long)a.nx * a.ny * a.nz;
    if (idx >= nvox) return;
    int x = (int)(idx % a.nx);
    long long rest = idx / a.nx;
    int y = (int)(rest % a.ny);
    int z = (int)(rest / a.ny);
    long long i0 = (long long)(z + a.pz) * a.gpitch_z + (long long)(y + a.py) * a.gpitch_y + (x + a.px);
    const float m = a.mult[z];
    const float raw0 = a.raw_pad[i0];
    float acc = 0.0f, wsum = 0.0f, wmax = 0.0f;
    for (int s = 0; s < a.S; s++) {
        long long i1 = i0 + a.search_off[s];
        float dist = 0.0f;
        for (int q = 0; q < a.P; q++) {
            long long po = a.patch_off[q];
            float t = __fsub_rn(a.prev_pad[i1 + po], a.prev_pad[i0 + po]);
            dist = __fadd_rn(dist, __fmul_rn(__fmul_rn(t, t), a.weights[q]));
        }
        float wt = pade_weight_exact(__fmul_rn(dist, m));
        acc = __fadd_rn(acc, __fmul_rn(wt, a.raw_pad[i1]));
        wsum = __fadd_rn(wsum, wt);
        wmax = fmaxf(wmax, wt);
    }
    float res = raw0;
    if (wmax > 0.0f) res = __fdiv_rn(__fadd_rn(acc, __fmul_rn(wmax, raw0)), __fadd_rn(wsum, wmax));
    a.out[idx] = res;
}

// ---- reflective padding (iternlm_prepare.cpp:6-48 / iternlm_gpu.cu:27) ----
__global__ void pad_reflective_kernel(const float* __restrict__ in, int nx, int ny, int nz,
                                      float* __restrict__ out, int px, int py, int pz,
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
        // mirror without edge repeat, repeated while out of range; the host
        // rejects axes of length 1 that would need padding, so this ends
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
        out[z1 * pitch_z + y1 * pitch_y + x1] = in[((long long)z0 * ny + y0) * nx + x0];
    }
}

__global__ void sigma_to_mult_kernel(const float* __restrict__ sigma, float beta,
                                     float* __restrict__ mult, int nz) {
    int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z < nz) {
        float s = sigma[z];
        // -1.f/(sigma*sigma*beta), iternlm_cpu.cpp:95
        mult[z] = __fdiv_rn(-1.f, __fmul_rn(__fmul_rn(s, s), beta));
    }
}

__global__ void sigma_blend_kernel(const float* __restrict__ sigma0, float* __restrict__ sigma1,
                                   float alpha, int nz) {
    int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z < nz) {
        // alpha*sigma0 + (1-alpha)*sigma1, main.cpp:442-443
        sigma1[z] = __fadd_rn(__fmul_rn(alpha, sigma0[z]),
                              __fmul_rn(__fsub_rn(1.f, alpha), sigma1[z]));
    }
}

// ---- host-side dispatch ----

template <int RX, int RY, int RZ, int TZ, bool RAW_SMEM>
static size_t smem_bytes_for(const TileArgs& a) {
    using G = TileGeom<RX, RY, RZ, TZ>;
    size_t pb = round_up32(a.pbx * a.pby * a.pbz);
    size_t rb = RAW_SMEM ? round_up32(a.rplane * a.rbz) : 0;
    size_t d = round_up32(G::DPLANE * G::DD);
    // the 16-deep kernel keeps one D buffer (one offset per barrier step)
    return 128 + 4 * (pb + rb + (TZ == 16 ? 1 : kOffGroup) * d);
}

template <int RX, int RY, int RZ, bool SLAB>
static cudaError_t launch_z2(const CUtensorMap* tmp, const TileArgs& a, int tiles_z, size_t smem,
                             cudaStream_t st) {
    auto kern = nlm_tile_f32_z2_kernel<RX, RY, RZ, SLAB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid(a.tiles_x, a.tiles_y, tiles_z);
    kern<<<grid, 256, smem, st>>>(*tmp, a);
    return cudaGetLastError();
}

template <int RX, int RY, int RZ, int TZ, bool RAW_SMEM, bool FUSED = false, bool SLAB = false>
static cudaError_t launch_inst(const CUtensorMap* tmp, const CUtensorMap* tmr, const TileArgs& a,
                               int tiles_z, size_t smem, cudaStream_t st) {
    (void)tmr;
    auto kern = nlm_tile_f32_kernel<RX, RY, RZ, TZ, RAW_SMEM, FUSED, SLAB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid(a.tiles_x, a.tiles_y, tiles_z);
    kern<<<grid, 32 * TZ, smem, st>>>(*tmp, a);
    return cudaGetLastError();
}

int batch_kind(const TileConfig& c) {
    if (c.tz != 8) return -1;
    if (c.rx == 1 && c.ry == 1 && c.rz == 1)
        return c.raw_slab ? kBatchP111Slab : c.raw_smem ? kBatchP111Smem : kBatchP111Glob;
    if (c.rx == 2 && c.ry == 2 && c.rz == 2)
        return c.raw_slab ? kBatchP222Slab : c.raw_smem ? kBatchP222Smem : kBatchP222Glob;
    if (c.rx == 3 && c.ry == 3 && c.rz == 3)
        return c.raw_slab ? kBatchP333Slab : c.raw_smem ? kBatchP333Smem : kBatchP333Glob;
    return -1;
}

template <int R, bool RAW, bool SLAB = false>
static cudaError_t batch_setup_r(size_t smem, int* ctas_per_sm) {
    cudaError_t e = cudaFuncSetAttribute(nlm_batch_f32_kernel<R, RAW, SLAB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, nlm_batch_f32_kernel<R, RAW, SLAB>,
                                                         256, smem);
}

cudaError_t batch_kernel_setup(int kind, size_t smem, int* ctas_per_sm) {
    switch (kind) {
        case kBatchP111Smem: return batch_setup_r<1, true>(smem, ctas_per_sm);
        case kBatchP111Glob: return batch_setup_r<1, false>(smem, ctas_per_sm);
        case kBatchP222Smem: return batch_setup_r<2, true>(smem, ctas_per_sm);
        case kBatchP222Glob: return batch_setup_r<2, false>(smem, ctas_per_sm);
        case kBatchP333Smem: return batch_setup_r<3, true>(smem, ctas_per_sm);
        case kBatchP333Glob: return batch_setup_r<3, false>(smem, ctas_per_sm);
        case kBatchP111Slab: return batch_setup_r<1, true, true>(smem, ctas_per_sm);
        case kBatchP222Slab: return batch_setup_r<2, true, true>(smem, ctas_per_sm);
        case kBatchP333Slab: return batch_setup_r<3, true, true>(smem, ctas_per_sm);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_batch_kernel(int kind, const BatchParams& bp, int ctas, size_t smem,
                                cudaStream_t st) {
    switch (kind) {
        case kBatchP111Smem: nlm_batch_f32_kernel<1, true><<<ctas, 256, smem, st>>>(bp); break;
        case kBatchP111Glob: nlm_batch_f32_kernel<1, false><<<ctas, 256, smem, st>>>(bp); break;
        case kBatchP222Smem: nlm_batch_f32_kernel<2, true><<<ctas, 256, smem, st>>>(bp); break;
        case kBatchP222Glob: nlm_batch_f32_kernel<2, false><<<ctas, 256, smem, st>>>(bp); break;
        case kBatchP333Smem: nlm_batch_f32_kernel<3, true><<<ctas, 256, smem, st>>>(bp); break;
        case kBatchP333Glob: nlm_batch_f32_kernel<3, false><<<ctas, 256, smem, st>>>(bp); break;
        case kBatchP111Slab: nlm_batch_f32_kernel<1, true, true><<<ctas, 256, smem, st>>>(bp); break;
        case kBatchP222Slab: nlm_batch_f32_kernel<2, true, true><<<ctas, 256, smem, st>>>(bp); break;
        case kBatchP333Slab: nlm_batch_f32_kernel<3, true, true><<<ctas, 256, smem, st>>>(bp); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

#define INLM_FOR_EACH_SHAPE(X) \
    X(1, 1, 1) X(1, 1, 2) X(1, 1, 3) X(2, 2, 1) X(2, 2, 2) X(3, 3, 1) X(3, 3, 2) X(3, 3, 3)

bool tile_kernel_available(int rx, int ry, int rz) {
#define X(a, b, c) \
    if (rx == a && ry == b && rz == c) return true;
    INLM_FOR_EACH_SHAPE(X)
#undef X
    return false;
}

size_t tile_smem_bytes(const TileConfig& c, const TileArgs& a) {
#define X(A, B, C)                                                                    \
    if (c.rx == A && c.ry == B && c.rz == C) {                                        \
        if (c.tz == 16 && c.raw_smem) return smem_bytes_for<A, B, C, 16, true>(a);   \
        if (c.tz == 8 && c.raw_smem) return smem_bytes_for<A, B, C, 8, true>(a);     \
        if (c.tz == 8 && !c.raw_smem) return smem_bytes_for<A, B, C, 8, false>(a);   \
        if (c.tz == 4 && !c.raw_smem) return smem_bytes_for<A, B, C, 4, false>(a);   \
    }
    INLM_FOR_EACH_SHAPE(X)
#undef X
    return 0;
}

size_t tile_ws_smem_bytes(const TileConfig& c, const TileArgs& a) {
    // raw box and three single-offset buffers, or raw from global and two pairs
#define X(A, B, C)                                                                  \
    if (c.rx == A && c.ry == B && c.rz == C) {                                      \
        using G = TileGeom<A, B, C, 8>;                                             \
        const size_t rb = c.raw_smem ? round_up32(a.rplane * a.rbz) : 0;           \
        return 128 + 4 * (round_up32(a.pbx * a.pby * a.pbz) + rb +                  \
                          (c.raw_smem ? 3 : 4) * (size_t)round_up32(G::DPLANE * G::DD)); \
    }
    INLM_FOR_EACH_SHAPE(X)
#undef X
    return 0;
}

template <int RX, int RY, int RZ>
static cudaError_t launch_ws(const CUtensorMap* tmp, const TileArgs& a, int tiles_z, size_t smem, bool raw_smem,
                             bool fused, cudaStream_t st) {
    auto kern = fused ? (raw_smem ? nlm_tile_f32_ws_kernel<RX, RY, RZ, true, true>
                                  : nlm_tile_f32_ws_kernel<RX, RY, RZ, false, true>)
                      : (raw_smem ? nlm_tile_f32_ws_kernel<RX, RY, RZ, true, false>
                                  : nlm_tile_f32_ws_kernel<RX, RY, RZ, false, false>);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid(a.tiles_x, a.tiles_y, tiles_z);
    kern<<<grid, WsThreads<RX>::N, smem, st>>>(*tmp, a);
    return cudaGetLastError();
}

cudaError_t launch_tile_kernel(const TileConfig& c, const CUtensorMap* tm_prev,
                               const CUtensorMap* tm_raw, const TileArgs& a, int tiles_z,
                               cudaStream_t st) {
    if (c.column) return launch_column_kernel(c, tm_prev, a, tiles_z, st);
    if (c.ws) {
#define X(A, B, C) \
        if (c.rx == A && c.ry == B && c.rz == C)                                                      \
            return launch_ws<A, B, C>(tm_prev, a, tiles_z, c.smem_bytes, c.raw_smem, c.fused, st);
        INLM_FOR_EACH_SHAPE(X)
#undef X
        return cudaErrorInvalidConfiguration;
    }
#define X(A, B, C)                                                                             \
    if (c.rx == A && c.ry == B && c.rz == C) {                                                 \
        if (c.tz == 16 && c.raw_smem && !c.fused)                                              \
            return c.raw_slab ? launch_z2<A, B, C, true>(tm_prev, a, tiles_z, c.smem_bytes, st)   \
                              : launch_z2<A, B, C, false>(tm_prev, a, tiles_z, c.smem_bytes, st); \
        if (c.raw_slab && c.tz == 8 && c.raw_smem)                                             \
            return c.fused ? launch_inst<A, B, C, 8, true, true, true>(tm_prev, tm_raw, a, tiles_z,  \
                                                                      c.smem_bytes, st)        \
                           : launch_inst<A, B, C, 8, true, false, true>(tm_prev, tm_raw, a, tiles_z, \
                                                                       c.smem_bytes, st);      \
        if (c.raw_slab) return cudaErrorInvalidConfiguration;                                  \
        if (c.fused && c.tz == 8 && c.raw_smem)                                                \
            return launch_inst<A, B, C, 8, true, true>(tm_prev, tm_raw, a, tiles_z, c.smem_bytes, st); \
        if (c.fused && c.tz == 8 && !c.raw_smem)                                               \
            return launch_inst<A, B, C, 8, false, true>(tm_prev, tm_raw, a, tiles_z, c.smem_bytes, st); \
        if (c.fused) return cudaErrorInvalidConfiguration;                                     \
        if (c.tz == 8 && c.raw_smem)                                                           \
            return launch_inst<A, B, C, 8, true>(tm_prev, tm_raw, a, tiles_z, c.smem_bytes, st);  \
        if (c.tz == 8 && !c.raw_smem)                                                          \
            return launch_inst<A, B, C, 8, false>(tm_prev, tm_raw, a, tiles_z, c.smem_bytes, st); \
        if (c.tz == 4 && !c.raw_smem)                                                          \
            return launch_inst<A, B, C, 4, false>(tm_prev, tm_raw, a, tiles_z, c.smem_bytes, st); \
    }
    INLM_FOR_EACH_SHAPE(X)
#undef X
    return cudaErrorInvalidConfiguration;
}

template <int RX, int RY, int RZ>
static int tap_order_impl(int* xyz, int max_taps) {
    constexpr PatchRows rows = make_patch_rows(RX, RY, RZ);
    int n = 0;
    auto put = [&](int x, int y, int z) {
        if (n < max_taps) {
            xyz[3 * n] = x;
            xyz[3 * n + 1] = y;
            xyz[3 * n + 2] = z;
        }
        n++;
    };
    put(0, 0, 0);
    for (int ri = 0; ri < rows.n; ri++)
        for (int xp = -rows.e[ri]; xp <= rows.e[ri]; xp++)
            if (!(rows.zp[ri] == 0 && rows.yp[ri] == 0 && xp == 0)) put(xp, rows.yp[ri], rows.zp[ri]);
    return n;
}

int tile_kernel_tap_order(int rx, int ry, int rz, int* xyz, int max_taps) {
#define X(A, B, C) \
    if (rx == A && ry == B && rz == C) return tap_order_impl<A, B, C>(xyz, max_taps);
    INLM_FOR_EACH_SHAPE(X)
#undef X
    return -1;
}

cudaError_t launch_generic_kernel(const GenericArgs& a, cudaStream_t st) {
    long long nvox = (long long)a.nx * a.ny * a.nz;
    int blocks = (int)((nvox + 255) / 256);
    nlm_generic_f32_kernel<<<blocks, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_pad_reflective(const float* in, int nx, int ny, int nz, float* out, int px,
                                  int py, int pz, long long pitch_y, long long pitch_z,
                                  cudaStream_t st) {
    pad_reflective_kernel<<<148 * 8, 256, 0, st>>>(in, nx, ny, nz, out, px, py, pz, pitch_y,
                                                   pitch_z);
    return cudaGetLastError();
}

cudaError_t launch_sigma_to_mult(const float* sigma, float beta, float* mult, int nz,
                                 cudaStream_t st) {
    sigma_to_mult_kernel<<<(nz + 255) / 256, 256, 0, st>>>(sigma, beta, mult, nz);
    return cudaGetLastError();
}

cudaError_t launch_sigma_blend(const float* sigma0, float* sigma1, float alpha, int nz,
                               cudaStream_t st) {
    sigma_blend_kernel<<<(nz + 255) / 256, 256, 0, st>>>(sigma0, sigma1, alpha, nz);
    return cudaGetLastError();
}

// ---- failure-path self-test of the bounded wait ----
// One CTA arms an mbarrier for 1024 bytes that no copy delivers and waits on
// it with mbar_wait_bounded, the wait every TMA-staged kernel uses, under a
// budget of `cycles`: the wait gives up, the CTA agrees on it as the filter
// kernels do and records DEV_TMA_TIMEOUT, and the kernel returns. No copy is
// in flight, so nothing is left pending when the CTA exits.
__global__ void __launch_bounds__(32) selftest_wait_kernel(int* err, long long cycles) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 1024u);
    const bool arrived = mbar_wait_bounded(&bar, 0, cycles);
    if (!__syncthreads_and(arrived) && threadIdx.x == 0) set_error(err, DEV_TMA_TIMEOUT);
}

cudaError_t launch_selftest_wait(int* err, long long cycles, cudaStream_t st) {
    selftest_wait_kernel<<<1, 32, 0, st>>>(err, cycles);
    return cudaGetLastError();
}

}  // namespace inlm

