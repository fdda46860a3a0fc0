// Tile geometry shared by the FP32 and FP16 tiled filter kernels.
#pragma once

#include "filter_kernels.cuh"
#include "geometry.hpp"

namespace inlm {

// D-plane row pitch: a multiple of 4 floats with an odd number of 16-byte
// chunks, so the 8 y-lanes x 4 x-lanes of a warp hit distinct bank quads.
constexpr int dpitch(int w) {
    int p = (w + 3) / 4 * 4;
    return ((p / 4) % 2 == 0) ? p + 4 : p;
}
constexpr int round_up32(int v) { return (v + 31) / 32 * 32; }

// TX: CTA width in x (32, or 8 for one 8^3 tile per CTA); 8 voxels per thread.
template <int RX, int RY, int RZ, int TZ, int TX = kTX>
struct TileGeom {
    static constexpr PatchRows rows = make_patch_rows(RX, RY, RZ);
    static constexpr int DW = TX + 2 * RX;
    static constexpr int DH = kTY + 2 * RY;
    static constexpr int DD = TZ + 2 * RZ;
    static constexpr int DP = dpitch(DW);
    static constexpr int DPLANE = DP * DH;
    static constexpr int ND = DW * DH * DD;
    static constexpr int NT = TX * TZ;
};

// Tap counts of the reference geometry (float32 ellipsoid test).
static_assert(make_patch_rows(1, 1, 1).ntaps == 7, "p111");
static_assert(make_patch_rows(1, 1, 2).ntaps == 9, "p112");
static_assert(make_patch_rows(1, 1, 3).ntaps == 11, "p113");
static_assert(make_patch_rows(2, 2, 1).ntaps == 15, "p221");
static_assert(make_patch_rows(2, 2, 2).ntaps == 33, "p222");
static_assert(make_patch_rows(3, 3, 1).ntaps == 31, "p331");
static_assert(make_patch_rows(3, 3, 2).ntaps == 73, "p332");
static_assert(make_patch_rows(3, 3, 3).ntaps == 115, "p333");

// Index of the first tap (xp = -e) of row RI in the reference tap list.
template <int RX, int RY, int RZ, int RI>
struct RowFirst {
    static constexpr PatchRows rows = make_patch_rows(RX, RY, RZ);
    static constexpr int value =
        RowFirst<RX, RY, RZ, RI - 1>::value + 2 * rows.e[RI - 1] + 1 -
        ((rows.zp[RI - 1] == 0 && rows.yp[RI - 1] == 0) ? 1 : 0);
};
template <int RX, int RY, int RZ>
struct RowFirst<RX, RY, RZ, 0> {
    static constexpr int value = 1;
};

}  // namespace inlm
