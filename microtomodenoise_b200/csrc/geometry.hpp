// Search-space and patch-space geometry of the iterNLM filter.
//
// Host tables follow Denoiser/iternlm_prepare.cpp:102-262 with float32
// arithmetic exactly as written there (compiled with -ffp-contract=off):
//   * ellipsoid test (x/rx)^2+(y/ry)^2+(z/rz)^2 <= 1 in float, rx = max(r,1);
//   * z clipped to |z| <= nslices/2;
//   * search: z, y, x ascending, centre excluded;
//   * patch: centre first, then z, y, x ascending;
//   * weights 1/(2d+1)^2, d = sqrtf(x^2+y^2 + z^2 aniso^2), tap 0 = max weight,
//     all 1/7 for radius (1,1,1).
// The reference CPU filter dispatches (iternlm_cpu.cpp:97-114) eight patch
// shapes to kernels with literal weight tables (iternlm_cpu_kernels.cpp) that
// are the distweight values printed to 6 significant digits (p111: 1/7);
// filter_weights() rebuilds that table.
#pragma once

#include <vector>

namespace inlm {

struct Offset3 {
    int x, y, z;
};

struct Geometry {
    int search_radius[3];
    int patch_radius[3];
    int nslices;
    int pad[3];                 // symmetric padding per axis
    std::vector<Offset3> search;  // S offsets, reference order
    std::vector<Offset3> taps;    // P taps, tap 0 = centre
    std::vector<float> weights;   // P weights actually applied by the filter
    bool specialised;             // one of the eight reference CPU kernels
};

// Builds the tables; weight_table: 0 = reference CPU filter table,
// 1 = setup_distweight values. nz_padded feeds the radius-1 special case
// (iternlm_prepare.cpp:257).
Geometry make_geometry(const int search_radius[3], const int patch_radius[3], int nslices,
                       float z_anisotropy, int weight_table, int nz_padded);

// ---- compile-time patch rows for the tiled kernels ----
//
// The patch of radius (RX,RY,RZ) decomposes into rows of constant (zp, yp)
// with xp in [-e, e]; in reference tap order the rows come z-major then y
// (the centre tap is applied first and skipped inside its row).

constexpr bool ell_member(int x, int y, int z, float rx, float ry, float rz) {
    float a = float(x) / rx;
    float b = float(y) / ry;
    float c = float(z) / rz;
    float v = a * a + b * b;
    v = v + c * c;
    return v <= 1.f;
}

struct PatchRows {
    int n;
    int zp[64];
    int yp[64];
    int e[64];
    int ntaps;
};

constexpr PatchRows make_patch_rows(int rx, int ry, int rz) {
    PatchRows r{};
    float fx = float(rx < 1 ? 1 : rx), fy = float(ry < 1 ? 1 : ry), fz = float(rz < 1 ? 1 : rz);
    r.n = 0;
    r.ntaps = 1;
    for (int zp = -rz; zp <= rz; zp++)
        for (int yp = -ry; yp <= ry; yp++) {
            if (!ell_member(0, yp, zp, fx, fy, fz)) continue;
            int e = 0;
            while (e + 1 <= rx && ell_member(e + 1, yp, zp, fx, fy, fz)) e++;
            r.zp[r.n] = zp;
            r.yp[r.n] = yp;
            r.e[r.n] = e;
            r.n++;
            r.ntaps += 2 * e + 1 - ((zp == 0 && yp == 0) ? 1 : 0);
        }
    return r;
}

}  // namespace inlm
