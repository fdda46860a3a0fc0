// Host geometry tables; see geometry.hpp. Built with -ffp-contract=off so the
// float expressions round as the reference's g++ build rounds them.
#include "geometry.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>

namespace inlm {

static bool in_ellipsoid(int x, int y, int z, float rx, float ry, float rz) {
    // iternlm_prepare.cpp:139 / :191
    volatile float a = (float)x / rx, b = (float)y / ry, c = (float)z / rz;
    volatile float v = a * a;
    v = v + b * b;
    v = v + c * c;
    return v <= 1.f;
}

static bool is_specialised_shape(const int* r) {
    static const int shapes[8][3] = {{1, 1, 1}, {1, 1, 2}, {1, 1, 3}, {2, 2, 1},
                                     {2, 2, 2}, {3, 3, 1}, {3, 3, 2}, {3, 3, 3}};
    for (auto& s : shapes)
        if (r[0] == s[0] && r[1] == s[1] && r[2] == s[2]) return true;
    return false;
}

Geometry make_geometry(const int sr[3], const int pr[3], int nslices, float z_anisotropy,
                       int weight_table, int nz_padded) {
    Geometry g;
    for (int i = 0; i < 3; i++) {
        g.search_radius[i] = sr[i];
        g.patch_radius[i] = pr[i];
    }
    g.nslices = nslices;
    // iternlm_cpu.cpp:18-23
    g.pad[0] = sr[0] + pr[0];
    g.pad[1] = sr[1] + pr[1];
    g.pad[2] = std::min(nslices / 2, sr[2]) + pr[2];

    // setup_searchspace, iternlm_prepare.cpp:102-150
    {
        float rx = (float)std::max(sr[0], 1), ry = (float)std::max(sr[1], 1),
              rz = (float)std::max(sr[2], 1);
        for (int zs = -sr[2]; zs <= sr[2]; zs++)
            for (int ys = -sr[1]; ys <= sr[1]; ys++)
                for (int xs = -sr[0]; xs <= sr[0]; xs++) {
                    if (std::abs(zs) > nslices / 2) continue;
                    if (zs == 0 && ys == 0 && xs == 0) continue;
                    if (in_ellipsoid(xs, ys, zs, rx, ry, rz)) g.search.push_back({xs, ys, zs});
                }
    }
    // setup_patchspace :152-202 and setup_distweight :204-262
    {
        float rx = (float)std::max(pr[0], 1), ry = (float)std::max(pr[1], 1),
              rz = (float)std::max(pr[2], 1);
        volatile float sq_an = z_anisotropy * z_anisotropy;
        float maxweight = 0.0f;
        g.taps.push_back({0, 0, 0});
        g.weights.push_back(1.f);
        for (int zp = -pr[2]; zp <= pr[2]; zp++)
            for (int yp = -pr[1]; yp <= pr[1]; yp++)
                for (int xp = -pr[0]; xp <= pr[0]; xp++) {
                    if (std::abs(zp) > nslices / 2) continue;
                    if (zp == 0 && yp == 0 && xp == 0) continue;
                    if (in_ellipsoid(xp, yp, zp, rx, ry, rz)) {
                        volatile float zz = (float)(zp * zp) * sq_an;
                        volatile float s = (float)(xp * xp + yp * yp) + zz;
                        volatile float d = sqrtf(s);
                        volatile float t = 2.f * d;
                        t = t + 1.f;
                        volatile float tt = t * t;
                        float wt = 1.f / tt;
                        if (wt > maxweight) maxweight = wt;
                        g.taps.push_back({xp, yp, zp});
                        g.weights.push_back(wt);
                    }
                }
        g.weights[0] = maxweight;
        if (rx == 1.f && ry == 1.f && rz == 1.f && nz_padded > 1)
            for (auto& w : g.weights) w = 1.f / 7.f;
    }
    g.specialised = is_specialised_shape(pr);
    if (weight_table == 0 && g.specialised) {
        // the specialised kernels carry the isotropic table; z_anisotropy
        // does not reach them
        if (z_anisotropy != 1.f)
            g.weights = make_geometry(sr, pr, nslices, 1.f, 1, nz_padded).weights;
        bool r111 = pr[0] == 1 && pr[1] == 1 && pr[2] == 1;
        for (auto& w : g.weights) {
            if (r111) {
                w = 0.142857143f;  // iternlm_cpu_kernels.cpp:57-63
            } else {
                char buf[64];
                std::snprintf(buf, sizeof buf, "%g", (double)w);
                w = std::strtof(buf, nullptr);
            }
        }
    }
    return g;
}

}  // namespace inlm
