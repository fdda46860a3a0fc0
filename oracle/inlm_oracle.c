/*
 * inlm_oracle.c — TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * Plain-C restatement of the reference iterNLM_v0.3 hot path. Each function
 * cites the reference file:line it restates. Compiled with
 * -ffp-contract=off and no fast-math so float expressions round exactly as
 * the reference's g++ -O3 (SSE, no FMA) build rounds them.
 *
 * Parity pinned bit-for-bit against the reference CPU build (oracle/_ref) and
 * against fixtures generated from it (tests/golden/).
 */
#include "inlm_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }

void ora_padding(const ora_params* p, int pad[3]) {
    /* iternlm_cpu.cpp:18-23 */
    pad[0] = p->search_radius[0] + p->patch_radius[0];
    pad[1] = p->search_radius[1] + p->patch_radius[1];
    pad[2] = imin(p->nslices / 2, p->search_radius[2]) + p->patch_radius[2];
}

/* float32 ellipsoid membership as written at iternlm_prepare.cpp:139 / :191 */
static int in_ellipsoid(int x, int y, int z, float rx, float ry, float rz) {
    float a = (float)x / rx, b = (float)y / ry, c = (float)z / rz;
    float v = a * a + b * b;
    v = v + c * c;
    return v <= 1.f;
}

int ora_search_offsets(const ora_params* p, int* dx, int* dy, int* dz, int max_n) {
    /* iternlm_prepare.cpp:102-150 */
    const int* r = p->search_radius;
    float rx = (float)imax(r[0], 1), ry = (float)imax(r[1], 1), rz = (float)imax(r[2], 1);
    int n = 0;
    for (int zs = -r[2]; zs <= r[2]; zs++)
        for (int ys = -r[1]; ys <= r[1]; ys++)
            for (int xs = -r[0]; xs <= r[0]; xs++) {
                if (abs(zs) > p->nslices / 2) continue;
                if (zs == 0 && ys == 0 && xs == 0) continue;
                if (in_ellipsoid(xs, ys, zs, rx, ry, rz)) {
                    if (n < max_n) { dx[n] = xs; dy[n] = ys; dz[n] = zs; }
                    n++;
                }
            }
    return n;
}

int ora_patch_taps(const ora_params* p, int* dx, int* dy, int* dz, int max_n) {
    /* iternlm_prepare.cpp:152-202 */
    const int* r = p->patch_radius;
    float rx = (float)imax(r[0], 1), ry = (float)imax(r[1], 1), rz = (float)imax(r[2], 1);
    int n = 0;
    if (max_n > 0) { dx[0] = dy[0] = dz[0] = 0; }
    n = 1;
    for (int zp = -r[2]; zp <= r[2]; zp++)
        for (int yp = -r[1]; yp <= r[1]; yp++)
            for (int xp = -r[0]; xp <= r[0]; xp++) {
                if (abs(zp) > p->nslices / 2) continue;
                if (zp == 0 && yp == 0 && xp == 0) continue;
                if (in_ellipsoid(xp, yp, zp, rx, ry, rz)) {
                    if (n < max_n) { dx[n] = xp; dy[n] = yp; dz[n] = zp; }
                    n++;
                }
            }
    return n;
}

int ora_distweight(const ora_params* p, int nz, float* w, int max_n) {
    /* iternlm_prepare.cpp:204-262 */
    const int* r = p->patch_radius;
    float rx = (float)imax(r[0], 1), ry = (float)imax(r[1], 1), rz = (float)imax(r[2], 1);
    float sq_an = p->z_anisotropy * p->z_anisotropy;
    float maxweight = 0.0f;
    int n = 1;
    for (int zp = -r[2]; zp <= r[2]; zp++)
        for (int yp = -r[1]; yp <= r[1]; yp++)
            for (int xp = -r[0]; xp <= r[0]; xp++) {
                if (abs(zp) > p->nslices / 2) continue;
                if (zp == 0 && yp == 0 && xp == 0) continue;
                if (in_ellipsoid(xp, yp, zp, rx, ry, rz)) {
                    /* (xp*xp)+(yp*yp) is integer arithmetic in the reference */
                    float d = sqrtf((float)(xp * xp + yp * yp) + (float)(zp * zp) * sq_an);
                    float t = 2.f * d + 1.f;
                    float wt = 1.f / (t * t);
                    if (wt > maxweight) maxweight = wt;
                    if (n < max_n) w[n] = wt;
                    n++;
                }
            }
    if (max_n > 0) w[0] = maxweight;
    /* padded nz > 1 (:257) */
    if (rx == 1.f && ry == 1.f && rz == 1.f && nz > 1)
        for (int i = 0; i < n && i < max_n; i++) w[i] = 1.f / 7.f;
    return n;
}

static int is_specialised(const int* r) {
    /* dispatch iternlm_cpu.cpp:97-114 */
    static const int shapes[8][3] = {{1, 1, 1}, {1, 1, 2}, {1, 1, 3}, {2, 2, 1},
                                     {2, 2, 2}, {3, 3, 1}, {3, 3, 2}, {3, 3, 3}};
    for (int i = 0; i < 8; i++)
        if (r[0] == shapes[i][0] && r[1] == shapes[i][1] && r[2] == shapes[i][2]) return 1;
    return 0;
}

int ora_filter_weights(const ora_params* p, int nz, float* w, int max_n, int* specialised) {
    int spec = is_specialised(p->patch_radius);
    if (specialised) *specialised = spec;
    if (!spec) return ora_distweight(p, nz, w, max_n);
    /* the specialised kernels carry the isotropic table: z_anisotropy does
     * not reach them */
    ora_params iso = *p;
    iso.z_anisotropy = 1.0f;
    int n = ora_distweight(&iso, nz, w, max_n);
    int r111 = p->patch_radius[0] == 1 && p->patch_radius[1] == 1 && p->patch_radius[2] == 1;
    for (int i = 0; i < n && i < max_n; i++) {
        if (r111) {
            /* iternlm_cpu_kernels.cpp:57-63: 0.142857143f for every tap */
            w[i] = 0.142857143f;
        } else {
            /* the specialised kernels hold the table as printed by the
             * reference's own generator (iternlm_gpu.cu:1500, default ostream
             * precision = 6 significant digits) */
            char buf[64];
            snprintf(buf, sizeof buf, "%g", (double)w[i]);
            w[i] = strtof(buf, NULL);
        }
    }
    return n;
}

void ora_pad_reflective(const float* in, const int shape[3], const int pad[3], float* out) {
    /* iternlm_prepare.cpp:6-48 (symmetric padding) */
    int nx0 = shape[0], ny0 = shape[1], nz0 = shape[2];
    int nx1 = nx0 + 2 * pad[0], ny1 = ny0 + 2 * pad[1], nz1 = nz0 + 2 * pad[2];
    long long nslice0 = (long long)nx0 * ny0;
#pragma omp parallel for
    for (int z1 = 0; z1 < nz1; z1++)
        for (int y1 = 0; y1 < ny1; y1++)
            for (int x1 = 0; x1 < nx1; x1++) {
                int z0 = z1 - pad[2], y0 = y1 - pad[1], x0 = x1 - pad[0];
                while (z0 < 0 || z0 >= nz0 || y0 < 0 || y0 >= ny0 || x0 < 0 || x0 >= nx0) {
                    if (z0 < 0) z0 = -z0;
                    if (y0 < 0) y0 = -y0;
                    if (x0 < 0) x0 = -x0;
                    if (z0 >= nz0) z0 = 2 * nz0 - z0 - 2;
                    if (y0 >= ny0) y0 = 2 * ny0 - y0 - 2;
                    if (x0 >= nx0) x0 = 2 * nx0 - x0 - 2;
                }
                out[((long long)z1 * ny1 + y1) * nx1 + x1] = in[z0 * nslice0 + (long long)y0 * nx0 + x0];
            }
}

#define ORA_MAXS 20000
#define ORA_MAXP 1000

/* 3rd-order Pade of exp, iternlm_cpu.h:125; cutoff iternlm_cpu.h:126 */
static float pade_f32(float x) {
    return (120.f + 60.f * x + 12.f * x * x + x * x * x) /
           (120.f - 60.f * x + 12.f * x * x - x * x * x);
}
static const float PADE_CUTOFF = -3.56648f;
static double pade_f64(double x) {
    return (120.0 + 60.0 * x + 12.0 * x * x + x * x * x) /
           (120.0 - 60.0 * x + 12.0 * x * x - x * x * x);
}

void ora_filter_f32(const float* raw_pad, const float* prev_pad, const int shape[3],
                    const ora_params* p, const float* mult, float* out) {
    int pad[3];
    ora_padding(p, pad);
    int nx = shape[0], ny = shape[1], nz = shape[2];
    long long nxp = nx + 2 * pad[0], nyp = ny + 2 * pad[1];
    long long nsl = nxp * nyp;
    static int sdx[ORA_MAXS], sdy[ORA_MAXS], sdz[ORA_MAXS];
    int pdx[ORA_MAXP], pdy[ORA_MAXP], pdz[ORA_MAXP];
    float w[ORA_MAXP];
    int ns = ora_search_offsets(p, sdx, sdy, sdz, ORA_MAXS);
    int np = ora_patch_taps(p, pdx, pdy, pdz, ORA_MAXP);
    ora_filter_weights(p, nz + 2 * pad[2], w, ORA_MAXP, NULL);
    long long* soff = (long long*)malloc(sizeof(long long) * ns);
    long long poff[ORA_MAXP];
    for (int s = 0; s < ns; s++) soff[s] = sdz[s] * nsl + sdy[s] * nxp + sdx[s];
    for (int q = 0; q < np; q++) poff[q] = pdz[q] * nsl + pdy[q] * nxp + pdx[q];

#pragma omp parallel for schedule(dynamic)
    for (int z = 0; z < nz; z++) {
        float m = mult[z];
        float vorig[ORA_MAXP];
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                long long idx0 = (z + pad[2]) * nsl + (y + pad[1]) * nxp + (x + pad[0]);
                float raw0 = raw_pad[idx0];
                for (int q = 0; q < np; q++) vorig[q] = prev_pad[idx0 + poff[q]];
                float acc = 0.0f, wsum = 0.0f, wmax = 0.0f;
                for (int s = 0; s < ns; s++) {
                    long long idx1 = idx0 + soff[s];
                    float rs = raw_pad[idx1];
                    float dist = 0.0f;
                    for (int q = 0; q < np; q++) {
                        float t = prev_pad[idx1 + poff[q]] - vorig[q];
                        float sq = t * t;
                        float term = sq * w[q];
                        dist = dist + term;
                    }
                    dist = dist * m;
                    float wt = (dist > PADE_CUTOFF) ? pade_f32(dist) : 0.0f;
                    float prod = wt * rs;
                    acc = acc + prod;
                    wsum = wsum + wt;
                    if (wt > wmax) wmax = wt;
                }
                float r;
                if (wmax > 0.0f) {
                    float prod = wmax * raw0;
                    acc = acc + prod;
                    wsum = wsum + wmax;
                    r = acc / wsum;
                } else {
                    r = raw0;
                }
                out[((long long)z * ny + y) * nx + x] = r;
            }
    }
    free(soff);
}

void ora_filter_f64(const double* raw_pad, const double* prev_pad, const int shape[3],
                    const ora_params* p, const double* mult, double* out) {
    int pad[3];
    ora_padding(p, pad);
    int nx = shape[0], ny = shape[1], nz = shape[2];
    long long nxp = nx + 2 * pad[0], nyp = ny + 2 * pad[1];
    long long nsl = nxp * nyp;
    static int sdx[ORA_MAXS], sdy[ORA_MAXS], sdz[ORA_MAXS];
    int pdx[ORA_MAXP], pdy[ORA_MAXP], pdz[ORA_MAXP];
    float wf[ORA_MAXP];
    double w[ORA_MAXP];
    int ns = ora_search_offsets(p, sdx, sdy, sdz, ORA_MAXS);
    int np = ora_patch_taps(p, pdx, pdy, pdz, ORA_MAXP);
    ora_filter_weights(p, nz + 2 * pad[2], wf, ORA_MAXP, NULL);
    for (int q = 0; q < np; q++) w[q] = (double)wf[q];
    long long* soff = (long long*)malloc(sizeof(long long) * ns);
    long long poff[ORA_MAXP];
    for (int s = 0; s < ns; s++) soff[s] = sdz[s] * nsl + sdy[s] * nxp + sdx[s];
    for (int q = 0; q < np; q++) poff[q] = pdz[q] * nsl + pdy[q] * nxp + pdx[q];
    const double cut = (double)PADE_CUTOFF;
#pragma omp parallel for schedule(dynamic)
    for (int z = 0; z < nz; z++) {
        double m = mult[z];
        double vorig[ORA_MAXP];
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                long long idx0 = (z + pad[2]) * nsl + (y + pad[1]) * nxp + (x + pad[0]);
                double raw0 = raw_pad[idx0];
                for (int q = 0; q < np; q++) vorig[q] = prev_pad[idx0 + poff[q]];
                double acc = 0.0, wsum = 0.0, wmax = 0.0;
                for (int s = 0; s < ns; s++) {
                    long long idx1 = idx0 + soff[s];
                    double dist = 0.0;
                    for (int q = 0; q < np; q++) {
                        double t = prev_pad[idx1 + poff[q]] - vorig[q];
                        dist += t * t * w[q];
                    }
                    dist *= m;
                    double wt = (dist > cut) ? pade_f64(dist) : 0.0;
                    acc += wt * raw_pad[idx1];
                    wsum += wt;
                    if (wt > wmax) wmax = wt;
                }
                out[((long long)z * ny + y) * nx + x] =
                    (wmax > 0.0) ? (acc + wmax * raw0) / (wsum + wmax) : raw0;
            }
    }
    free(soff);
}

static void sigma_to_mult_f32(const float* sigma, int nz, float beta, float* mult) {
    /* iternlm_cpu.cpp:94-95 */
    for (int z = 0; z < nz; z++) {
        float s = sigma[z];
        mult[z] = -1.f / (s * s * beta);
    }
}

void ora_denoise_f32(const float* raw, const int shape[3], const ora_params* p,
                     const float* sigmas, int n_iter, float* out_last, float* out_all) {
    int pad[3];
    ora_padding(p, pad);
    int pshape[3] = {shape[0] + 2 * pad[0], shape[1] + 2 * pad[1], shape[2] + 2 * pad[2]};
    long long nvox = (long long)shape[0] * shape[1] * shape[2];
    long long npad = (long long)pshape[0] * pshape[1] * pshape[2];
    float* raw_pad = (float*)malloc(npad * sizeof(float));
    float* prev_pad = (float*)malloc(npad * sizeof(float));
    float* cur = (float*)malloc(nvox * sizeof(float));
    float* mult = (float*)malloc(shape[2] * sizeof(float));
    ora_pad_reflective(raw, shape, pad, raw_pad);
    memcpy(prev_pad, raw_pad, npad * sizeof(float));
    for (int it = 1; it <= n_iter; it++) {
        if (it > 1) ora_pad_reflective(cur, shape, pad, prev_pad);
        sigma_to_mult_f32(sigmas + (long long)(it - 1) * shape[2], shape[2], p->beta, mult);
        ora_filter_f32(raw_pad, prev_pad, shape, p, mult, cur);
        if (out_all) memcpy(out_all + (long long)(it - 1) * nvox, cur, nvox * sizeof(float));
    }
    memcpy(out_last, cur, nvox * sizeof(float));
    free(raw_pad); free(prev_pad); free(cur); free(mult);
}

static void pad_reflective_f64(const double* in, const int shape[3], const int pad[3], double* out) {
    int nx0 = shape[0], ny0 = shape[1], nz0 = shape[2];
    int nx1 = nx0 + 2 * pad[0], ny1 = ny0 + 2 * pad[1], nz1 = nz0 + 2 * pad[2];
#pragma omp parallel for
    for (int z1 = 0; z1 < nz1; z1++)
        for (int y1 = 0; y1 < ny1; y1++)
            for (int x1 = 0; x1 < nx1; x1++) {
                int z0 = z1 - pad[2], y0 = y1 - pad[1], x0 = x1 - pad[0];
                while (z0 < 0 || z0 >= nz0 || y0 < 0 || y0 >= ny0 || x0 < 0 || x0 >= nx0) {
                    if (z0 < 0) z0 = -z0;
                    if (y0 < 0) y0 = -y0;
                    if (x0 < 0) x0 = -x0;
                    if (z0 >= nz0) z0 = 2 * nz0 - z0 - 2;
                    if (y0 >= ny0) y0 = 2 * ny0 - y0 - 2;
                    if (x0 >= nx0) x0 = 2 * nx0 - x0 - 2;
                }
                out[((long long)z1 * ny1 + y1) * nx1 + x1] =
                    in[((long long)z0 * ny0 + y0) * nx0 + x0];
            }
}

void ora_denoise_f64(const float* raw, const int shape[3], const ora_params* p,
                     const float* sigmas, int n_iter, double* out_last) {
    int pad[3];
    ora_padding(p, pad);
    int pshape[3] = {shape[0] + 2 * pad[0], shape[1] + 2 * pad[1], shape[2] + 2 * pad[2]};
    long long nvox = (long long)shape[0] * shape[1] * shape[2];
    long long npad = (long long)pshape[0] * pshape[1] * pshape[2];
    double* rawd = (double*)malloc(nvox * sizeof(double));
    double* raw_pad = (double*)malloc(npad * sizeof(double));
    double* prev_pad = (double*)malloc(npad * sizeof(double));
    double* mult = (double*)malloc(shape[2] * sizeof(double));
    for (long long i = 0; i < nvox; i++) rawd[i] = raw[i];
    pad_reflective_f64(rawd, shape, pad, raw_pad);
    memcpy(prev_pad, raw_pad, npad * sizeof(double));
    for (int it = 1; it <= n_iter; it++) {
        if (it > 1) pad_reflective_f64(out_last, shape, pad, prev_pad);
        for (int z = 0; z < shape[2]; z++) {
            double s = sigmas[(long long)(it - 1) * shape[2] + z];
            mult[z] = -1.0 / (s * s * (double)p->beta);
        }
        ora_filter_f64(raw_pad, prev_pad, shape, p, mult, out_last);
    }
    free(rawd); free(raw_pad); free(prev_pad); free(mult);
}

/* ---------------- noise ---------------- */

void ora_srand(ora_rand_state* st, unsigned int seed) {
    /* glibc random_r.c __srandom_r, TYPE_3: Schrage's method for 16807*r mod
     * (2^31-1), then 310 discarded outputs. Kept as a 34-entry sliding
     * history of r[i-34..i-1]. */
    int32_t r[34];
    if (seed == 0) seed = 1;
    r[0] = (int32_t)seed;
    int32_t word = (int32_t)seed; /* 32-bit state word, 64-bit hi/lo */
    for (int i = 1; i < 31; i++) {
        int64_t hi = word / 127773;
        int64_t lo = word % 127773;
        word = (int32_t)(16807 * lo - 2836 * hi);
        if (word < 0) word += 2147483647;
        r[i] = word;
    }
    for (int i = 31; i < 34; i++) r[i] = r[i - 31];
    for (int i = 0; i < 34; i++) st->r[i] = (uint32_t)r[i];
    st->k = 0; /* number of values generated beyond r[33] */
    for (int i = 0; i < 310; i++) (void)ora_rand(st);
}

int ora_rand(ora_rand_state* st) {
    /* r[i] = r[i-3] + r[i-31] (mod 2^32); output r[i] >> 1 */
    uint32_t v = st->r[34 - 3] + st->r[34 - 31];
    memmove(st->r, st->r + 1, 33 * sizeof(uint32_t));
    st->r[33] = v;
    st->k++;
    return (int)(v >> 1);
}

static int cmp_i64(const void* a, const void* b) {
    int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
    return (x > y) - (x < y);
}

void ora_draw_samples(const int shape[3], int64_t n_samples, int patchsize,
                      int circular_mask_diameter, unsigned int seed, int64_t* out) {
    /* noiselevel.cpp:192-234, sequential rand() order */
    int nx = shape[0], ny = shape[1], nz = shape[2];
    long long nslice = (long long)nx * ny;
    float maxradiussq = (float)(circular_mask_diameter / 2.f - sqrt((double)(2 * patchsize * patchsize)));
    maxradiussq *= maxradiussq;
    ora_rand_state st;
    ora_srand(&st, seed);
    for (int64_t s = 0; s < n_samples; s++) {
        int x = ora_rand(&st) % (nx - patchsize);
        int y = ora_rand(&st) % (ny - patchsize);
        int z = ora_rand(&st) % nz;
        if (circular_mask_diameter > 0) {
            float radiussq = (float)((x - nx / 2) * (x - nx / 2) + (y - ny / 2) * (y - ny / 2));
            while (radiussq > maxradiussq) {
                x = ora_rand(&st) % (nx - patchsize);
                y = ora_rand(&st) % (ny - patchsize);
                radiussq = (float)((x - nx / 2) * (x - nx / 2) + (y - ny / 2) * (y - ny / 2));
            }
        }
        out[s] = z * nslice + (long long)y * nx + x;
    }
    qsort(out, (size_t)n_samples, sizeof(int64_t), cmp_i64);
}

void ora_patchstd(const float* stack, const int shape[3], const int64_t* samples, int64_t n,
                  int patchsize, float* out) {
    /* noiselevel.cpp:235-283 */
    int nx = shape[0];
    long long nslice = (long long)shape[0] * shape[1];
    int patchlength = patchsize * patchsize;
#pragma omp parallel for
    for (int64_t s = 0; s < n; s++) {
        long long idx = samples[s];
        int z0 = (int)(idx / nslice);
        int y0 = (int)((idx - z0 * nslice) / nx);
        int x0 = (int)(idx - z0 * nslice - (long long)y0 * nx);
        float sum = 0;
        for (int y = y0; y < y0 + patchsize; y++) {
            long long pos0 = z0 * nslice + (long long)y * nx + x0;
            for (int x = 0; x < patchsize; x++) sum += stack[pos0 + x];
        }
        float mean = sum / patchlength;
        float sq_sum = 0.0f;
        for (int y = y0; y < y0 + patchsize; y++) {
            long long pos0 = z0 * nslice + (long long)y * nx + x0;
            for (int x = 0; x < patchsize; x++) {
                float val = stack[pos0 + x];
                float d = val - mean;
                sq_sum += d * d;
            }
        }
        float variance = sq_sum / patchlength;
        out[s] = sqrtf(variance);
    }
}

/* membership probability as written at noiselevel.cpp:456-457: the 1./ is a
 * double division, the product is rounded to float on assignment */
static float cluster_prob(float val, float mean, float var) {
    const float PI = 3.141592654f;
    float d = val - mean;
    float e = expf(-(d * d / (2 * var)));
    return (float)(1. / (sqrtf(var * 2 * PI)) * (double)e);
}

void ora_create2clusters_f32(const float* values, int n_samples, int firstpos, int lastpos,
                             float out[2]) {
    /* noiselevel.cpp:366-528 */
    int fs = 0, ls = n_samples - 1;
    if (firstpos != -1) fs = firstpos;
    if (lastpos != -1) ls = lastpos;
    float minimum = 1e20f, maximum = -1e20f;
    for (int i = fs; i <= ls; i++) {
        float v = values[i];
        if (v < minimum) minimum = v;
        if (v > maximum) maximum = v;
    }
    float mean1 = (float)((double)minimum + 0.25 * (double)(maximum - minimum));
    float mean2 = (float)((double)maximum - 0.25 * (double)(maximum - minimum));
    int* a = (int*)malloc(sizeof(int) * (size_t)(n_samples > 0 ? n_samples : 1));
    float cs1 = 0.f, cs2 = 0.f, n1 = 0.f, n2 = 0.f;
    for (int i = fs; i <= ls; i++) {
        float v = values[i];
        if (v == 0.0f) a[i] = -1;
        else if (fabsf(v - mean1) < fabsf(v - mean2)) { cs1 += v; n1++; a[i] = 0; }
        else { cs2 += v; n2++; a[i] = 1; }
    }
    if (n1 > 0.0f) mean1 = cs1 / n1;
    if (n2 > 0.0f) mean2 = cs2 / n2;
    if (n1 == 0 && n2 == 0) { free(a); out[0] = 0.f; out[1] = 0.f; return; }
    float var1 = 0.f, var2 = 0.f;
    for (int i = fs; i <= ls; i++) {
        float v = values[i];
        if (a[i] == 0) { float d = v - mean1; var1 += d * d; }
        else if (a[i] == 1) { float d = v - mean2; var2 += d * d; }
    }
    var1 /= (n1 > 1.0f ? n1 : 1.0f);
    var2 /= (n2 > 1.0f ? n2 : 1.0f);
    int change = 1;
    unsigned long long iters = 0, maxiters = 1000;
    while (change && var1 > 0.0f && var2 > 0.0f) {
        change = 0;
        iters++;
        cs1 = cs2 = n1 = n2 = 0.0f;
        for (int i = fs; i <= ls; i++) {
            float v = values[i];
            if (v == 0.0f) continue;
            float p1 = cluster_prob(v, mean1, var1);
            float p2 = cluster_prob(v, mean2, var2);
            if (p2 > p1) {
                if (a[i] != 1) { change = 1; a[i] = 1; }
                cs2 += v; n2++;
            } else {
                if (a[i] != 0) { change = 1; a[i] = 0; }
                cs1 += v; n1++;
            }
        }
        if (n1 > 0.0f) mean1 = cs1 / n1;
        if (n2 > 0.0f) mean2 = cs2 / n2;
        var1 = 0.f; var2 = 0.f;
        for (int i = fs; i <= ls; i++) {
            float v = values[i];
            if (a[i] == 0) { float d = v - mean1; var1 += d * d; }
            else if (a[i] == 1) { float d = v - mean2; var2 += d * d; }
        }
        var1 /= (n1 > 1.0f ? n1 : 1.0f);
        var2 /= (n2 > 1.0f ? n2 : 1.0f);
        if (iters == maxiters) break;
    }
    free(a);
    if (mean1 <= mean2 || var2 <= 0.0) { out[0] = mean1; out[1] = sqrtf(var1); }
    else { out[0] = mean2; out[1] = sqrtf(var2); }
}

void ora_create2clusters_f64acc(const float* values, int n_samples, int firstpos, int lastpos,
                                float out[2]) {
    int fs = 0, ls = n_samples - 1;
    if (firstpos != -1) fs = firstpos;
    if (lastpos != -1) ls = lastpos;
    float minimum = 1e20f, maximum = -1e20f;
    for (int i = fs; i <= ls; i++) {
        float v = values[i];
        if (v < minimum) minimum = v;
        if (v > maximum) maximum = v;
    }
    float mean1 = (float)((double)minimum + 0.25 * (double)(maximum - minimum));
    float mean2 = (float)((double)maximum - 0.25 * (double)(maximum - minimum));
    int* a = (int*)malloc(sizeof(int) * (size_t)(n_samples > 0 ? n_samples : 1));
    double cs1 = 0, cs2 = 0;
    long long n1 = 0, n2 = 0;
    for (int i = fs; i <= ls; i++) {
        float v = values[i];
        if (v == 0.0f) a[i] = -1;
        else if (fabsf(v - mean1) < fabsf(v - mean2)) { cs1 += v; n1++; a[i] = 0; }
        else { cs2 += v; n2++; a[i] = 1; }
    }
    if (n1 > 0) mean1 = (float)(cs1 / (double)n1);
    if (n2 > 0) mean2 = (float)(cs2 / (double)n2);
    if (n1 == 0 && n2 == 0) { free(a); out[0] = 0.f; out[1] = 0.f; return; }
    double v1 = 0, v2 = 0;
    for (int i = fs; i <= ls; i++) {
        float v = values[i];
        if (a[i] == 0) { float d = v - mean1; v1 += (double)(d * d); }
        else if (a[i] == 1) { float d = v - mean2; v2 += (double)(d * d); }
    }
    float var1 = (float)(v1 / (double)(n1 > 1 ? n1 : 1));
    float var2 = (float)(v2 / (double)(n2 > 1 ? n2 : 1));
    int change = 1;
    int iters = 0;
    while (change && var1 > 0.0f && var2 > 0.0f) {
        change = 0;
        iters++;
        cs1 = cs2 = 0; n1 = n2 = 0;
        for (int i = fs; i <= ls; i++) {
            float v = values[i];
            if (v == 0.0f) continue;
            float p1 = cluster_prob(v, mean1, var1);
            float p2 = cluster_prob(v, mean2, var2);
            if (p2 > p1) {
                if (a[i] != 1) { change = 1; a[i] = 1; }
                cs2 += v; n2++;
            } else {
                if (a[i] != 0) { change = 1; a[i] = 0; }
                cs1 += v; n1++;
            }
        }
        if (n1 > 0) mean1 = (float)(cs1 / (double)n1);
        if (n2 > 0) mean2 = (float)(cs2 / (double)n2);
        v1 = 0; v2 = 0;
        for (int i = fs; i <= ls; i++) {
            float v = values[i];
            if (a[i] == 0) { float d = v - mean1; v1 += (double)(d * d); }
            else if (a[i] == 1) { float d = v - mean2; v2 += (double)(d * d); }
        }
        var1 = (float)(v1 / (double)(n1 > 1 ? n1 : 1));
        var2 = (float)(v2 / (double)(n2 > 1 ? n2 : 1));
        if (iters == 1000) break;
    }
    free(a);
    if (mean1 <= mean2 || var2 <= 0.0f) { out[0] = mean1; out[1] = sqrtf(var1); }
    else { out[0] = mean2; out[1] = sqrtf(var2); }
}

void ora_zwindows(const int64_t* samples, int64_t n, const int shape[3], int windowsize,
                  int* start, int* end) {
    /* noiselevel.cpp:538-546. The end index stops on the first sample past
     * the window (it is included in the inclusive range), as in the
     * reference. The start scan is bounded to the array (the reference reads
     * past the end only when every sample lies below the window). */
    long long nslice = (long long)shape[0] * shape[1];
    int startpos = 0, endpos = 0;
    for (int pos = 0; pos < shape[2]; pos++) {
        while (startpos < n - 1 && samples[startpos] / nslice <= (pos - windowsize / 2)) startpos++;
        while ((endpos < (int)(n - 1)) && (samples[endpos] / nslice <= (pos + windowsize / 2))) endpos++;
        start[pos] = startpos;
        end[pos] = endpos;
    }
}

void ora_fill_empty_slices(float* mean, float* sd, int nz) {
    /* noiselevel.cpp:571-603 */
    float max_std = -1.f;
    int zero = 0;
    for (int i = 0; i < nz; i++) {
        if (mean[i] > max_std) max_std = mean[i];
        if (mean[i] == 0.0f) zero = 1;
    }
    if (!(zero && max_std > 0.0f)) return;
    while (zero) {
        zero = 0;
        for (int i = 0; i < nz; i++) {
            float this_var = mean[i];
            if (this_var == 0.0f) {
                float nv = 0.0f, nvs = 0.0f;
                int count = 0;
                if (i > 0 && mean[i - 1] > 0.0f) { nv += mean[i - 1]; nvs += sd[i - 1]; count++; }
                if (i < nz - 1 && mean[i + 1] > 0.0f) { nv += mean[i + 1]; nvs += sd[i + 1]; count++; }
                if (count > 0) {
                    this_var = nv / count;
                    mean[i] = this_var;
                    sd[i] = nvs / count;
                }
            }
            if (this_var == 0.0f) zero = 1;
        }
    }
}

void ora_noise_from_patchstd(const float* patchstd, const int64_t* samples, int64_t n,
                             const int shape[3], int mode, int zwindow, float stds_from_mean,
                             int f64acc, float* sigma) {
    int nz = shape[2];
    float ms[2];
    if (mode == 0) {
        /* noiselevel.cpp:55-61 */
        if (f64acc) ora_create2clusters_f64acc(patchstd, (int)n, -1, -1, ms);
        else ora_create2clusters_f32(patchstd, (int)n, -1, -1, ms);
        for (int z = 0; z < nz; z++) sigma[z] = ms[0] + stds_from_mean * ms[1];
        return;
    }
    /* noiselevel.cpp:45-53, 529-606 */
    int* st = (int*)malloc(sizeof(int) * nz);
    int* en = (int*)malloc(sizeof(int) * nz);
    float* mean = (float*)malloc(sizeof(float) * nz);
    float* sd = (float*)malloc(sizeof(float) * nz);
    ora_zwindows(samples, n, shape, zwindow, st, en);
#pragma omp parallel for schedule(dynamic)
    for (int z = 0; z < nz; z++) {
        float r[2];
        if (f64acc) ora_create2clusters_f64acc(patchstd, (int)n, st[z], en[z], r);
        else ora_create2clusters_f32(patchstd, (int)n, st[z], en[z], r);
        mean[z] = r[0];
        sd[z] = r[1];
    }
    ora_fill_empty_slices(mean, sd, nz);
    for (int z = 0; z < nz; z++) sigma[z] = mean[z] + stds_from_mean * sd[z];
    free(st); free(en); free(mean); free(sd);
}

void ora_filter_f32_voxels(const float* raw_pad, const float* prev_pad, const int shape[3],
                           const ora_params* p, const float* mult, int64_t n,
                           const int64_t* voxels, float* out) {
    /* the FP32 filter of ora_filter_f32 evaluated at the given unpadded linear
     * voxel indices only (for sampled parity on full-size volumes) */
    int pad[3];
    ora_padding(p, pad);
    int nx = shape[0], ny = shape[1], nz = shape[2];
    long long nxp = nx + 2 * pad[0], nyp = ny + 2 * pad[1];
    long long nsl = nxp * nyp;
    static int sdx[ORA_MAXS], sdy[ORA_MAXS], sdz[ORA_MAXS];
    int pdx[ORA_MAXP], pdy[ORA_MAXP], pdz[ORA_MAXP];
    float w[ORA_MAXP];
    int ns = ora_search_offsets(p, sdx, sdy, sdz, ORA_MAXS);
    int np = ora_patch_taps(p, pdx, pdy, pdz, ORA_MAXP);
    ora_filter_weights(p, nz + 2 * pad[2], w, ORA_MAXP, NULL);
    long long* soff = (long long*)malloc(sizeof(long long) * ns);
    long long poff[ORA_MAXP];
    for (int s = 0; s < ns; s++) soff[s] = sdz[s] * nsl + sdy[s] * nxp + sdx[s];
    for (int q = 0; q < np; q++) poff[q] = pdz[q] * nsl + pdy[q] * nxp + pdx[q];
#pragma omp parallel for schedule(dynamic)
    for (int64_t i = 0; i < n; i++) {
        int64_t v = voxels[i];
        int x = (int)(v % nx);
        int y = (int)((v / nx) % ny);
        int z = (int)(v / ((int64_t)nx * ny));
        float m = mult[z];
        float vorig[ORA_MAXP];
        long long idx0 = (z + pad[2]) * nsl + (y + pad[1]) * nxp + (x + pad[0]);
        float raw0 = raw_pad[idx0];
        for (int q = 0; q < np; q++) vorig[q] = prev_pad[idx0 + poff[q]];
        float acc = 0.0f, wsum = 0.0f, wmax = 0.0f;
        for (int s = 0; s < ns; s++) {
            long long idx1 = idx0 + soff[s];
            float dist = 0.0f;
            for (int q = 0; q < np; q++) {
                float t = prev_pad[idx1 + poff[q]] - vorig[q];
                float sq = t * t;
                float term = sq * w[q];
                dist = dist + term;
            }
            dist = dist * m;
            float wt = (dist > PADE_CUTOFF) ? pade_f32(dist) : 0.0f;
            float prod = wt * raw_pad[idx1];
            acc = acc + prod;
            wsum = wsum + wt;
            if (wt > wmax) wmax = wt;
        }
        if (wmax > 0.0f) {
            float prod = wmax * raw0;
            acc = acc + prod;
            wsum = wsum + wmax;
            out[i] = acc / wsum;
        } else {
            out[i] = raw0;
        }
    }
    free(soff);
}

void ora_sigma_to_mult(const float* sigma, int nz, float beta, float* mult) {
    sigma_to_mult_f32(sigma, nz, beta, mult);
}

void ora_denoise_f64_plan(const float* raw, const int shape[3], const ora_params* p,
                          const float* sigmas, int n_iter, const int tile[3],
                          const unsigned char* keep, long long keep_iter_stride, double* out_last) {
    /* ora_denoise_f64 with the search restricted, per tile of tile[0] x
     * tile[1] x tile[2] voxels (x fastest tile index), to the offsets whose
     * keep[tile * S + s] is set; wmax is taken over the kept offsets. */
    int pad[3];
    ora_padding(p, pad);
    int nx = shape[0], ny = shape[1], nz = shape[2];
    long long nxp = nx + 2 * pad[0], nyp = ny + 2 * pad[1], nzp = nz + 2 * pad[2];
    long long nsl = nxp * nyp, npad = nsl * nzp, nvox = (long long)nx * ny * nz;
    static int sdx[ORA_MAXS], sdy[ORA_MAXS], sdz[ORA_MAXS];
    int pdx[ORA_MAXP], pdy[ORA_MAXP], pdz[ORA_MAXP];
    float wf[ORA_MAXP];
    double w[ORA_MAXP];
    int ns = ora_search_offsets(p, sdx, sdy, sdz, ORA_MAXS);
    int np = ora_patch_taps(p, pdx, pdy, pdz, ORA_MAXP);
    ora_filter_weights(p, nz + 2 * pad[2], wf, ORA_MAXP, NULL);
    for (int q = 0; q < np; q++) w[q] = (double)wf[q];
    long long* soff = (long long*)malloc(sizeof(long long) * ns);
    long long poff[ORA_MAXP];
    for (int s = 0; s < ns; s++) soff[s] = sdz[s] * nsl + sdy[s] * nxp + sdx[s];
    for (int q = 0; q < np; q++) poff[q] = pdz[q] * nsl + pdy[q] * nxp + pdx[q];
    int ntx = (nx + tile[0] - 1) / tile[0], nty = (ny + tile[1] - 1) / tile[1];
    double* rawd = (double*)malloc(nvox * sizeof(double));
    double* raw_pad = (double*)malloc(npad * sizeof(double));
    double* prev_pad = (double*)malloc(npad * sizeof(double));
    int sh[3] = {nx, ny, nz};
    for (long long i = 0; i < nvox; i++) rawd[i] = raw[i];
    pad_reflective_f64(rawd, sh, pad, raw_pad);
    memcpy(prev_pad, raw_pad, npad * sizeof(double));
    const double cut = (double)PADE_CUTOFF;
    for (int it = 1; it <= n_iter; it++) {
        if (it > 1) pad_reflective_f64(out_last, sh, pad, prev_pad);
#pragma omp parallel for schedule(dynamic)
        for (int z = 0; z < nz; z++) {
            double sgm = sigmas[(long long)(it - 1) * nz + z];
            double m = -1.0 / (sgm * sgm * (double)p->beta);
            double vorig[ORA_MAXP];
            for (int y = 0; y < ny; y++)
                for (int x = 0; x < nx; x++) {
                    long long t = ((long long)(z / tile[2]) * nty + y / tile[1]) * ntx + x / tile[0];
                    const unsigned char* kp = keep + (it - 1) * keep_iter_stride + t * ns;
                    long long idx0 = (z + pad[2]) * nsl + (y + pad[1]) * nxp + (x + pad[0]);
                    double raw0 = raw_pad[idx0];
                    for (int q = 0; q < np; q++) vorig[q] = prev_pad[idx0 + poff[q]];
                    double acc = 0.0, wsum = 0.0, wmax = 0.0;
                    for (int s = 0; s < ns; s++) {
                        if (!kp[s]) continue;
                        long long idx1 = idx0 + soff[s];
                        double dist = 0.0;
                        for (int q = 0; q < np; q++) {
                            double tt = prev_pad[idx1 + poff[q]] - vorig[q];
                            dist += tt * tt * w[q];
                        }
                        dist *= m;
                        double wt = (dist > cut) ? pade_f64(dist) : 0.0;
                        acc += wt * raw_pad[idx1];
                        wsum += wt;
                        if (wt > wmax) wmax = wt;
                    }
                    out_last[((long long)z * ny + y) * nx + x] =
                        (wmax > 0.0) ? (acc + wmax * raw0) / (wsum + wmax) : raw0;
                }
        }
    }
    free(soff); free(rawd); free(raw_pad); free(prev_pad);
}

void ora_weight_mass_f64(const float* prev, const int shape[3], const ora_params* p,
                         const float* sigma, const int tile[3], double* out) {
    /* the weights of ora_filter_f64 (iternlm_cpu.cpp:758-843 in double) */
    int pad[3];
    ora_padding(p, pad);
    int nx = shape[0], ny = shape[1], nz = shape[2];
    long long nxp = nx + 2 * pad[0], nyp = ny + 2 * pad[1], nzp = nz + 2 * pad[2];
    long long nsl = nxp * nyp, npad = nsl * nzp, nvox = (long long)nx * ny * nz;
    static int sdx[ORA_MAXS], sdy[ORA_MAXS], sdz[ORA_MAXS];
    int pdx[ORA_MAXP], pdy[ORA_MAXP], pdz[ORA_MAXP];
    float wf[ORA_MAXP];
    double w[ORA_MAXP];
    int ns = ora_search_offsets(p, sdx, sdy, sdz, ORA_MAXS);
    int np = ora_patch_taps(p, pdx, pdy, pdz, ORA_MAXP);
    ora_filter_weights(p, nz + 2 * pad[2], wf, ORA_MAXP, NULL);
    for (int q = 0; q < np; q++) w[q] = (double)wf[q];
    long long* soff = (long long*)malloc(sizeof(long long) * ns);
    long long poff[ORA_MAXP];
    for (int s = 0; s < ns; s++) soff[s] = sdz[s] * nsl + sdy[s] * nxp + sdx[s];
    for (int q = 0; q < np; q++) poff[q] = pdz[q] * nsl + pdy[q] * nxp + pdx[q];
    int ntx = (nx + tile[0] - 1) / tile[0], nty = (ny + tile[1] - 1) / tile[1];
    int ntz = (nz + tile[2] - 1) / tile[2];
    long long ntiles = (long long)ntx * nty * ntz;
    double* prevd = (double*)malloc(nvox * sizeof(double));
    double* prev_pad = (double*)malloc(npad * sizeof(double));
    int sh[3] = {nx, ny, nz};
    for (long long i = 0; i < nvox; i++) prevd[i] = prev[i];
    pad_reflective_f64(prevd, sh, pad, prev_pad);
    memset(out, 0, sizeof(double) * ntiles * ns);
    const double cut = (double)PADE_CUTOFF;
    double* wt = (double*)malloc(sizeof(double) * ns);
    for (int z = 0; z < nz; z++) {
        double sgm = sigma[z];
        double m = -1.0 / (sgm * sgm * (double)p->beta);
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                long long t = ((long long)(z / tile[2]) * nty + y / tile[1]) * ntx + x / tile[0];
                long long idx0 = (z + pad[2]) * nsl + (y + pad[1]) * nxp + (x + pad[0]);
                double sum = 0.0;
                for (int s = 0; s < ns; s++) {
                    long long idx1 = idx0 + soff[s];
                    double dist = 0.0;
                    for (int q = 0; q < np; q++) {
                        double tt = prev_pad[idx1 + poff[q]] - prev_pad[idx0 + poff[q]];
                        dist += tt * tt * w[q];
                    }
                    dist *= m;
                    wt[s] = (dist > cut) ? pade_f64(dist) : 0.0;
                    sum += wt[s];
                }
                if (sum > 0.0)
                    for (int s = 0; s < ns; s++) out[t * ns + s] += wt[s] / sum;
            }
    }
    for (long long t = 0; t < ntiles; t++) {
        double sum = 0.0;
        for (int s = 0; s < ns; s++) sum += out[t * ns + s];
        if (sum > 0.0)
            for (int s = 0; s < ns; s++) out[t * ns + s] /= sum;
    }
    free(wt); free(soff); free(prevd); free(prev_pad);
}

/* ---- colour path ---- */

void ora_filter_rgb(const float* const raw[3], const float* const prev[3], int nx, int ny,
                    const ora_params* p2d, const float mult[3], int independent, float* const out[3]) {
    /* IterativeNLM_CPU::filterslice_3channels (iternlm_cpu.cpp:932-1075) on one
     * 2D image: p2d has z radii 0 and nslices 1; the weights are
     * setup_distweight's (iternlm_prepare.cpp:204-262) for a one-slice stack. */
    int pad[3];
    ora_padding(p2d, pad);
    const int shape[3] = {nx, ny, 1};
    long long nxp = nx + 2 * pad[0], nyp = ny + 2 * pad[1];
    static int sdx[ORA_MAXS], sdy[ORA_MAXS], sdz[ORA_MAXS];
    int pdx[ORA_MAXP], pdy[ORA_MAXP], pdz[ORA_MAXP];
    float w[ORA_MAXP];
    int ns = ora_search_offsets(p2d, sdx, sdy, sdz, ORA_MAXS);
    int np = ora_patch_taps(p2d, pdx, pdy, pdz, ORA_MAXP);
    ora_distweight(p2d, 1, w, ORA_MAXP);
    float* rp[3];
    float* pp[3];
    for (int c = 0; c < 3; c++) {
        rp[c] = (float*)malloc(sizeof(float) * nxp * nyp);
        pp[c] = (float*)malloc(sizeof(float) * nxp * nyp);
        ora_pad_reflective(raw[c], shape, pad, rp[c]);
        ora_pad_reflective(prev[c], shape, pad, pp[c]);
    }
#pragma omp parallel for schedule(dynamic)
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
            long long i0 = (y + pad[1]) * nxp + (x + pad[0]);
            float fv[3] = {0.f, 0.f, 0.f}, fw[3] = {0.f, 0.f, 0.f}, mw[3] = {0.f, 0.f, 0.f};
            for (int s = 0; s < ns; s++) {
                long long i1 = i0 + sdy[s] * nxp + sdx[s];
                float d[3] = {0.f, 0.f, 0.f};
                for (int q = 0; q < np; q++) {
                    long long po = pdy[q] * nxp + pdx[q];
                    for (int c = 0; c < 3; c++) {
                        float t = pp[c][i1 + po] - pp[c][i0 + po];
                        float sq = t * t;
                        float term = sq * w[q];
                        d[c] = d[c] + term;
                    }
                }
                for (int c = 0; c < 3; c++) d[c] = d[c] * mult[c];
                if (!independent) {
                    float sum = d[0] + d[1];
                    sum = sum + d[2];
                    float ds = sum / 3.f;
                    float wt = (ds > PADE_CUTOFF) ? pade_f32(ds) : 0.0f;
                    for (int c = 0; c < 3; c++) {
                        float prod = wt * rp[c][i1];
                        fv[c] = fv[c] + prod;
                    }
                    fw[0] = fw[0] + wt;
                    if (wt > mw[0]) mw[0] = wt;
                } else {
                    for (int c = 0; c < 3; c++) {
                        float wt = (d[c] > PADE_CUTOFF) ? pade_f32(d[c]) : 0.0f;
                        float prod = wt * rp[c][i1];
                        fv[c] = fv[c] + prod;
                        fw[c] = fw[c] + wt;
                        if (wt > mw[c]) mw[c] = wt;
                    }
                }
            }
            long long o = (long long)y * nx + x;
            for (int c = 0; c < 3; c++) {
                float r0 = rp[c][i0];
                if (!independent) {
                    if (mw[0] > 0.0f) {
                        float prod = mw[0] * r0;
                        float num = fv[c] + prod;
                        float den = fw[0] + mw[0];
                        out[c][o] = num / den;
                    } else {
                        out[c][o] = r0;
                    }
                } else {
                    out[c][o] = (mw[c] > 0.0f) ? fv[c] / fw[c] : r0;
                }
            }
        }
    for (int c = 0; c < 3; c++) {
        free(rp[c]);
        free(pp[c]);
    }
}

void ora_anscombe(float* v, int64_t n, int inverse) {
    /* colorspace.h:83-125: 2 sqrt(v + 3/8), and (v/2)^2 - 3/8 */
    for (int64_t i = 0; i < n; i++) {
        float r = v[i];
        if (inverse) {
            float h = r / 2.f;
            float sq = h * h;
            v[i] = sq - 3.f / 8.f;
        } else {
            float s = sqrtf(r + 3.f / 8.f);
            v[i] = 2.f * s;
        }
    }
}
