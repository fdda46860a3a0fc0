// The colour path: 2D RGB images denoised with one joint (or per-channel)
// weight per search offset, after an Anscombe transform that turns Poisson
// counts into unit-variance Gaussian values. Replaces
// color_denoise::run_colorimage_denoising (Color/color_denoising.h:19-150),
// IterativeNLM_CPU::Run_GaussianNoise_3channels (Denoiser/iternlm_cpu.cpp:272-400)
// and NoiseLevel::get_noiselevel_2D_RGB (Noise/noiselevel.cpp:96-191).
#include <cmath>
#include <vector>

#include "api_internal.hpp"
#include "color_kernels.cuh"
#include "noise_kernels.cuh"
#include "sampling.hpp"

using namespace inlm;

namespace {

struct RgbJob {
    int device = 0;
    cudaStream_t st = nullptr;
    float* ch[3][3] = {};          // [buffer: raw, a, b][channel]
    long long* d_samples = nullptr;
    float* d_ps = nullptr;         // 3 * ns patch stds
    int2* d_win = nullptr;
    long long* d_off = nullptr;
    signed char* d_assign = nullptr;
    float* d_mean = nullptr;
    float* d_sd = nullptr;
    int2* d_search = nullptr;
    int2* d_taps = nullptr;
    float* d_w = nullptr;
    std::vector<float> host;       // one channel-triple staging area
    ~RgbJob() {
        for (auto& b : ch)
            for (float* p : b) device_free(p);
        device_free(d_samples);
        device_free(d_ps);
        device_free(d_win);
        device_free(d_off);
        device_free(d_assign);
        device_free(d_mean);
        device_free(d_sd);
        device_free(d_search);
        device_free(d_taps);
        device_free(d_w);
        if (st) cudaStreamDestroy(st);
    }
};

// NoiseLevel state of one image: samples drawn on the first call, the
// semimanual reference samples per channel, the call count for manual mode.
struct RgbNoise {
    std::vector<long long> samples;
    long long ref[3] = {0, 0, 0};
    int ncalls = 0;
};

}  // namespace

// get_noiselevel_2D_RGB on the three device planes in J.ch[buf]
static int rgb_noise(RgbJob& J, RgbNoise& N, inlm_params* p, int nx, int ny, int buf, float sig[3]) {
    const int mode = p->noise_mode;
    if (mode == INLM_NOISE_MANUAL) {
        const float v = p->sigma[N.ncalls > 0 ? 1 : 0];
        sig[0] = sig[1] = sig[2] = v;
        N.ncalls++;
        return INLM_OK;
    }
    if (mode != INLM_NOISE_ZADAPTIVE && mode != INLM_NOISE_GLOBAL && mode != INLM_NOISE_SEMIMANUAL)
        return fail(INLM_ERR_ARG, "unknown noise mode %d", mode);
    const bool first = N.samples.empty();
    const int shape[3] = {nx, ny, 1};
    if (first) {
        N.samples = draw_noise_samples(shape, p->n_samples, p->noise_patchsize, p->circular_mask_diameter,
                                       p->noise_seed);
        const long long ns = (long long)N.samples.size();
        if (ns == 0) return fail(INLM_ERR_ARG, "no noise samples fit a %dx%d image", nx, ny);
        CUDA_TRY(dalloc(&J.d_samples, ns));
        CUDA_TRY(dalloc(&J.d_ps, 3 * ns));
        CUDA_TRY(dalloc(&J.d_assign, 3 * ns));
        CUDA_TRY(dalloc(&J.d_win, 3));
        CUDA_TRY(dalloc(&J.d_off, 3));
        CUDA_TRY(dalloc(&J.d_mean, 3));
        CUDA_TRY(dalloc(&J.d_sd, 3));
        const int2 w[3] = {make_int2(0, (int)ns - 1), make_int2((int)ns, (int)(2 * ns - 1)),
                           make_int2((int)(2 * ns), (int)(3 * ns - 1))};
        const long long off[3] = {0, ns, 2 * ns};
        CUDA_TRY(cudaMemcpyAsync(J.d_samples, N.samples.data(), ns * 8, cudaMemcpyHostToDevice, J.st));
        CUDA_TRY(cudaMemcpyAsync(J.d_win, w, sizeof w, cudaMemcpyHostToDevice, J.st));
        CUDA_TRY(cudaMemcpyAsync(J.d_off, off, sizeof off, cudaMemcpyHostToDevice, J.st));
        CUDA_TRY(cudaStreamSynchronize(J.st));
    }
    const long long ns = (long long)N.samples.size();
    const long long plane = (long long)nx * ny;
    for (int c = 0; c < 3; c++)
        CUDA_TRY(launch_noise_patchstd(J.ch[buf][c], nx, plane, nx, plane, J.d_samples, ns,
                                       p->noise_patchsize, J.d_ps + c * ns, J.st));
    if (mode == INLM_NOISE_SEMIMANUAL) {
        // noiselevel.cpp:125-169: the sample nearest sigma[0] per channel on the
        // first call; later calls return those samples' stds
        std::vector<float> ps(3 * ns);
        CUDA_TRY(cudaMemcpyAsync(ps.data(), J.d_ps, 3 * ns * 4, cudaMemcpyDeviceToHost, J.st));
        CUDA_TRY(cudaStreamSynchronize(J.st));
        if (first) {
            const float v = p->sigma[0];
            for (int c = 0; c < 3; c++) {
                float best = 1e9f;
                for (long long i = 0; i < ns; i++) {
                    const float d = std::fabs(ps[c * ns + i] - v);
                    if (d < best) {
                        best = d;
                        N.ref[c] = i;
                    }
                }
                sig[c] = v;
            }
        } else {
            for (int c = 0; c < 3; c++) sig[c] = ps[c * ns + N.ref[c]];
            p->sigma[1] = sig[0];
        }
        N.ncalls++;
        return INLM_OK;
    }
    // global two-cluster estimate per channel (z-adaptive is global for one slice)
    CUDA_TRY(launch_noise_em(J.d_ps, J.d_win, 3, J.d_off, J.d_assign, J.d_mean, J.d_sd, J.st));
    float mean[3], sd[3];
    CUDA_TRY(cudaMemcpyAsync(mean, J.d_mean, 12, cudaMemcpyDeviceToHost, J.st));
    CUDA_TRY(cudaMemcpyAsync(sd, J.d_sd, 12, cudaMemcpyDeviceToHost, J.st));
    CUDA_TRY(cudaStreamSynchronize(J.st));
    for (int c = 0; c < 3; c++) sig[c] = mean[c] + p->stds_from_mean * sd[c];
    N.ncalls++;
    return INLM_OK;
}

extern "C" int inlm_rgb_denoise(int nx, int ny, const inlm_params* params, const inlm_color_params* color,
                                const float* r, const float* g, const float* b, float* out_r, float* out_g,
                                float* out_b, inlm_rgb_iteration_fn on_iteration, void* user,
                                float sigma_first[3], float sigma_last[3]) {
    if (!params || !color || !r || !g || !b || !out_r || !out_g || !out_b)
        return fail(INLM_ERR_ARG, "null argument");
    inlm_params p = *params;
    // the colour driver's fixed settings (color_denoising.h:25-28); the sample
    // count is the caller's (the reference driver passes 2048)
    p.search_radius[2] = 0;
    p.patch_radius[2] = 0;
    p.nslices = 1;
    const int hx = p.search_radius[0] + p.patch_radius[0], hy = p.search_radius[1] + p.patch_radius[1];
    if (nx < 1 || ny < 1 || p.search_radius[0] < 0 || p.search_radius[1] < 0 || p.patch_radius[0] < 0 ||
        p.patch_radius[1] < 0)
        return fail(INLM_ERR_ARG, "bad image %dx%d or radii", nx, ny);
    if ((nx == 1 && hx > 0) || (ny == 1 && hy > 0))
        return fail(INLM_ERR_ARG, "an axis of length 1 cannot be padded reflectively");
    if (p.maxiterations < 1) return fail(INLM_ERR_ARG, "maxiterations must be >= 1");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(INLM_ERR_NODEVICE, "no CUDA device");
    }
    CUDA_TRY(cudaSetDevice(p.device_id));

    Geometry geo = make_geometry(p.search_radius, p.patch_radius, 1, p.z_anisotropy, INLM_WEIGHTS_DISTWEIGHT, 1);
    RgbArgs a{};
    a.nx = nx;
    a.ny = ny;
    a.S = (int)geo.search.size();
    a.P = (int)geo.taps.size();
    a.hx = hx;
    a.hy = hy;
    a.sx = p.search_radius[0];
    a.sy = p.search_radius[1];
    a.independent = color->independent_channels ? 1 : 0;
    // the unrolled kernel when its compile-time tap order is the table's
    a.tap_radius = 0;
    if (p.patch_radius[0] == p.patch_radius[1] && p.patch_radius[0] >= 1) {
        std::vector<int> order(2 * 64);
        const int nt = rgb_tap_order(p.patch_radius[0], order.data(), 64);
        bool same = nt == a.P;
        for (int q = 0; same && q < nt; q++)
            same = order[2 * q] == geo.taps[q].x && order[2 * q + 1] == geo.taps[q].y && geo.taps[q].z == 0;
        if (same) a.tap_radius = p.patch_radius[0];
    }
    if (rgb_smem_bytes(a) > 227u * 1024)
        return fail(INLM_ERR_UNSUPPORTED, "search + patch radius too large for the tile (%zu bytes)",
                    rgb_smem_bytes(a));

    RgbJob J;
    J.device = p.device_id;
    CUDA_TRY(cudaStreamCreateWithFlags(&J.st, cudaStreamNonBlocking));
    const long long plane = (long long)nx * ny;
    for (auto& bufs : J.ch)
        for (float*& q : bufs) CUDA_TRY(dalloc(&q, plane));
    {
        std::vector<int2> s(a.S), t(a.P);
        for (int i = 0; i < a.S; i++) s[i] = make_int2(geo.search[i].x, geo.search[i].y);
        for (int i = 0; i < a.P; i++) t[i] = make_int2(geo.taps[i].x, geo.taps[i].y);
        CUDA_TRY(dalloc(&J.d_search, a.S));
        CUDA_TRY(dalloc(&J.d_taps, a.P));
        CUDA_TRY(dalloc(&J.d_w, a.P));
        CUDA_TRY(cudaMemcpyAsync(J.d_search, s.data(), a.S * sizeof(int2), cudaMemcpyHostToDevice, J.st));
        CUDA_TRY(cudaMemcpyAsync(J.d_taps, t.data(), a.P * sizeof(int2), cudaMemcpyHostToDevice, J.st));
        CUDA_TRY(cudaMemcpyAsync(J.d_w, geo.weights.data(), a.P * 4, cudaMemcpyHostToDevice, J.st));
        CUDA_TRY(cudaStreamSynchronize(J.st));
    }
    a.search = J.d_search;
    a.taps = J.d_taps;
    a.w = J.d_w;

    const float* in[3] = {r, g, b};
    for (int c = 0; c < 3; c++)
        CUDA_TRY(cudaMemcpyAsync(J.ch[0][c], in[c], plane * 4, cudaMemcpyHostToDevice, J.st));
    const bool stab = color->stabilize_variance != 0;
    auto transform = [&](int buf, bool inverse) -> int {
        for (int c = 0; c < 3; c++) CUDA_TRY(launch_anscombe(J.ch[buf][c], plane, inverse, J.st));
        return INLM_OK;
    };
    if (stab) {
        int rc = transform(0, false);
        if (rc) return rc;
    }
    RgbNoise N;
    auto average = [&](float s[3]) {
        if (color->average_channelsigma) s[0] = s[1] = s[2] = (s[0] + s[1] + s[2]) / 3.f;
    };
    float sig0[3], sig1[3];
    int rc = rgb_noise(J, N, &p, nx, ny, 0, sig0);
    if (rc) return rc;
    average(sig0);
    if (sigma_first) std::copy(sig0, sig0 + 3, sigma_first);

    J.host.resize(3 * plane);
    // hands the caller an iteration's result (inverse-transformed, as the
    // reference saves it) and, under the transform, re-applies it in place
    // exactly as the reference does between its saves (color_denoising.h:73-84)
    auto report = [&](int iter, int buf) -> int {
        if (!on_iteration) return INLM_OK;
        if (stab) {
            int e = transform(buf, true);
            if (e) return e;
        }
        for (int c = 0; c < 3; c++)
            CUDA_TRY(cudaMemcpyAsync(J.host.data() + c * plane, J.ch[buf][c], plane * 4,
                                     cudaMemcpyDeviceToHost, J.st));
        CUDA_TRY(cudaStreamSynchronize(J.st));
        on_iteration(iter, J.host.data(), J.host.data() + plane, J.host.data() + 2 * plane, user);
        if (stab) return transform(buf, false);
        return INLM_OK;
    };
    auto blend = [&](const float s1[3]) {
        for (int c = 0; c < 3; c++) sig0[c] = p.alpha * sig0[c] + (1.f - p.alpha) * s1[c];
    };

    int prev = 0, next = 1;
    for (int iter = 1; iter <= p.maxiterations; iter++) {
        for (int c = 0; c < 3; c++) {
            a.raw[c] = J.ch[0][c];
            a.prev[c] = J.ch[prev][c];
            a.out[c] = J.ch[next][c];
            // -1.f / (sigma * sigma * beta), iternlm_cpu.cpp:377-379
            a.mult[c] = -1.f / (sig0[c] * sig0[c] * p.beta);
        }
        CUDA_TRY(launch_rgb_filter(a, J.st));
        rc = report(iter, next);
        if (rc) return rc;
        if ((iter == 1 && p.maxiterations > 1) || (iter > 1 && p.continuous_estimate)) {
            // get texture level (color_denoising.h:88-100, 118-126)
            rc = rgb_noise(J, N, &p, nx, ny, next, sig1);
            if (rc) return rc;
            average(sig1);
            blend(sig1);
        }
        prev = next;
        next = (next == 1) ? 2 : 1;
    }
    if (sigma_last) std::copy(sig0, sig0 + 3, sigma_last);
    if (stab) {
        rc = transform(prev, true);
        if (rc) return rc;
    }
    float* outs[3] = {out_r, out_g, out_b};
    for (int c = 0; c < 3; c++)
        CUDA_TRY(cudaMemcpyAsync(outs[c], J.ch[prev][c], plane * 4, cudaMemcpyDeviceToHost, J.st));
    CUDA_TRY(cudaStreamSynchronize(J.st));
    return INLM_OK;
}
