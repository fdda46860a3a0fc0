// Test-only C entry points over the reference's own CPU implementation.
//
// This translation unit is compiled together with the UNMODIFIED reference
// sources (Denoiser/iternlm_cpu.cpp, Denoiser/iternlm_cpu_kernels.cpp,
// Denoiser/iternlm_prepare.cpp, Noise/noiselevel.cpp, Geometry/auxiliary.cpp)
// into oracle/_ref/libiternlm_ref.so by oracle/Makefile. It is the checker
// and the timed CPU baseline; the product never links it.
//
// Determinism recipe (reference has no seed control):
//   * filter: sigma is passed in directly, as main.cpp:366/462 does after
//     NoiseLevel::get_noiselevel; the whole-stack path
//     IterativeNLM_CPU::Run_GaussianNoise (iternlm_cpu.cpp:8) is used with
//     params.cpu.blockwise = false and io.resume = false.
//   * noise: NoiseLevel's constructor calls srand(time(NULL))
//     (noiselevel.h:24); we call srand(seed) right after it and run the first
//     get_noiselevel with one OpenMP thread so drawsamples' rand() sequence
//     (noiselevel.cpp:206-229) is the sequential glibc sequence.

// Standard headers first, so that the access override below only touches the
// reference's own class definitions.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <utility>
#include <vector>
#include <omp.h>

// Private members (NoiseLevel::samples, create2clusters) are read for parity
// checks of the sample positions and the two-cluster EM.
#define private public
#include "Denoiser/iternlm_cpu.h"
#include "Denoiser/iternlm_prepare.h"
#include "Noise/noiselevel.h"
#undef private
#include "Color/colorspace.h"

extern "C" {

struct ref_params {
    int search_radius[3];
    int patch_radius[3];
    int nslices;
    float beta;
    float z_anisotropy;
};

static void fill_params(protocol::DenoiseParameters* p, const ref_params* rp) {
    for (int i = 0; i < 3; i++) {
        p->radius_searchspace[i] = rp->search_radius[i];
        p->radius_patchspace[i] = rp->patch_radius[i];
    }
    p->nslices = rp->nslices;
    p->beta = rp->beta;
    p->z_anisotropy = rp->z_anisotropy;
    p->cpu.blockwise = false;
    p->cpu.unrolled_patchspace = false;
    p->io.resume = false;
    p->gpu.n_gpus = 0;
}

// Runs n_iter iterations of IterativeNLM_CPU::Run_GaussianNoise.
// sigmas: n_iter * nz floats, row k is the sigma list for iteration k+1.
// out_last: nx*ny*nz result of the last iteration.
// out_all (nullable): n_iter * nx*ny*nz, every iterate.
// n_threads <= 0 keeps the OpenMP default.
// Returns the seconds spent inside Run_GaussianNoise (all iterations).
double ref_denoise(const float* raw_in, const int* shape_in, const ref_params* rp,
                   const float* sigmas, int n_iter, float* out_last, float* out_all,
                   int n_threads) {
    protocol::DenoiseParameters params;
    fill_params(&params, rp);
    int shape[3] = {shape_in[0], shape_in[1], shape_in[2]};
    long long nvox = (long long)shape[0] * shape[1] * shape[2];
    int saved_threads = omp_get_max_threads();
    if (n_threads > 0) omp_set_num_threads(n_threads);
    params.cpu.max_threads = omp_get_max_threads();

    float* raw = (float*)malloc(nvox * sizeof(float));
    std::memcpy(raw, raw_in, nvox * sizeof(float));
    float* prev = nullptr;
    float* out = nullptr;
    denoise::IterativeNLM_CPU nlm;
    // Run_GaussianNoise prints a progress line per slice; keep stdout quiet.
    std::streambuf* saved_buf = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    double seconds = 0.0;
    for (int it = 1; it <= n_iter; it++) {
        float* sig = const_cast<float*>(sigmas + (long long)(it - 1) * shape[2]);
        auto t0 = std::chrono::steady_clock::now();
        if (it == 1) {
            out = nlm.Run_GaussianNoise(1, raw, prev, sig, shape, &params);
        } else {
            out = nlm.Run_GaussianNoise(it, raw, out, sig, shape, &params);
        }
        auto t1 = std::chrono::steady_clock::now();
        seconds += std::chrono::duration<double>(t1 - t0).count();
        if (out_all) std::memcpy(out_all + (long long)(it - 1) * nvox, out, nvox * sizeof(float));
    }
    std::cout.rdbuf(saved_buf);
    std::memcpy(out_last, out, nvox * sizeof(float));
    free(out);
    free(raw);  // padded raw (the original was swapped and freed at iteration 1)
    if (n_threads > 0) omp_set_num_threads(saved_threads);
    return seconds;
}

// Reference geometry tables for a padded shape: search and patch index deltas
// (iternlm_prepare.cpp:102,152) and distance weights (:204).
// Sizes are returned in *ns, *np; arrays must hold at least max_n entries.
int ref_tables(const int* shape_padded, const ref_params* rp, long long* search, int* ns,
               long long* patch, int* np, float* distweight, int max_n) {
    protocol::DenoiseParameters params;
    fill_params(&params, rp);
    int sp[3] = {shape_padded[0], shape_padded[1], shape_padded[2]};
    int nsearch = 0, npatch = 0;
    long long* s = denoise::setup_searchspace(sp, &params, nsearch);
    long long* p = denoise::setup_patchspace(sp, &params, npatch);
    float* w = denoise::setup_distweight(sp, &params);
    *ns = nsearch;
    *np = npatch;
    if (nsearch > max_n || npatch > max_n) {
        free(s); free(p); free(w);
        return -1;
    }
    std::memcpy(search, s, nsearch * sizeof(long long));
    std::memcpy(patch, p, npatch * sizeof(long long));
    std::memcpy(distweight, w, npatch * sizeof(float));
    free(s); free(p); free(w);
    return 0;
}

// Reference reflective padding (iternlm_prepare.cpp:6).
void ref_pad_reflective(const float* in, const int* shape, const int* padding6, float* out) {
    int outshape[3];
    int pad[6];
    for (int i = 0; i < 6; i++) pad[i] = padding6[i];
    float* r = denoise::pad_reflective(const_cast<float*>(in), pad, shape, outshape);
    long long n = (long long)outshape[0] * outshape[1] * outshape[2];
    std::memcpy(out, r, n * sizeof(float));
    free(r);
}

struct ref_noise_params {
    const char* mode;  // "global", "z-adaptive", "manual", "semimanual"
    int zwindow;
    float sigma[2];
    float stds_from_mean;
    int circular_mask_diameter;
};

struct ref_noise_state {
    noise::NoiseLevel* nl;
    protocol::DenoiseParameters params;
    std::vector<std::string> filelist;
};

void* ref_noise_create(const int* shape_in, unsigned long long n_samples, int patchsize,
                       unsigned int seed) {
    int shape[3] = {shape_in[0], shape_in[1], shape_in[2]};
    ref_noise_state* st = new ref_noise_state();
    st->nl = new noise::NoiseLevel((uint64_t)n_samples, patchsize, shape);
    srand(seed);  // after the constructor's srand(time(NULL)) (noiselevel.h:24)
    st->params.cpu.blockwise = false;
    st->params.gpu.n_gpus = 0;
    st->params.io.resume = false;
    return st;
}

// One NoiseLevel::get_noiselevel call (noiselevel.cpp:9). The first call draws
// the samples with a single OpenMP thread. sigma_out: nz floats.
int ref_noise_estimate(void* handle, const float* stack, const ref_noise_params* np,
                       float* sigma_out) {
    ref_noise_state* st = (ref_noise_state*)handle;
    st->params.noiselevel.mode = np->mode;
    st->params.noiselevel.zwindow = np->zwindow;
    st->params.noiselevel.sigma[0] = np->sigma[0];
    st->params.noiselevel.sigma[1] = np->sigma[1];
    st->params.noiselevel.stds_from_mean = np->stds_from_mean;
    st->params.noiselevel.circular_mask_diameter = np->circular_mask_diameter;
    int saved_threads = omp_get_max_threads();
    bool first = st->nl->samples.empty();
    if (first) omp_set_num_threads(1);
    std::streambuf* saved_buf = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());
    float* s = st->nl->get_noiselevel(const_cast<float*>(stack), st->filelist, &st->params);
    std::cout.rdbuf(saved_buf);
    if (first) omp_set_num_threads(saved_threads);
    std::memcpy(sigma_out, s, st->nl->datashape[2] * sizeof(float));
    free(s);
    return 0;
}

// Sample positions drawn by the first estimate (sorted linear indices).
long long ref_noise_samples(void* handle, long long* out, long long max_n) {
    ref_noise_state* st = (ref_noise_state*)handle;
    long long n = (long long)st->nl->samples.size();
    for (long long i = 0; i < n && i < max_n; i++) out[i] = st->nl->samples[i];
    return n;
}

// semimanual-mode second-call value written back into params (noiselevel.cpp:74)
float ref_noise_sigma1(void* handle) {
    return ((ref_noise_state*)handle)->params.noiselevel.sigma[1];
}

void ref_noise_destroy(void* handle) {
    ref_noise_state* st = (ref_noise_state*)handle;
    delete st->nl;
    delete st;
}

// Per-sample patch std (noiselevel.cpp:235) for given sample positions.
void ref_patchstd(const float* stack, const int* shape_in, const long long* samples,
                  long long n, int patchsize, float* out) {
    int shape[3] = {shape_in[0], shape_in[1], shape_in[2]};
    noise::NoiseLevel nl(0, patchsize, shape);
    std::vector<long long int> s(samples, samples + n);
    float* r = nl.get_patchstd(s, const_cast<float*>(stack));
    std::memcpy(out, r, n * sizeof(float));
    free(r);
}

// Two-cluster EM (noiselevel.cpp:366) over values[first..last].
void ref_create2clusters(const float* values, int n, int first, int last, float* mean_std) {
    int shape[3] = {1, 1, 1};
    noise::NoiseLevel nl(0, 15, shape);
    std::pair<float, float> r = nl.create2clusters(const_cast<float*>(values), n, first, last);
    mean_std[0] = r.first;
    mean_std[1] = r.second;
}

// ---- colour path (Color/color_denoising.h:19-150) ----

struct ref_rgb_params {
    float alpha;
    int maxiterations;
    const char* mode;
    float sigma[2];
    unsigned long long n_samples;
    int patchsize;
    float stds_from_mean;
    int continuous_estimate;
    int circular_mask_diameter;
    unsigned int seed;
    int stabilize_variance;
    int independent_channels;
    int average_channelsigma;
    int keep_iterations;  // the run without --cleanup: every iteration is saved
};

// The colour driver's schedule for one image with the reference's own
// pieces (colorspace.h transforms, NoiseLevel::get_noiselevel_2D_RGB,
// IterativeNLM_CPU::Run_GaussianNoise_3channels); file IO left out. With
// keep_iterations, iter_out (nullable, maxiterations x 3 x nx*ny) receives
// each iteration's planes as they would be saved (before the uint8 cast),
// and the buffers go through the same inverse/forward transform the saves
// apply. out_*: the final planes before the uint8 cast.
int ref_rgb_job(const float* r, const float* g, const float* b, int nx, int ny, const ref_params* rp,
                const ref_rgb_params* cp, float* out_r, float* out_g, float* out_b, float* iter_out,
                float* sigma_first, float* sigma_last) {
    protocol::DenoiseParameters params;
    fill_params(&params, rp);
    params.radius_patchspace[2] = 0;
    params.radius_searchspace[2] = 0;
    params.nslices = 1;
    params.alpha = cp->alpha;
    params.maxiterations = cp->maxiterations;
    params.noiselevel.mode = cp->mode;
    params.noiselevel.sigma[0] = cp->sigma[0];
    params.noiselevel.sigma[1] = cp->sigma[1];
    params.noiselevel.n_samples = cp->n_samples;
    params.noiselevel.patchsize = cp->patchsize;
    params.noiselevel.stds_from_mean = cp->stds_from_mean;
    params.noiselevel.continuous_estimate = cp->continuous_estimate != 0;
    params.noiselevel.circular_mask_diameter = cp->circular_mask_diameter;
    params.color.stabilize_variance = cp->stabilize_variance != 0;
    params.color.independent_channels = cp->independent_channels != 0;
    params.color.average_channelsigma = cp->average_channelsigma != 0;
    params.io.cleanup = cp->keep_iterations == 0;

    int shape[3] = {nx, ny, 1};
    const long long n = (long long)nx * ny;
    float* R = (float*)malloc(n * 4);
    float* G = (float*)malloc(n * 4);
    float* B = (float*)malloc(n * 4);
    std::memcpy(R, r, n * 4);
    std::memcpy(G, g, n * 4);
    std::memcpy(B, b, n * 4);
    std::streambuf* saved_buf = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());

    if (params.color.stabilize_variance) color::anscombe_transform(R, G, B, shape);
    denoise::IterativeNLM_CPU nlm;
    std::vector<float*> raw = {R, G, B};
    std::vector<float*> res;
    noise::NoiseLevel noise(params.noiselevel.n_samples, params.noiselevel.patchsize, shape);
    srand(cp->seed);
    int saved_threads = omp_get_max_threads();
    omp_set_num_threads(1);  // the first estimate draws the samples
    std::vector<float> s0 = noise.get_noiselevel_2D_RGB(R, G, B, &params);
    omp_set_num_threads(saved_threads);
    auto average = [&](std::vector<float>& s) {
        if (params.color.average_channelsigma) s[0] = s[1] = s[2] = (s[0] + s[1] + s[2]) / 3.f;
    };
    auto blend = [&](const std::vector<float>& s1) {
        for (int c = 0; c < 3; c++) s0[c] = params.alpha * s0[c] + (1.f - params.alpha) * s1[c];
    };
    average(s0);
    if (sigma_first)
        for (int c = 0; c < 3; c++) sigma_first[c] = s0[c];
    auto save = [&](int iter) {
        if (params.io.cleanup) return;
        if (params.color.stabilize_variance) color::inverse_anscombe_transform(res[0], res[1], res[2], shape);
        if (iter_out)
            for (int c = 0; c < 3; c++)
                std::memcpy(iter_out + ((long long)(iter - 1) * 3 + c) * n, res[c], n * 4);
        if (params.color.stabilize_variance) color::anscombe_transform(res[0], res[1], res[2], shape);
    };
    for (int iter = 1; iter <= params.maxiterations; iter++) {
        nlm.Run_GaussianNoise_3channels(iter, raw, res, s0, shape, &params);
        save(iter);
        if ((iter == 1 && params.maxiterations > 1) || (iter > 1 && params.noiselevel.continuous_estimate)) {
            std::vector<float> s1 = noise.get_noiselevel_2D_RGB(res[0], res[1], res[2], &params);
            average(s1);
            blend(s1);
        }
    }
    if (sigma_last)
        for (int c = 0; c < 3; c++) sigma_last[c] = s0[c];
    if (params.color.stabilize_variance) color::inverse_anscombe_transform(res[0], res[1], res[2], shape);
    std::cout.rdbuf(saved_buf);
    std::memcpy(out_r, res[0], n * 4);
    std::memcpy(out_g, res[1], n * 4);
    std::memcpy(out_b, res[2], n * 4);
    for (float* q : raw) free(q);
    for (float* q : res) free(q);
    return 0;
}

}  // extern "C"
