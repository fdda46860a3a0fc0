// Test-only C entry point over the reference's own GPU class.
//
// Compiled by oracle/Makefile (target ref_gpu) together with the UNMODIFIED
// reference sources Denoiser/iternlm_gpu.cu, Denoiser/iternlm_prepare.cpp and
// Geometry/auxiliary.cpp, for sm_100a, into oracle/_ref/libiternlm_gpu_ref.so.
// It is the reference GPU kernel the product is measured beside; the product
// never links it.
//
// The call follows the reference driver's whole-stack GPU path
// (main.cpp:311-545 with n_parallelslices >= nz): configure_device, then per
// iteration set_sigma and Run_GaussianNoise (iternlm_gpu.cu:1651-1728, which
// synchronises the device before it returns), then get_result. As shipped,
// Run_GaussianNoise launches the patch-specific kernel and then, for every
// patch shape but 1/1/3, apply_filter_generic as well (the `if` at
// iternlm_gpu.cu:1717); its weights use expf where the CPU filter uses the
// Pade approximation, so its results differ from the CPU reference.
#include <chrono>
#include <iostream>
#include <sstream>

#include "Denoiser/iternlm_gpu.h"

extern "C" {

// shape = {nx, ny, nz}; raw: nz*ny*nx floats (x fastest); sigma: iters rows of
// nz floats (the sigma of each iteration); out: nz*ny*nx floats or null.
// ms_per_iter[iters]: host wall time of each Run_GaussianNoise call.
// Returns 0, -1 (no GPU), -2 (CUDA error reported by configure_device) or
// -3 (the stack does not fit the device in one pass: the whole-stack path the
// reference takes only when it fits).
int ref_gpu_run(const int shape_in[3], int patch_radius, int search_radius, int nslices, float beta,
                const float* raw, const float* sigma, int iters, float* out, double* ms_per_iter) {
    protocol::DenoiseParameters p;
    for (int a = 0; a < 3; a++) {
        p.radius_patchspace[a] = patch_radius;
        p.radius_searchspace[a] = search_radius;
    }
    p.nslices = nslices;
    p.beta = beta;
    p.maxiterations = iters;
    p.gpu.n_gpus = 1;
    p.gpu.deviceID = 0;
    p.io.resume = false;
    int shape[3] = {shape_in[0], shape_in[1], shape_in[2]};

    // the reference prints progress on std::cout; keep the caller's stdout clean
    std::ostringstream sink;
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
    denoise::IterativeNLM_GPU g;
    const int n = g.configure_device(shape, &p);
    int rc = 0;
    if (n < 0) {
        rc = n;
    } else if (n < shape[2]) {
        rc = -3;
        g.free_device();
    } else {
        const long long nz = shape[2];
        for (int it = 1; it <= iters; it++) {
            g.set_sigma(const_cast<float*>(sigma + (it - 1) * nz), shape);
            const auto t0 = std::chrono::high_resolution_clock::now();
            g.Run_GaussianNoise(it, const_cast<float*>(raw), shape, &p);
            const auto t1 = std::chrono::high_resolution_clock::now();
            if (ms_per_iter) ms_per_iter[it - 1] = std::chrono::duration<double, std::milli>(t1 - t0).count();
        }
        if (out) g.get_result(out, shape);
        g.free_device();
    }
    std::cout.rdbuf(old);
    return rc;
}

}  // extern "C"
