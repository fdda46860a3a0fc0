// C ABI (include/inlm.h): denoiser and noise-level handles over the sm_100a
// kernels. Host orchestration follows IterativeNLM_GPU (Denoiser/iternlm_gpu.cu:
// configure_device :1440, Run_GaussianNoise :1651, prepare_iteration1 :2117,
// prepare_nextiteration :2230, set_sigma :2341, get_result :2356) and
// NoiseLevel::get_noiselevel (Noise/noiselevel.cpp:9), on one device and one
// stream per handle, without the reference's per-step device synchronisation.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "api_internal.hpp"
#include "noise_kernels.cuh"
#include "common.cuh"
#include "sampling.hpp"

using namespace inlm;

// ---------------- error plumbing ----------------

static thread_local std::string g_last_error;

int inlm::fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

extern "C" const char* inlm_last_error(void) { return g_last_error.c_str(); }

// ---------------- device allocations ----------------

// Live device allocations of the library, and the allocation-failure
// injection of the tests: with g_fail_after = n >= 0 the allocation after n
// further successful ones fails (once) as cudaMalloc does when memory runs out.
static std::atomic<long long> g_live_allocations{0};
static std::atomic<long long> g_fail_after{-1};

cudaError_t inlm::device_malloc(void** p, size_t bytes) {
    *p = nullptr;
    long long n = g_fail_after.load();
    while (n >= 0) {
        if (g_fail_after.compare_exchange_weak(n, n - 1)) {
            if (n == 0) return cudaErrorMemoryAllocation;  // now -1: disarmed
            break;
        }
    }
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) g_live_allocations++;
    return e;
}

cudaError_t inlm::device_free(void* p) {
    if (!p) return cudaSuccess;
    g_live_allocations--;
    return cudaFree(p);
}

extern "C" int inlm_debug_fail_allocation(int64_t after) {
    g_fail_after.store(after < 0 ? -1 : after);
    return INLM_OK;
}

extern "C" int inlm_debug_wait_expiry(inlm_denoiser* d, int64_t cycles) {
    if (!d) return fail(INLM_ERR_ARG, "null handle");
    if (cycles < 0 || cycles > kWaitCycles) return fail(INLM_ERR_ARG, "cycles outside 0..%lld", kWaitCycles);
    CUDA_TRY(cudaSetDevice(d->device));
    CUDA_TRY(launch_selftest_wait(d->d_err, (long long)cycles, d->stream));
    d->launches++;
    return check_device_error(d);
}

extern "C" int inlm_debug_live_allocations(int64_t* n) {
    if (!n) return fail(INLM_ERR_ARG, "null argument");
    *n = g_live_allocations.load();
    return INLM_OK;
}

extern "C" void inlm_default_params(inlm_params* p) {
    // protocol::DenoiseParameters defaults, denoise_parameters.h:11-73
    std::memset(p, 0, sizeof *p);
    p->alpha = 0.5f;
    p->maxiterations = 4;
    p->nslices = 11;
    for (int i = 0; i < 3; i++) {
        p->search_radius[i] = 10;
        p->patch_radius[i] = 1;
    }
    p->beta = 1.f;
    p->z_anisotropy = 1.f;
    p->noise_mode = INLM_NOISE_ZADAPTIVE;
    p->zwindow = 100;
    p->sigma[0] = p->sigma[1] = 0.0f;
    p->n_samples = 100000;
    p->noise_patchsize = 15;
    p->stds_from_mean = 1.f;
    p->continuous_estimate = 0;
    p->circular_mask_diameter = 0;
    p->noise_seed = 0;
    p->device_id = 0;
    p->precision = INLM_PRECISION_F32;
    p->weight_table = INLM_WEIGHTS_CPU;
}

// ---------------- TMA descriptor encoding ----------------

typedef CUresult (*PFN_encodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                    const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                    const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                    CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiled get_encode_fn() {
    static PFN_encodeTiled fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_encodeTiled)p;
    }
    return fn;
}

// 3D float32 map over a padded volume (pitch in elements), box (bx,by,bz).
static int encode_map_3d(CUtensorMap* tm, const void* base, int ex, int ey, int ez,
                         long long pitch_y, long long pitch_z, int bx, int by, int bz,
                         int esize = 4) {
    PFN_encodeTiled enc = get_encode_fn();
    if (!enc) return fail(INLM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[3] = {(cuuint64_t)ex, (cuuint64_t)ey, (cuuint64_t)ez};
    cuuint64_t strides[2] = {(cuuint64_t)pitch_y * esize, (cuuint64_t)pitch_z * esize};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(tm, esize == 2 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                     3, (void*)base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(INLM_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return INLM_OK;
}

// ---------------- noise handle ----------------

void inlm::noise_free(inlm_noise* n) {
    if (!n) return;
    cudaSetDevice(n->device);
    device_free(n->d_samples);
    device_free(n->d_patchstd);
    device_free(n->d_stack);
    device_free(n->d_windows);
    device_free(n->d_scratch_off);
    device_free(n->d_assign);
    device_free(n->d_mean);
    device_free(n->d_sd);
    device_free(n->d_sigma);
    if (n->own_stream && n->stream) cudaStreamDestroy(n->stream);
}

extern "C" int inlm_noise_create(const int shape[3], uint64_t n_samples, int patchsize,
                                 unsigned int seed, int device_id, inlm_noise** out) {
    if (!shape || !out) return fail(INLM_ERR_ARG, "null argument");
    *out = nullptr;
    if (shape[0] <= patchsize || shape[1] <= patchsize || shape[2] < 1)
        return fail(INLM_ERR_ARG, "shape %dx%dx%d too small for noise patch %d", shape[0], shape[1],
                    shape[2], patchsize);
    if (n_samples == 0 || n_samples > (1ull << 31))
        return fail(INLM_ERR_ARG, "n_samples out of range");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return fail(INLM_ERR_NODEVICE, "no CUDA device");
    if (device_id < 0 || device_id >= ndev) return fail(INLM_ERR_ARG, "bad device id");
    inlm_noise* n = new inlm_noise();
    for (int i = 0; i < 3; i++) n->shape[i] = shape[i];
    n->n_samples = n_samples;
    n->patchsize = patchsize;
    n->seed = seed;
    n->device = device_id;
    cudaSetDevice(device_id);
    cudaError_t e = cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete n;
        return fail(INLM_ERR_CUDA, "stream create: %s", cudaGetErrorString(e));
    }
    n->own_stream = true;
    int nz = shape[2];
    if (dalloc(&n->d_samples, n_samples) != cudaSuccess || dalloc(&n->d_patchstd, n_samples) != cudaSuccess ||
        dalloc(&n->d_windows, nz) != cudaSuccess || dalloc(&n->d_scratch_off, nz) != cudaSuccess ||
        dalloc(&n->d_mean, nz) != cudaSuccess || dalloc(&n->d_sd, nz) != cudaSuccess ||
        dalloc(&n->d_sigma, nz) != cudaSuccess) {
        noise_free(n);
        delete n;
        return fail(INLM_ERR_NOMEM, "noise buffers");
    }
    *out = n;
    return INLM_OK;
}

extern "C" int inlm_noise_destroy(inlm_noise* n) {
    noise_free(n);
    delete n;
    return INLM_OK;
}

// Runs the estimate for a device stack (pitches in elements); the result stays
// in n->d_sigma. Host-side decisions (manual, semimanual) fill host_sigma.
// Draws the sample positions on the first call and uploads the EM windows of
// the mode (z-adaptive: one per slice; global: one); *nwin gets their count
// (0 for the manual modes), *first whether the samples were drawn now.
int inlm::noise_prepare(inlm_noise* n, const inlm_params* p, int* nwin, bool* first_out) {
    const int nz = n->shape[2];
    const int mode = p->noise_mode;
    const bool first = n->samples.empty();
    if (first_out) *first_out = first;
    *nwin = 0;
    if (first) {
        n->samples = draw_noise_samples(n->shape, n->n_samples, n->patchsize,
                                        p->circular_mask_diameter, n->seed);
        CUDA_TRY(cudaMemcpyAsync(n->d_samples, n->samples.data(), n->samples.size() * 8,
                                 cudaMemcpyHostToDevice, n->stream));
        CUDA_TRY(cudaStreamSynchronize(n->stream));  // the host vector may be replaced later
    }
    const long long ns = (long long)n->samples.size();
    if (mode == INLM_NOISE_ZADAPTIVE) {
        if (n->zwindow_cached != p->zwindow || first) {
            std::vector<int> st, en;
            noise_zwindows(n->samples, n->shape, p->zwindow, st, en);
            std::vector<int2> w(nz);
            std::vector<long long> off(nz);
            long long total = 0;
            for (int z = 0; z < nz; z++) {
                w[z] = make_int2(st[z], en[z]);
                off[z] = total;
                total += std::max(0, en[z] - st[z] + 1);
            }
            if ((size_t)total > n->assign_cap) {
                device_free(n->d_assign);
                n->d_assign = nullptr;
                n->assign_cap = 0;
                CUDA_TRY(dalloc(&n->d_assign, (size_t)total));
                n->assign_cap = (size_t)total;
            }
            CUDA_TRY(cudaMemcpyAsync(n->d_windows, w.data(), nz * sizeof(int2),
                                     cudaMemcpyHostToDevice, n->stream));
            CUDA_TRY(cudaMemcpyAsync(n->d_scratch_off, off.data(), nz * 8, cudaMemcpyHostToDevice,
                                     n->stream));
            CUDA_TRY(cudaStreamSynchronize(n->stream));  // host vectors go out of scope
            n->zwindow_cached = p->zwindow;
            n->mean_window = nz > 0 ? total / nz : 0;
        }
        *nwin = nz;
    } else if (mode == INLM_NOISE_GLOBAL) {
        if (n->zwindow_cached != -2) {
            int2 w = make_int2(0, (int)ns - 1);
            long long off = 0;
            if ((size_t)ns > n->assign_cap) {
                device_free(n->d_assign);
                n->d_assign = nullptr;
                n->assign_cap = 0;
                CUDA_TRY(dalloc(&n->d_assign, (size_t)ns));
                n->assign_cap = (size_t)ns;
            }
            CUDA_TRY(cudaMemcpyAsync(n->d_windows, &w, sizeof w, cudaMemcpyHostToDevice, n->stream));
            CUDA_TRY(cudaMemcpyAsync(n->d_scratch_off, &off, 8, cudaMemcpyHostToDevice, n->stream));
            CUDA_TRY(cudaStreamSynchronize(n->stream));
            n->zwindow_cached = -2;
            n->mean_window = ns;
        }
        *nwin = 1;
    }
    return INLM_OK;
}

// EM over the patch stds in n->d_patchstd and the per-slice sigma into
// n->d_sigma (device work only).
int inlm::noise_em_finish(inlm_noise* n, const inlm_params* p, int nwin) {
    CUDA_TRY(launch_noise_em(n->d_patchstd, n->d_windows, nwin, n->d_scratch_off, n->d_assign,
                             n->d_mean, n->d_sd, n->stream, n->mean_window));
    CUDA_TRY(launch_noise_finalize(n->d_mean, n->d_sd, n->shape[2],
                                   p->noise_mode == INLM_NOISE_ZADAPTIVE ? 1 : 0, p->stds_from_mean,
                                   n->d_sigma, n->stream));
    n->ncalls++;
    return INLM_OK;
}

// d_stack NULL: the stack is in host memory (h_stack) and larger than the
// device holds; its samples' patch stds are taken slab by slab through the
// staging buffer n->d_stack (n->stack_slices slices).
static int noise_estimate_device(inlm_noise* n, inlm_params* p, const float* d_stack,
                                 long long pitch_y, long long pitch_z, std::vector<float>* host_sigma,
                                 bool* sigma_on_host, const float* h_stack = nullptr) {
    const int nz = n->shape[2];
    *sigma_on_host = false;
    const int mode = p->noise_mode;
    if (mode == INLM_NOISE_MANUAL) {
        // noiselevel.cpp:84-91
        float v = p->sigma[n->ncalls > 0 ? 1 : 0];
        host_sigma->assign(nz, v);
        *sigma_on_host = true;
        n->ncalls++;
        return INLM_OK;
    }
    if (mode != INLM_NOISE_ZADAPTIVE && mode != INLM_NOISE_GLOBAL && mode != INLM_NOISE_SEMIMANUAL)
        return fail(INLM_ERR_ARG, "unknown noise mode %d", mode);
    int nwin = 0;
    bool first = false;
    int rc = noise_prepare(n, p, &nwin, &first);
    if (rc) return rc;
    const long long ns = (long long)n->samples.size();
    const long long plane = (long long)n->shape[0] * n->shape[1];
    if (d_stack) {
        CUDA_TRY(launch_noise_patchstd(d_stack, pitch_y, pitch_z, n->shape[0], plane, n->d_samples, ns,
                                       n->patchsize, n->d_patchstd, n->stream));
    } else {
        // patches lie within one slice, so each slab gives its own samples' stds
        const int S = std::max(1, n->stack_slices);
        for (int z0 = 0; z0 < nz; z0 += S) {
            const int z1 = std::min(nz, z0 + S);
            const long long i0 = std::lower_bound(n->samples.begin(), n->samples.end(), z0 * plane) -
                                 n->samples.begin();
            const long long i1 = std::lower_bound(n->samples.begin(), n->samples.end(), z1 * plane) -
                                 n->samples.begin();
            if (i1 == i0) continue;
            CUDA_TRY(cudaMemcpyAsync(n->d_stack, h_stack + z0 * plane, (size_t)(z1 - z0) * plane * 4,
                                     cudaMemcpyHostToDevice, n->stream));
            CUDA_TRY(launch_noise_patchstd(n->d_stack, n->shape[0], plane, n->shape[0], plane,
                                           n->d_samples + i0, i1 - i0, n->patchsize, n->d_patchstd + i0,
                                           n->stream, z0));
        }
    }
    if (mode == INLM_NOISE_SEMIMANUAL) {
        // noiselevel.cpp:62-79
        std::vector<float> ps(ns);
        CUDA_TRY(cudaMemcpyAsync(ps.data(), n->d_patchstd, ns * 4, cudaMemcpyDeviceToHost, n->stream));
        CUDA_TRY(cudaStreamSynchronize(n->stream));
        float v;
        if (first) {
            float best = 1e9f;
            v = p->sigma[0];
            for (long long i = 0; i < ns; i++) {
                float d = std::fabs(ps[i] - v);
                if (d < best) {
                    best = d;
                    n->ref_sample_semimanual = i;
                }
            }
        } else {
            v = ps[n->ref_sample_semimanual];
            p->sigma[1] = v;
        }
        host_sigma->assign(nz, v);
        *sigma_on_host = true;
        n->ncalls++;
        return INLM_OK;
    }
    return noise_em_finish(n, p, nwin);
}

extern "C" int inlm_noise_estimate(inlm_noise* n, inlm_params* p, const float* stack,
                                   int on_device, float* sigma_out) {
    if (!n || !p || !stack || !sigma_out) return fail(INLM_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(n->device));
    const long long nvox = (long long)n->shape[0] * n->shape[1] * n->shape[2];
    const float* d_stack = stack;
    if (!on_device) {
        const long long plane = (long long)n->shape[0] * n->shape[1];
        if (!n->d_stack) {
            // the whole stack where it fits, else a staging slab of <= 256 MiB
            if (dalloc(&n->d_stack, nvox) == cudaSuccess) {
                n->stack_slices = n->shape[2];
            } else {
                cudaGetLastError();
                n->d_stack = nullptr;
                n->stack_slices = (int)std::max<long long>(1, std::min<long long>(n->shape[2], (256ll << 20) / (plane * 4)));
                CUDA_TRY(dalloc(&n->d_stack, n->stack_slices * plane));
            }
        }
        if (n->stack_slices == n->shape[2]) {
            CUDA_TRY(cudaMemcpyAsync(n->d_stack, stack, nvox * 4, cudaMemcpyHostToDevice, n->stream));
            d_stack = n->d_stack;
        } else {
            d_stack = nullptr;  // slab by slab from the host
        }
    }
    std::vector<float> hs;
    bool on_host = false;
    int rc = noise_estimate_device(n, p, d_stack, n->shape[0], (long long)n->shape[0] * n->shape[1],
                                   &hs, &on_host, on_device ? nullptr : stack);
    if (rc != INLM_OK) return rc;
    if (on_host) {
        std::memcpy(sigma_out, hs.data(), n->shape[2] * 4);
    } else {
        CUDA_TRY(cudaMemcpyAsync(sigma_out, n->d_sigma, n->shape[2] * 4, cudaMemcpyDeviceToHost,
                                 n->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(n->stream));
    return INLM_OK;
}

extern "C" int inlm_noise_samples(inlm_noise* n, int64_t* out, uint64_t max_n, uint64_t* n_out) {
    if (!n) return fail(INLM_ERR_ARG, "null handle");
    if (n_out) *n_out = n->samples.size();
    if (out)
        for (uint64_t i = 0; i < max_n && i < n->samples.size(); i++) out[i] = n->samples[i];
    return INLM_OK;
}

extern "C" int inlm_noise_patchstd(inlm_noise* n, float* out, uint64_t max_n) {
    if (!n || !out) return fail(INLM_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(n->device));
    uint64_t cnt = std::min<uint64_t>(max_n, n->samples.size());
    CUDA_TRY(cudaMemcpyAsync(out, n->d_patchstd, cnt * 4, cudaMemcpyDeviceToHost, n->stream));
    CUDA_TRY(cudaStreamSynchronize(n->stream));
    return INLM_OK;
}

extern "C" int inlm_noise_patchstd_slab(inlm_noise* n, const inlm_params* p, const float* slab,
                                        int on_device, int z_base, int n_slices, float* patchstd_host,
                                        uint64_t n_values) {
    if (!n || !p || !slab || !patchstd_host) return fail(INLM_ERR_ARG, "null argument");
    const int nz = n->shape[2];
    if (z_base < 0 || n_slices < 1 || z_base + n_slices > nz)
        return fail(INLM_ERR_ARG, "slices %d..%d outside the stack of %d", z_base, z_base + n_slices - 1, nz);
    CUDA_TRY(cudaSetDevice(n->device));
    int nwin = 0;
    int rc = noise_prepare(n, p, &nwin, nullptr);  // draws the samples on the first call
    if (rc) return rc;
    const uint64_t ns = n->samples.size();
    if (n_values < ns) return fail(INLM_ERR_ARG, "patchstd_host holds %llu values, %llu samples drawn",
                                   (unsigned long long)n_values, (unsigned long long)ns);
    const long long plane = (long long)n->shape[0] * n->shape[1];
    const float* d_slab = slab;
    if (!on_device) {
        if (!n->d_stack || n->stack_slices < n_slices) {
            CUDA_TRY(cudaStreamSynchronize(n->stream));
            device_free(n->d_stack);
            n->d_stack = nullptr;
            CUDA_TRY(dalloc(&n->d_stack, plane * nz));
            n->stack_slices = nz;
        }
        CUDA_TRY(cudaMemcpyAsync(n->d_stack, slab, plane * n_slices * 4, cudaMemcpyHostToDevice, n->stream));
        d_slab = n->d_stack;
    }
    // samples are sorted by linear index: the slab's samples are one range
    const long long i0 = std::lower_bound(n->samples.begin(), n->samples.end(), (long long)z_base * plane) -
                         n->samples.begin();
    const long long i1 = std::lower_bound(n->samples.begin(), n->samples.end(),
                                          (long long)(z_base + n_slices) * plane) - n->samples.begin();
    std::fill(patchstd_host, patchstd_host + ns, 0.0f);
    if (i1 > i0) {
        CUDA_TRY(launch_noise_patchstd(d_slab, n->shape[0], plane, n->shape[0], plane, n->d_samples + i0,
                                       i1 - i0, n->patchsize, n->d_patchstd + i0, n->stream, z_base));
        CUDA_TRY(cudaMemcpyAsync(patchstd_host + i0, n->d_patchstd + i0, (i1 - i0) * 4,
                                 cudaMemcpyDeviceToHost, n->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(n->stream));
    return INLM_OK;
}

extern "C" int inlm_noise_estimate_from_patchstd(inlm_noise* n, inlm_params* p, const float* patchstd_host,
                                                 uint64_t n_values, float* sigma_out) {
    if (!n || !p || !sigma_out) return fail(INLM_ERR_ARG, "null argument");
    const int nz = n->shape[2];
    if (p->noise_mode == INLM_NOISE_MANUAL) {
        // noiselevel.cpp:84-91
        std::fill(sigma_out, sigma_out + nz, p->sigma[n->ncalls > 0 ? 1 : 0]);
        n->ncalls++;
        return INLM_OK;
    }
    if (p->noise_mode != INLM_NOISE_ZADAPTIVE && p->noise_mode != INLM_NOISE_GLOBAL &&
        p->noise_mode != INLM_NOISE_SEMIMANUAL)
        return fail(INLM_ERR_ARG, "unknown noise mode %d", p->noise_mode);
    if (!patchstd_host) return fail(INLM_ERR_ARG, "null patch stds");
    if (n->samples.empty()) return fail(INLM_ERR_STATE, "no samples drawn: run inlm_noise_patchstd_slab first");
    const uint64_t ns = n->samples.size();
    if (n_values != ns)
        return fail(INLM_ERR_ARG, "%llu patch stds for %llu samples", (unsigned long long)n_values,
                    (unsigned long long)ns);
    CUDA_TRY(cudaSetDevice(n->device));
    if (p->noise_mode == INLM_NOISE_SEMIMANUAL) {
        // noiselevel.cpp:62-79, as inlm_noise_estimate decides it
        float v;
        if (n->ncalls == 0) {
            float best = 1e9f;
            v = p->sigma[0];
            for (uint64_t i = 0; i < ns; i++) {
                const float d = std::fabs(patchstd_host[i] - v);
                if (d < best) {
                    best = d;
                    n->ref_sample_semimanual = (long long)i;
                }
            }
        } else {
            v = patchstd_host[n->ref_sample_semimanual];
            p->sigma[1] = v;
        }
        std::fill(sigma_out, sigma_out + nz, v);
        n->ncalls++;
        return INLM_OK;
    }
    int nwin = 0;
    int rc = noise_prepare(n, p, &nwin, nullptr);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(n->d_patchstd, patchstd_host, ns * 4, cudaMemcpyHostToDevice, n->stream));
    rc = noise_em_finish(n, p, nwin);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(sigma_out, n->d_sigma, nz * 4, cudaMemcpyDeviceToHost, n->stream));
    CUDA_TRY(cudaStreamSynchronize(n->stream));
    return INLM_OK;
}

// ---------------- denoiser handle ----------------

static void denoiser_free(inlm_denoiser* d) {
    if (!d) return;
    cudaSetDevice(d->device);
    if (d->stream) cudaStreamSynchronize(d->stream);
    for (auto& t : d->pending) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    for (auto& t : d->event_pool) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    device_free(d->d_raw_pad);
    device_free(d->d_prev_pad);
    device_free(d->d_next);
    device_free(d->d_sigma);
    device_free(d->d_sigma0);
    device_free(d->d_mult);
    device_free(d->d_err);
    device_free(d->d_search_delta);
    device_free(d->d_group_zb);
    device_free(d->d_search_off);
    device_free(d->d_patch_off);
    device_free(d->d_weights);
    device_free(d->d_raw_h);
    device_free(d->d_prev_h);
    device_free(d->d_plan_start);
    device_free(d->d_plan_off);
    device_free(d->d_search_delta8);
    device_free(d->d_search_delta_c);
    proposal_release(d);
    d->aux.release();
    if (d->noise) {
        noise_free(d->noise);
        delete d->noise;
    }
    if (d->own_stream && d->stream) cudaStreamDestroy(d->stream);
}

// Plane pitch (floats) of the raw box: the smallest padding of rpx * rby for
// which the phase-B raw reads of a warp (8 rows j, 4 planes pstride apart,
// one column) fall in distinct banks.
static int raw_plane_pitch(int rpx, int rby, int pstride = 1) {
    const int base = rpx * rby;
    for (int pad = 0; pad < 32; pad++) {
        const int pl = base + pad;
        bool ok = true;
        for (int col = 0; col < 8 && ok; col++) {
            unsigned used = 0;
            for (int l = 0; l < 32; l++) {
                const unsigned bank = (unsigned)((l >> 3) * pstride * pl + (l & 7) * rpx + col) % 32u;
                if (used & (1u << bank)) {
                    ok = false;
                    break;
                }
                used |= 1u << bank;
            }
        }
        if (ok) return pl;
    }
    return base;
}

// Tiled FP32 configuration for one candidate (CTA depth tz, raw staged in
// shared memory or read from global; tz 0: the column form, patch radius 1,
// at its own depth): tables, kernel arguments, TMA map.
// *ok = false when the candidate does not apply or does not fit.
// Raw-slab schedule: for each group of kOffGroup consecutive offsets, the z
// offset from which the TZ + 1 staged raw planes start. The search list must
// run z-major (the reference order does: iternlm_prepare.cpp:102-150), so a
// group spans at most two z offsets; the slab moves only when a group needs a
// plane past it. Returns false if the list is not z-major or the slab would
// not be smaller than the whole box.
static bool raw_slab_table(const Geometry& g, int szc, int tz, std::vector<int>* out) {
    const int S = (int)g.search.size();
    if (S == 0 || tz + 1 >= tz + 2 * szc) return false;
    for (int s = 1; s < S; s++)
        if (g.search[s].z < g.search[s - 1].z) return false;
    out->clear();
    int zb = g.search[0].z;
    for (int s = 0; s < S; s += kOffGroup) {
        const int lo = g.search[s].z, hi = g.search[std::min(s + kOffGroup, S) - 1].z;
        if (hi - lo > 1) return false;
        if (lo < zb || hi > zb + 1) zb = lo;
        out->push_back(zb);
    }
    return true;
}

int inlm::tile_config_try(inlm_denoiser* d, int tz, bool raw_smem, bool* ok, bool ws) {
    const Geometry& g = d->geo;
    const int* pr = g.patch_radius;
    *ok = false;
    if (!tile_kernel_available(pr[0], pr[1], pr[2])) return INLM_OK;
    if (d->p.nslices / 2 < pr[2]) return INLM_OK;           // z-clipped patch
    if ((int)g.taps.size() > kMaxTaps) return INLM_OK;
    // the kernel's compile-time tap order must equal the host table
    std::vector<int> order(3 * kMaxTaps);
    int nt = tile_kernel_tap_order(pr[0], pr[1], pr[2], order.data(), kMaxTaps);
    if (nt != (int)g.taps.size()) return INLM_OK;
    for (int t = 0; t < nt; t++)
        if (order[3 * t] != g.taps[t].x || order[3 * t + 1] != g.taps[t].y ||
            order[3 * t + 2] != g.taps[t].z)
            return INLM_OK;
    const bool fused = d->p.precision == INLM_PRECISION_F32_FMA;
    const bool column = tz == 0;
    if (column) {
        tz = column_kernel_depth(pr[0], pr[1], pr[2]);
        if (tz == 0) return INLM_OK;
        raw_smem = false;
    }
    if (ws) {  // the warp-specialised 8-deep kernel: raw box staged or read from global memory
        if (column) return INLM_OK;
        tz = 8;
    }
    // tz 16: the two-planes-per-thread kernel (raw staged in shared memory)
    if (!column && !((tz == 8) || (tz == 4 && !raw_smem) || (tz == 16 && raw_smem))) return INLM_OK;
    if (fused && !column && tz != 8) return INLM_OK;  // the fused tile form is instantiated at depth 8

    TileArgs a{};
    a.nx = d->shape[0];
    a.ny = d->shape[1];
    a.nz = d->shape[2];
    a.px = g.pad[0];
    a.py = g.pad[1];
    a.pz = g.pad[2];
    a.sxr = g.search_radius[0];
    a.syr = g.search_radius[1];
    a.szc = std::min(d->p.nslices / 2, g.search_radius[2]);
    a.S = (int)g.search.size();
    a.gpitch_y = d->pitch_y;
    a.gpitch_z = d->pitch_z;
    a.pbx = (kTX + 2 * a.px + 3) / 4 * 4;
    a.pby = kTY + 2 * a.py;
    a.rbx = (pr[0] + kTX + 2 * a.sxr + 3) / 4 * 4;
    a.rby = kTY + 2 * a.syr;
    for (int t = 0; t < nt; t++) a.w[t] = g.weights[t];
    a.pbz = tz + 2 * a.pz;
    a.rbz = tz + 2 * a.szc;
    if (a.pbx > 256 || a.pby > 256 || a.pbz > 256) return INLM_OK;
    if ((long long)a.pbx * a.pby * a.pbz >= 65536) return INLM_OK;  // 16-bit index table
    a.rplane = raw_plane_pitch(a.rbx + 1, a.rby, tz == 16 ? 2 : 1);
    int smem_max = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, d->device));
    TileConfig tc{pr[0], pr[1], pr[2], tz, raw_smem, 0, fused};
    tc.column = column;
    tc.ws = ws;
    size_t sm = column ? column_smem_bytes(a) : ws ? tile_ws_smem_bytes(tc, a) : tile_smem_bytes(tc, a);
    a.raw_slab = 0;
    a.group_zb = nullptr;
    std::vector<int> zb;
    if (raw_smem && !ws && (tz == 8 || tz == 16) && (sm == 0 || sm > (size_t)smem_max) &&
        raw_slab_table(g, a.szc, tz, &zb)) {
        // the whole raw box does not fit: stage TZ + 1 planes per z offset pair
        a.rbz = tz + 1;
        a.raw_slab = 1;
        tc.raw_slab = true;
        sm = tile_smem_bytes(tc, a);
    }
    if (sm == 0 || sm > (size_t)smem_max) return INLM_OK;
    if (a.raw_slab) {
        device_free(d->d_group_zb);
        d->d_group_zb = nullptr;
        CUDA_TRY(dalloc(&d->d_group_zb, zb.size()));
        CUDA_TRY(cudaMemcpy(d->d_group_zb, zb.data(), zb.size() * sizeof(int), cudaMemcpyHostToDevice));
        a.group_zb = d->d_group_zb;
    }
    tc.smem_bytes = sm;
    a.tiles_x = (d->shape[0] + kTX - 1) / kTX;
    a.tiles_y = (d->shape[1] + kTY - 1) / kTY;
    // search deltas inside the shared-memory boxes (raw: box or global)
    std::vector<int2> dl(a.S);
    const int rpx = a.rbx + 1;  // odd shared-memory row pitch of the raw box
    const int pplane = a.pbx * a.pby, rplane = a.rplane;
    for (int s = 0; s < a.S; s++) {
        const Offset3& o = g.search[s];
        dl[s].x = o.z * pplane + o.y * a.pbx + o.x;
        dl[s].y = raw_smem ? o.z * rplane + o.y * rpx + o.x
                           : (int)(o.z * d->pitch_z + o.y * d->pitch_y + o.x);
    }
    if (!d->d_search_delta) CUDA_TRY(dalloc(&d->d_search_delta, a.S));
    CUDA_TRY(cudaMemcpy(d->d_search_delta, dl.data(), a.S * sizeof(int2), cudaMemcpyHostToDevice));
    a.search_delta = d->d_search_delta;
    a.raw_pad = d->d_raw_pad;
    a.out = d->d_next;
    a.mult = d->d_mult;
    a.err = d->d_err;
    int rc = encode_map_3d(&d->tm_prev, d->d_prev_pad, d->nxp, d->nyp, d->nzp, d->pitch_y, d->pitch_z,
                           a.pbx, a.pby, a.pbz);
    if (rc) return rc;
    d->tm_raw = d->tm_prev;  // raw is staged with plain loads; the map is unused
    d->targs = a;
    d->tcfg = tc;
    d->use_tile = true;
    *ok = true;
    return INLM_OK;
}

// Default choice (before any autotuning): the first candidate that fits.
// form: 0 every candidate, 1 the tiled kernels only, 2 the column form only,
// 3 the warp-specialised kernel only. In form 0 the warp-specialised kernel
// leads when patch sums dominate the work (at least 100 patch taps, or at
// least 30 taps and 400 offsets). With fewer than 100 taps its raw-global
// variant comes after the tiled kernels that stage the whole raw box (and
// before those that restage raw slabs). Measured on B200 (256^3 launches):
// faster at patch radius 2 with search radius 5 (5 %) and 7 (3 %, raw global
// against the slab), at patch radius 3 with search radius 3 (8 %) and 4 (7 %,
// raw global against the 8-deep raw box); slower at patch radius 2 with search
// radius 3 and 4 (114 and 256 offsets, 4 %) and, reading raw from global
// memory, at search radius 6 against the 8-deep kernel's raw box (7 %); the
// column form leads at patch radius 1. The fused FP32 form takes the
// warp-specialised kernel only with the raw box and fewer than 100 taps:
// measured 7 % faster at patch radius 2 / search radius 5, but 9 % slower
// reading raw from global memory (search radius 7, against the raw slab) and
// 2 % slower at patch radius 3 / search radius 3.
static int choose_tile_config(inlm_denoiser* d, int form = 0) {
    d->use_tile = false;
    struct Cand {
        int tz;
        bool raw;
        bool ws;
        bool box_only;  // accept only with the whole raw box staged (no slab)
    };
    const int P = (int)d->geo.taps.size(), S = (int)d->geo.search.size();
    const bool fused = d->p.precision == INLM_PRECISION_F32_FMA;
    const bool ws_first =
        form == 0 && (fused ? (P >= 30 && P < 100 && S >= 400) : (P >= 100 || (P >= 30 && S >= 400)));
    const Cand base[] = {{0, false, false, false}, {16, true, false, false}, {8, true, false, false},
                         {8, false, false, false}, {4, false, false, false}, {8, true, true, false},
                         {8, false, true, false}};
    const Cand lead[] = {{0, false, false, false}, {8, true, true, true},   {16, true, false, true},
                         {8, true, false, true},   {8, false, true, false}, {16, true, false, false},
                         {8, true, false, false},  {8, false, false, false}, {4, false, false, false}};
    const Cand* cands = ws_first ? lead : base;
    const int n = ws_first ? 9 : 7;
    for (int i = 0; i < n; i++) {
        const Cand c = cands[i];
        if (c.box_only && !c.ws && P >= 100) continue;  // many taps: the raw-global variant first
        if (form == 0 && fused && c.ws && !c.raw) continue;
        if ((form == 1 && (c.tz == 0 || c.ws)) || (form == 2 && c.tz != 0) || (form == 3 && !c.ws) ||
            (form == 0 && c.ws && !ws_first))
            continue;
        bool ok = false;
        int rc = tile_config_try(d, c.tz, c.raw, &ok, c.ws);
        if (rc) return rc;
        if (ok && c.box_only && d->tcfg.raw_slab) {
            d->use_tile = false;
            continue;
        }
        if (ok) return INLM_OK;
    }
    return INLM_OK;
}

// FP16-storage kernel configurations: CTA width tx = 32 (full search) and
// tx = 8 (one 8^3 tile per CTA, for per-tile offset plans); prev box in
// halves arriving by TMA, raw staged in halves with an odd pitch. tx = 0:
// the column form at its own CTA depth (32 x 8 x depth voxels, raw from
// global memory, no raw box).
static int build_fast_config(inlm_denoiser* d, int tx, FastConfig* cfg, FastArgs* args,
                             CUtensorMap* tm, int2** d_delta, bool* ok) {
    const Geometry& g = d->geo;
    const int* pr = g.patch_radius;
    *ok = false;
    if (!tile_kernel_available(pr[0], pr[1], pr[2])) return INLM_OK;
    if (d->p.nslices / 2 < pr[2]) return INLM_OK;
    if ((int)g.taps.size() > kMaxTaps) return INLM_OK;
    std::vector<int> order(3 * kMaxTaps);
    int nt = tile_kernel_tap_order(pr[0], pr[1], pr[2], order.data(), kMaxTaps);
    if (nt != (int)g.taps.size()) return INLM_OK;
    for (int t = 0; t < nt; t++)
        if (order[3 * t] != g.taps[t].x || order[3 * t + 1] != g.taps[t].y ||
            order[3 * t + 2] != g.taps[t].z)
            return INLM_OK;
    FastArgs& a = *args;
    a = FastArgs{};
    a.nx = d->shape[0];
    a.ny = d->shape[1];
    a.nz = d->shape[2];
    a.px = g.pad[0];
    a.py = g.pad[1];
    a.pz = g.pad[2];
    a.sxr = g.search_radius[0];
    a.syr = g.search_radius[1];
    a.szc = std::min(d->p.nslices / 2, g.search_radius[2]);
    a.S = (int)g.search.size();
    a.gpitch_y = d->pitch_y;
    a.gpitch_z = d->pitch_z;
    const bool column = tx == 0;
    const int cdepth = column ? column_kernel_depth(pr[0], pr[1], pr[2]) : 0;
    if (column && cdepth == 0) return INLM_OK;
    const int txw = column ? kTX : tx;  // CTA width in x
    a.pbx = (txw + 2 * a.px + 7) / 8 * 8;  // halves, 16-byte TMA rows
    a.pby = kTY + 2 * a.py;
    a.rbx = (pr[0] + txw + 2 * a.sxr + 3) / 4 * 4;
    a.rby = kTY + 2 * a.syr;
    for (int t = 0; t < nt; t++) {
        a.w[t] = g.weights[t];
        const __half h = __float2half_rn(g.weights[t]);
        a.wh[t] = __halves2half2(h, h);
    }
    int smem_max = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, d->device));
    const bool dh = d->p.precision == INLM_PRECISION_F16;
    const int tzs[] = {8, 4};
    if (column) {
        a.pbz = cdepth + 2 * a.pz;
        a.rbz = 0;
        FastConfig fc{pr[0], pr[1], pr[2], cdepth, kTX, dh, 0};
        fc.column = true;
        const size_t sm = 128 + (size_t)a.pbx * a.pby * a.pbz * 2;
        if (a.pbx <= 256 && a.pby <= 256 && a.pbz <= 256 && sm <= (size_t)smem_max) {
            fc.smem_bytes = sm;
            *cfg = fc;
            *ok = true;
        }
    }
    for (int tz : tzs) {
        if (column) break;
        if (tz == 4 && (!dh || tx != 32)) continue;
        a.pbz = tz + 2 * a.pz;
        a.rbz = tz + 2 * a.szc;
        if (a.pbx > 256 || a.pby > 256 || a.pbz > 256) continue;
        if ((long long)a.pbx * a.pby * a.pbz >= (1ll << 24)) continue;
        FastConfig fc{pr[0], pr[1], pr[2], tz, tx, dh, 0};
        size_t sm = fast_smem_bytes(fc, a);
        if (sm == 0 || sm > (size_t)smem_max) continue;
        fc.smem_bytes = sm;
        *cfg = fc;
        *ok = true;
        break;
    }
    if (!*ok) return INLM_OK;
    a.tiles_x = (d->shape[0] + txw - 1) / txw;
    a.tiles_y = (d->shape[1] + kTY - 1) / kTY;
    std::vector<int2> dl(a.S);
    const int rpx = a.rbx + 1;
    for (int si = 0; si < a.S; si++) {
        const Offset3& o = g.search[si];
        dl[si].x = o.z * a.pbx * a.pby + o.y * a.pbx + o.x;
        // raw: shared-box delta (tx = 32) or padded global delta (tx = 8, column)
        dl[si].y = (tx == 8 || column) ? (int)(o.z * d->pitch_z + o.y * d->pitch_y + o.x)
                                       : o.z * rpx * a.rby + o.y * rpx + o.x;
    }
    CUDA_TRY(dalloc(d_delta, a.S));
    CUDA_TRY(cudaMemcpy(*d_delta, dl.data(), a.S * sizeof(int2), cudaMemcpyHostToDevice));
    a.search_delta = *d_delta;
    a.plan_offsets = nullptr;
    a.plan_start = nullptr;
    a.plan_count = nullptr;
    a.raw_pad = (const __half*)d->d_raw_h;
    a.out = d->d_next;
    a.mult = d->d_mult;
    a.err = d->d_err;
    return encode_map_3d(tm, d->d_prev_h, d->nxp, d->nyp, d->nzp, d->pitch_y, d->pitch_z, a.pbx,
                         a.pby, a.pbz, 2);
}

static int choose_fast_config(inlm_denoiser* d) {
    bool ok32 = false, ok8 = false;
    int rc = build_fast_config(d, 32, &d->fcfg, &d->fargs, &d->tm_prev_h, &d->d_search_delta, &ok32);
    if (rc) return rc;
    d->use_fast = ok32;
    if (!ok32) return INLM_OK;
    d->n_cta = d->fargs.tiles_x * d->fargs.tiles_y * ((d->shape[2] + d->fcfg.tz - 1) / d->fcfg.tz);
    rc = build_fast_config(d, 8, &d->fcfg8, &d->fargs8, &d->tm_prev_h8, &d->d_search_delta8, &ok8);
    if (rc) return rc;
    d->use_tile8 = ok8;
    // the column form for full search at patch radius 1, scaled as the
    // 32-wide kernel's tiles so both round every voxel alike
    bool okc = false;
    rc = build_fast_config(d, 0, &d->fcfgc, &d->fargsc, &d->tm_prev_hc, &d->d_search_delta_c, &okc);
    if (rc) return rc;
    d->fargsc.scale_tz = d->fcfg.tz;
    d->use_colf = okc;
    return INLM_OK;
}

extern "C" int inlm_denoiser_create(const int shape[3], const inlm_params* p, inlm_denoiser** out) {
    if (!shape || !p || !out) return fail(INLM_ERR_ARG, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return fail(INLM_ERR_NODEVICE, "no CUDA device");
    if (p->device_id < 0 || p->device_id >= ndev) return fail(INLM_ERR_ARG, "bad device id");
    for (int i = 0; i < 3; i++) {
        if (shape[i] < 1) return fail(INLM_ERR_ARG, "shape must be positive");
        if (p->search_radius[i] < 0 || p->patch_radius[i] < 0)
            return fail(INLM_ERR_ARG, "radii must be >= 0");
    }
    if (p->nslices < 1) return fail(INLM_ERR_ARG, "nslices must be >= 1");
    const bool f16 = p->precision == INLM_PRECISION_F16 || p->precision == INLM_PRECISION_F16_DF32;
    if (p->precision != INLM_PRECISION_F32 && p->precision != INLM_PRECISION_F32_FMA && !f16)
        return fail(INLM_ERR_ARG, "unknown precision %d", p->precision);

    inlm_denoiser* d = new inlm_denoiser();
    d->p = *p;
    d->device = p->device_id;
    for (int i = 0; i < 3; i++) d->shape[i] = shape[i];
    cudaSetDevice(d->device);
    int pad0[3] = {p->search_radius[0] + p->patch_radius[0], p->search_radius[1] + p->patch_radius[1],
                   std::min(p->nslices / 2, p->search_radius[2]) + p->patch_radius[2]};
    for (int i = 0; i < 3; i++)
        if (shape[i] == 1 && pad0[i] > 0) {
            delete d;
            return fail(INLM_ERR_ARG,
                        "axis %d has length 1 but needs padding %d: set its search and patch "
                        "radius to 0 (the reference does so for single slices, main.cpp:268-272)",
                        i, pad0[i]);
        }
    d->geo = make_geometry(p->search_radius, p->patch_radius, p->nslices, p->z_anisotropy,
                           p->weight_table, shape[2] + 2 * pad0[2]);
    const Geometry& g = d->geo;
    d->nxp = shape[0] + 2 * g.pad[0];
    d->nyp = shape[1] + 2 * g.pad[1];
    d->nzp = shape[2] + 2 * g.pad[2];
    d->pitch_y = (d->nxp + 31) / 32 * 32;
    d->pitch_z = d->pitch_y * d->nyp;
    // Tiles that stick out of the volume (z up to TZ-1 planes with TZ <= 16,
    // y up to TY-1 rows, x up to 31 columns past the end) read raw from global
    // memory at positions they never store; kSlackPlanes zeroed planes after
    // the padded volume keep every such read inside the allocation.
    const long long kSlackPlanes = 17;
    const long long npad = d->pitch_z * (d->nzp + kSlackPlanes);
    const long long nvox = (long long)shape[0] * shape[1] * shape[2];
    int rc = INLM_OK;
    auto bail = [&](int code) {
        denoiser_free(d);
        delete d;
        return code;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(fail(INLM_ERR_CUDA, "stream: %s", cudaGetErrorString(e)));
    d->own_stream = true;
    if (dalloc(&d->d_next, nvox) != cudaSuccess || dalloc(&d->d_sigma, shape[2]) != cudaSuccess ||
        dalloc(&d->d_sigma0, shape[2]) != cudaSuccess || dalloc(&d->d_mult, shape[2]) != cudaSuccess ||
        dalloc(&d->d_err, 1) != cudaSuccess || cudaMemset(d->d_err, 0, 4) != cudaSuccess)
        return bail(fail(INLM_ERR_NOMEM, "device allocation failed"));
    if (f16) {
        if (device_malloc(&d->d_raw_h, npad * 2) != cudaSuccess ||
            device_malloc(&d->d_prev_h, npad * 2) != cudaSuccess)
            return bail(fail(INLM_ERR_NOMEM, "device allocation of %.2f GB failed",
                             (2.0 * npad * 2 + nvox * 4) / 1e9));
        if (cudaMemset(d->d_raw_h, 0, npad * 2) != cudaSuccess ||
            cudaMemset(d->d_prev_h, 0, npad * 2) != cudaSuccess)
            return bail(fail(INLM_ERR_CUDA, "memset failed"));
        rc = choose_fast_config(d);
        if (rc != INLM_OK) return bail(rc);
        if (!d->use_fast)
            return bail(fail(INLM_ERR_UNSUPPORTED,
                             "the FP16 form covers patch radii (1,1,1) (1,1,2) (1,1,3) (2,2,1) "
                             "(2,2,2) (3,3,1) (3,3,2) (3,3,3) with nslices/2 >= z radius"));
    } else {
        if (dalloc(&d->d_raw_pad, npad) != cudaSuccess || dalloc(&d->d_prev_pad, npad) != cudaSuccess)
            return bail(fail(INLM_ERR_NOMEM, "device allocation of %.2f GB failed",
                             (2.0 * npad + nvox) * 4 / 1e9));
        // pitch padding columns stay zero
        if (cudaMemset(d->d_raw_pad, 0, npad * 4) != cudaSuccess ||
            cudaMemset(d->d_prev_pad, 0, npad * 4) != cudaSuccess)
            return bail(fail(INLM_ERR_CUDA, "memset failed"));
        // generic-kernel tables (padded-linear offsets)
        {
            std::vector<long long> so(g.search.size()), po(g.taps.size());
            for (size_t s = 0; s < g.search.size(); s++)
                so[s] = g.search[s].z * d->pitch_z + g.search[s].y * d->pitch_y + g.search[s].x;
            for (size_t q = 0; q < g.taps.size(); q++)
                po[q] = g.taps[q].z * d->pitch_z + g.taps[q].y * d->pitch_y + g.taps[q].x;
            if (dalloc(&d->d_search_off, so.size()) != cudaSuccess ||
                dalloc(&d->d_patch_off, po.size()) != cudaSuccess ||
                dalloc(&d->d_weights, g.weights.size()) != cudaSuccess)
                return bail(fail(INLM_ERR_NOMEM, "table allocation"));
            cudaMemcpy(d->d_search_off, so.data(), so.size() * 8, cudaMemcpyHostToDevice);
            cudaMemcpy(d->d_patch_off, po.data(), po.size() * 8, cudaMemcpyHostToDevice);
            cudaMemcpy(d->d_weights, g.weights.data(), g.weights.size() * 4, cudaMemcpyHostToDevice);
            GenericArgs& ga = d->gargs;
            ga.nx = shape[0];
            ga.ny = shape[1];
            ga.nz = shape[2];
            ga.px = g.pad[0];
            ga.py = g.pad[1];
            ga.pz = g.pad[2];
            ga.gpitch_y = d->pitch_y;
            ga.gpitch_z = d->pitch_z;
            ga.S = (int)g.search.size();
            ga.P = (int)g.taps.size();
            ga.search_off = d->d_search_off;
            ga.patch_off = d->d_patch_off;
            ga.weights = d->d_weights;
            ga.raw_pad = d->d_raw_pad;
            ga.prev_pad = d->d_prev_pad;
            ga.out = d->d_next;
            ga.mult = d->d_mult;
        }

        rc = choose_tile_config(d);
        if (rc != INLM_OK) return bail(rc);
    }
    if (shape[0] > p->noise_patchsize && shape[1] > p->noise_patchsize && p->n_samples > 0) {
        rc = inlm_noise_create(shape, p->n_samples, p->noise_patchsize, p->noise_seed, d->device,
                               &d->noise);
        if (rc != INLM_OK) return bail(rc);
        cudaStreamDestroy(d->noise->stream);
        d->noise->stream = d->stream;  // one stream per job
        d->noise->own_stream = false;
    }
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return bail(fail(INLM_ERR_CUDA, "configure: %s", cudaGetErrorString(e)));
    *out = d;
    return INLM_OK;
}

extern "C" int inlm_denoiser_destroy(inlm_denoiser* d) {
    denoiser_free(d);
    delete d;
    return INLM_OK;
}

extern "C" int inlm_set_stream(inlm_denoiser* d, void* stream) {
    if (!d) return fail(INLM_ERR_ARG, "null handle");
    CUDA_TRY(cudaSetDevice(d->device));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    if (stream) {
        if (d->own_stream) cudaStreamDestroy(d->stream);
        d->stream = (cudaStream_t)stream;
        d->own_stream = false;
    } else if (!d->own_stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking));
        d->own_stream = true;
    }
    if (d->noise) d->noise->stream = d->stream;
    return INLM_OK;
}

int inlm::upload_sigma_device(inlm_denoiser* d) {
    CUDA_TRY(launch_sigma_to_mult(d->d_sigma, d->p.beta, d->d_mult, d->shape[2], d->stream));
    d->launches++;
    d->sigma_set = true;
    return INLM_OK;
}

extern "C" int inlm_set_sigma(inlm_denoiser* d, const float* sigma_host) {
    if (!d || !sigma_host) return fail(INLM_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(d->device));
    CUDA_TRY(cudaMemcpyAsync(d->d_sigma, sigma_host, d->shape[2] * 4, cudaMemcpyHostToDevice,
                             d->stream));
    int rc = upload_sigma_device(d);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    return INLM_OK;
}

int inlm::launch_filter(inlm_denoiser* d) {
    TimedLaunch t;
    if (!d->event_pool.empty()) {
        t = d->event_pool.back();
        d->event_pool.pop_back();
    } else {
        CUDA_TRY(cudaEventCreate(&t.a));
        CUDA_TRY(cudaEventCreate(&t.b));
    }
    CUDA_TRY(cudaEventRecord(t.a, d->stream));
    if (d->use_fast && d->plan_active && d->plan_cta32) {
        // per-CTA plans of the learned proposal at 4 tiles per plan: full-width CTAs
        int tiles_z = (d->shape[2] + d->fcfg.tz - 1) / d->fcfg.tz;
        CUDA_TRY(launch_fast_kernel(d->fcfg, &d->tm_prev_h, d->fargs_plan, tiles_z, d->stream));
    } else if (d->use_fast && d->plan_active) {
        // per-tile plans: one 8^3 tile per CTA
        int tiles_z = (d->shape[2] + d->fcfg8.tz - 1) / d->fcfg8.tz;
        CUDA_TRY(launch_fast_kernel(d->fcfg8, &d->tm_prev_h8, d->fargs8, tiles_z, d->stream));
    } else if (d->use_fast && d->use_colf) {
        // full search at patch radius 1: the column form
        int tiles_z = (d->shape[2] + d->fcfgc.tz - 1) / d->fcfgc.tz;
        CUDA_TRY(launch_column_fast_kernel(d->fcfgc, &d->tm_prev_hc, d->fargsc, tiles_z, d->stream));
    } else if (d->use_fast) {
        int tiles_z = (d->shape[2] + d->fcfg.tz - 1) / d->fcfg.tz;
        CUDA_TRY(launch_fast_kernel(d->fcfg, &d->tm_prev_h, d->fargs, tiles_z, d->stream));
    } else if (d->use_tile) {
        int tiles_z = (d->shape[2] + d->tcfg.tz - 1) / d->tcfg.tz;
        CUDA_TRY(launch_tile_kernel(d->tcfg, &d->tm_prev, &d->tm_raw, d->targs, tiles_z, d->stream));
    } else {
        CUDA_TRY(launch_generic_kernel(d->gargs, d->stream));
    }
    CUDA_TRY(cudaEventRecord(t.b, d->stream));
    d->pending.push_back(t);
    d->launches++;
    return INLM_OK;
}

// Pads the unpadded volume `src` (device) into the FP16 padded buffer `dst`.
int inlm::pad_into_half(inlm_denoiser* d, const float* src, void* dst) {
    const Geometry& g = d->geo;
    CUDA_TRY(launch_pad_reflective_half(src, d->shape[0], d->shape[1], d->shape[2], dst, g.pad[0],
                                        g.pad[1], g.pad[2], d->pitch_y, d->pitch_z, d->stream));
    d->launches++;
    return INLM_OK;
}

// Pads the unpadded volume `src` (device) into the padded buffer `dst`.
int inlm::pad_into(inlm_denoiser* d, const float* src, float* dst) {
    const Geometry& g = d->geo;
    CUDA_TRY(launch_pad_reflective(src, d->shape[0], d->shape[1], d->shape[2], dst, g.pad[0],
                                   g.pad[1], g.pad[2], d->pitch_y, d->pitch_z, d->stream));
    d->launches++;
    return INLM_OK;
}

int inlm::check_device_error(inlm_denoiser* d) {
    int h = 0;
    CUDA_TRY(cudaMemcpyAsync(&h, d->d_err, 4, cudaMemcpyDeviceToHost, d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    if (h != 0) {
        cudaMemsetAsync(d->d_err, 0, 4, d->stream);
        return fail(INLM_ERR_TIMEOUT, "device wait gave up (code %d)", h);
    }
    return INLM_OK;
}

// Enqueues one iteration; raw_dev is the unpadded raw volume on the device
// (iteration 1 only). No host synchronisation.
static int enqueue_iteration(inlm_denoiser* d, int iter, const float* raw_dev) {
    if (iter < 1) return fail(INLM_ERR_ARG, "iteration must be >= 1");
    if (!d->sigma_set) return fail(INLM_ERR_STATE, "set_sigma before running an iteration");
    int rc;
    if (d->use_fast) {
        if (iter == 1) {
            if (!raw_dev) return fail(INLM_ERR_ARG, "iteration 1 needs the raw volume");
            rc = pad_into_half(d, raw_dev, d->d_raw_h);
            if (rc) return rc;
            CUDA_TRY(cudaMemcpyAsync(d->d_prev_h, d->d_raw_h, d->pitch_z * d->nzp * 2,
                                     cudaMemcpyDeviceToDevice, d->stream));
        } else {
            if (d->last_iter < 1) return fail(INLM_ERR_STATE, "iteration %d before iteration 1", iter);
            rc = pad_into_half(d, d->d_next, d->d_prev_h);
            if (rc) return rc;
        }
        if (d->prop.net) {
            rc = proposal_prepare_iteration(d, iter);
            if (rc) return rc;
        }
        rc = launch_filter(d);
        if (rc) return rc;
        d->last_iter = iter;
        return INLM_OK;
    }
    if (iter == 1) {
        if (!raw_dev) return fail(INLM_ERR_ARG, "iteration 1 needs the raw volume");
        rc = pad_into(d, raw_dev, d->d_raw_pad);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(d->d_prev_pad, d->d_raw_pad, d->pitch_z * d->nzp * 4,
                                 cudaMemcpyDeviceToDevice, d->stream));
    } else {
        if (d->last_iter < 1) return fail(INLM_ERR_STATE, "iteration %d before iteration 1", iter);
        rc = pad_into(d, d->d_next, d->d_prev_pad);
        if (rc) return rc;
    }
    rc = launch_filter(d);
    if (rc) return rc;
    d->last_iter = iter;
    return INLM_OK;
}

extern "C" int inlm_run_iteration(inlm_denoiser* d, int iter, const float* raw_host) {
    if (!d) return fail(INLM_ERR_ARG, "null handle");
    CUDA_TRY(cudaSetDevice(d->device));
    const long long nvox = (long long)d->shape[0] * d->shape[1] * d->shape[2];
    if (iter == 1) {
        if (!raw_host) return fail(INLM_ERR_ARG, "iteration 1 needs the raw volume");
        // stage through the result buffer, as prepare_iteration1 does
        CUDA_TRY(cudaMemcpyAsync(d->d_next, raw_host, nvox * 4, cudaMemcpyHostToDevice, d->stream));
        int rc = enqueue_iteration(d, 1, d->d_next);
        if (rc) return rc;
    } else {
        int rc = enqueue_iteration(d, iter, nullptr);
        if (rc) return rc;
    }
    return check_device_error(d);
}

extern "C" int inlm_run_iteration_device(inlm_denoiser* d, int iter, const float* raw_dev) {
    if (!d) return fail(INLM_ERR_ARG, "null handle");
    CUDA_TRY(cudaSetDevice(d->device));
    int rc = enqueue_iteration(d, iter, raw_dev);
    if (rc) return rc;
    return check_device_error(d);
}

extern "C" int inlm_get_result(inlm_denoiser* d, float* out_host) {
    if (!d || !out_host) return fail(INLM_ERR_ARG, "null argument");
    if (d->last_iter < 1) return fail(INLM_ERR_STATE, "no iteration has run");
    CUDA_TRY(cudaSetDevice(d->device));
    const long long nvox = (long long)d->shape[0] * d->shape[1] * d->shape[2];
    CUDA_TRY(cudaMemcpyAsync(out_host, d->d_next, nvox * 4, cudaMemcpyDeviceToHost, d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    return check_device_error(d);
}

extern "C" int inlm_set_result(inlm_denoiser* d, int iter, const float* result_host,
                               const float* raw_host) {
    if (!d || !result_host) return fail(INLM_ERR_ARG, "null argument");
    if (iter < 1) return fail(INLM_ERR_ARG, "iteration must be >= 1");
    if (iter > 1 && d->last_iter < 1) return fail(INLM_ERR_STATE, "iteration %d before iteration 1", iter);
    CUDA_TRY(cudaSetDevice(d->device));
    const long long nvox = (long long)d->shape[0] * d->shape[1] * d->shape[2];
    if (iter == 1) {
        if (!raw_host) return fail(INLM_ERR_ARG, "iteration 1 needs the raw volume");
        // raw is padded once and kept, as prepare_iteration1 does
        CUDA_TRY(cudaMemcpyAsync(d->d_next, raw_host, nvox * 4, cudaMemcpyHostToDevice, d->stream));
        const int rc = d->use_fast ? pad_into_half(d, d->d_next, d->d_raw_h)
                                   : pad_into(d, d->d_next, d->d_raw_pad);
        if (rc) return rc;
    }
    CUDA_TRY(cudaMemcpyAsync(d->d_next, result_host, nvox * 4, cudaMemcpyHostToDevice, d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    d->last_iter = iter;
    return check_device_error(d);
}

static int result_slices(inlm_denoiser* d, int z0, int n_slices, const void* src, void* dst, bool to_result,
                         int on_device) {
    if (!d || !(to_result ? src : dst)) return fail(INLM_ERR_ARG, "null argument");
    if (d->last_iter < 1) return fail(INLM_ERR_STATE, "no iteration has run");
    if (z0 < 0 || n_slices < 0 || z0 + n_slices > d->shape[2])
        return fail(INLM_ERR_ARG, "slices %d..%d outside 0..%d", z0, z0 + n_slices - 1, d->shape[2] - 1);
    if (n_slices == 0) return INLM_OK;
    CUDA_TRY(cudaSetDevice(d->device));
    const size_t plane = (size_t)d->shape[0] * d->shape[1];
    float* res = d->d_next + plane * z0;
    const size_t bytes = plane * n_slices * 4;
    const cudaMemcpyKind kind = to_result ? (on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice)
                                          : (on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost);
    CUDA_TRY(cudaMemcpyAsync(to_result ? (void*)res : dst, to_result ? src : (const void*)res, bytes, kind,
                             d->stream));
    // host copies complete before returning; device copies are ordered on the stream
    if (!on_device) CUDA_TRY(cudaStreamSynchronize(d->stream));
    return INLM_OK;
}

extern "C" int inlm_get_result_slices(inlm_denoiser* d, int z0, int n_slices, float* dst, int on_device) {
    return result_slices(d, z0, n_slices, nullptr, dst, false, on_device);
}

extern "C" int inlm_set_result_slices(inlm_denoiser* d, int z0, int n_slices, const float* src,
                                      int on_device) {
    return result_slices(d, z0, n_slices, src, nullptr, true, on_device);
}

extern "C" int inlm_get_result_device(inlm_denoiser* d, float* out_dev) {
    if (!d || !out_dev) return fail(INLM_ERR_ARG, "null argument");
    if (d->last_iter < 1) return fail(INLM_ERR_STATE, "no iteration has run");
    CUDA_TRY(cudaSetDevice(d->device));
    const long long nvox = (long long)d->shape[0] * d->shape[1] * d->shape[2];
    CUDA_TRY(cudaMemcpyAsync(out_dev, d->d_next, nvox * 4, cudaMemcpyDeviceToDevice, d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    return check_device_error(d);
}

// Noise estimate of a device volume into d->d_sigma (or sigma0 buffer).
int inlm::estimate_into(inlm_denoiser* d, const float* vol_dev, float* d_dst, std::vector<float>* host_copy) {
    if (!d->noise) return fail(INLM_ERR_ARG, "volume too small for the noise patch");
    std::vector<float> hs;
    bool on_host = false;
    int rc = noise_estimate_device(d->noise, &d->p, vol_dev, d->shape[0],
                                   (long long)d->shape[0] * d->shape[1], &hs, &on_host);
    if (rc) return rc;
    if (!on_host) d->launches += 3;  // patch std, EM, finalize
    const int nz = d->shape[2];
    if (on_host) {
        CUDA_TRY(cudaMemcpyAsync(d_dst, hs.data(), nz * 4, cudaMemcpyHostToDevice, d->stream));
        CUDA_TRY(cudaStreamSynchronize(d->stream));
    } else {
        CUDA_TRY(cudaMemcpyAsync(d_dst, d->noise->d_sigma, nz * 4, cudaMemcpyDeviceToDevice, d->stream));
    }
    if (host_copy) {
        host_copy->resize(nz);
        CUDA_TRY(cudaMemcpyAsync(host_copy->data(), d_dst, nz * 4, cudaMemcpyDeviceToHost, d->stream));
    }
    return INLM_OK;
}

extern "C" int inlm_denoise(inlm_denoiser* d, const float* raw, float* out, int on_device,
                            float* sigma0_out, float* sigma1_out) {
    if (!d || !raw || !out) return fail(INLM_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(d->device));
    const long long nvox = (long long)d->shape[0] * d->shape[1] * d->shape[2];
    const int nz = d->shape[2];
    const float* raw_dev = raw;
    if (!on_device) {
        CUDA_TRY(cudaMemcpyAsync(d->d_next, raw, nvox * 4, cudaMemcpyHostToDevice, d->stream));
        raw_dev = d->d_next;
    }
    // sigma0 on the raw data (main.cpp:327-351)
    std::vector<float> s0h, s1h;
    int rc = estimate_into(d, raw_dev, d->d_sigma0, sigma0_out ? &s0h : nullptr);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(d->d_sigma, d->d_sigma0, nz * 4, cudaMemcpyDeviceToDevice, d->stream));
    rc = upload_sigma_device(d);
    if (rc) return rc;
    rc = enqueue_iteration(d, 1, raw_dev);
    if (rc) return rc;
    const int maxit = d->p.maxiterations;
    if (maxit > 1) {
        // sigma1 on the first result, blended with sigma0 (main.cpp:422-448)
        rc = estimate_into(d, d->d_next, d->d_sigma, sigma1_out ? &s1h : nullptr);
        if (rc) return rc;
        CUDA_TRY(launch_sigma_blend(d->d_sigma0, d->d_sigma, d->p.alpha, nz, d->stream));
        d->launches++;
        rc = upload_sigma_device(d);
        if (rc) return rc;
    }
    for (int it = 2; it <= maxit; it++) {
        rc = enqueue_iteration(d, it, nullptr);
        if (rc) return rc;
        // --continuous (main.cpp:517-544)
        if (d->p.continuous_estimate && maxit > it + 1) {
            rc = estimate_into(d, d->d_next, d->d_sigma, nullptr);
            if (rc) return rc;
            CUDA_TRY(launch_sigma_blend(d->d_sigma0, d->d_sigma, d->p.alpha, nz, d->stream));
            d->launches++;
            rc = upload_sigma_device(d);
            if (rc) return rc;
        }
    }
    if (on_device) {
        CUDA_TRY(cudaMemcpyAsync(out, d->d_next, nvox * 4, cudaMemcpyDeviceToDevice, d->stream));
    } else {
        CUDA_TRY(cudaMemcpyAsync(out, d->d_next, nvox * 4, cudaMemcpyDeviceToHost, d->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    if (sigma0_out) std::memcpy(sigma0_out, s0h.data(), nz * 4);
    if (sigma1_out && maxit > 1) {
        // the pre-blend estimate is what the reference reports (main.cpp:438)
        std::memcpy(sigma1_out, s1h.data(), nz * 4);
    }
    return check_device_error(d);
}

extern "C" int inlm_filter_kernel_ms(inlm_denoiser* d, double* avg_ms, int* n_launches) {
    if (!d) return fail(INLM_ERR_ARG, "null handle");
    CUDA_TRY(cudaSetDevice(d->device));
    double tot = 0.0;
    int n = 0;
    for (auto& t : d->pending) {
        CUDA_TRY(cudaEventSynchronize(t.b));
        float ms = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&ms, t.a, t.b));
        tot += ms;
        n++;
        d->event_pool.push_back(t);
    }
    d->pending.clear();
    if (avg_ms) *avg_ms = n ? tot / n : 0.0;
    if (n_launches) *n_launches = n;
    return INLM_OK;
}

extern "C" int inlm_select_tile_form(inlm_denoiser* d, int form) {
    if (!d) return fail(INLM_ERR_ARG, "null handle");
    if (form < 0 || form > 3) return fail(INLM_ERR_ARG, "form must be 0, 1, 2 or 3");
    if (!d->use_tile) return fail(INLM_ERR_UNSUPPORTED, "the plain FP32 tiled kernels do not cover this configuration");
    CUDA_TRY(cudaSetDevice(d->device));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    int rc = choose_tile_config(d, form);
    if (rc) return rc;
    if (!d->use_tile) {
        choose_tile_config(d, 0);  // keep the handle usable
        return fail(INLM_ERR_UNSUPPORTED, "no kernel of form %d fits this configuration", form);
    }
    return INLM_OK;
}

extern "C" int inlm_describe(inlm_denoiser* d, char* buf, size_t len) {
    if (!d || !buf) return fail(INLM_ERR_ARG, "null argument");
    const Geometry& g = d->geo;
    if (d->use_fast) {
        const bool col = !d->plan_active && d->use_colf;
        const FastConfig& c = (d->plan_active && !d->plan_cta32) ? d->fcfg8 : col ? d->fcfgc : d->fcfg;
        snprintf(buf, len,
                 "nlm_%s_fast<%d,%d,%d> tx=%d tz=%d d_planes=%s smem=%zu S=%zu P=%zu plan=%s "
                 "pad=%d,%d,%d",
                 col ? "column" : "tile", c.rx, c.ry, c.rz, c.tx, c.tz, c.d_half ? "f16" : "f32", c.smem_bytes,
                 g.search.size(), g.taps.size(),
                 d->plan_active ? (d->plan_cta32 ? "per-cta" : "per-tile") : "full", g.pad[0],
                 g.pad[1], g.pad[2]);
    }
    else if (d->use_tile)
        snprintf(buf, len,
                 "nlm_%s_f32%s<%d,%d,%d> tz=%d raw_%s smem=%zu S=%zu P=%zu weights=%s pad=%d,%d,%d",
                 d->tcfg.column ? "column" : d->tcfg.ws ? "tile_ws" : "tile", d->tcfg.fused ? "_fused" : "",
                 d->tcfg.rx, d->tcfg.ry, d->tcfg.rz, d->tcfg.tz,
                 d->tcfg.raw_smem ? (d->targs.raw_slab ? "slab" : "smem") : "global",
                 d->tcfg.smem_bytes, g.search.size(), g.taps.size(),
                 g.specialised && d->p.weight_table == INLM_WEIGHTS_CPU ? "cpu-table" : "distweight",
                 g.pad[0], g.pad[1], g.pad[2]);
    else
        snprintf(buf, len, "nlm_generic_f32 S=%zu P=%zu pad=%d,%d,%d", g.search.size(), g.taps.size(),
                 g.pad[0], g.pad[1], g.pad[2]);
    return INLM_OK;
}

// ---------------- host-only helpers ----------------

extern "C" int inlm_geometry(const inlm_params* p, int nz, int* search_xyz, int* n_search,
                             int* patch_xyz, float* weights, int* n_patch, int pad3[3]) {
    if (!p) return fail(INLM_ERR_ARG, "null params");
    int pad2 = std::min(p->nslices / 2, p->search_radius[2]) + p->patch_radius[2];
    Geometry g = make_geometry(p->search_radius, p->patch_radius, p->nslices, p->z_anisotropy,
                               p->weight_table, nz + 2 * pad2);
    if (n_search) *n_search = (int)g.search.size();
    if (n_patch) *n_patch = (int)g.taps.size();
    if (pad3)
        for (int i = 0; i < 3; i++) pad3[i] = g.pad[i];
    if (search_xyz)
        for (size_t s = 0; s < g.search.size(); s++) {
            search_xyz[3 * s] = g.search[s].x;
            search_xyz[3 * s + 1] = g.search[s].y;
            search_xyz[3 * s + 2] = g.search[s].z;
        }
    if (patch_xyz)
        for (size_t q = 0; q < g.taps.size(); q++) {
            patch_xyz[3 * q] = g.taps[q].x;
            patch_xyz[3 * q + 1] = g.taps[q].y;
            patch_xyz[3 * q + 2] = g.taps[q].z;
        }
    if (weights)
        for (size_t q = 0; q < g.weights.size(); q++) weights[q] = g.weights[q];
    return INLM_OK;
}

extern "C" int inlm_noise_draw_samples(const int shape[3], uint64_t n_samples, int patchsize,
                                       int circular_mask_diameter, unsigned int seed, int64_t* out) {
    if (!shape || !out) return fail(INLM_ERR_ARG, "null argument");
    if (shape[0] <= patchsize || shape[1] <= patchsize || shape[2] < 1)
        return fail(INLM_ERR_ARG, "shape too small for the noise patch");
    std::vector<long long> s =
        draw_noise_samples(shape, n_samples, patchsize, circular_mask_diameter, seed);
    for (size_t i = 0; i < s.size(); i++) out[i] = s[i];
    return INLM_OK;
}

extern "C" int inlm_kernel_launches(inlm_denoiser* d, uint64_t* count) {
    if (!d || !count) return fail(INLM_ERR_ARG, "null argument");
    *count = d->launches;
    return INLM_OK;
}

// ---------------- allocation-free EM ----------------

extern "C" int inlm_noise_em_noalloc(void* stream, const float* values_dev, int64_t n_values,
                                     const int64_t* windows_host, int n_windows, float* mean_dev,
                                     float* sd_dev) {
    if (!values_dev || !windows_host || !mean_dev || !sd_dev)
        return fail(INLM_ERR_ARG, "null argument");
    if (n_values <= 0 || n_values > INT32_MAX) return fail(INLM_ERR_ARG, "n_values out of range");
    if (n_windows <= 0 || n_windows > kNoAllocMaxWindows)
        return fail(INLM_ERR_ARG, "n_windows %d outside 1..%d (static window table size)", n_windows,
                    kNoAllocMaxWindows);
    long long total = 0;
    for (int w = 0; w < n_windows; w++) {
        int64_t f = windows_host[2 * w], l = windows_host[2 * w + 1];
        if (l < f) continue;
        if (f < 0 || l >= n_values)
            return fail(INLM_ERR_ARG, "window %d [%lld, %lld] outside 0..%lld", w, (long long)f,
                        (long long)l, (long long)(n_values - 1));
        total += l - f + 1;
    }
    if (total > kNoAllocAssignBytes)
        return fail(INLM_ERR_ARG,
                    "windows cover %lld samples in total; the static scratch holds at most %lld",
                    total, (long long)kNoAllocAssignBytes);
    int dev = -1;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(launch_noise_em_noalloc(dev, values_dev, (const long long*)windows_host, n_windows,
                                     mean_dev, sd_dev, (cudaStream_t)stream));
    return INLM_OK;
}


// ---------------- per-tile offset plans ----------------

extern "C" int inlm_tile_grid(inlm_denoiser* d, int tile_shape[3], int tiles[3]) {
    if (!d) return fail(INLM_ERR_ARG, "null handle");
    int tz = d->use_fast ? d->fcfg.tz : (d->use_tile ? d->tcfg.tz : 1);
    if (tile_shape) {
        tile_shape[0] = kTX;
        tile_shape[1] = kTY;
        tile_shape[2] = tz;
    }
    if (tiles) {
        tiles[0] = (d->shape[0] + kTX - 1) / kTX;
        tiles[1] = (d->shape[1] + kTY - 1) / kTY;
        tiles[2] = (d->shape[2] + tz - 1) / tz;
    }
    return INLM_OK;
}

extern "C" int inlm_set_offset_plan(inlm_denoiser* d, const int* start, const int* count,
                                    const int* offsets, int n_offsets, int on_device) {
    if (!d) return fail(INLM_ERR_ARG, "null handle");
    if (!d->use_fast || !d->use_tile8)
        return fail(INLM_ERR_UNSUPPORTED, "offset plans need the FP16 form");
    if (d->prop.net) return fail(INLM_ERR_STATE, "a proposal network is attached; detach it first");
    CUDA_TRY(cudaSetDevice(d->device));
    d->plan_cta32 = false;
    if (!start) {
        d->plan_active = false;
        d->fargs8.plan_start = nullptr;
        d->fargs8.plan_count = nullptr;
        d->fargs8.plan_offsets = nullptr;
        return INLM_OK;
    }
    if (!count || !offsets || n_offsets < 0) return fail(INLM_ERR_ARG, "null plan array");
    // one list per 8^3 tile (the tx = 8 grid)
    const long long n = (long long)d->fargs8.tiles_x * d->fargs8.tiles_y *
                        ((d->shape[2] + d->fcfg8.tz - 1) / d->fcfg8.tz);
    if (!on_device) {
        for (long long c = 0; c < n; c++)
            if (start[c] < 0 || count[c] < 0 || count[c] > d->fargs8.S ||
                (long long)start[c] + count[c] > n_offsets)
                return fail(INLM_ERR_ARG, "plan tile %lld has a bad offset range", c);
        for (int i = 0; i < n_offsets; i++)
            if (offsets[i] < 0 || offsets[i] >= d->fargs8.S)
                return fail(INLM_ERR_ARG, "plan entry %d out of range", offsets[i]);
    }
    if (!d->d_plan_start) CUDA_TRY(dalloc(&d->d_plan_start, 2 * (size_t)n));
    if (d->plan_cap < std::max(n_offsets, 1)) {
        device_free(d->d_plan_off);
        d->d_plan_off = nullptr;
        d->plan_cap = 0;
        CUDA_TRY(dalloc(&d->d_plan_off, (size_t)std::max(n_offsets, 1)));
        d->plan_cap = std::max(n_offsets, 1);
    }
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CUDA_TRY(cudaMemcpyAsync(d->d_plan_start, start, (size_t)n * 4, kind, d->stream));
    CUDA_TRY(cudaMemcpyAsync(d->d_plan_start + n, count, (size_t)n * 4, kind, d->stream));
    CUDA_TRY(cudaMemcpyAsync(d->d_plan_off, offsets, (size_t)n_offsets * 4, kind, d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    d->fargs8.plan_start = d->d_plan_start;
    d->fargs8.plan_count = d->d_plan_start + n;
    d->fargs8.plan_offsets = d->d_plan_off;
    d->plan_active = true;
    return INLM_OK;
}
