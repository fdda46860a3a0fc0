// One stack split in z across several GPUs of this process: the n_gpus mode of
// IterativeNLM_GPU::Run_GaussianNoise_GPUBlocks (Denoiser/iternlm_gpu.cu:
// 1732-2115), where the reference hands each GPU a block of slices.
//
// Device i owns slices [z0_i, z1_i) (8-slice units, split evenly) and filters
// them as a sub-volume with h slices of each neighbour (h = the z padding
// rounded up to 8). After every iteration each device's boundary slices are
// copied device to device into its neighbours' halos, so every owned voxel
// reads exactly the previous iterate the single-GPU job reads; raw halos come
// with the sub-volume. Noise estimates: every device measures the patch stds
// of the samples in its own slices (the sample positions are the same on
// every device: same seed, whole-stack shape), the host sums the disjoint
// parts and one EM runs on the first device. Owned results equal inlm_denoise
// bit for bit in every precision form. Devices may repeat in the list (two
// sub-volumes on one GPU), which is how a one-GPU machine runs this path.
#include <algorithm>
#include <memory>
#include <thread>
#include <vector>

#include "api_internal.hpp"

using namespace inlm;

namespace {

struct Part {
    int device = 0;
    int z0 = 0, z1 = 0;      // owned slices
    int a = 0, b = 0;        // sub-volume slices [a, b)
    inlm_denoiser* d = nullptr;
    inlm_noise* noise = nullptr;
    float* d_stage = nullptr;  // own raw slices (device) for the first estimate
    ~Part() {
        if (d) inlm_denoiser_destroy(d);
        if (noise) inlm_noise_destroy(noise);
        if (d_stage) {
            cudaSetDevice(device);
            device_free(d_stage);
        }
    }
};

// Runs fn(i) for every part on its own host thread (the C ABI calls of one
// part block on that part's stream); returns the first error.
template <typename Fn>
int each_part(std::vector<Part>& parts, Fn fn) {
    std::vector<int> rc(parts.size(), INLM_OK);
    std::vector<std::string> err(parts.size());
    std::vector<std::thread> th;
    for (size_t i = 0; i < parts.size(); i++)
        th.emplace_back([&, i]() {
            cudaSetDevice(parts[i].device);
            rc[i] = fn(i);
            if (rc[i] != INLM_OK) err[i] = inlm_last_error();
        });
    for (auto& t : th) t.join();
    for (size_t i = 0; i < parts.size(); i++)
        if (rc[i] != INLM_OK) return fail(rc[i], "device part %zu: %s", i, err[i].c_str());
    return INLM_OK;
}

}  // namespace

extern "C" int inlm_denoise_multi(const int shape[3], const inlm_params* p, const float* raw_host,
                                  float* out_host, int n_parts, const int* device_ids, float* sigma0_out,
                                  float* sigma1_out) {
    if (!shape || !p || !raw_host || !out_host || !device_ids) return fail(INLM_ERR_ARG, "null argument");
    if (n_parts < 1) return fail(INLM_ERR_ARG, "n_parts must be >= 1");
    if (p->maxiterations < 1) return fail(INLM_ERR_ARG, "maxiterations < 1");
    const int nx = shape[0], ny = shape[1], nz = shape[2];
    const long long plane = (long long)nx * ny;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(INLM_ERR_NODEVICE, "no CUDA device");
    }
    for (int i = 0; i < n_parts; i++)
        if (device_ids[i] < 0 || device_ids[i] >= ndev)
            return fail(INLM_ERR_ARG, "device %d of %d", device_ids[i], ndev);
    // slabs: 8-slice units split evenly, lower parts taking the remainder
    const int units = (nz + 7) / 8;
    if (units < n_parts) return fail(INLM_ERR_ARG, "%d slices give fewer than %d slabs of 8", nz, n_parts);
    const int pz = std::min(p->nslices / 2, p->search_radius[2]) + p->patch_radius[2];
    const int halo = (std::max(pz, 1) + 7) / 8 * 8;
    std::vector<Part> parts(n_parts);
    {
        int u = 0;
        for (int i = 0; i < n_parts; i++) {
            const int n = units / n_parts + (i < units % n_parts ? 1 : 0);
            Part& q = parts[i];
            q.device = device_ids[i];
            q.z0 = std::min(nz, 8 * u);
            q.z1 = std::min(nz, 8 * (u + n));
            u += n;
            q.a = std::max(0, q.z0 - halo);
            q.b = std::min(nz, q.z1 + halo);
            if (n_parts > 1 && q.z1 - q.z0 < halo)
                return fail(INLM_ERR_ARG, "slab %d..%d is shallower than the halo of %d slices", q.z0,
                            q.z1 - 1, halo);
        }
    }
    const bool manual = p->noise_mode == INLM_NOISE_MANUAL;
    if (!manual && p->noise_mode != INLM_NOISE_GLOBAL && p->noise_mode != INLM_NOISE_ZADAPTIVE)
        return fail(INLM_ERR_UNSUPPORTED, "noise modes across GPUs: global, z-adaptive, manual");

    // peer access where the devices allow it (copies work without it too)
    for (int i = 0; i + 1 < n_parts; i++) {
        const int a = parts[i].device, b = parts[i + 1].device;
        if (a == b) continue;
        int ok = 0;
        if (cudaDeviceCanAccessPeer(&ok, a, b) == cudaSuccess && ok) {
            cudaSetDevice(a);
            cudaDeviceEnablePeerAccess(b, 0);
            cudaSetDevice(b);
            cudaDeviceEnablePeerAccess(a, 0);
        }
        cudaGetLastError();  // "already enabled" is not an error here
    }

    inlm_params q0 = *p;
    int rc = each_part(parts, [&](size_t i) -> int {
        Part& q = parts[i];
        inlm_params qi = q0;
        qi.device_id = q.device;
        qi.n_samples = 0;  // the parts' noise handles cover the whole stack
        const int sh[3] = {nx, ny, q.b - q.a};
        int r = inlm_denoiser_create(sh, &qi, &q.d);
        if (r) return r;
        if (!manual) {
            r = inlm_noise_create(shape, p->n_samples, p->noise_patchsize, p->noise_seed, q.device, &q.noise);
            if (r) return r;
            CUDA_TRY(dalloc(&q.d_stage, (size_t)plane * (q.z1 - q.z0)));
            CUDA_TRY(cudaMemcpy(q.d_stage, raw_host + q.z0 * plane, plane * (q.z1 - q.z0) * 4,
                                cudaMemcpyHostToDevice));
        }
        return INLM_OK;
    });
    if (rc) return rc;

    // a noise estimate over all parts: patch stds of own slices, summed on the host
    std::vector<std::vector<float>> ps(n_parts);
    auto estimate = [&](bool on_raw, float* sigma) -> int {
        uint64_t ns = 0;
        int r = each_part(parts, [&](size_t i) -> int {
            Part& q = parts[i];
            const float* slab = on_raw ? q.d_stage : q.d->d_next + (long long)(q.z0 - q.a) * plane;
            if (!on_raw) CUDA_TRY(cudaStreamSynchronize(q.d->stream));
            ps[i].assign(std::max<uint64_t>(p->n_samples, 1), 0.0f);
            return inlm_noise_patchstd_slab(q.noise, p, slab, 1, q.z0, q.z1 - q.z0, ps[i].data(),
                                            ps[i].size());
        });
        if (r) return r;
        uint64_t drawn = 0;
        r = inlm_noise_samples(parts[0].noise, nullptr, 0, &drawn);
        if (r) return r;
        ns = drawn;
        std::vector<float> all(ns, 0.0f);
        for (int i = 0; i < n_parts; i++)
            for (uint64_t k = 0; k < ns; k++) all[k] += ps[i][k];
        inlm_params qe = q0;
        CUDA_TRY(cudaSetDevice(parts[0].device));
        return inlm_noise_estimate_from_patchstd(parts[0].noise, &qe, all.data(), ns, sigma);
    };
    // halos: every part's halo slices from its neighbours' owned results
    auto exchange = [&]() -> int {
        for (int i = 0; i < n_parts; i++) {
            CUDA_TRY(cudaSetDevice(parts[i].device));
            CUDA_TRY(cudaStreamSynchronize(parts[i].d->stream));
        }
        for (int i = 0; i < n_parts; i++) {
            Part& q = parts[i];
            CUDA_TRY(cudaSetDevice(q.device));
            if (q.z0 > q.a) {  // lower halo from part i-1
                const Part& s = parts[i - 1];
                const int h = q.z0 - q.a;
                CUDA_TRY(cudaMemcpyPeerAsync(q.d->d_next, q.device,
                                             s.d->d_next + (long long)(q.z0 - h - s.a) * plane, s.device,
                                             (size_t)h * plane * 4, q.d->stream));
            }
            if (q.b > q.z1) {  // upper halo from part i+1
                const Part& s = parts[i + 1];
                const int h = q.b - q.z1;
                CUDA_TRY(cudaMemcpyPeerAsync(q.d->d_next + (long long)(q.z1 - q.a) * plane, q.device,
                                             s.d->d_next + (long long)(q.z1 - s.a) * plane, s.device,
                                             (size_t)h * plane * 4, q.d->stream));
            }
        }
        for (int i = 0; i < n_parts; i++) {
            CUDA_TRY(cudaSetDevice(parts[i].device));
            CUDA_TRY(cudaStreamSynchronize(parts[i].d->stream));
        }
        return INLM_OK;
    };
    auto set_sigma = [&](const std::vector<float>& sig) -> int {
        return each_part(parts, [&](size_t i) -> int {
            return inlm_set_sigma(parts[i].d, sig.data() + parts[i].a);
        });
    };
    auto blend = [&](const std::vector<float>& s0, const std::vector<float>& s1) {
        std::vector<float> out(nz);
        for (int z = 0; z < nz; z++) out[z] = p->alpha * s0[z] + (1.f - p->alpha) * s1[z];
        return out;
    };

    std::vector<float> s0(nz), s1(nz, 0.0f);
    if (manual) {
        std::fill(s0.begin(), s0.end(), p->sigma[0]);
    } else {
        rc = estimate(true, s0.data());
        if (rc) return rc;
    }
    rc = set_sigma(s0);
    if (rc) return rc;
    rc = each_part(parts, [&](size_t i) -> int {
        return inlm_run_iteration(parts[i].d, 1, raw_host + parts[i].a * plane);
    });
    if (rc) return rc;
    for (int it = 2; it <= p->maxiterations; it++) {
        rc = exchange();
        if (rc) return rc;
        if (it == 2 || (p->continuous_estimate && p->maxiterations > it)) {
            // sigma1 on iteration 1's result (main.cpp:422-448); --continuous
            // re-estimates before later iterations (main.cpp:517-544)
            std::vector<float> est(nz);
            if (manual) {
                std::fill(est.begin(), est.end(), p->sigma[1]);
            } else {
                rc = estimate(false, est.data());
                if (rc) return rc;
            }
            if (it == 2) s1 = est;
            rc = set_sigma(blend(s0, est));
            if (rc) return rc;
        }
        rc = each_part(parts, [&](size_t i) -> int { return inlm_run_iteration(parts[i].d, it, nullptr); });
        if (rc) return rc;
    }
    // owned slices back to the host
    rc = each_part(parts, [&](size_t i) -> int {
        Part& q = parts[i];
        return inlm_get_result_slices(q.d, q.z0 - q.a, q.z1 - q.z0, out_host + q.z0 * plane, 0);
    });
    if (rc) return rc;
    if (sigma0_out) std::copy(s0.begin(), s0.end(), sigma0_out);
    if (sigma1_out) std::copy(s1.begin(), s1.end(), sigma1_out);
    return INLM_OK;
}

extern "C" int inlm_device_count(int* n) {
    if (!n) return fail(INLM_ERR_ARG, "null argument");
    *n = 0;
    if (cudaGetDeviceCount(n) != cudaSuccess) {
        cudaGetLastError();
        *n = 0;
    }
    return INLM_OK;
}

// ---------------- per-iteration engine over several devices ----------------
//
// The same split, one iteration per call with the caller's sigma and buffers
// (the n_gpus blocks of IterativeNLM_GPU::Run_GaussianNoise_GPUBlocks,
// Denoiser/iternlm_gpu.cu:1729-1886): iteration 1 takes each part's slices of
// raw; a later iteration installs each part's sub-volume of the previous
// iterate from host memory (its halos included, so no device-to-device
// exchange is needed) and filters it; every part's owned slices go to the
// output.
namespace {

struct MultiBlocks final : BlocksBackend {
    std::vector<Part> parts;
    long long plane = 0;
    int depth = 0;
    int slab_depth() const override { return depth; }
    int set_sigma(const float* sigma) override {
        return each_part(parts, [&](size_t i) -> int { return inlm_set_sigma(parts[i].d, sigma + parts[i].a); });
    }
    int iteration(int it, const float* raw, const float* prev, float* out) override {
        return each_part(parts, [&](size_t i) -> int {
            Part& q = parts[i];
            const long long off = (long long)q.a * plane;
            int r;
            if (it == 1) {
                r = inlm_run_iteration(q.d, 1, raw + off);
            } else {
                // the whole sub-volume, halos included, from the caller's previous
                // iterate (raw is padded once, with the first installed result)
                // (installing iteration 1 pads raw with it, so it takes raw)
                r = (q.d->last_iter < 1 || it - 1 == 1) ? inlm_set_result(q.d, 1, prev + off, raw + off)
                                                        : inlm_set_result(q.d, it - 1, prev + off, nullptr);
                if (!r) r = inlm_run_iteration(q.d, it, nullptr);
            }
            if (r) return r;
            return inlm_get_result_slices(q.d, q.z0 - q.a, q.z1 - q.z0, out + (long long)q.z0 * plane, 0);
        });
    }
};

}  // namespace

int inlm::make_multi_blocks(const int shape[3], const inlm_params* p, int n_parts, const int* device_ids,
                            BlocksBackend** out) {
    if (n_parts < 1 || !device_ids) return fail(INLM_ERR_ARG, "n_parts must be >= 1");
    const int nz = shape[2];
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(INLM_ERR_NODEVICE, "no CUDA device");
    }
    for (int i = 0; i < n_parts; i++)
        if (device_ids[i] < 0 || device_ids[i] >= ndev)
            return fail(INLM_ERR_ARG, "device %d of %d", device_ids[i], ndev);
    const int units = (nz + 7) / 8;
    if (units < n_parts) return fail(INLM_ERR_ARG, "%d slices give fewer than %d slabs of 8", nz, n_parts);
    const int pz = std::min(p->nslices / 2, p->search_radius[2]) + p->patch_radius[2];
    const int halo = (std::max(pz, 1) + 7) / 8 * 8;
    auto* b = new MultiBlocks();
    std::unique_ptr<MultiBlocks> guard(b);
    b->plane = (long long)shape[0] * shape[1];
    b->parts.resize(n_parts);
    int u = 0;
    for (int i = 0; i < n_parts; i++) {
        const int n = units / n_parts + (i < units % n_parts ? 1 : 0);
        Part& q = b->parts[i];
        q.device = device_ids[i];
        q.z0 = std::min(nz, 8 * u);
        q.z1 = std::min(nz, 8 * (u + n));
        u += n;
        q.a = std::max(0, q.z0 - halo);
        q.b = std::min(nz, q.z1 + halo);
        b->depth = std::max(b->depth, q.z1 - q.z0);
        if (n_parts > 1 && q.z1 - q.z0 < halo)
            return fail(INLM_ERR_ARG, "slab %d..%d is shallower than the halo of %d slices", q.z0, q.z1 - 1, halo);
    }
    const inlm_params q0 = *p;
    int rc = each_part(b->parts, [&](size_t i) -> int {
        Part& q = b->parts[i];
        inlm_params qi = q0;
        qi.device_id = q.device;
        qi.n_samples = 0;  // the caller estimates the noise
        const int sh[3] = {shape[0], shape[1], q.b - q.a};
        return inlm_denoiser_create(sh, &qi, &q.d);
    });
    if (rc) return rc;
    *out = guard.release();
    return INLM_OK;
}

extern "C" int inlm_device_memory(int device, size_t* free_bytes, size_t* total_bytes) {
    if (!free_bytes || !total_bytes) return fail(INLM_ERR_ARG, "null argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(INLM_ERR_NODEVICE, "no CUDA device");
    }
    if (device < 0 || device >= ndev) return fail(INLM_ERR_ARG, "device %d of %d", device, ndev);
    CUDA_TRY(cudaSetDevice(device));
    CUDA_TRY(cudaMemGetInfo(free_bytes, total_bytes));
    return INLM_OK;
}
