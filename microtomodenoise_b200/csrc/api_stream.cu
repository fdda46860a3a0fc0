// z-slab streaming of a host-resident volume (include/inlm.h). The reference
// streams volumes that do not fit its GPUs in blocks of slices
// (IterativeNLM_GPU::Run_GaussianNoise_GPUBlocks, Denoiser/iternlm_gpu.cu:
// 1887-2115); here the volume stays in host memory and every iteration walks
// it in z-slabs:
//   * slab [z0, z1) is filtered as the sub-volume [z0 - h, z1 + h) (h >= the
//     filter's z padding, clipped at the volume's faces), so every voxel of
//     the slab reads exactly the values the whole-volume filter reads; the
//     faces of the sub-volume pad like the whole volume's only where they are
//     the volume's own faces;
//   * h and the slab starts are multiples of 8, so the FP16 form's tiles and
//     the learned proposal's 8^3 tiles fall where they fall in the whole
//     volume, and h >= 16 with a proposal (its 15-voxel receptive field);
//   * two denoisers per sub-volume depth alternate on their own streams, so
//     one slab's copies overlap the other's kernels;
//   * the noise estimates take each sample's patch std from the slab holding
//     it (on the device, right after the slab's filter for sigma1) and run the
//     EM once over all samples.
// Results equal the in-memory schedule (inlm_denoise) bit for bit.
#include <map>
#include <memory>

#include "api_internal.hpp"
#include "noise_kernels.cuh"

using namespace inlm;

namespace {

struct SlabPair {
    inlm_denoiser* d[2] = {nullptr, nullptr};
    float* stage[2] = {nullptr, nullptr};  // unpadded raw sub-volume
};

struct StreamJob {
    int shape[3];
    long long plane = 0;
    std::map<int, SlabPair> pairs;  // by sub-volume depth
    inlm_noise* noise = nullptr;
    float* d_sig0 = nullptr;  // sigma0 per slice
    float* d_sig = nullptr;   // sigma of the current iteration
    float* tmp_host = nullptr;
    bool reg_raw = false, reg_out = false;
    const float* raw_host = nullptr;
    float* out_host = nullptr;
    cudaStream_t main = nullptr;
    int tiles_x = 1;  // proposal lists per 8^3 tile (1) or per 32 x 8 x 8 block (4)
    float rel_mass = 0.f;  // relative fallback (the mean over each sub-volume's lists)
    std::vector<int> sched_k;  // per-iteration schedule (inlm_proposal_schedule), or empty
    std::vector<float> sched_rel;

    ~StreamJob() {
        for (auto& kv : pairs)
            for (int j = 0; j < 2; j++) {
                if (kv.second.d[j]) inlm_denoiser_destroy(kv.second.d[j]);
                device_free(kv.second.stage[j]);
            }
        if (noise) inlm_noise_destroy(noise);
        device_free(d_sig0);
        device_free(d_sig);
        if (tmp_host) cudaFreeHost(tmp_host);
        if (reg_raw) cudaHostUnregister(const_cast<float*>(raw_host));
        if (reg_out) cudaHostUnregister(out_host);
        if (main) cudaStreamDestroy(main);
    }
};

int round_up8(int v) { return (v + 7) / 8 * 8; }

// Sample index range [i0, i1) of slices [z0, z1) (samples are sorted).
void sample_range(const std::vector<long long>& s, long long plane, int z0, int z1, long long* i0,
                  long long* i1) {
    *i0 = std::lower_bound(s.begin(), s.end(), (long long)z0 * plane) - s.begin();
    *i1 = std::lower_bound(s.begin(), s.end(), (long long)z1 * plane) - s.begin();
}

int get_pair(StreamJob& J, const inlm_params& p, int depth, inlm_proposal* net, int k,
             float min_mass, SlabPair** out) {
    auto it = J.pairs.find(depth);
    if (it != J.pairs.end()) {
        *out = &it->second;
        return INLM_OK;
    }
    SlabPair& sp = J.pairs[depth];
    inlm_params q = p;
    q.n_samples = 0;  // the job's own noise handle covers the whole volume
    const int sh[3] = {J.shape[0], J.shape[1], depth};
    for (int j = 0; j < 2; j++) {
        int rc = inlm_denoiser_create(sh, &q, &sp.d[j]);
        if (rc) return rc;
        CUDA_TRY(dalloc(&sp.stage[j], (size_t)J.plane * depth));
        if (net) {
            rc = inlm_attach_proposal_ex(sp.d[j], net, k, min_mass, J.rel_mass, J.tiles_x);
            if (rc) return rc;
            if (!J.sched_k.empty()) {
                rc = inlm_proposal_schedule(sp.d[j], (int)J.sched_k.size(), J.sched_k.data(),
                                            J.sched_rel.data());
                if (rc) return rc;
            }
        }
    }
    *out = &sp;
    return INLM_OK;
}

// One iteration over every slab: slab [z0, z1) is filtered as the sub-volume
// [z0 - halo, z1 + halo) on one of the two denoisers of its depth (they
// alternate, so one slab's copies overlap the other's kernels); raw from
// raw_host, the previous iterate from prev_host (iteration > 1), the slab's
// result to next_host. With patchstd, each slab's result also gives the
// patch stds of the samples in its own slices. J.d_sig holds the sigma of
// this iteration; every slab's stream waits for the event `ready` first.
int stream_pass(StreamJob& J, const inlm_params& p, int it, const std::vector<int>& z0s, int sd,
                int halo, inlm_proposal* net, int k, float min_mass, const float* raw_host,
                const float* prev_host, float* next_host, bool patchstd, cudaEvent_t ready,
                double* h2d, double* d2h) {
    const int nz = J.shape[2];
    int s = 0;
    for (int z0 : z0s) {
        const int z1 = std::min(nz, z0 + sd);
        const int a = std::max(0, z0 - halo), b = std::min(nz, z1 + halo);
        SlabPair* sp;
        int rc = get_pair(J, p, b - a, net, k, min_mass, &sp);
        if (rc) return rc;
        const int j = s++ & 1;
        inlm_denoiser* d = sp->d[j];
        cudaStream_t st = d->stream;
        const size_t sub = (size_t)(b - a) * J.plane * 4;
        // the sub-volume's sigma slice and multiplier
        CUDA_TRY(cudaStreamWaitEvent(st, ready, 0));
        CUDA_TRY(cudaMemcpyAsync(d->d_sigma, J.d_sig + a, (b - a) * 4, cudaMemcpyDeviceToDevice, st));
        rc = upload_sigma_device(d);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(sp->stage[j], raw_host + a * J.plane, sub, cudaMemcpyHostToDevice, st));
        *h2d += sub;
        if (it > 1) {
            CUDA_TRY(cudaMemcpyAsync(d->d_next, prev_host + a * J.plane, sub, cudaMemcpyHostToDevice, st));
            *h2d += sub;
        }
        if (d->use_fast) {
            rc = pad_into_half(d, sp->stage[j], d->d_raw_h);
            if (rc) return rc;
            if (it == 1) {
                CUDA_TRY(cudaMemcpyAsync(d->d_prev_h, d->d_raw_h, d->pitch_z * d->nzp * 2,
                                         cudaMemcpyDeviceToDevice, st));
            } else {
                rc = pad_into_half(d, d->d_next, d->d_prev_h);
                if (rc) return rc;
            }
            if (d->prop.net) {
                rc = proposal_prepare_iteration(d, it);
                if (rc) return rc;
            }
        } else {
            rc = pad_into(d, sp->stage[j], d->d_raw_pad);
            if (rc) return rc;
            if (it == 1) {
                CUDA_TRY(cudaMemcpyAsync(d->d_prev_pad, d->d_raw_pad, d->pitch_z * d->nzp * 4,
                                         cudaMemcpyDeviceToDevice, st));
            } else {
                rc = pad_into(d, d->d_next, d->d_prev_pad);
                if (rc) return rc;
            }
        }
        rc = launch_filter(d);
        if (rc) return rc;
        d->last_iter = it;
        CUDA_TRY(cudaMemcpyAsync(next_host + z0 * J.plane, d->d_next + (z0 - a) * J.plane,
                                 (z1 - z0) * J.plane * 4, cudaMemcpyDeviceToHost, st));
        *d2h += (z1 - z0) * J.plane * 4.0;
        if (patchstd) {
            long long i0, i1;
            sample_range(J.noise->samples, J.plane, z0, z1, &i0, &i1);
            CUDA_TRY(launch_noise_patchstd(d->d_next, J.shape[0], J.plane, J.shape[0], J.plane,
                                           J.noise->d_samples + i0, i1 - i0, J.noise->patchsize,
                                           J.noise->d_patchstd + i0, st, a));
        }
    }
    return INLM_OK;
}

}  // namespace

extern "C" int inlm_stream_denoise(const int shape[3], const inlm_params* p, const float* raw_host,
                                   float* out_host, int slab_depth, inlm_proposal* net, int k,
                                   float min_mass, float* sigma0_out, float* sigma1_out,
                                   double* stats) {
    return inlm_stream_denoise_grouped(shape, p, raw_host, out_host, slab_depth, net, k, min_mass, 1,
                                       sigma0_out, sigma1_out, stats);
}

extern "C" int inlm_stream_denoise_grouped(const int shape[3], const inlm_params* p,
                                           const float* raw_host, float* out_host, int slab_depth,
                                           inlm_proposal* net, int k, float min_mass, int tiles_x,
                                           float* sigma0_out, float* sigma1_out, double* stats) {
    return inlm_stream_denoise_ex(shape, p, raw_host, out_host, slab_depth, net, k, min_mass, 0.f, tiles_x,
                                  sigma0_out, sigma1_out, stats);
}

extern "C" int inlm_stream_denoise_ex(const int shape[3], const inlm_params* p, const float* raw_host,
                                      float* out_host, int slab_depth, inlm_proposal* net, int k,
                                      float min_mass, float rel_mass, int tiles_x, float* sigma0_out,
                                      float* sigma1_out, double* stats) {
    return inlm_stream_denoise_sched(shape, p, raw_host, out_host, slab_depth, net, 1, &k, &rel_mass,
                                     min_mass, tiles_x, sigma0_out, sigma1_out, stats);
}

extern "C" int inlm_stream_denoise_sched(const int shape[3], const inlm_params* p, const float* raw_host,
                                         float* out_host, int slab_depth, inlm_proposal* net, int n_sched,
                                         const int* k_sched, const float* rel_sched, float min_mass,
                                         int tiles_x, float* sigma0_out, float* sigma1_out, double* stats) {
    if (!shape || !p || !raw_host || !out_host) return fail(INLM_ERR_ARG, "null argument");
    if (n_sched < 1 || n_sched > 1024 || !k_sched || !rel_sched)
        return fail(INLM_ERR_ARG, "a schedule of 1..1024 entries is required");
    int k = 0;
    for (int i = 0; i < n_sched; i++) {
        if (k_sched[i] < 0) return fail(INLM_ERR_ARG, "schedule k must be >= 0 (0: full search)");
        if (!(rel_sched[i] >= 0.f && rel_sched[i] <= 1.f))
            return fail(INLM_ERR_ARG, "schedule rel_mass must be in 0..1");
        k = std::max(k, k_sched[i]);
    }
    if (net && k < 1) return fail(INLM_ERR_ARG, "a schedule needs one iteration with k >= 1");
    const float rel_mass = rel_sched[n_sched - 1];
    if (!(rel_mass >= 0.f && rel_mass <= 1.f)) return fail(INLM_ERR_ARG, "rel_mass must be in 0..1");
    if (tiles_x != 1 && tiles_x != 4) return fail(INLM_ERR_ARG, "tiles_x must be 1 or 4");
    if (slab_depth < 1) return fail(INLM_ERR_ARG, "slab depth must be >= 1");
    if (p->noise_mode != INLM_NOISE_GLOBAL && p->noise_mode != INLM_NOISE_ZADAPTIVE &&
        p->noise_mode != INLM_NOISE_MANUAL)
        return fail(INLM_ERR_UNSUPPORTED, "streamed noise modes are global, z-adaptive and manual");
    if (p->maxiterations < 1) return fail(INLM_ERR_ARG, "maxiterations < 1");
    if (net && p->precision == INLM_PRECISION_F32)
        return fail(INLM_ERR_UNSUPPORTED, "the proposal drives the FP16 form");
    const bool manual = p->noise_mode == INLM_NOISE_MANUAL;
    CUDA_TRY(cudaSetDevice(p->device_id));
    StreamJob J;
    J.tiles_x = tiles_x;
    J.rel_mass = rel_mass;
    if (n_sched > 1) {
        J.sched_k.assign(k_sched, k_sched + n_sched);
        J.sched_rel.assign(rel_sched, rel_sched + n_sched);
    }
    for (int i = 0; i < 3; i++) J.shape[i] = shape[i];
    J.plane = (long long)shape[0] * shape[1];
    J.raw_host = raw_host;
    J.out_host = out_host;
    const int nz = shape[2];
    const long long nvox = J.plane * nz;
    CUDA_TRY(cudaStreamCreateWithFlags(&J.main, cudaStreamNonBlocking));

    // halo and slab grid
    const int pz = std::min(p->nslices / 2, p->search_radius[2]) + p->patch_radius[2];
    int halo = round_up8(std::max(pz, 1));
    if (net) halo = std::max(halo, 16);
    const int sd = round_up8(slab_depth);
    std::vector<int> z0s;
    for (int z = 0; z < nz; z += sd) z0s.push_back(z);

    // host buffers: page-locked for asynchronous copies
    cudaError_t e = cudaHostRegister(const_cast<float*>(raw_host), nvox * 4, cudaHostRegisterPortable);
    if (e == cudaSuccess) J.reg_raw = true;
    else cudaGetLastError();  // already page-locked (or not registrable): copies still work
    e = cudaHostRegister(out_host, nvox * 4, cudaHostRegisterPortable);
    if (e == cudaSuccess) J.reg_out = true;
    else cudaGetLastError();
    if (p->maxiterations > 1) CUDA_TRY(cudaMallocHost(&J.tmp_host, nvox * 4));

    CUDA_TRY(dalloc(&J.d_sig0, nz));
    CUDA_TRY(dalloc(&J.d_sig, nz));
    int nwin = 0;
    if (!manual) {
        int rc = inlm_noise_create(shape, p->n_samples, p->noise_patchsize, p->noise_seed,
                                   p->device_id, &J.noise);
        if (rc) return rc;
        cudaStreamDestroy(J.noise->stream);
        J.noise->stream = J.main;
        J.noise->own_stream = false;
        rc = noise_prepare(J.noise, p, &nwin, nullptr);
        if (rc) return rc;
    }
    double h2d = 0, d2h = 0;
    cudaEvent_t t0, t1;
    CUDA_TRY(cudaEventCreate(&t0));
    CUDA_TRY(cudaEventCreate(&t1));
    CUDA_TRY(cudaEventRecord(t0, J.main));

    auto sync_all = [&]() -> int {
        for (auto& kv : J.pairs)
            for (int j = 0; j < 2; j++) CUDA_TRY(cudaStreamSynchronize(kv.second.d[j]->stream));
        CUDA_TRY(cudaStreamSynchronize(J.main));
        return INLM_OK;
    };
    // patch stds of the samples in slices [z0, z1) of a device slab holding
    // slices from zb on, on stream st
    auto slab_patchstd = [&](const float* slab, int zb, int z0, int z1, cudaStream_t st) -> int {
        long long i0, i1;
        sample_range(J.noise->samples, J.plane, z0, z1, &i0, &i1);
        CUDA_TRY(launch_noise_patchstd(slab, shape[0], J.plane, shape[0], J.plane,
                                       J.noise->d_samples + i0, i1 - i0, J.noise->patchsize,
                                       J.noise->d_patchstd + i0, st, zb));
        return INLM_OK;
    };

    // sigma0 (main.cpp:327-351): the raw volume's samples, slab by slab
    std::vector<float> s0h(nz), s1h(nz);
    if (manual) {
        std::vector<float> v(nz, p->sigma[0]);
        CUDA_TRY(cudaMemcpy(J.d_sig0, v.data(), nz * 4, cudaMemcpyHostToDevice));
    } else {
        int s = 0;
        for (int z0 : z0s) {
            const int z1 = std::min(nz, z0 + sd);
            SlabPair* sp;
            int rc = get_pair(J, *p, std::min(nz, z1 + halo) - std::max(0, z0 - halo), net, k,
                              min_mass, &sp);
            if (rc) return rc;
            const int j = s++ & 1;
            cudaStream_t st = sp->d[j]->stream;
            CUDA_TRY(cudaMemcpyAsync(sp->stage[j], raw_host + z0 * J.plane, (z1 - z0) * J.plane * 4,
                                     cudaMemcpyHostToDevice, st));
            h2d += (z1 - z0) * J.plane * 4.0;
            rc = slab_patchstd(sp->stage[j], z0, z0, z1, st);
            if (rc) return rc;
        }
        int rc = sync_all();
        if (rc) return rc;
        rc = noise_em_finish(J.noise, p, nwin);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(J.d_sig0, J.noise->d_sigma, nz * 4, cudaMemcpyDeviceToDevice, J.main));
    }
    CUDA_TRY(cudaMemcpyAsync(J.d_sig, J.d_sig0, nz * 4, cudaMemcpyDeviceToDevice, J.main));
    CUDA_TRY(cudaMemcpyAsync(s0h.data(), J.d_sig0, nz * 4, cudaMemcpyDeviceToHost, J.main));
    CUDA_TRY(cudaStreamSynchronize(J.main));

    const int maxit = p->maxiterations;
    const float* prev_host = raw_host;
    for (int it = 1; it <= maxit; it++) {
        // the last iteration writes the caller's buffer
        float* next_host = ((maxit - it) % 2 == 0) ? out_host : J.tmp_host;
        const bool estimate = (it == 1 && maxit > 1) || (it > 1 && p->continuous_estimate && maxit > it + 1);
        int rc = stream_pass(J, *p, it, z0s, sd, halo, net, k, min_mass, raw_host, prev_host, next_host,
                             estimate && !manual, t0, &h2d, &d2h);
        if (rc) return rc;
        rc = sync_all();
        if (rc) return rc;
        for (auto& kv : J.pairs)
            for (int j = 0; j < 2; j++) {
                rc = check_device_error(kv.second.d[j]);
                if (rc) return rc;
            }
        if (estimate) {
            // sigma1 on this result, blended with sigma0 (main.cpp:422-448, 517-544)
            if (manual) {
                std::vector<float> v(nz, p->sigma[1]);
                CUDA_TRY(cudaMemcpy(J.d_sig, v.data(), nz * 4, cudaMemcpyHostToDevice));
            } else {
                rc = noise_em_finish(J.noise, p, nwin);
                if (rc) return rc;
                CUDA_TRY(cudaMemcpyAsync(J.d_sig, J.noise->d_sigma, nz * 4, cudaMemcpyDeviceToDevice,
                                         J.main));
            }
            if (it == 1) CUDA_TRY(cudaMemcpyAsync(s1h.data(), J.d_sig, nz * 4, cudaMemcpyDeviceToHost, J.main));
            CUDA_TRY(launch_sigma_blend(J.d_sig0, J.d_sig, p->alpha, nz, J.main));
            CUDA_TRY(cudaStreamSynchronize(J.main));
        }
        prev_host = next_host;
    }
    CUDA_TRY(cudaEventRecord(t1, J.main));
    CUDA_TRY(cudaEventSynchronize(t1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (sigma0_out) std::memcpy(sigma0_out, s0h.data(), nz * 4);
    if (sigma1_out && maxit > 1) std::memcpy(sigma1_out, s1h.data(), nz * 4);
    if (stats) {
        stats[0] = ms;
        stats[1] = h2d;
        stats[2] = d2h;
        stats[3] = (double)z0s.size();
        stats[4] = halo;
        stats[5] = sd;
    }
    return INLM_OK;
}

// ---------------- per-iteration engine on one device ----------------
//
// The same slab walk, one iteration per call, with the caller's sigma and the
// caller's buffers: what the host-RAM overload of
// IterativeNLM_GPU::Run_GaussianNoise_GPUBlocks (Denoiser/iternlm_gpu.cu:
// 1729-1886) does for each block of slices. The caller's volumes are
// page-locked for the duration of a call.
namespace {

struct HostPin {
    std::vector<void*> regs;
    void pin(const void* ptr, size_t bytes) {
        for (void* r : regs)
            if (r == ptr) return;
        if (cudaHostRegister(const_cast<void*>(ptr), bytes, cudaHostRegisterPortable) == cudaSuccess)
            regs.push_back(const_cast<void*>(ptr));
        else
            cudaGetLastError();  // already page-locked, or not registrable: copies still work
    }
    ~HostPin() {
        for (void* r : regs) cudaHostUnregister(r);
    }
};

struct StreamBlocks final : BlocksBackend {
    StreamJob J;
    inlm_params p;
    std::vector<int> z0s;
    int sd = 0, halo = 0;
    cudaEvent_t ready = nullptr;
    inlm_proposal* net = nullptr;
    int k = 0;
    float min_mass = 0.f;

    ~StreamBlocks() override {
        cudaSetDevice(p.device_id);
        for (auto& kv : J.pairs)
            for (int j = 0; j < 2; j++)
                if (kv.second.d[j]) cudaStreamSynchronize(kv.second.d[j]->stream);
        if (ready) cudaEventDestroy(ready);
    }
    int slab_depth() const override { return sd; }
    int proposal_schedule(int n, const int* ks, const float* rels) override {
        if (!net) return fail(INLM_ERR_STATE, "attach a proposal first");
        J.sched_k.assign(ks, ks + n);
        J.sched_rel.assign(rels, rels + n);
        for (auto& kv : J.pairs)
            for (int j = 0; j < 2; j++)
                if (kv.second.d[j]) {
                    int rc = inlm_proposal_schedule(kv.second.d[j], n, ks, rels);
                    if (rc) return rc;
                }
        return INLM_OK;
    }
    int attach_proposal(inlm_proposal* n, int kk, float mm, float rel, int tiles_x) override {
        if (net) return fail(INLM_ERR_STATE, "a proposal is attached already");
        if (p.precision == INLM_PRECISION_F32 || p.precision == INLM_PRECISION_F32_FMA)
            return fail(INLM_ERR_UNSUPPORTED, "the proposal drives the FP16 form");
        if (tiles_x != 1 && tiles_x != 4) return fail(INLM_ERR_ARG, "tiles_x must be 1 or 4");
        // the sub-volume denoisers are rebuilt with the proposal attached;
        // halos of >= 16 slices cover its receptive field
        for (auto& kv : J.pairs)
            for (int j = 0; j < 2; j++) {
                if (kv.second.d[j]) inlm_denoiser_destroy(kv.second.d[j]);
                device_free(kv.second.stage[j]);
            }
        J.pairs.clear();
        net = n;
        k = kk;
        min_mass = mm;
        J.tiles_x = tiles_x;
        J.rel_mass = rel;
        halo = std::max(halo, 16);
        const int nz = J.shape[2];
        for (int z0 : z0s) {
            const int z1 = std::min(nz, z0 + sd);
            SlabPair* sp;
            int rc = get_pair(J, p, std::min(nz, z1 + halo) - std::max(0, z0 - halo), net, k, min_mass, &sp);
            if (rc) return rc;
        }
        return INLM_OK;
    }
    int set_sigma(const float* sigma) override {
        CUDA_TRY(cudaSetDevice(p.device_id));
        CUDA_TRY(cudaMemcpyAsync(J.d_sig, sigma, J.shape[2] * 4, cudaMemcpyHostToDevice, J.main));
        CUDA_TRY(cudaEventRecord(ready, J.main));
        CUDA_TRY(cudaStreamSynchronize(J.main));
        return INLM_OK;
    }
    int iteration(int it, const float* raw, const float* prev, float* out) override {
        CUDA_TRY(cudaSetDevice(p.device_id));
        const size_t bytes = (size_t)J.plane * J.shape[2] * 4;
        HostPin pin;
        pin.pin(raw, bytes);
        if (it > 1) pin.pin(prev, bytes);
        pin.pin(out, bytes);
        double h2d = 0, d2h = 0;
        int rc = stream_pass(J, p, it, z0s, sd, halo, net, k, min_mass, raw, prev, out, false, ready, &h2d,
                             &d2h);
        // every slab's copies finish before the buffers are unpinned
        for (auto& kv : J.pairs)
            for (int j = 0; j < 2; j++) {
                cudaError_t e = cudaStreamSynchronize(kv.second.d[j]->stream);
                if (rc == INLM_OK && e != cudaSuccess) rc = fail(INLM_ERR_CUDA, "%s", cudaGetErrorString(e));
                if (rc == INLM_OK) rc = check_device_error(kv.second.d[j]);
            }
        return rc;
    }
};

}  // namespace

int inlm::make_stream_blocks(const int shape[3], const inlm_params* p, int slab_depth, BlocksBackend** out) {
    if (slab_depth < 1) return fail(INLM_ERR_ARG, "slab depth must be >= 1");
    CUDA_TRY(cudaSetDevice(p->device_id));
    auto* b = new StreamBlocks();
    std::unique_ptr<StreamBlocks> guard(b);
    b->p = *p;
    for (int i = 0; i < 3; i++) b->J.shape[i] = shape[i];
    b->J.plane = (long long)shape[0] * shape[1];
    const int nz = shape[2];
    const int pz = std::min(p->nslices / 2, p->search_radius[2]) + p->patch_radius[2];
    b->halo = round_up8(std::max(pz, 1));
    b->sd = round_up8(slab_depth);
    for (int z = 0; z < nz; z += b->sd) b->z0s.push_back(z);
    CUDA_TRY(cudaStreamCreateWithFlags(&b->J.main, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&b->ready, cudaEventDisableTiming));
    CUDA_TRY(dalloc(&b->J.d_sig0, nz));
    CUDA_TRY(dalloc(&b->J.d_sig, nz));
    // the denoisers of every sub-volume depth, created now so that a device
    // too small for them fails here rather than in the first iteration
    for (int z0 : b->z0s) {
        const int z1 = std::min(nz, z0 + b->sd);
        SlabPair* sp;
        int rc = get_pair(b->J, *p, std::min(nz, z1 + b->halo) - std::max(0, z0 - b->halo), nullptr, 0, 0.f,
                          &sp);
        if (rc) return rc;
    }
    *out = guard.release();
    return INLM_OK;
}
