// C ABI of the per-iteration engine over host-resident volumes (include/inlm.h,
// inlm_blocks_*): the host-RAM overload of
// IterativeNLM_GPU::Run_GaussianNoise_GPUBlocks (Denoiser/iternlm_gpu.h:31,
// Denoiser/iternlm_gpu.cu:1729-1886), which the reference driver calls once
// per iteration when the stack does not fit one GPU or runs on several
// (main.cpp:379, 472). One device: z-slab streaming (api_stream.cu); several:
// the stack split over them (api_multi.cu).
#include <memory>

#include "api_internal.hpp"

using namespace inlm;

extern "C" int inlm_blocks_create(const int shape[3], const inlm_params* p, int n_devices,
                                  const int* device_ids, int slab_depth, inlm_blocks** out) {
    if (!shape || !p || !out) return fail(INLM_ERR_ARG, "null argument");
    *out = nullptr;
    for (int i = 0; i < 3; i++)
        if (shape[i] < 1) return fail(INLM_ERR_ARG, "empty shape");
    if (n_devices < 1) return fail(INLM_ERR_ARG, "n_devices must be >= 1");
    if (p->maxiterations < 1) return fail(INLM_ERR_ARG, "maxiterations < 1");
    auto b = std::make_unique<inlm_blocks>();
    for (int i = 0; i < 3; i++) b->shape[i] = shape[i];
    int rc;
    if (n_devices == 1) {
        inlm_params q = *p;
        if (device_ids) q.device_id = device_ids[0];
        rc = make_stream_blocks(shape, &q, slab_depth, &b->be);
    } else {
        if (!device_ids) return fail(INLM_ERR_ARG, "device_ids needed for several devices");
        rc = make_multi_blocks(shape, p, n_devices, device_ids, &b->be);
    }
    if (rc) return rc;
    *out = b.release();
    return INLM_OK;
}

extern "C" int inlm_blocks_destroy(inlm_blocks* b) {
    delete b;
    return INLM_OK;
}

extern "C" int inlm_blocks_slab_depth(const inlm_blocks* b, int* depth) {
    if (!b || !depth) return fail(INLM_ERR_ARG, "null argument");
    *depth = b->be->slab_depth();
    return INLM_OK;
}

extern "C" int inlm_blocks_attach_proposal(inlm_blocks* b, inlm_proposal* net, int k, float min_mass,
                                           float rel_mass, int tiles_x) {
    if (!b || !net) return fail(INLM_ERR_ARG, "null argument");
    if (k < 1) return fail(INLM_ERR_ARG, "k must be >= 1");
    if (!(rel_mass >= 0.f && rel_mass <= 1.f)) return fail(INLM_ERR_ARG, "rel_mass must be in 0..1");
    if (b->last_iter > 0) return fail(INLM_ERR_STATE, "attach the proposal before the first iteration");
    return b->be->attach_proposal(net, k, min_mass, rel_mass, tiles_x);
}

extern "C" int inlm_blocks_proposal_schedule(inlm_blocks* b, int n, const int* k, const float* rel_mass) {
    if (!b) return fail(INLM_ERR_ARG, "null handle");
    if (n < 0 || n > 1024) return fail(INLM_ERR_ARG, "schedule length must be in 0..1024");
    if (n > 0 && (!k || !rel_mass)) return fail(INLM_ERR_ARG, "null schedule");
    for (int i = 0; i < n; i++) {
        if (k[i] < 0) return fail(INLM_ERR_ARG, "schedule k must be >= 0 (0: full search)");
        if (!(rel_mass[i] >= 0.f && rel_mass[i] <= 1.f))
            return fail(INLM_ERR_ARG, "schedule rel_mass must be in 0..1");
    }
    if (b->last_iter > 0) return fail(INLM_ERR_STATE, "set the schedule before the first iteration");
    return b->be->proposal_schedule(n, k, rel_mass);
}

extern "C" int inlm_blocks_set_sigma(inlm_blocks* b, const float* sigma_host) {
    if (!b || !sigma_host) return fail(INLM_ERR_ARG, "null argument");
    int rc = b->be->set_sigma(sigma_host);
    if (rc) return rc;
    b->sigma_set = true;
    return INLM_OK;
}

extern "C" int inlm_blocks_run_iteration(inlm_blocks* b, int iter, const float* raw_host,
                                         const float* prev_host, float* out_host) {
    if (!b || !raw_host || !out_host) return fail(INLM_ERR_ARG, "null argument");
    if (iter < 1) return fail(INLM_ERR_ARG, "iteration must be >= 1");
    if (!b->sigma_set) return fail(INLM_ERR_STATE, "set sigma before the first iteration");
    if (iter > 1) {
        if (!prev_host) return fail(INLM_ERR_ARG, "iteration %d needs the previous iterate", iter);
        if (prev_host == out_host) return fail(INLM_ERR_ARG, "prev_host and out_host must be distinct");
    }
    int rc = b->be->iteration(iter, raw_host, prev_host, out_host);
    if (rc) return rc;
    b->last_iter = iter;
    return INLM_OK;
}
