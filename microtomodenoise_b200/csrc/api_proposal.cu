// C ABI of the learned search-offset proposal (include/inlm.h). The reference
// has no counterpart: its filter always evaluates every search offset
// (Denoiser/iternlm_cpu.cpp:758-843). The proposal only changes which offsets
// a tile of the FP16 form evaluates; the arithmetic per offset is unchanged.
#include "api_internal.hpp"

using namespace inlm;

static cudaError_t prop_levels_alloc(DevBuf* a1, DevBuf* a2, DevBuf* a3, DevBuf* a4, int nx, int ny,
                                     int nz) {
    Dim3i lv[4];
    net_levels(nx, ny, nz, lv);
    auto bytes = [](Dim3i d) { return (size_t)d.x * d.y * d.z * kNetC * sizeof(float); };
    cudaError_t e;
    if ((e = a1->ensure(bytes(lv[1]))) != cudaSuccess) return e;
    if ((e = a2->ensure(bytes(lv[2]))) != cudaSuccess) return e;
    if ((e = a3->ensure(bytes(lv[3]))) != cudaSuccess) return e;
    return a4->ensure(bytes(lv[3]));
}

static void proposal_free(inlm_proposal* p) {
    if (!p) return;
    cudaSetDevice(p->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    device_free(p->d_w);
    device_free(p->d_m);
    device_free(p->d_v);
    device_free(p->d_g);
    device_free(p->d_wb);
    device_free(p->d_loss);
    device_free(p->d_err);
    for (DevBuf* b : {&p->pad, &p->a1, &p->a2, &p->a3, &p->a4, &p->glog, &p->d1, &p->d2, &p->d3,
                      &p->d4, &p->counters})
        b->release();
    if (p->stream) cudaStreamDestroy(p->stream);
}

extern "C" int inlm_proposal_create(int n_offsets, int device_id, inlm_proposal** out) {
    if (!out) return fail(INLM_ERR_ARG, "null argument");
    *out = nullptr;
    if (n_offsets < 1 || n_offsets > 65535) return fail(INLM_ERR_ARG, "n_offsets must be 1..65535");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return fail(INLM_ERR_NODEVICE, "no CUDA device");
    if (device_id < 0 || device_id >= ndev) return fail(INLM_ERR_ARG, "bad device id");
    inlm_proposal* p = new inlm_proposal();
    p->device = device_id;
    p->L = net_layout(n_offsets);
    cudaSetDevice(device_id);
    const long long n = p->L.total;
    if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess ||
        dalloc(&p->d_w, n) != cudaSuccess || dalloc(&p->d_m, n) != cudaSuccess ||
        dalloc(&p->d_v, n) != cudaSuccess || dalloc(&p->d_g, n) != cudaSuccess ||
        dalloc(&p->d_wb, n) != cudaSuccess || dalloc(&p->d_loss, 1) != cudaSuccess ||
        dalloc(&p->d_err, 1) != cudaSuccess || cudaMemset(p->d_err, 0, 4) != cudaSuccess ||
        cudaMemset(p->d_w, 0, n * 4) != cudaSuccess || cudaMemset(p->d_m, 0, n * 4) != cudaSuccess ||
        cudaMemset(p->d_v, 0, n * 4) != cudaSuccess || cudaMemset(p->d_wb, 0, n * 2) != cudaSuccess) {
        proposal_free(p);
        delete p;
        return fail(INLM_ERR_NOMEM, "proposal allocation failed");
    }
    *out = p;
    return INLM_OK;
}

extern "C" int inlm_proposal_destroy(inlm_proposal* p) {
    proposal_free(p);
    delete p;
    return INLM_OK;
}

extern "C" int inlm_proposal_n_params(const inlm_proposal* p, int64_t* n) {
    if (!p || !n) return fail(INLM_ERR_ARG, "null argument");
    *n = p->L.total;
    return INLM_OK;
}

extern "C" int inlm_proposal_set_params(inlm_proposal* p, const float* params, int64_t n) {
    if (!p || !params) return fail(INLM_ERR_ARG, "null argument");
    if (n != p->L.total) return fail(INLM_ERR_ARG, "expected %lld parameters", p->L.total);
    CUDA_TRY(cudaSetDevice(p->device));
    CUDA_TRY(cudaMemcpyAsync(p->d_w, params, n * 4, cudaMemcpyHostToDevice, p->stream));
    CUDA_TRY(cudaMemsetAsync(p->d_m, 0, n * 4, p->stream));
    CUDA_TRY(cudaMemsetAsync(p->d_v, 0, n * 4, p->stream));
    CUDA_TRY(net_round_bf16(p->d_w, p->d_wb, n, p->stream));
    CUDA_TRY(cudaStreamSynchronize(p->stream));
    p->step = 0;
    return INLM_OK;
}

extern "C" int inlm_proposal_get_params(inlm_proposal* p, float* params, int64_t n) {
    if (!p || !params) return fail(INLM_ERR_ARG, "null argument");
    if (n != p->L.total) return fail(INLM_ERR_ARG, "expected %lld parameters", p->L.total);
    CUDA_TRY(cudaSetDevice(p->device));
    CUDA_TRY(cudaMemcpyAsync(params, p->d_w, n * 4, cudaMemcpyDeviceToHost, p->stream));
    CUDA_TRY(cudaStreamSynchronize(p->stream));
    return INLM_OK;
}

// The tensor-core layers' bounded waits report through p->d_err.
static int proposal_check_error(inlm_proposal* p) {
    int h = 0;
    CUDA_TRY(cudaMemcpyAsync(&h, p->d_err, 4, cudaMemcpyDeviceToHost, p->stream));
    CUDA_TRY(cudaStreamSynchronize(p->stream));
    if (h != 0) {
        cudaMemsetAsync(p->d_err, 0, 4, p->stream);
        return fail(INLM_ERR_TIMEOUT, "device wait gave up (code %d)", h);
    }
    return INLM_OK;
}

extern "C" int inlm_proposal_set_tensor_cores(inlm_proposal* p, int mode) {
    if (!p) return fail(INLM_ERR_ARG, "null handle");
    if (mode < 0 || mode > 3) return fail(INLM_ERR_ARG, "mode must be 0..3");
    p->tc = (mode & 1) != 0;
    p->train_tc = (mode & 2) != 0;
    return INLM_OK;
}

static int check_shape(const int shape[3]) {
    if (!shape) return fail(INLM_ERR_ARG, "null shape");
    for (int i = 0; i < 3; i++)
        if (shape[i] < 2) return fail(INLM_ERR_ARG, "every axis needs at least 2 voxels");
    return INLM_OK;
}

// Pads an unpadded FP32 example by one voxel (reflective) into p->pad.
static int example_input(inlm_proposal* p, const float* vol, const float* scale, const int shape[3],
                         NetIn* in) {
    const int nx = shape[0], ny = shape[1], nz = shape[2];
    const long long py = nx + 2, pz = py * (ny + 2);
    CUDA_TRY(p->pad.ensure((size_t)pz * (nz + 2) * 4));
    CUDA_TRY(launch_pad_reflective(vol, nx, ny, nz, p->pad.as<float>(), 1, 1, 1, py, pz, p->stream));
    in->base = p->pad.as<float>() + pz + py + 1;
    in->half = false;
    in->py = py;
    in->pz = pz;
    in->nx = nx;
    in->ny = ny;
    in->nz = nz;
    in->scale = scale;
    return INLM_OK;
}

static NetActs prop_acts(inlm_proposal* p) {
    return NetActs{p->a1.as<float>(), p->a2.as<float>(), p->a3.as<float>(), p->a4.as<float>()};
}

extern "C" int inlm_proposal_logits(inlm_proposal* p, const float* vol, const float* scale,
                                    const int shape[3], float* logits) {
    if (!p || !vol || !scale || !logits) return fail(INLM_ERR_ARG, "null argument");
    int rc = check_shape(shape);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(p->device));
    NetIn in;
    rc = example_input(p, vol, scale, shape, &in);
    if (rc) return rc;
    CUDA_TRY(prop_levels_alloc(&p->a1, &p->a2, &p->a3, &p->a4, shape[0], shape[1], shape[2]));
    CUDA_TRY(net_forward(p->L, p->d_wb, p->d_w, in, prop_acts(p), p->stream, NetTc{p->tc, p->d_err}));
    Dim3i lv[4];
    net_levels(shape[0], shape[1], shape[2], lv);
    CUDA_TRY(net_logits(p->L, p->d_wb, p->d_w, p->a4.as<float>(), lv[3].x * lv[3].y * lv[3].z, logits,
                        p->stream));
    return proposal_check_error(p);
}

extern "C" int inlm_proposal_train(inlm_proposal* p, int n_examples, const float* const* vols,
                                   const float* const* scales, const float* const* targets,
                                   const int* shapes, float lr, double* loss_out, float* grad_host) {
    if (!p || n_examples < 1 || !vols || !scales || !targets || !shapes)
        return fail(INLM_ERR_ARG, "null argument");
    for (int e = 0; e < n_examples; e++) {
        int rc = check_shape(shapes + 3 * e);
        if (rc) return rc;
        if (!vols[e] || !scales[e] || !targets[e]) return fail(INLM_ERR_ARG, "null example %d", e);
    }
    CUDA_TRY(cudaSetDevice(p->device));
    long long total_tiles = 0;
    for (int e = 0; e < n_examples; e++) {
        Dim3i lv[4];
        net_levels(shapes[3 * e], shapes[3 * e + 1], shapes[3 * e + 2], lv);
        total_tiles += (long long)lv[3].x * lv[3].y * lv[3].z;
    }
    const float inv_n = (float)(1.0 / (double)total_tiles);
    const long long np = p->L.total;
    CUDA_TRY(cudaMemsetAsync(p->d_g, 0, np * 4, p->stream));
    CUDA_TRY(cudaMemsetAsync(p->d_loss, 0, 8, p->stream));
    for (int e = 0; e < n_examples; e++) {
        const int* sh = shapes + 3 * e;
        NetIn in;
        int rc = example_input(p, vols[e], scales[e], sh, &in);
        if (rc) return rc;
        CUDA_TRY(prop_levels_alloc(&p->a1, &p->a2, &p->a3, &p->a4, sh[0], sh[1], sh[2]));
        CUDA_TRY(prop_levels_alloc(&p->d1, &p->d2, &p->d3, &p->d4, sh[0], sh[1], sh[2]));
        Dim3i lv[4];
        net_levels(sh[0], sh[1], sh[2], lv);
        const long long nt = (long long)lv[3].x * lv[3].y * lv[3].z;
        CUDA_TRY(p->glog.ensure((size_t)nt * p->L.S * 4));
        const NetTc ttc{p->train_tc, p->d_err};
        CUDA_TRY(net_forward(p->L, p->d_wb, p->d_w, in, prop_acts(p), p->stream, ttc));
        NetGradScratch gs{p->glog.as<float>(), p->d1.as<float>(), p->d2.as<float>(),
                          p->d3.as<float>(), p->d4.as<float>()};
        CUDA_TRY(net_backward(p->L, p->d_wb, p->d_w, in, prop_acts(p), targets[e], inv_n, gs, p->d_g,
                              p->d_loss, p->stream, ttc));
    }
    if (grad_host) {
        CUDA_TRY(cudaMemcpyAsync(grad_host, p->d_g, np * 4, cudaMemcpyDeviceToHost, p->stream));
    } else {
        p->step++;
        const float b1 = 0.9f, b2 = 0.999f;
        const float bc1 = (float)(1.0 - std::pow((double)b1, (double)p->step));
        const float bc2 = (float)(1.0 - std::pow((double)b2, (double)p->step));
        CUDA_TRY(net_adam(p->d_w, p->d_m, p->d_v, p->d_g, p->d_wb, np, lr, b1, b2, 1e-8f, bc1, bc2,
                          p->stream));
    }
    double loss = 0.0;
    CUDA_TRY(cudaMemcpyAsync(&loss, p->d_loss, 8, cudaMemcpyDeviceToHost, p->stream));
    CUDA_TRY(cudaStreamSynchronize(p->stream));
    if (loss_out) *loss_out = loss;
    return proposal_check_error(p);
}

extern "C" int inlm_proposal_select(inlm_proposal* p, const float* vol, const float* scale,
                                    const int shape[3], int k, float min_mass, uint32_t* bitmap,
                                    float* pred_mass, int* n_fallback) {
    if (!p || !vol || !scale || !bitmap || !pred_mass) return fail(INLM_ERR_ARG, "null argument");
    if (k < 1) return fail(INLM_ERR_ARG, "k must be >= 1");
    int rc = check_shape(shape);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(p->device));
    NetIn in;
    rc = example_input(p, vol, scale, shape, &in);
    if (rc) return rc;
    CUDA_TRY(prop_levels_alloc(&p->a1, &p->a2, &p->a3, &p->a4, shape[0], shape[1], shape[2]));
    CUDA_TRY(p->counters.ensure(16));
    CUDA_TRY(cudaMemsetAsync(p->counters.p, 0, 16, p->stream));
    CUDA_TRY(net_forward(p->L, p->d_wb, p->d_w, in, prop_acts(p), p->stream, NetTc{p->tc, p->d_err}));
    Dim3i lv[4];
    net_levels(shape[0], shape[1], shape[2], lv);
    const int nt = lv[3].x * lv[3].y * lv[3].z;
    const int nwords = (p->L.S + 31) / 32;
    CUDA_TRY(net_select(p->L, p->d_wb, p->d_w, p->a4.as<float>(), nt, k, min_mass, bitmap, nwords,
                        pred_mass, p->counters.as<int>(), p->stream));
    int cnt[4] = {0, 0, 0, 0};
    CUDA_TRY(cudaMemcpyAsync(cnt, p->counters.p, 16, cudaMemcpyDeviceToHost, p->stream));
    CUDA_TRY(cudaStreamSynchronize(p->stream));
    if (n_fallback) *n_fallback = cnt[0];
    return proposal_check_error(p);
}

extern "C" int inlm_proposal_select_grouped(inlm_proposal* p, const float* vol, const float* scale,
                                            const int shape[3], int tiles_x, int k, float min_mass,
                                            uint32_t* bitmap, float* pred_mass, int* n_fallback) {
    if (tiles_x == 1) return inlm_proposal_select(p, vol, scale, shape, k, min_mass, bitmap, pred_mass, n_fallback);
    if (!p || !vol || !scale || !bitmap || !pred_mass) return fail(INLM_ERR_ARG, "null argument");
    if (k < 1 || tiles_x < 1) return fail(INLM_ERR_ARG, "k and tiles_x must be >= 1");
    int rc = check_shape(shape);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(p->device));
    NetIn in;
    rc = example_input(p, vol, scale, shape, &in);
    if (rc) return rc;
    CUDA_TRY(prop_levels_alloc(&p->a1, &p->a2, &p->a3, &p->a4, shape[0], shape[1], shape[2]));
    CUDA_TRY(p->counters.ensure(16));
    CUDA_TRY(cudaMemsetAsync(p->counters.p, 0, 16, p->stream));
    CUDA_TRY(net_forward(p->L, p->d_wb, p->d_w, in, prop_acts(p), p->stream, NetTc{p->tc, p->d_err}));
    Dim3i lv[4];
    net_levels(shape[0], shape[1], shape[2], lv);
    CUDA_TRY(net_select_group(p->L, p->d_wb, p->d_w, p->a4.as<float>(), lv[3], tiles_x, k, min_mass, bitmap,
                              (p->L.S + 31) / 32, pred_mass, p->counters.as<int>(), p->stream));
    int cnt[4] = {0, 0, 0, 0};
    CUDA_TRY(cudaMemcpyAsync(cnt, p->counters.p, 16, cudaMemcpyDeviceToHost, p->stream));
    CUDA_TRY(cudaStreamSynchronize(p->stream));
    if (n_fallback) *n_fallback = cnt[0];
    return proposal_check_error(p);
}

// ---------------- denoiser side ----------------

void inlm::proposal_release(inlm_denoiser* d) {
    ProposalRun& r = d->prop;
    for (DevBuf* b : {&r.a1, &r.a2, &r.a3, &r.a4, &r.bitmap, &r.pmass, &r.counters, &r.scale,
                      &r.plan_start, &r.plan_off, &r.mass_sum})
        b->release();
    r.net = nullptr;
}

extern "C" int inlm_attach_proposal(inlm_denoiser* d, inlm_proposal* p, int k, float min_mass) {
    return inlm_attach_proposal_grouped(d, p, k, min_mass, 1);
}

extern "C" int inlm_attach_proposal_grouped(inlm_denoiser* d, inlm_proposal* p, int k, float min_mass,
                                            int tiles_x) {
    return inlm_attach_proposal_ex(d, p, k, min_mass, 0.f, tiles_x);
}

extern "C" int inlm_attach_proposal_ex(inlm_denoiser* d, inlm_proposal* p, int k, float min_mass,
                                       float rel_mass, int tiles_x) {
    if (!d) return fail(INLM_ERR_ARG, "null handle");
    CUDA_TRY(cudaSetDevice(d->device));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    if (!p) {
        if (d->prop.net) {
            d->plan_active = false;
            d->plan_cta32 = false;
            d->fargs8.plan_start = nullptr;
            d->fargs8.plan_count = nullptr;
            d->fargs8.plan_offsets = nullptr;
        }
        proposal_release(d);
        return INLM_OK;
    }
    if (tiles_x != 1 && tiles_x != 4) return fail(INLM_ERR_ARG, "tiles_x must be 1 or 4");
    if (tiles_x == 4 && (d->fcfg.tx != 32 || d->fcfg.tz != 8))
        return fail(INLM_ERR_UNSUPPORTED, "no 32 x 8 x 8 FP16 kernel for this patch shape");
    if (!d->use_fast || !d->use_tile8)
        return fail(INLM_ERR_UNSUPPORTED, "the proposal drives the FP16 form only");
    if (d->plan_active && !d->prop.net)
        return fail(INLM_ERR_STATE, "an offset plan is set; clear it first");
    if (p->device != d->device) return fail(INLM_ERR_ARG, "proposal and denoiser on different devices");
    if (p->L.S != d->fargs.S)
        return fail(INLM_ERR_ARG, "proposal trained for %d offsets, the denoiser searches %d", p->L.S,
                    d->fargs.S);
    if (k < 1) return fail(INLM_ERR_ARG, "k must be >= 1");
    if (!(rel_mass >= 0.f && rel_mass <= 1.f)) return fail(INLM_ERR_ARG, "rel_mass must be in 0..1");
    ProposalRun& r = d->prop;
    r.k = k;
    r.min_mass = min_mass;
    r.rel_mass = rel_mass;
    r.nwords = (p->L.S + 31) / 32;
    Dim3i lv[4];
    net_levels(d->shape[0], d->shape[1], d->shape[2], lv);
    r.t8 = lv[3];
    r.n_tiles = (long long)lv[3].x * lv[3].y * lv[3].z;
    r.group = tiles_x;
    // one plan list per 8^3 tile (a CTA of the tx = 8 configuration) or per
    // group of 4 tiles along x (a CTA of the tx = 32 configuration)
    r.n_plan = (long long)((lv[3].x + tiles_x - 1) / tiles_x) * lv[3].y * lv[3].z;
    const long long n = r.n_plan;
    CUDA_TRY(prop_levels_alloc(&r.a1, &r.a2, &r.a3, &r.a4, d->shape[0], d->shape[1], d->shape[2]));
    CUDA_TRY(r.bitmap.ensure((size_t)n * r.nwords * 4));
    CUDA_TRY(r.pmass.ensure((size_t)n * 4));
    CUDA_TRY(r.counters.ensure(16));
    CUDA_TRY(r.scale.ensure((size_t)d->shape[2] * 4));
    CUDA_TRY(r.plan_start.ensure((size_t)2 * n * 4));
    CUDA_TRY(r.plan_off.ensure((size_t)n * p->L.S * 4));
    CUDA_TRY(r.mass_sum.ensure(8));
    if ((long long)n * p->L.S >= (1ll << 31))
        return fail(INLM_ERR_ARG, "volume too large for one plan table; stream it in z-slabs");
    std::vector<int> st(n);
    for (long long c = 0; c < n; c++) st[c] = (int)(c * p->L.S);
    CUDA_TRY(cudaMemcpyAsync(r.plan_start.p, st.data(), (size_t)n * 4, cudaMemcpyHostToDevice,
                             d->stream));
    CUDA_TRY(cudaMemsetAsync(r.counters.p, 0, 16, d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    r.net = p;
    return INLM_OK;
}

void inlm::proposal_step(const ProposalRun& r, int iter, int* k, float* rel_mass) {
    if (r.sched_k.empty()) {
        *k = r.k;
        *rel_mass = r.rel_mass;
        return;
    }
    const size_t i = (size_t)std::max(1, std::min(iter, (int)r.sched_k.size())) - 1;
    *k = r.sched_k[i];
    *rel_mass = r.sched_rel[i];
}

extern "C" int inlm_proposal_schedule(inlm_denoiser* d, int n, const int* k, const float* rel_mass) {
    if (!d) return fail(INLM_ERR_ARG, "null handle");
    if (!d->prop.net) return fail(INLM_ERR_STATE, "attach a proposal first");
    if (n < 0 || n > 1024) return fail(INLM_ERR_ARG, "schedule length must be in 0..1024");
    if (n > 0 && (!k || !rel_mass)) return fail(INLM_ERR_ARG, "null schedule");
    for (int i = 0; i < n; i++) {
        if (k[i] < 0) return fail(INLM_ERR_ARG, "schedule k must be >= 0 (0: full search)");
        if (!(rel_mass[i] >= 0.f && rel_mass[i] <= 1.f))
            return fail(INLM_ERR_ARG, "schedule rel_mass must be in 0..1");
    }
    CUDA_TRY(cudaSetDevice(d->device));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    d->prop.sched_k.assign(k, k + n);
    d->prop.sched_rel.assign(rel_mass, rel_mass + n);
    return INLM_OK;
}

int inlm::proposal_prepare_iteration(inlm_denoiser* d, int iter) {
    int k = 0;
    float rel = 0.f;
    proposal_step(d->prop, iter, &k, &rel);
    if (k > 0) return proposal_enqueue(d, iter);
    // this iteration of the schedule searches every offset
    d->plan_active = false;
    d->plan_cta32 = false;
    return INLM_OK;
}

int inlm::proposal_enqueue(inlm_denoiser* d, int iter) {
    ProposalRun& r = d->prop;
    inlm_proposal* p = r.net;
    int k = r.k;
    float rel = r.rel_mass;
    proposal_step(r, iter, &k, &rel);
    if (k < 1) return fail(INLM_ERR_STATE, "iteration %d runs the full search", iter);
    const Geometry& g = d->geo;
    CUDA_TRY(net_scale_from_mult(d->d_mult, d->shape[2], r.scale.as<float>(), d->stream));
    NetIn in;
    in.base = static_cast<const __half*>(d->d_prev_h) + g.pad[2] * d->pitch_z + g.pad[1] * d->pitch_y +
              g.pad[0];
    in.half = true;
    in.py = d->pitch_y;
    in.pz = d->pitch_z;
    in.nx = d->shape[0];
    in.ny = d->shape[1];
    in.nz = d->shape[2];
    in.scale = r.scale.as<float>();
    NetActs act{r.a1.as<float>(), r.a2.as<float>(), r.a3.as<float>(), r.a4.as<float>()};
    CUDA_TRY(net_forward(p->L, p->d_wb, p->d_w, in, act, d->stream, NetTc{p->tc, d->d_err}));
    CUDA_TRY(cudaMemsetAsync(r.counters.p, 0, 16, d->stream));
    if (r.group == 1)
        CUDA_TRY(net_select(p->L, p->d_wb, p->d_w, act.a4, (int)r.n_tiles, k, r.min_mass,
                            r.bitmap.as<unsigned>(), r.nwords, r.pmass.as<float>(), r.counters.as<int>(),
                            d->stream));
    else
        CUDA_TRY(net_select_group(p->L, p->d_wb, p->d_w, act.a4, r.t8, r.group, k, r.min_mass,
                                  r.bitmap.as<unsigned>(), r.nwords, r.pmass.as<float>(),
                                  r.counters.as<int>(), d->stream));
    int* ps = r.plan_start.as<int>();
    CUDA_TRY(net_plan_tiles(r.bitmap.as<unsigned>(), r.nwords, r.n_plan, p->L.S,
                            r.plan_off.as<int>(), ps + r.n_plan, r.counters.as<int>(), d->stream,
                            r.pmass.as<float>(), r.mass_sum.as<double>(), rel));
    d->launches += rel > 0.f ? 8 : 7;  // scale, 4 layers, select, (mass sum,) plan
    if (r.group == 1) {
        d->fargs8.plan_start = ps;
        d->fargs8.plan_count = ps + r.n_plan;
        d->fargs8.plan_offsets = r.plan_off.as<int>();
        d->plan_cta32 = false;
    } else {
        d->fargs_plan = d->fargs;
        d->fargs_plan.plan_start = ps;
        d->fargs_plan.plan_count = ps + r.n_plan;
        d->fargs_plan.plan_offsets = r.plan_off.as<int>();
        d->plan_cta32 = true;
    }
    d->plan_active = true;
    return INLM_OK;
}

extern "C" int inlm_proposal_stats(inlm_denoiser* d, int64_t stats[5]) {
    if (!d || !stats) return fail(INLM_ERR_ARG, "null argument");
    if (!d->prop.net) return fail(INLM_ERR_STATE, "no proposal attached");
    CUDA_TRY(cudaSetDevice(d->device));
    int cnt[4] = {0, 0, 0, 0};
    CUDA_TRY(cudaMemcpyAsync(cnt, d->prop.counters.p, 16, cudaMemcpyDeviceToHost, d->stream));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    stats[0] = d->prop.n_plan;
    stats[1] = cnt[0];
    stats[2] = cnt[1];
    stats[3] = (int64_t)d->prop.n_plan * d->fargs.S;
    stats[4] = d->fargs.S;
    return INLM_OK;
}

extern "C" int inlm_weight_map(inlm_denoiser* d, float* map) {
    if (!d || !map) return fail(INLM_ERR_ARG, "null argument");
    if (!d->use_fast) return fail(INLM_ERR_UNSUPPORTED, "weight maps come from the FP16 form");
    if (d->last_iter < 1) return fail(INLM_ERR_STATE, "no iteration has run");
    CUDA_TRY(cudaSetDevice(d->device));
    const long long nvox = (long long)d->shape[0] * d->shape[1] * d->shape[2];
    CUDA_TRY(d->aux.ensure((size_t)nvox * 4));
    Dim3i lv[4];
    net_levels(d->shape[0], d->shape[1], d->shape[2], lv);
    const long long nt = (long long)lv[3].x * lv[3].y * lv[3].z;
    const int S = d->fargs.S;
    FastArgs a = d->fargs;  // full search over the last iteration's inputs
    a.plan_start = nullptr;
    a.plan_count = nullptr;
    a.plan_offsets = nullptr;
    a.aux = d->aux.as<float>();
    a.map = map;
    a.t8x = lv[3].x;
    a.t8y = lv[3].y;
    const int tiles_z = (d->shape[2] + d->fcfg.tz - 1) / d->fcfg.tz;
    CUDA_TRY(launch_fast_kernel(d->fcfg, &d->tm_prev_h, a, tiles_z, d->stream, false));
    CUDA_TRY(cudaMemsetAsync(map, 0, (size_t)nt * S * 4, d->stream));
    CUDA_TRY(launch_fast_kernel(d->fcfg, &d->tm_prev_h, a, tiles_z, d->stream, true));
    CUDA_TRY(normalise_rows(map, nt, S, d->stream));
    d->launches += 3;
    return check_device_error(d);
}

extern "C" int inlm_net_input(inlm_denoiser* d, float* vol, float* scale) {
    if (!d || !vol || !scale) return fail(INLM_ERR_ARG, "null argument");
    if (!d->use_fast) return fail(INLM_ERR_UNSUPPORTED, "the proposal reads the FP16 form");
    if (d->last_iter < 1) return fail(INLM_ERR_STATE, "no iteration has run");
    CUDA_TRY(cudaSetDevice(d->device));
    const Geometry& g = d->geo;
    CUDA_TRY(unpad_half_to_float(d->d_prev_h, d->pitch_y, d->pitch_z, g.pad[0], g.pad[1], g.pad[2],
                                 d->shape[0], d->shape[1], d->shape[2], vol, d->stream));
    CUDA_TRY(net_scale_from_mult(d->d_mult, d->shape[2], scale, d->stream));
    d->launches += 2;
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    return INLM_OK;
}
