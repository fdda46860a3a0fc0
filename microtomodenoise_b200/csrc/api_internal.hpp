// Internal state of the C ABI handles, shared by the translation units that
// implement include/inlm.h (api.cu, api_proposal.cu).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/inlm.h"
#include "filter_fast.cuh"
#include "filter_kernels.cuh"
#include "geometry.hpp"
#include "proposal.cuh"

namespace inlm {

// Records the calling thread's error text (inlm_last_error) and returns code.
int fail(int code, const char* fmt, ...);

// Every device allocation and release of the library goes through these two:
// they keep the live-allocation count and carry the allocation-failure
// injection of the tests (inlm_debug_fail_allocation). device_free(NULL) is a
// no-op.
cudaError_t device_malloc(void** p, size_t bytes);
cudaError_t device_free(void* p);

template <typename T>
static inline cudaError_t dalloc(T** p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    return device_malloc((void**)p, n * sizeof(T));
}

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        device_free(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = device_malloc(&p, n ? n : 1);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    void release() {
        device_free(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

struct TimedLaunch {
    cudaEvent_t a, b;
};

}  // namespace inlm

#define CUDA_TRY(expr)                                                                         \
    do {                                                                                       \
        cudaError_t _e = (expr);                                                               \
        if (_e != cudaSuccess) {                                                               \
            int _code = (_e == cudaErrorMemoryAllocation) ? INLM_ERR_NOMEM : INLM_ERR_CUDA;    \
            return inlm::fail(_code, "%s: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__, \
                              __LINE__);                                                       \
        }                                                                                      \
    } while (0)

struct inlm_noise {
    int shape[3] = {0, 0, 0};
    uint64_t n_samples = 0;
    int patchsize = 15;
    unsigned int seed = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int mask_drawn = -1;
    std::vector<long long> samples;
    long long* d_samples = nullptr;
    float* d_patchstd = nullptr;
    float* d_stack = nullptr;  // staging for host stacks
    int stack_slices = 0;      // slices d_stack holds: nz, or a slab when the stack does not fit
    int zwindow_cached = -1;
    int2* d_windows = nullptr;
    long long* d_scratch_off = nullptr;
    signed char* d_assign = nullptr;
    size_t assign_cap = 0;
    float* d_mean = nullptr;
    float* d_sd = nullptr;
    float* d_sigma = nullptr;
    int ncalls = 0;
    long long ref_sample_semimanual = 0;
    long long mean_window = 0;  // average samples per EM window (picks the EM's CTA size)
};

// Proposal network: FP32 master parameters, BF16 copy, Adam state, training
// scratch.
struct inlm_proposal {
    int device = 0;
    inlm::NetLayout L;
    cudaStream_t stream = nullptr;
    float* d_w = nullptr;
    float* d_m = nullptr;
    float* d_v = nullptr;
    float* d_g = nullptr;
    __nv_bfloat16* d_wb = nullptr;
    double* d_loss = nullptr;
    int* d_err = nullptr;  // device error word of the tensor-core layers' bounded waits
    bool tc = true;         // inference layers 2-4 on the tensor cores
    bool train_tc = false;  // training forward and input gradients of layers 2-4 on the tensor cores
    long long step = 0;
    inlm::DevBuf pad, a1, a2, a3, a4, glog, d1, d2, d3, d4, counters;
};

// Per-denoiser inference state of an attached proposal.
struct ProposalRun {
    inlm_proposal* net = nullptr;
    int k = 0;
    float min_mass = 0.95f;
    float rel_mass = 0.f;  // > 0: fallback below rel_mass x the mean predicted kept mass
    // per-iteration schedule (inlm_proposal_schedule): iteration i uses entry
    // min(i, n) - 1; k 0 = full search that iteration. Empty: k, rel_mass.
    std::vector<int> sched_k;
    std::vector<float> sched_rel;
    int nwords = 0;
    long long n_tiles = 0;
    inlm::Dim3i t8{0, 0, 0};
    int group = 1;         // 8^3 tiles per plan along x: 1, or 4 (the 32 x 8 x 8 CTA)
    long long n_plan = 0;  // plan lists (tiles / groups)
    inlm::DevBuf a1, a2, a3, a4, bitmap, pmass, counters, scale, plan_start, plan_off, mass_sum;
};

struct inlm_denoiser {
    int shape[3] = {0, 0, 0};
    inlm_params p;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    inlm::Geometry geo;
    int nxp = 0, nyp = 0, nzp = 0;
    long long pitch_y = 0, pitch_z = 0;
    float* d_raw_pad = nullptr;
    float* d_prev_pad = nullptr;
    float* d_next = nullptr;
    float* d_sigma = nullptr;
    float* d_sigma0 = nullptr;
    float* d_mult = nullptr;
    int* d_err = nullptr;
    int2* d_search_delta = nullptr;
    int* d_group_zb = nullptr;  // raw-slab form: first z offset of the slab per offset group
    long long* d_search_off = nullptr;
    long long* d_patch_off = nullptr;
    float* d_weights = nullptr;
    bool use_tile = false;
    bool use_fast = false;       // FP16-storage kernel
    inlm::FastConfig fcfg{};
    inlm::FastArgs fargs{};
    void* d_raw_h = nullptr;     // padded FP16 raw / previous iterate
    void* d_prev_h = nullptr;
    CUtensorMap tm_prev_h{};
    // one 8^3 tile per CTA (tx = 8), the configuration per-tile plans run on
    bool use_tile8 = false;
    inlm::FastConfig fcfg8{};
    inlm::FastArgs fargs8{};
    CUtensorMap tm_prev_h8{};
    int2* d_search_delta8 = nullptr;
    // the FP16 column form (patch radius 1): full search without plans
    bool use_colf = false;
    inlm::FastConfig fcfgc{};
    inlm::FastArgs fargsc{};
    CUtensorMap tm_prev_hc{};
    int2* d_search_delta_c = nullptr;
    bool plan_active = false;     // fargs8 carries a per-tile plan
    bool plan_cta32 = false;      // ... or fargs_plan a per-32x8x8-CTA plan (proposal, group 4)
    inlm::FastArgs fargs_plan{};
    int* d_plan_start = nullptr;  // per-tile offset lists set by inlm_set_offset_plan
    int* d_plan_off = nullptr;
    int plan_cap = 0;
    int n_cta = 0;                // CTAs of the full-search (tx = 32) configuration
    ProposalRun prop;             // attached proposal network (prop.net != NULL)
    inlm::DevBuf aux;             // weight-mass maps: 1 / weight sum per voxel
    inlm::TileConfig tcfg{};
    inlm::TileArgs targs{};
    inlm::GenericArgs gargs{};
    CUtensorMap tm_prev{}, tm_raw{};
    int last_iter = 0;
    bool sigma_set = false;
    uint64_t launches = 0;
    std::vector<inlm::TimedLaunch> pending;
    std::vector<inlm::TimedLaunch> event_pool;
    double timed_ms = 0.0;
    int timed_n = 0;
    inlm_noise* noise = nullptr;
};

namespace inlm {
void noise_free(inlm_noise* n);
int launch_filter(inlm_denoiser* d);
int check_device_error(inlm_denoiser* d);
int tile_config_try(inlm_denoiser* d, int tz, bool raw_smem, bool* ok, bool ws = false);
int upload_sigma_device(inlm_denoiser* d);
int pad_into(inlm_denoiser* d, const float* src, float* dst);
int pad_into_half(inlm_denoiser* d, const float* src, void* dst);
// Noise estimate of a device volume into d_dst (nz floats, device); host_copy
// (nullable) gets a host copy after a stream synchronisation.
int estimate_into(inlm_denoiser* d, const float* vol_dev, float* d_dst,
                  std::vector<float>* host_copy);
// Parts of a device noise estimate (global / z-adaptive): sample draw and EM
// windows, then patch stds into n->d_patchstd (by the caller), then EM and
// per-slice sigma into n->d_sigma.
int noise_prepare(inlm_noise* n, const inlm_params* p, int* nwin, bool* first);
int noise_em_finish(inlm_noise* n, const inlm_params* p, int nwin);
// Runs the attached proposal on the padded previous iterate and points the
// filter's plan at its per-CTA lists (api_proposal.cu).
// k and relative threshold of iteration iter (1-based) under the schedule.
void proposal_step(const ProposalRun& r, int iter, int* k, float* rel_mass);
// Inference, selection and plans of iteration iter (its k must be > 0).
int proposal_enqueue(inlm_denoiser* d, int iter);
// Before iteration iter's filter launch: the proposal's plans, or the full
// search where the schedule's k is 0.
int proposal_prepare_iteration(inlm_denoiser* d, int iter);
void proposal_release(inlm_denoiser* d);

// Per-iteration engines over host-resident volumes (inlm_blocks_*): z-slab
// streaming on one device (api_stream.cu) or the stack split over several
// devices (api_multi.cu).
struct BlocksBackend {
    virtual ~BlocksBackend() {}
    virtual int set_sigma(const float* sigma_host) = 0;
    virtual int iteration(int iter, const float* raw_host, const float* prev_host, float* out_host) = 0;
    virtual int slab_depth() const = 0;
    virtual int attach_proposal(inlm_proposal*, int, float, float, int) {
        return fail(INLM_ERR_UNSUPPORTED, "the proposal runs on the one-device blocks only");
    }
    virtual int proposal_schedule(int, const int*, const float*) {
        return fail(INLM_ERR_UNSUPPORTED, "the proposal runs on the one-device blocks only");
    }
};
int make_stream_blocks(const int shape[3], const inlm_params* p, int slab_depth, BlocksBackend** out);
int make_multi_blocks(const int shape[3], const inlm_params* p, int n_parts, const int* device_ids,
                      BlocksBackend** out);
}  // namespace inlm

struct inlm_blocks {
    inlm::BlocksBackend* be = nullptr;
    int shape[3] = {0, 0, 0};
    int last_iter = 0;
    bool sigma_set = false;
    ~inlm_blocks() { delete be; }
};
