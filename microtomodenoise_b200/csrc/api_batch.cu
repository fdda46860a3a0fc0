// Batched form and tile-configuration autotuner (include/inlm.h). No
// counterpart in the reference, which filters one stack at a time
// (main.cpp:311-545); every volume of a batch follows that driver's schedule
// (sigma0 on the raw volume, iteration 1, sigma1 on its result blended with
// sigma0, iterations 2..n) with the plain FP32 filter, bit-identical to a
// single-volume run.
//
// Per iteration, one persistent kernel per patch shape filters the tiles of
// every volume of that shape, whatever its size and search radius (heaviest
// tiles first, each volume with the tile configuration the autotuner chose);
// the whole schedule of all volumes (noise estimates, padding, filter
// launches) is captured once in a CUDA graph and replayed.
#include <array>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>

#include "api_internal.hpp"

using namespace inlm;

// ---------------- autotuner ----------------

namespace {

struct TuneKey {
    int pr[3], sr[3], nslices, batch;
    bool operator<(const TuneKey& o) const {
        return std::lexicographical_compare(&pr[0], &pr[0] + 8, &o.pr[0], &o.pr[0] + 8);
    }
};
static_assert(sizeof(TuneKey) == 8 * sizeof(int), "TuneKey is eight ints");

struct TuneResult {
    int tz = 8;
    bool raw_smem = true;
    bool ws = false;  // the warp-specialised 8-deep kernel
    std::string report;
};

std::mutex g_tune_mu;
std::map<TuneKey, TuneResult> g_tune;
bool g_tune_loaded = false;

TuneKey tune_key(const inlm_params& p, bool batch) {
    TuneKey k{};
    for (int i = 0; i < 3; i++) {
        k.pr[i] = p.patch_radius[i];
        k.sr[i] = p.search_radius[i];
    }
    k.nslices = p.nslices;
    k.batch = batch ? 1 : 0;
    return k;
}

// Cache file (INLM_AUTOTUNE_CACHE): one line per class,
// "pr0 pr1 pr2 sr0 sr1 sr2 nslices batch tz raw_smem".
void load_cache_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = std::getenv("INLM_AUTOTUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    TuneKey k{};
    int tz = 0, raw = 0;
    while (std::fscanf(f, "%d %d %d %d %d %d %d %d %d %d", &k.pr[0], &k.pr[1], &k.pr[2], &k.sr[0],
                       &k.sr[1], &k.sr[2], &k.nslices, &k.batch, &tz, &raw) == 10) {
        TuneResult r;
        r.tz = tz;
        r.raw_smem = (raw & 1) != 0;  // bit 0: raw staged, bit 1: warp-specialised
        r.ws = (raw & 2) != 0;
        r.report = "cached";
        g_tune[k] = r;
    }
    std::fclose(f);
}

void save_cache_locked() {
    const char* path = std::getenv("INLM_AUTOTUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "w");
    if (!f) return;
    for (auto& kv : g_tune)
        std::fprintf(f, "%d %d %d %d %d %d %d %d %d %d\n", kv.first.pr[0], kv.first.pr[1],
                     kv.first.pr[2], kv.first.sr[0], kv.first.sr[1], kv.first.sr[2], kv.first.nslices,
                     kv.first.batch, kv.second.tz, (kv.second.raw_smem ? 1 : 0) | (kv.second.ws ? 2 : 0));
    std::fclose(f);
}

// Times every tiled configuration of a parameter class on a probe volume of
// 128 x 128 x 64 voxels (several CTA waves on 148 SMs; the kernel's work does
// not depend on the data) and returns the fastest. batch = true restricts the
// candidates to the CTA depth the persistent batch kernel runs (tz 8, not the
// warp-specialised kernel).
int tune_class(const inlm_params& p0, bool batch, TuneResult* out) {
    inlm_params p = p0;
    p.precision = INLM_PRECISION_F32;
    p.n_samples = 0;  // no noise handle
    const int shape[3] = {128, 128, 64};
    inlm_denoiser* d = nullptr;
    int rc = inlm_denoiser_create(shape, &p, &d);
    if (rc) return rc;
    struct Cand {
        int tz;
        bool raw;
        bool ws;
    };
    // tz 0: the column form (patch radius 1); ws: the warp-specialised kernel
    const Cand cands[] = {{0, false, false}, {16, true, false}, {8, true, false}, {8, false, false},
                          {4, false, false}, {8, true, true},   {8, false, true}};
    double best = 1e30;
    TuneResult res;
    bool any = false;
    char line[160];
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto cleanup = [&](int code) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        inlm_denoiser_destroy(d);
        return code;
    };
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return cleanup(fail(INLM_ERR_CUDA, "event creation failed"));
    std::vector<float> ones(shape[2], 1.0f);
    if (cudaMemcpy(d->d_sigma, ones.data(), shape[2] * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return cleanup(fail(INLM_ERR_CUDA, "sigma upload failed"));
    rc = upload_sigma_device(d);
    if (rc) return cleanup(rc);
    for (const Cand& c : cands) {
        if (batch && (c.tz != 8 || c.ws)) continue;
        bool ok = false;
        rc = tile_config_try(d, c.tz, c.raw, &ok, c.ws);
        if (rc) return cleanup(rc);
        if (!ok) continue;
        const int tiles_z = (shape[2] + d->tcfg.tz - 1) / d->tcfg.tz;
        float ms = 0.f;
        for (int rep = 0; rep < 3; rep++) {  // one warm-up, two timed
            if (rep == 1) cudaEventRecord(e0, d->stream);
            if (launch_tile_kernel(d->tcfg, &d->tm_prev, &d->tm_raw, d->targs, tiles_z, d->stream) !=
                cudaSuccess)
                return cleanup(fail(INLM_ERR_CUDA, "autotune launch failed"));
        }
        cudaEventRecord(e1, d->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess)
            return cleanup(fail(INLM_ERR_CUDA, "autotune timing failed"));
        cudaEventElapsedTime(&ms, e0, e1);
        ms *= 0.5f;
        std::snprintf(line, sizeof line, "tz=%d%s raw_%s: %.3f ms; ", c.tz, c.ws ? " ws" : "",
                      c.raw ? "smem" : "global", ms);
        res.report += line;
        if (ms < best) {
            best = ms;
            res.tz = c.tz;
            res.raw_smem = c.raw;
            res.ws = c.ws;
            any = true;
        }
    }
    rc = check_device_error(d);
    if (rc) return cleanup(rc);
    if (!any) return cleanup(fail(INLM_ERR_UNSUPPORTED, "no tiled configuration for this class"));
    std::snprintf(line, sizeof line, "chosen tz=%d%s raw_%s", res.tz, res.ws ? " ws" : "",
                  res.raw_smem ? "smem" : "global");
    res.report += line;
    *out = res;
    return cleanup(INLM_OK);
}

int tuned_config(const inlm_params& p, bool batch, TuneResult* out) {
    const TuneKey k = tune_key(p, batch);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        load_cache_locked();
        auto it = g_tune.find(k);
        if (it != g_tune.end()) {
            *out = it->second;
            return INLM_OK;
        }
    }
    TuneResult r;
    int rc = tune_class(p, batch, &r);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[k] = r;
    save_cache_locked();
    *out = r;
    return INLM_OK;
}

}  // namespace

extern "C" int inlm_autotune(inlm_denoiser* d, char* report, size_t len) {
    if (!d) return fail(INLM_ERR_ARG, "null handle");
    if (!d->use_tile) return fail(INLM_ERR_UNSUPPORTED, "the tiled FP32 kernel does not cover this configuration");
    CUDA_TRY(cudaSetDevice(d->device));
    CUDA_TRY(cudaStreamSynchronize(d->stream));
    TuneResult r;
    int rc = tuned_config(d->p, false, &r);
    if (rc) return rc;
    bool ok = false;
    rc = tile_config_try(d, r.tz, r.raw_smem, &ok, r.ws);
    if (rc) return rc;
    if (!ok) return fail(INLM_ERR_STATE, "tuned configuration does not fit this volume");
    if (report && len) std::snprintf(report, len, "%s", r.report.c_str());
    return INLM_OK;
}

// ---------------- batch ----------------

struct inlm_batch {
    int n = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<inlm_denoiser*> d;
    std::vector<float*> in;            // owned input volumes (the graph reads these)
    std::vector<float*> sigma_manual;  // manual mode: sigma[1] per slice
    std::vector<int> kind;             // batch body per volume (-1: own launch)
    std::vector<int> order;            // batched volumes, heaviest tiles first
    // persistent launch groups: volumes of one patch shape whose shared
    // memory allows the same number of CTAs per SM
    struct Group {
        int shape = 0;  // batch kind (BatchKind: patch radius and raw placement)
        int occ = 1;    // CTAs per SM
        size_t smem = 0;
        int ctas = 0;
        std::vector<int> vols;  // heaviest tiles first
    };
    std::vector<Group> groups;
    std::vector<std::vector<BatchParams>> launches;  // [iteration][group]
    std::vector<cudaStream_t> branch;                // one graph branch per group
    std::vector<cudaEvent_t> join;
    cudaEvent_t fork = nullptr;
    unsigned* d_counters = nullptr;
    int maxit = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    size_t graph_nodes = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::string tune_report;
};

static void batch_free(inlm_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (inlm_denoiser* d : b->d)
        if (d) inlm_denoiser_destroy(d);
    for (float* p : b->in) device_free(p);
    for (float* p : b->sigma_manual) device_free(p);
    device_free(b->d_counters);
    for (cudaStream_t s : b->branch) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->join) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    if (b->stream) cudaStreamDestroy(b->stream);
}

static long long nvox_of(const inlm_denoiser* d) {
    return (long long)d->shape[0] * d->shape[1] * d->shape[2];
}

// The filter launch of one volume outside the persistent kernel.
static int own_filter_launch(inlm_denoiser* d, cudaStream_t st) {
    if (d->use_tile) {
        const int tiles_z = (d->shape[2] + d->tcfg.tz - 1) / d->tcfg.tz;
        CUDA_TRY(launch_tile_kernel(d->tcfg, &d->tm_prev, &d->tm_raw, d->targs, tiles_z, st));
    } else {
        CUDA_TRY(launch_generic_kernel(d->gargs, st));
    }
    return INLM_OK;
}

// sigma for the next iterations: estimate on `vol` (or the manual value),
// blend with sigma0, multiplier.
static int batch_sigma1(inlm_batch* b, int v, const float* vol) {
    inlm_denoiser* d = b->d[v];
    const int nz = d->shape[2];
    if (d->p.noise_mode == INLM_NOISE_MANUAL) {
        CUDA_TRY(cudaMemcpyAsync(d->d_sigma, b->sigma_manual[v], nz * 4, cudaMemcpyDeviceToDevice,
                                 b->stream));
    } else {
        int rc = estimate_into(d, vol, d->d_sigma, nullptr);
        if (rc) return rc;
    }
    CUDA_TRY(launch_sigma_blend(d->d_sigma0, d->d_sigma, d->p.alpha, nz, b->stream));
    return upload_sigma_device(d);
}

// Enqueues the whole schedule of every volume on b->stream (captured).
static int batch_enqueue(inlm_batch* b) {
    cudaStream_t st = b->stream;
    for (int v = 0; v < b->n; v++) {
        inlm_denoiser* d = b->d[v];
        const int nz = d->shape[2];
        if (d->p.noise_mode != INLM_NOISE_MANUAL) {
            int rc = estimate_into(d, b->in[v], d->d_sigma0, nullptr);
            if (rc) return rc;
        }
        CUDA_TRY(cudaMemcpyAsync(d->d_sigma, d->d_sigma0, nz * 4, cudaMemcpyDeviceToDevice, st));
        int rc = upload_sigma_device(d);
        if (rc) return rc;
        rc = pad_into(d, b->in[v], d->d_raw_pad);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(d->d_prev_pad, d->d_raw_pad, d->pitch_z * d->nzp * 4,
                                 cudaMemcpyDeviceToDevice, st));
    }
    for (int it = 1; it <= b->maxit; it++) {
        if (it > 1) {
            for (int v = 0; v < b->n; v++) {
                inlm_denoiser* d = b->d[v];
                if (it > d->p.maxiterations) continue;
                int rc = pad_into(d, d->d_next, d->d_prev_pad);
                if (rc) return rc;
            }
        }
        // the groups run as parallel branches: a group's CTAs start on SMs
        // another group's tail frees
        CUDA_TRY(cudaEventRecord(b->fork, st));
        for (size_t gi = 0; gi < b->groups.size(); gi++) {
            const BatchParams& bp = b->launches[it - 1][gi];
            if (bp.n == 0) continue;
            const auto& grp = b->groups[gi];
            cudaStream_t bs = b->branch[gi];
            CUDA_TRY(cudaStreamWaitEvent(bs, b->fork, 0));
            CUDA_TRY(cudaMemsetAsync(bp.counter, 0, sizeof(unsigned), bs));
            CUDA_TRY(launch_batch_kernel(grp.shape, bp, grp.ctas, grp.smem, bs));
            CUDA_TRY(cudaEventRecord(b->join[gi], bs));
        }
        // volumes with their own launch run on the main stream beside the
        // persistent groups
        for (int v = 0; v < b->n; v++) {
            inlm_denoiser* d = b->d[v];
            if (it > d->p.maxiterations || b->kind[v] >= 0) continue;
            int rc = own_filter_launch(d, st);
            if (rc) return rc;
        }
        for (size_t gi = 0; gi < b->groups.size(); gi++)
            if (b->launches[it - 1][gi].n > 0) CUDA_TRY(cudaStreamWaitEvent(st, b->join[gi], 0));
        for (int v = 0; v < b->n; v++) {
            inlm_denoiser* d = b->d[v];
            const int mi = d->p.maxiterations;
            if (it > mi) continue;
            // sigma1 after iteration 1 (main.cpp:422-448); re-estimates under
            // continuous_estimate (main.cpp:517-544)
            if ((it == 1 && mi > 1) || (it > 1 && d->p.continuous_estimate && mi > it + 1)) {
                int rc = batch_sigma1(b, v, d->d_next);
                if (rc) return rc;
            }
        }
    }
    return INLM_OK;
}

extern "C" int inlm_batch_create(int n, const int* shapes, const inlm_params* params,
                                 inlm_batch** out) {
    if (!out || !shapes || !params || n < 1) return fail(INLM_ERR_ARG, "null argument or empty batch");
    *out = nullptr;
    const int dev = params[0].device_id;
    for (int v = 0; v < n; v++) {
        const inlm_params& p = params[v];
        if (p.device_id != dev) return fail(INLM_ERR_ARG, "a batch runs on one device");
        if (p.precision != INLM_PRECISION_F32)
            return fail(INLM_ERR_UNSUPPORTED, "the batched form runs the plain FP32 filter");
        if (p.noise_mode != INLM_NOISE_GLOBAL && p.noise_mode != INLM_NOISE_ZADAPTIVE &&
            p.noise_mode != INLM_NOISE_MANUAL)
            return fail(INLM_ERR_UNSUPPORTED, "volume %d: batched noise modes are global, "
                                              "z-adaptive and manual", v);
        if (p.maxiterations < 1) return fail(INLM_ERR_ARG, "volume %d: maxiterations < 1", v);
    }
    inlm_batch* b = new inlm_batch();
    b->n = n;
    b->device = dev;
    auto bail = [&](int code) {
        batch_free(b);
        delete b;
        return code;
    };
    cudaSetDevice(dev);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess)
        return bail(fail(INLM_ERR_CUDA, "stream/event creation failed"));
    b->d.assign(n, nullptr);
    b->in.assign(n, nullptr);
    b->sigma_manual.assign(n, nullptr);
    b->kind.assign(n, -1);
    int sms_dev = 148;
    cudaDeviceGetAttribute(&sms_dev, cudaDevAttrMultiProcessorCount, dev);
    for (int v = 0; v < n; v++) {
        int rc = inlm_denoiser_create(shapes + 3 * v, &params[v], &b->d[v]);
        if (rc) return bail(rc);
        inlm_denoiser* d = b->d[v];
        rc = inlm_set_stream(d, b->stream);
        if (rc) return bail(rc);
        if (dalloc(&b->in[v], (size_t)nvox_of(d)) != cudaSuccess ||
            cudaMemset(b->in[v], 0, nvox_of(d) * 4) != cudaSuccess)
            return bail(fail(INLM_ERR_NOMEM, "batch input allocation failed"));
        b->maxit = std::max(b->maxit, d->p.maxiterations);
        const int nz = d->shape[2];
        if (d->p.noise_mode == INLM_NOISE_MANUAL) {
            std::vector<float> s0(nz, d->p.sigma[0]), s1(nz, d->p.sigma[1]);
            if (dalloc(&b->sigma_manual[v], nz) != cudaSuccess ||
                cudaMemcpy(d->d_sigma0, s0.data(), nz * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(b->sigma_manual[v], s1.data(), nz * 4, cudaMemcpyHostToDevice) !=
                    cudaSuccess)
                return bail(fail(INLM_ERR_NOMEM, "manual sigma upload failed"));
        } else {
            if (!d->noise)
                return bail(fail(INLM_ERR_ARG, "volume %d is too small for the noise patch", v));
            // first estimate draws the samples and uploads the windows (host
            // work the graph cannot hold); later ones are device-only
            rc = estimate_into(d, b->in[v], d->d_sigma0, nullptr);
            if (rc) return bail(rc);
        }
        // A volume whose own configuration is the column form, the 16-deep
        // CTA or the warp-specialised kernel (faster than the persistent
        // depth-8 body) and which fills the GPU by itself (>= 4 waves of CTAs)
        // keeps it and runs its own launch beside the persistent groups.
        if (d->use_tile && (d->tcfg.column || d->tcfg.tz == 16 || d->tcfg.ws)) {
            const long long ctas = (long long)d->targs.tiles_x * d->targs.tiles_y *
                                   ((d->shape[2] + d->tcfg.tz - 1) / d->tcfg.tz);
            if (ctas >= 4LL * sms_dev) continue;  // kind stays -1
        }
        // tile configuration from the autotuner (depth 8: the persistent body)
        if (d->use_tile) {
            TuneResult r;
            rc = tuned_config(d->p, true, &r);
            if (rc == INLM_OK) {
                bool ok = false;
                rc = tile_config_try(d, r.tz, r.raw_smem, &ok, r.ws);
                if (rc) return bail(rc);
                char line[256];
                std::snprintf(line, sizeof line, "[p%d%d%d s%d%d%d] %s\n", d->p.patch_radius[0],
                              d->p.patch_radius[1], d->p.patch_radius[2], d->p.search_radius[0],
                              d->p.search_radius[1], d->p.search_radius[2], r.report.c_str());
                if (b->tune_report.find(line) == std::string::npos) b->tune_report += line;
            } else if (rc != INLM_ERR_UNSUPPORTED) {
                return bail(rc);
            }
            if (d->use_tile) b->kind[v] = batch_kind(d->tcfg);
        }
    }
    if (cudaStreamSynchronize(b->stream) != cudaSuccess)
        return bail(fail(INLM_ERR_CUDA, "batch setup failed"));

    // batched volumes, heaviest tile first (longest-processing-time order)
    int nb = 0;
    for (int v = 0; v < n; v++)
        if (b->kind[v] >= 0) b->order.push_back(v);
    std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
        const inlm_denoiser* dx = b->d[x];
        const inlm_denoiser* dy = b->d[y];
        return (double)dx->geo.search.size() * dx->geo.taps.size() >
               (double)dy->geo.search.size() * dy->geo.taps.size();
    });
    nb = (int)b->order.size();
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (int shape = 0; shape < kBatchKinds; shape++) {
        size_t smax = 0;
        for (int v : b->order)
            if (b->kind[v] == shape) smax = std::max(smax, b->d[v]->tcfg.smem_bytes);
        if (smax == 0) continue;
        int occ_max = 0;
        if (batch_kernel_setup(shape, smax, &occ_max) != cudaSuccess || occ_max < 1)
            return bail(fail(INLM_ERR_UNSUPPORTED, "persistent kernel does not fit (%zu bytes)", smax));
        for (int v : b->order) {  // keeps the heaviest-first order inside groups
            if (b->kind[v] != shape) continue;
            int occ = 0;
            if (batch_kernel_setup(shape, b->d[v]->tcfg.smem_bytes, &occ) != cudaSuccess || occ < 1)
                return bail(fail(INLM_ERR_CUDA, "occupancy query failed"));
            // a group's volumes share the patch weights (the kernel reads them
            // from its first volume's parameters: constant-bank operands)
            const inlm_denoiser* dv = b->d[v];
            auto it = std::find_if(b->groups.begin(), b->groups.end(), [&](const inlm_batch::Group& g) {
                const inlm_denoiser* d0 = b->d[g.vols[0]];
                return g.shape == shape && g.occ == occ && d0->geo.taps.size() == dv->geo.taps.size() &&
                       std::memcmp(d0->targs.w, dv->targs.w, dv->geo.taps.size() * sizeof(float)) == 0;
            });
            if (it == b->groups.end()) {
                b->groups.push_back(inlm_batch::Group{});
                it = b->groups.end() - 1;
                it->shape = shape;
                it->occ = occ;
            }
            it->vols.push_back(v);
            it->smem = std::max(it->smem, b->d[v]->tcfg.smem_bytes);
        }
        // the function attribute covers the largest group of this shape
        int dummy = 0;
        batch_kernel_setup(shape, smax, &dummy);
    }
    for (auto& g : b->groups) {
        if ((int)g.vols.size() > kBatchMax)
            return bail(fail(INLM_ERR_ARG, "at most %d volumes per launch group", kBatchMax));
        g.ctas = g.occ * sms;
    }
    (void)nb;
    const size_t ng = b->groups.size();
    if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(INLM_ERR_CUDA, "event creation failed"));
    b->branch.assign(ng, nullptr);
    b->join.assign(ng, nullptr);
    for (size_t gi = 0; gi < ng; gi++)
        if (cudaStreamCreateWithFlags(&b->branch[gi], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->join[gi], cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(INLM_ERR_CUDA, "branch stream creation failed"));
    if (dalloc(&b->d_counters, (size_t)b->maxit * std::max<size_t>(ng, 1)) != cudaSuccess)
        return bail(fail(INLM_ERR_NOMEM, "counter allocation failed"));
    b->launches.assign(b->maxit, std::vector<BatchParams>(ng));
    for (int it = 1; it <= b->maxit; it++) {
        for (size_t gi = 0; gi < ng; gi++) {
            BatchParams& bp = b->launches[it - 1][gi];
            std::memset(&bp, 0, sizeof bp);
            bp.counter = b->d_counters + ng * (it - 1) + gi;
            int items = 0;
            for (int v : b->groups[gi].vols) {
                const inlm_denoiser* d = b->d[v];
                if (it > d->p.maxiterations) continue;
                const int i = bp.n++;
                bp.maps[i] = d->tm_prev;
                bp.args[i] = d->targs;
                bp.kind[i] = b->kind[v];
                bp.item_begin[i] = items;
                items += d->targs.tiles_x * d->targs.tiles_y * ((d->shape[2] + 7) / 8);
            }
            bp.item_begin[bp.n] = items;
        }
    }

    // capture the schedule once
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return bail(fail(INLM_ERR_CUDA, "stream capture could not start"));
    int rc = batch_enqueue(b);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return bail(rc);
    }
    if (ce != cudaSuccess || !g)
        return bail(fail(INLM_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(ce)));
    b->graph = g;
    if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess)
        return bail(fail(INLM_ERR_CUDA, "graph instantiation failed"));
    cudaGraphGetNodes(g, nullptr, &b->graph_nodes);
    *out = b;
    return INLM_OK;
}

extern "C" int inlm_batch_destroy(inlm_batch* b) {
    batch_free(b);
    delete b;
    return INLM_OK;
}

extern "C" int inlm_batch_run(inlm_batch* b, const float* const* raws, float* const* outs,
                              int on_device, float* ms_out) {
    if (!b || !raws || !outs) return fail(INLM_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(b->device));
    const cudaMemcpyKind kin = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind kout = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    for (int v = 0; v < b->n; v++) {
        if (!raws[v] || !outs[v]) return fail(INLM_ERR_ARG, "null volume %d", v);
        CUDA_TRY(cudaMemcpyAsync(b->in[v], raws[v], nvox_of(b->d[v]) * 4, kin, b->stream));
    }
    CUDA_TRY(cudaEventRecord(b->e0, b->stream));
    CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
    CUDA_TRY(cudaEventRecord(b->e1, b->stream));
    for (int v = 0; v < b->n; v++)
        CUDA_TRY(cudaMemcpyAsync(outs[v], b->d[v]->d_next, nvox_of(b->d[v]) * 4, kout, b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    if (ms_out) CUDA_TRY(cudaEventElapsedTime(ms_out, b->e0, b->e1));
    for (int v = 0; v < b->n; v++) {
        int rc = check_device_error(b->d[v]);
        if (rc) return rc;
    }
    return INLM_OK;
}

extern "C" int inlm_batch_describe(inlm_batch* b, char* buf, size_t len) {
    if (!b || !buf || !len) return fail(INLM_ERR_ARG, "null argument");
    static const char* kinds[kBatchKinds] = {"p111/raw_smem", "p111/raw_global", "p222/raw_smem",
                                             "p222/raw_global", "p333/raw_smem", "p333/raw_global",
                                             "p111/raw_slab",  "p222/raw_slab",   "p333/raw_slab"};
    std::string s;
    char line[256];
    std::snprintf(line, sizeof line, "graph of %zu nodes; %d volumes\n", b->graph_nodes, b->n);
    s += line;
    for (const auto& g : b->groups) {
        const bool slab = g.shape >= kBatchP111Slab;
        const int r = slab ? g.shape - kBatchP111Slab + 1 : g.shape / 2 + 1;
        std::snprintf(line, sizeof line,
                      "persistent nlm_batch_f32<p%d%d%d, raw_%s>: %d volumes, %d CTAs x 256 threads "
                      "(%d per SM), %zu B shared\n",
                      r, r, r, slab ? "slab" : g.shape % 2 ? "global" : "smem", (int)g.vols.size(), g.ctas,
                      g.occ, g.smem);
        s += line;
    }
    for (int v = 0; v < b->n; v++) {
        const inlm_denoiser* d = b->d[v];
        std::snprintf(line, sizeof line, "  %d: %dx%dx%d p%d%d%d s%d%d%d S=%zu P=%zu %s%s\n", v,
                      d->shape[0], d->shape[1], d->shape[2], d->p.patch_radius[0],
                      d->p.patch_radius[1], d->p.patch_radius[2], d->p.search_radius[0],
                      d->p.search_radius[1], d->p.search_radius[2], d->geo.search.size(),
                      d->geo.taps.size(), b->kind[v] >= 0 ? "batched " : "own launch ",
                      b->kind[v] >= 0 ? kinds[b->kind[v]]
                                      : (d->use_tile ? (d->tcfg.column ? "column"
                                                        : d->tcfg.ws      ? "tile ws"
                                                        : d->tcfg.tz == 16 ? "tile tz=16"
                                                                           : "tile")
                                                     : "generic"));
        s += line;
    }
    s += "autotuner: " + b->tune_report;
    std::snprintf(buf, len, "%s", s.c_str());
    return INLM_OK;
}
