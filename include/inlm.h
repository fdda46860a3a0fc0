/*
 * inlm.h — C ABI of the B200 iterNLM hot path (iterative 3D nonlocal means
 * filter and two-cluster noise estimators).
 *
 * Plain C types only: pointers, sizes, ints, floats. Every call returns an
 * int status (INLM_OK = 0, negative = error); inlm_last_error() gives the
 * text of the calling thread's last error. Handles are not thread-safe: one
 * host thread drives one handle, on that handle's own CUDA stream.
 *
 * Reference call surface each entry point replaces (file:line in
 * iterNLM_v0.3):
 *   inlm_denoiser_create   <- denoise::IterativeNLM_GPU::configure_device
 *                             (Denoiser/iternlm_gpu.h:27, iternlm_gpu.cu:1440)
 *   inlm_denoiser_destroy  <- IterativeNLM_GPU::free_device (iternlm_gpu.h:28,
 *                             iternlm_gpu.cu:1619)
 *   inlm_set_sigma         <- IterativeNLM_GPU::set_sigma (iternlm_gpu.h:34,
 *                             iternlm_gpu.cu:2341)
 *   inlm_run_iteration     <- IterativeNLM_GPU::Run_GaussianNoise (iternlm_gpu.h:30,
 *                             iternlm_gpu.cu:1651)
 *   inlm_get_result        <- IterativeNLM_GPU::get_result (iternlm_gpu.h:35,
 *                             iternlm_gpu.cu:2356)
 *   inlm_noise_create      <- noise::NoiseLevel::NoiseLevel (Noise/noiselevel.h:21)
 *   inlm_noise_estimate    <- noise::NoiseLevel::get_noiselevel (noiselevel.h:31,
 *                             noiselevel.cpp:9)
 *   inlm_denoise           <- the σ0/σ1 schedule and iteration loop of the
 *                             iterNLM driver (main.cpp:327-545)
 *
 * Shapes are {nx, ny, nz}, x fastest, as the reference stores stacks.
 */
#ifndef INLM_H
#define INLM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define INLM_OK 0
#define INLM_ERR_ARG -1        /* bad argument (shape, radius, null pointer) */
#define INLM_ERR_CUDA -2       /* CUDA runtime error (reference: configure_device -2) */
#define INLM_ERR_NODEVICE -3   /* no CUDA device (reference: configure_device -1) */
#define INLM_ERR_NOMEM -4      /* device allocation failed */
#define INLM_ERR_STATE -5      /* call out of order (e.g. iteration 2 before 1) */
#define INLM_ERR_TIMEOUT -6    /* a bounded device wait ran out */
#define INLM_ERR_UNSUPPORTED -7
#define INLM_ERR_IO -8         /* file missing, unreadable or not a TIFF */

/* noise estimation modes (denoise_parameters.h:22) */
#define INLM_NOISE_ZADAPTIVE 0
#define INLM_NOISE_GLOBAL 1
#define INLM_NOISE_MANUAL 2
#define INLM_NOISE_SEMIMANUAL 3

/* storage / arithmetic form of the filter */
#define INLM_PRECISION_F32 0   /* FP32, bit-identical to the reference CPU filter */
#define INLM_PRECISION_F16 1   /* FP16 volumes and squared-difference planes, FP32 accumulation */
#define INLM_PRECISION_F16_DF32 2 /* FP16 volumes, FP32 squared-difference planes */
#define INLM_PRECISION_F32_FMA 3  /* FP32 volumes, patch taps and Pade fused (FFMA), fast
                                     division: within a stated tolerance of the reference,
                                     not bit-identical */

/* patch-weight table */
#define INLM_WEIGHTS_CPU 0        /* the table the reference CPU filter applies (default) */
#define INLM_WEIGHTS_DISTWEIGHT 1 /* setup_distweight values for every shape */

typedef struct {
    /* filter (protocol::DenoiseParameters, denoise_parameters.h:11-20) */
    float alpha;             /* 0.5 */
    int maxiterations;       /* 4 */
    int nslices;             /* 11 */
    int search_radius[3];    /* {10,10,10} */
    int patch_radius[3];     /* {1,1,1} */
    float beta;              /* 1 */
    float z_anisotropy;      /* 1 */
    /* noise (denoise_parameters.h:20-34) */
    int noise_mode;          /* INLM_NOISE_ZADAPTIVE */
    int zwindow;             /* 100 */
    float sigma[2];          /* manual / semimanual values */
    uint64_t n_samples;      /* 100000 */
    int noise_patchsize;     /* 15 */
    float stds_from_mean;    /* 1 */
    int continuous_estimate; /* 0 */
    int circular_mask_diameter; /* 0 */
    unsigned int noise_seed; /* seed of the glibc-rand() sample draw (reference: time(NULL)) */
    /* device */
    int device_id;           /* 0 */
    int precision;           /* INLM_PRECISION_F32 */
    int weight_table;        /* INLM_WEIGHTS_CPU */
} inlm_params;

typedef struct inlm_denoiser inlm_denoiser;
typedef struct inlm_noise inlm_noise;

/* Fills the reference defaults (denoise_parameters.h). */
void inlm_default_params(inlm_params* p);

const char* inlm_last_error(void);

/* ---------------- denoiser (IterativeNLM_GPU) ---------------- */

/* Allocates the padded raw / previous-iterate volumes and the result on
 * device p->device_id and builds the search and patch tables.
 * Returns INLM_ERR_NODEVICE when no CUDA device exists (the reference's -1,
 * where its driver falls back to the CPU). */
int inlm_denoiser_create(const int shape[3], const inlm_params* p, inlm_denoiser** out);
int inlm_denoiser_destroy(inlm_denoiser* d);

/* Uploads nz sigma values (host) and derives the per-slice multiplier
 * -1/(sigma^2 beta) (iternlm_cpu.cpp:94-95). */
int inlm_set_sigma(inlm_denoiser* d, const float* sigma_host);

/* One iteration. iter == 1 needs raw_host (copied and padded on the device,
 * prepare_iteration1, iternlm_gpu.cu:2117); iter > 1 pads the previous result
 * (prepare_nextiteration, :2230) and raw_host may be NULL. */
int inlm_run_iteration(inlm_denoiser* d, int iter, const float* raw_host);

/* Copies the last iteration's nx*ny*nz result to host memory. */
int inlm_get_result(inlm_denoiser* d, float* out_host);

/* Device-resident forms (no host copies): raw_dev / out_dev are device
 * pointers on the denoiser's device. */
int inlm_run_iteration_device(inlm_denoiser* d, int iter, const float* raw_dev);
int inlm_get_result_device(inlm_denoiser* d, float* out_dev);

/* Whole job on the device, the driver's schedule (main.cpp:327-545):
 * sigma0 = noise(raw); iteration 1; sigma1 = noise(result);
 * sigma1 = alpha*sigma0 + (1-alpha)*sigma1; iterations 2..maxiterations
 * (re-estimating before each under continuous_estimate). raw and out are
 * host pointers when on_device == 0, device pointers otherwise.
 * sigma0_out / sigma1_out (nullable, host) receive the two estimates. */
int inlm_denoise(inlm_denoiser* d, const float* raw, float* out, int on_device,
                 float* sigma0_out, float* sigma1_out);

/* Stream the denoiser launches on (cudaStream_t as void*); NULL = its own. */
int inlm_set_stream(inlm_denoiser* d, void* stream);

/* Average duration in ms of the filter-kernel launches since the last call
 * (CUDA events on the launching stream); *n_launches gets their count. */
int inlm_filter_kernel_ms(inlm_denoiser* d, double* avg_ms, int* n_launches);

/* Description of the chosen filter kernel (name, tile, taps, offsets). */
int inlm_describe(inlm_denoiser* d, char* buf, size_t len);

/* Tiling of the full-search filter kernel: tile_shape = voxels per CTA
 * {x, y, z}, tiles = CTA counts {x, y, z}; index = (tz*tiles[1] + ty)*tiles[0] + tx. */
int inlm_tile_grid(inlm_denoiser* d, int tile_shape[3], int tiles[3]);

/* Per-tile offset plan for the FP16 form (the learned proposal's output):
 * 8^3 tile t (tiles ordered (tz*ceil(ny/8) + ty)*ceil(nx/8) + tx) evaluates
 * the search offsets offsets[start[t] .. start[t]+count[t]) (indices into
 * the reference-order search table, in the order given); the filter then
 * runs one 8^3 tile per CTA. start and count have one entry per tile,
 * offsets n_offsets; on_device = 1 when the three arrays are device memory
 * (they are copied; device plans are not range-checked, indices are clamped
 * to the table). start == NULL returns to full search. */
int inlm_set_offset_plan(inlm_denoiser* d, const int* start, const int* count, const int* offsets,
                         int n_offsets, int on_device);

/* Test hooks for the failure paths (no counterpart in the reference, whose
 * allocation failures surface as CUDA error strings, iternlm_gpu.cu:1608-1618).
 * inlm_debug_fail_allocation(n): the device allocation that follows n further
 * successful ones fails, once, as cudaMalloc fails when memory runs out (the
 * calling entry point then returns INLM_ERR_NOMEM and releases what it had
 * allocated); n < 0 disarms. inlm_debug_live_allocations: the number of device
 * allocations of this library not yet released (a leak check). */
int inlm_debug_fail_allocation(int64_t n);
int inlm_debug_live_allocations(int64_t* n);
/* Runs, on the handle's stream, a one-CTA kernel whose bounded mbarrier wait
 * (the wait of every TMA-staged filter kernel, ~1 s budget there) is never
 * satisfied, with a budget of `cycles` (0..2e9): the wait gives up, the kernel
 * records the timeout in the handle's error word and returns, and this call
 * returns INLM_ERR_TIMEOUT as a filter call would. The handle stays usable. */
int inlm_debug_wait_expiry(inlm_denoiser* d, int64_t cycles);

/* Number of kernels this handle has launched since creation. */
int inlm_kernel_launches(inlm_denoiser* d, uint64_t* count);

/* ---------------- noise level (NoiseLevel) ---------------- */

/* shape as above; n_samples random 2D patches of patchsize^2 voxels. The
 * sample positions are drawn on the first estimate and kept (the reference
 * caches them in NoiseLevel::samples). */
int inlm_noise_create(const int shape[3], uint64_t n_samples, int patchsize, unsigned int seed,
                      int device_id, inlm_noise** out);
int inlm_noise_destroy(inlm_noise* n);

/* NoiseLevel::get_noiselevel: sigma_out receives nz values (host).
 * stack is a host pointer when on_device == 0, else a device pointer.
 * Uses p->noise_mode, zwindow, sigma[], stds_from_mean,
 * circular_mask_diameter. In semimanual mode the second and later calls write
 * the chosen value to p->sigma[1], as the reference does (noiselevel.cpp:74). */
int inlm_noise_estimate(inlm_noise* n, inlm_params* p, const float* stack, int on_device,
                        float* sigma_out);

/* Sorted sample positions (linear voxel indices) drawn so far; returns the
 * count through *n_out. */
int inlm_noise_samples(inlm_noise* n, int64_t* out, uint64_t max_n, uint64_t* n_out);

/* Per-sample patch std of the last estimate (host copy). */
int inlm_noise_patchstd(inlm_noise* n, float* out, uint64_t max_n);

/* Two-cluster EM of the noise estimators for callers that cannot allocate
 * device memory. It has no counterpart in the reference (whose EM runs on
 * the host). It calls no cudaMalloc, cudaFree or other allocating routine:
 * its scratch (one byte per sample per window, and the window table) lives
 * in file-scope device arrays of this library, 16 MiB + 256 KiB, which every
 * GPU that loads the library holds until the process exits. Callers that
 * cannot allocate include code running while another thread captures a CUDA
 * graph in global capture mode (cudaMalloc is a prohibited call then) and
 * applications whose device memory is owned by their own pool.
 *
 * values_dev: n_values per-sample patch stds (device); windows_host: 2 values
 * per window (first, last sample index, inclusive; last < first = empty,
 * whose outputs are 0), host memory, read before the call returns;
 * mean_dev / sd_dev: n_windows outputs (device), the lower cluster's mean and
 * std per window, as inlm_noise_estimate computes them.
 * Runs on the calling thread's current device, on `stream`. The call only
 * enqueues kernels (the window table travels in their launch parameters): it
 * copies nothing from host memory and does not wait, so the outputs are
 * ready once `stream` reaches them. NULL is the legacy default stream, which
 * synchronises with every blocking stream of the context; while another
 * thread captures a stream, pass a stream created with
 * cudaStreamNonBlocking.
 * Limits: n_windows <= 16384 and the window lengths summing to at most
 * 16777216 samples; larger requests return INLM_ERR_ARG.
 * The first call on a device looks up the arrays' device addresses; make
 * it before any stream capture. Calls share the arrays and leave the last
 * call's contents behind: calls that overlap on the GPU race. */
int inlm_noise_em_noalloc(void* stream, const float* values_dev, int64_t n_values,
                          const int64_t* windows_host, int n_windows, float* mean_dev,
                          float* sd_dev);

/* ---------------- learned search-offset proposal ----------------
 * No counterpart in the reference, whose filter evaluates every search offset
 * for every voxel (Denoiser/iternlm_cpu.cpp:758-843, iternlm_gpu.cu:80-1437).
 * A small 3D conv net (4 conv layers of 16 channels with 3^3 kernels, BF16
 * weights, FP32 accumulation, a linear head and a softmax over the S search
 * offsets per 8^3 tile) predicts which offsets carry the filter weight; the
 * FP16 form then evaluates only each tile's top K, or every offset when the
 * predicted kept mass of the tile is below min_mass.
 *
 * Parameters are a flat float vector (inlm_proposal_n_params): conv weights
 * [27 taps][Cin][16] (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)) and biases [16] for
 * layers 1..4 (layer 1 has Cin = 1), head weights [S][16], head bias [S].
 * Network input: a volume (the filter's previous iterate) and a per-slice
 * scale 1/(sigma sqrt(beta)); layer 1 sees scale * (v(c+tap) - v(c)).
 * Example volumes are unpadded FP32 device arrays, x fastest, every axis >= 2. */
typedef struct inlm_proposal inlm_proposal;

int inlm_proposal_create(int n_offsets, int device_id, inlm_proposal** out);
int inlm_proposal_destroy(inlm_proposal* p);
int inlm_proposal_n_params(const inlm_proposal* p, int64_t* n);
/* Sets the FP32 parameters (host), rounds the weights to BF16 and resets the
 * optimiser state. */
int inlm_proposal_set_params(inlm_proposal* p, const float* params_host, int64_t n);
int inlm_proposal_get_params(inlm_proposal* p, float* params_host, int64_t n);
/* Forward pass of one example: logits_dev gets n_tiles x S values, tiles
 * ordered (tz*ty_n + ty)*tx_n + tx with tile counts ceil(n/8). */
int inlm_proposal_logits(inlm_proposal* p, const float* vol_dev, const float* scale_dev,
                         const int shape[3], float* logits_dev);
/* One optimiser step (Adam, beta 0.9/0.999) on the summed soft-target cross
 * entropy of n_examples examples, averaged over all their tiles. targets_dev[e]
 * holds n_tiles x S per-tile offset distributions (inlm_weight_map). shapes:
 * 3 ints per example. grad_host != NULL: store the gradient there instead of
 * updating the parameters. loss_out (nullable) gets the loss. */
int inlm_proposal_train(inlm_proposal* p, int n_examples, const float* const* vols_dev,
                        const float* const* scales_dev, const float* const* targets_dev,
                        const int* shapes, float lr, double* loss_out, float* grad_host);
/* Top-k selection of one example: bitmap_dev gets n_tiles x ceil(S/32) words
 * (bit k%32 of word k/32 = offset k evaluated), pred_mass_dev the predicted
 * kept mass per tile; tiles below min_mass select every offset (counted in
 * *n_fallback). */
int inlm_proposal_select(inlm_proposal* p, const float* vol_dev, const float* scale_dev,
                         const int shape[3], int k, float min_mass, uint32_t* bitmap_dev,
                         float* pred_mass_dev, int* n_fallback);
/* Layers 2-4 (3^3 convs, 16 -> 16 channels) on the tensor cores: tcgen05
 * implicit GEMMs with TF32 operands (the BF16 weights exact in TF32) and FP32
 * accumulation in tensor memory; else on the CUDA cores with FP32
 * activations (the reference of the tensor-core path). mode bit 0: inference
 * (set by default); bit 1: training, the forward pass and the input
 * gradients of inlm_proposal_train (clear by default; its weight gradients
 * always run on the CUDA cores). */
int inlm_proposal_set_tensor_cores(inlm_proposal* p, int mode);
/* Attaches a proposal to an FP16-form denoiser (p == NULL detaches): every
 * later iteration runs the network on its previous iterate and evaluates the
 * selected offsets per 8^3 tile. */
int inlm_attach_proposal(inlm_denoiser* d, inlm_proposal* p, int k, float min_mass);
/* The same with one offset list per tiles_x 8^3 tiles along x: 1 (as above,
 * one 8^3 tile per filter CTA), or 4: the offsets ranked by the sum of the
 * four tiles' softmax probabilities, one list per 32 x 8 x 8 block, run by
 * the full-width FP16 kernel (a coarser choice per offset, a faster kernel
 * per offset; the predicted kept mass is the mean over the four tiles). */
int inlm_attach_proposal_grouped(inlm_denoiser* d, inlm_proposal* p, int k, float min_mass,
                                 int tiles_x);
/* The same with a fallback threshold relative to the volume: a list whose
 * predicted kept mass is below rel_mass x the mean predicted kept mass of
 * all lists of the iteration (0 < rel_mass <= 1; 0: off) evaluates every
 * offset, as does one below min_mass. The mean adapts the threshold to k, S,
 * sigma and the data, so the fallback picks the lists whose kept mass is poor
 * for this volume, where an absolute threshold that a flat weight
 * distribution never reaches falls back everywhere. The mean is summed in a
 * fixed order: the same lists fall back on every run. */
int inlm_attach_proposal_ex(inlm_denoiser* d, inlm_proposal* p, int k, float min_mass, float rel_mass,
                            int tiles_x);
/* Per-iteration schedule for the attached proposal: iteration i (1-based)
 * keeps k[min(i, n) - 1] offsets per list with the relative fallback
 * rel_mass[min(i, n) - 1] (0: none); k = 0 runs that iteration's full
 * search. n = 0 returns to the attach call's k and rel_mass. The last
 * iteration's output carries the approximation directly, earlier ones are
 * re-filtered, so a schedule with small lists early and a larger list with
 * the fallback in the last iteration is both faster and closer to the full
 * search than one k throughout. Cleared by a new attach. */
int inlm_proposal_schedule(inlm_denoiser* d, int n, const int* k, const float* rel_mass);
/* inlm_proposal_select for groups of tiles_x 8^3 tiles along x: bitmap and
 * pred_mass hold one entry per group, groups ordered z, y, x. */
int inlm_proposal_select_grouped(inlm_proposal* p, const float* vol_dev, const float* scale_dev,
                                 const int shape[3], int tiles_x, int k, float min_mass,
                                 uint32_t* bitmap_dev, float* pred_mass_dev, int* n_fallback);
/* Last iteration of an attached proposal: stats = {plan lists (tiles or
 * groups), lists that fell back, offsets evaluated summed over filter CTAs,
 * lists * S (full search), S}. */
int inlm_proposal_stats(inlm_denoiser* d, int64_t stats[5]);
/* Training targets: the last iteration's per-8^3-tile weight mass of every
 * search offset (full search, FP16 form), each voxel's offset weights divided
 * by their sum, averaged over the tile's voxels; map_dev: n_tiles x S. */
int inlm_weight_map(inlm_denoiser* d, float* map_dev);
/* The last iteration's network input: its previous iterate (unpadded FP32,
 * the FP16 values the filter read) and the per-slice scale. */
int inlm_net_input(inlm_denoiser* d, float* vol_dev, float* scale_dev);

/* ---------------- autotuner and batched form ----------------
 * No counterpart in the reference, which runs one stack with one fixed
 * kernel configuration per run (main.cpp:311-545). */

/* Restricts the plain FP32 filter to one kernel family and picks its first
 * configuration that fits: form 0 = automatic (the column form for patch
 * radius 1 when it fits; the warp-specialised kernel where patch sums
 * dominate, at 100 or more patch taps or at 30 or more taps with 400 or more
 * search offsets; else the tiled kernels), 1 = the tiled kernels without warp
 * specialisation, 2 = the column form only, 3 = the warp-specialised kernel
 * only (INLM_ERR_UNSUPPORTED where the form has no instantiation or does not
 * fit). Results do not change: every form rounds each voxel identically. Call
 * between iterations, not while one runs. */
int inlm_select_tile_form(inlm_denoiser* d, int form);

/* Times the tiled FP32 kernel's configurations (the column form at patch
 * radius 1, CTA depth 16 with two planes per thread, CTA depth 8 with raw
 * staged in shared memory or read from global memory, depth 4, the
 * warp-specialised kernel with raw staged or from global memory) on a
 * 128x128x64 probe
 * of d's patch/search class, applies the fastest to d and caches the choice
 * per process (and in the file named by the INLM_AUTOTUNE_CACHE environment
 * variable when set). Results do not change: every configuration rounds each
 * voxel identically. report (nullable) gets the timings. */
int inlm_autotune(inlm_denoiser* d, char* report, size_t len);

typedef struct inlm_batch inlm_batch;

/* n volumes of different sizes and radii filtered together: shapes holds
 * {nx, ny, nz} per volume, params one inlm_params per volume (plain FP32,
 * noise mode global, z-adaptive or manual, one device). Each iteration of all
 * volumes runs as one persistent kernel over their tiles (heaviest tiles
 * first; tile configurations from the autotuner; volumes whose patch shape has
 * no batched body get their own launch), and the whole schedule (noise
 * estimates, padding, iterations) is captured once in a CUDA graph. At most 24
 * batched volumes. */
int inlm_batch_create(int n, const int* shapes, const inlm_params* params, inlm_batch** out);
int inlm_batch_destroy(inlm_batch* b);
/* Runs the schedule of every volume (inlm_denoise semantics per volume):
 * raws[v] / outs[v] are host pointers (on_device = 0) or device pointers;
 * ms_out (nullable) gets the graph's device time. */
int inlm_batch_run(inlm_batch* b, const float* const* raws, float* const* outs, int on_device,
                   float* ms_out);
int inlm_batch_describe(inlm_batch* b, char* buf, size_t len);

/* ---------------- z-slab streaming ----------------
 * replaces IterativeNLM_GPU::Run_GaussianNoise_GPUBlocks (iternlm_gpu.h:31-32,
 * iternlm_gpu.cu:1887-2115) for volumes held in host memory. */

/* The inlm_denoise schedule for a volume that stays in host memory (raw_host,
 * out_host: nx*ny*nz floats each; page-locked here for the call when they are
 * not already). Every iteration walks the volume in z-slabs of slab_depth
 * slices (rounded up to a multiple of 8), each filtered on the device as a
 * sub-volume with a halo of max(8, z padding rounded up to 8) slices (16 or
 * more with a proposal) on two alternating streams, so one slab's copies
 * overlap another's kernels; noise estimates gather each sample's patch std
 * from the slab holding it. Results equal inlm_denoise's bit for bit in every
 * form. p->precision selects the form; net (nullable, FP16 forms) attaches a
 * learned proposal with k offsets per tile and fallback below min_mass.
 * Noise modes: global, z-adaptive, manual. sigma0_out / sigma1_out (nullable,
 * host, nz floats) receive the estimates; stats (nullable, 6 doubles) =
 * {device ms, host-to-device bytes, device-to-host bytes, slabs, halo, slab
 * depth}. Needs one extra host volume (page-locked) for the iterations. */
int inlm_stream_denoise(const int shape[3], const inlm_params* p, const float* raw_host,
                        float* out_host, int slab_depth, inlm_proposal* net, int k, float min_mass,
                        float* sigma0_out, float* sigma1_out, double* stats);
/* The same with the proposal's lists per tiles_x 8^3 tiles along x (1 or 4,
 * as inlm_attach_proposal_grouped); slabs split z only, so the results equal
 * the in-memory schedule with the same grouping. */
int inlm_stream_denoise_grouped(const int shape[3], const inlm_params* p, const float* raw_host,
                                float* out_host, int slab_depth, inlm_proposal* net, int k,
                                float min_mass, int tiles_x, float* sigma0_out, float* sigma1_out,
                                double* stats);
/* The same with the relative fallback of inlm_attach_proposal_ex; its mean is
 * taken over each sub-volume's lists (so results with rel_mass > 0 depend on
 * the slab depth; with rel_mass = 0 they equal the in-memory schedule's). */
int inlm_stream_denoise_ex(const int shape[3], const inlm_params* p, const float* raw_host,
                           float* out_host, int slab_depth, inlm_proposal* net, int k, float min_mass,
                           float rel_mass, int tiles_x, float* sigma0_out, float* sigma1_out,
                           double* stats);
/* The same with a per-iteration schedule of (k, rel_mass) as in
 * inlm_proposal_schedule (n_sched >= 1 entries; one entry = one k
 * throughout). */
int inlm_stream_denoise_sched(const int shape[3], const inlm_params* p, const float* raw_host,
                              float* out_host, int slab_depth, inlm_proposal* net, int n_sched,
                              const int* k_sched, const float* rel_sched, float min_mass, int tiles_x,
                              float* sigma0_out, float* sigma1_out, double* stats);

/* ---------------- FP64 full-search reference on sub-blocks ----------------
 * No counterpart in the reference, whose filter computes in FP32. The
 * full-search result of the last of n_iter iterations in FP64 (every product,
 * sum and quotient a separately rounded double, iterates kept in double,
 * m = -1/(sigma*sigma*beta) in double; the reference's algorithm,
 * iternlm_cpu.cpp:795-834, and its reflective padding) on n_blocks blocks of
 * size[3] voxels (x, y, z) with lower corners corners[3*b..] (x, y, z), without
 * filtering the whole volume: iteration k runs on the block grown by
 * (n_iter - k) x the padding per side. raw: the unpadded FP32 volume, host
 * (on_device = 0) or device memory; sigmas: n_iter x nz (host); out_host:
 * n_blocks blocks of size[2] x size[1] x size[0] doubles, x fastest. The
 * precision reference of the FP16 and learned forms at volume sizes a CPU
 * cannot finish; it equals the oracle's FP64 restatement bit for bit. */
int inlm_denoise_f64_blocks(const int shape[3], const inlm_params* p, const float* raw, int on_device,
                            const float* sigmas, int n_iter, const int* corners, int n_blocks,
                            const int size[3], double* out_host);

/* ---------------- host-only helpers (no device needed) ---------------- */

/* Geometry of a parameter set (setup_searchspace / setup_patchspace /
 * setup_distweight, Denoiser/iternlm_prepare.cpp:102-262): offsets as
 * (x,y,z) triples in reference order and the patch weights the filter applies.
 * Pass NULL arrays to query the counts. pad3 gets the padding per axis. */
int inlm_geometry(const inlm_params* p, int nz, int* search_xyz, int* n_search, int* patch_xyz,
                  float* weights, int* n_patch, int pad3[3]);

/* NoiseLevel::drawsamples (Noise/noiselevel.cpp:192) with the glibc rand()
 * sequence of srand(seed), sorted ascending. */
int inlm_noise_draw_samples(const int shape[3], uint64_t n_samples, int patchsize,
                            int circular_mask_diameter, unsigned int seed, int64_t* out);

/* ---------------- one stack on several GPUs of this process ----------------
 * The n_gpus mode of IterativeNLM_GPU::Run_GaussianNoise_GPUBlocks
 * (iternlm_gpu.cu:1732-2115): the inlm_denoise schedule on a host-resident
 * stack split in z over n_parts sub-volumes, part i on device device_ids[i]
 * (ids may repeat). Every part owns a run of 8-slice units and keeps halos of
 * its neighbours' slices, copied device to device after every iteration;
 * noise estimates gather every part's patch stds and run one EM. The result
 * equals inlm_denoise's bit for bit in every precision form (no proposal).
 * Noise modes: global, z-adaptive, manual. sigma0_out / sigma1_out (nullable,
 * nz floats) as inlm_denoise reports them. Every slab must be at least one
 * halo deep (8 slices for z padding up to 8). */
int inlm_denoise_multi(const int shape[3], const inlm_params* p, const float* raw_host,
                       float* out_host, int n_parts, const int* device_ids, float* sigma0_out,
                       float* sigma1_out);
/* Number of CUDA devices this process sees (0 without a driver or device). */
int inlm_device_count(int* n);
/* Free and total memory of a device in bytes (cudaMemGetInfo; the reference
 * sizes its blocks from it, iternlm_gpu.cu:1537-1566). */
int inlm_device_memory(int device, size_t* free_bytes, size_t* total_bytes);

/* ---------------- one iteration at a time over host-resident volumes ----------------
 * replaces the host-RAM overload of IterativeNLM_GPU::Run_GaussianNoise_GPUBlocks
 * (iternlm_gpu.h:31, iternlm_gpu.cu:1729-1886), which the reference driver
 * calls once per iteration when the stack is larger than one GPU holds or
 * runs on several GPUs (main.cpp:379, 472). With one device the volume is
 * walked in z-slabs of slab_depth slices (rounded up to 8) as
 * inlm_stream_denoise does; with several, the stack is split over them as
 * inlm_denoise_multi does. The caller schedules sigma and the iterations (and
 * estimates the noise), as with the single-volume handle. Results equal
 * inlm_run_iteration's bit for bit in every precision form (no proposal).
 * Unlike the reference, which overwrites its previous-iterate buffer slab by
 * slab while later slabs still read it, a call reads prev_host and writes a
 * distinct out_host. */
typedef struct inlm_blocks inlm_blocks;
/* device_ids: n_devices ids (may repeat; NULL with one device: p->device_id). */
int inlm_blocks_create(const int shape[3], const inlm_params* p, int n_devices,
                       const int* device_ids, int slab_depth, inlm_blocks** out);
int inlm_blocks_destroy(inlm_blocks* b);
/* One device only, before the first iteration: the FP16 form evaluates the
 * offsets a learned proposal selects (as inlm_attach_proposal_ex; the slabs'
 * halos grow to >= 16 slices, the network's receptive field). */
int inlm_blocks_attach_proposal(inlm_blocks* b, inlm_proposal* net, int k, float min_mass,
                                float rel_mass, int tiles_x);
/* After the attach, before the first iteration: the per-iteration (k,
 * rel_mass) schedule of inlm_proposal_schedule. */
int inlm_blocks_proposal_schedule(inlm_blocks* b, int n, const int* k, const float* rel_mass);
/* Slices per slab (one device) or the deepest part (several). */
int inlm_blocks_slab_depth(const inlm_blocks* b, int* depth);
/* sigma of the following iterations, nz floats (host). */
int inlm_blocks_set_sigma(inlm_blocks* b, const float* sigma_host);
/* Iteration iter (>= 1) from raw_host and, for iter > 1, the previous iterate
 * prev_host, into out_host (nx*ny*nz floats each, host; out_host != prev_host).
 * The buffers are page-locked for the duration of the call where they are not
 * already. Returns once out_host holds the result. */
int inlm_blocks_run_iteration(inlm_blocks* b, int iter, const float* raw_host,
                              const float* prev_host, float* out_host);

/* ---------------- resume ---------------- */

/* Installs a finished iteration's result read back from disk instead of
 * computing it: the --resume branch of IterativeNLM_GPU::Run_GaussianNoise
 * (iternlm_gpu.cu:1665-1697), which uploads the saved result and, for
 * iteration 1, still prepares the raw volume. result_host holds nx*ny*nz
 * floats; raw_host is required when iter == 1 and ignored otherwise. */
int inlm_set_result(inlm_denoiser* d, int iter, const float* result_host, const float* raw_host);

/* ---------------- z-slab sharding across GPUs ----------------
 * Building blocks of the multi-GPU form of Run_GaussianNoise_GPUBlocks
 * (iternlm_gpu.cu:1732-2115, which splits the stack in z across n_gpus):
 * each rank filters its z-slab plus halos of its neighbours' slices, and the
 * noise estimate gathers the per-sample patch stds of all ranks before one
 * replicated EM. The exchange itself is the caller's (NCCL or any transport). */

/* Copies slices z0..z0+n_slices-1 of the last result out of (get) or into
 * (set) the denoiser; set overwrites them before the next iteration pads the
 * result into its previous-iterate volume. dst / src are host pointers when
 * on_device == 0 (the call returns when the copy is done), else device
 * pointers (the copy is queued on the denoiser's stream). */
int inlm_get_result_slices(inlm_denoiser* d, int z0, int n_slices, float* dst, int on_device);
int inlm_set_result_slices(inlm_denoiser* d, int z0, int n_slices, const float* src, int on_device);

/* get_patchstd (noiselevel.cpp:235-283) for the samples lying in slices
 * z_base..z_base+n_slices-1 of the noise handle's stack, read from slab (those
 * slices only, x fastest; host or device memory by on_device). Draws the
 * sample positions on the first call. patchstd_host receives one value per
 * drawn sample (n_values >= the count inlm_noise_samples reports): the
 * slab's samples get their std, all others 0, so that a sum over ranks
 * holding disjoint slabs yields every sample's std. */
int inlm_noise_patchstd_slab(inlm_noise* n, const inlm_params* p, const float* slab, int on_device,
                             int z_base, int n_slices, float* patchstd_host, uint64_t n_values);

/* The rest of get_noiselevel (noiselevel.cpp:9-95) for given patch stds
 * (host, one per drawn sample): the two-cluster EM of the mode, or the
 * semimanual / manual choice, into sigma_out (nz floats, host). Each call
 * counts as one estimate of the handle, as inlm_noise_estimate does. */
int inlm_noise_estimate_from_patchstd(inlm_noise* n, inlm_params* p, const float* patchstd_host,
                                      uint64_t n_values, float* sigma_out);

/* ---------------- TIFF sequence IO (hdcom::HdCommunication) ----------------
 * Uncompressed baseline TIFF without libtiff: greyscale slices of 8, 16 or 32
 * bits per sample (and 64-bit float), in strips, either byte order. path is a
 * directory of .tif / .tiff slice files, taken in sorted name order, or one
 * .tif / .tiff file whose pages are the slices (an ImageJ stack stored as one
 * directory with "images=N" included). Compressed, tiled and multi-sample
 * files return INLM_ERR_UNSUPPORTED; missing paths INLM_ERR_IO. */

/* GetFilelist_And_ImageSequenceDimensions (Geometry/hdcommunication.cpp:51):
 * shape receives {width, height, slices}; samples_per_pixel (nullable) the
 * first slice's samples per pixel. */
int inlm_tiff_shape(const char* path, int shape[3], int* samples_per_pixel);

/* Get3DTifSequence_32bitPointer (hdcommunication.cpp:975, :1022) and
 * GetTif_unknowndim_32bit (:106): slices first_slice..last_slice (inclusive,
 * clamped to the stack; -1, -1 = all) into out, x fastest; n_out is the
 * number of floats out holds. Integer samples convert by value (8- and
 * 16-bit unsigned as the reference reads them), IEEE samples as stored. */
int inlm_tiff_read(const char* path, int first_slice, int last_slice, float* out, uint64_t n_out);

/* SaveTifSequence_32bit / SaveTifSequence_as16bit (hdcommunication.cpp:1576,
 * :1602): shape[2] slices written as dir/<name><z0+i, 4 digits>.tif, dir
 * created as needed; 32-bit IEEE float, or with as_16bit unsigned 16-bit after
 * min(max(0, round(v)), 65535) (:1472). Strips of max(1, 2048 / width) rows. */
int inlm_tiff_write_sequence(const float* image, const int shape[3], int z0, const char* dir,
                             const char* name, int as_16bit);

/* ---------------- colour (2D RGB) path ----------------
 * color_denoise::run_colorimage_denoising (Color/color_denoising.h:19-150) for
 * one image: optional Anscombe transform 2 sqrt(v + 3/8) (colorspace.h:83-103),
 * noise per channel (NoiseLevel::get_noiselevel_2D_RGB, noiselevel.cpp:96-191),
 * optionally averaged over the channels, iterations of the three-channel
 * filter (IterativeNLM_CPU::Run_GaussianNoise_3channels, iternlm_cpu.cpp:272;
 * filterslice_3channels, :932-1075): one weight per search offset from the
 * mean of the three channels' patch distances, or one per channel with
 * independent_channels; the sigma of each later iteration is
 * alpha * sigma + (1 - alpha) * (the estimate on the previous result). */
typedef struct {
    int stabilize_variance;    /* Anscombe transform (reference default 1; --nopoisson: 0) */
    int independent_channels;  /* --independent */
    int average_channelsigma;  /* one sigma for all channels (default 1; --noaverage: 0) */
} inlm_color_params;

/* Called after each iteration with that iteration's result as the reference
 * saves it (inverse-transformed planes, host memory valid during the call).
 * Passing a callback also reproduces what the reference does to its buffers
 * around such a save under the transform (inverse, then forward again, in
 * place), so results equal the reference run that saves every iteration
 * (no --cleanup); pass NULL for the --cleanup run. */
typedef void (*inlm_rgb_iteration_fn)(int iter, const float* r, const float* g, const float* b,
                                      void* user);

/* r, g, b: nx*ny host planes (values as read, 0..255 for 8-bit images);
 * out_*: the final result, inverse-transformed, not clamped. p supplies the x
 * and y search / patch radii, alpha, beta, maxiterations, the noise knobs
 * (z-adaptive acts as global on one image; the reference driver passes
 * n_samples = 2048), noise_seed and device_id; z radii and nslices are
 * forced to 0 and 1. sigma_first / sigma_last (nullable, 3 floats) receive the
 * initial estimate and the sigma of the last iteration. */
int inlm_rgb_denoise(int nx, int ny, const inlm_params* p, const inlm_color_params* color,
                     const float* r, const float* g, const float* b, float* out_r, float* out_g,
                     float* out_b, inlm_rgb_iteration_fn on_iteration, void* user,
                     float sigma_first[3], float sigma_last[3]);

/* GetRGBTif_32bitChannels (hdcommunication.cpp:674): an 8- or 16-bit RGB(A)
 * TIFF into three float planes (alpha ignored); shape receives {nx, ny}; with
 * r = g = b = NULL only the shape is read. */
int inlm_tiff_read_rgb(const char* file, int shape[2], float* r, float* g, float* b, uint64_t n_out);

/* Save2DTifImage_RGB (hdcommunication.cpp:1487) of three float planes as
 * dir/<name>.tif, 8-bit interleaved, each value as (uint8_t) min(255, v)
 * (color_denoising.h:76-78), values below 0 as 0. */
int inlm_tiff_write_rgb(const char* dir, const char* name, const float* r, const float* g,
                        const float* b, int nx, int ny);

#ifdef __cplusplus
}
#endif
#endif /* INLM_H */
