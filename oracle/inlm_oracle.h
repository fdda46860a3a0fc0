/*
 * inlm_oracle — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference iterNLM_v0.3 algorithms on the hot
 * path: geometry tables, reflective padding, the per-voxel NLM filter (FP32
 * exactly as the reference CPU computes it, and an FP64 form), and the noise
 * estimators (glibc rand() sampling, 15x15 patch std, two-cluster EM, z
 * windows). Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it, as the checker. The product library never links it.
 *
 * Parity pin: every function here is checked bit-for-bit against the
 * reference's own CPU code compiled from its sources (oracle/_ref, built by
 * oracle/Makefile) in tests/test_oracle_pin.py, and against golden fixtures
 * generated from that build (tests/golden/).
 */
#ifndef INLM_ORACLE_H
#define INLM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int search_radius[3];
    int patch_radius[3];
    int nslices;
    float beta;
    float z_anisotropy;
} ora_params;

/* padding = {sr_x+pr_x, sr_y+pr_y, min(nslices/2, sr_z)+pr_z} both sides
 * (iternlm_cpu.cpp:18-23). */
void ora_padding(const ora_params* p, int pad[3]);

/* Search offsets in reference order (iternlm_prepare.cpp:102-150): z, y, x
 * ascending, float32 ellipsoid test, |z| <= nslices/2, centre excluded. */
int ora_search_offsets(const ora_params* p, int* dx, int* dy, int* dz, int max_n);

/* Patch taps (iternlm_prepare.cpp:152-202): centre first, then z, y, x
 * ascending, float32 ellipsoid test, |z| <= nslices/2. */
int ora_patch_taps(const ora_params* p, int* dx, int* dy, int* dz, int max_n);

/* setup_distweight (iternlm_prepare.cpp:204-262): 1/(2d+1)^2, tap 0 = max,
 * all 1/7 for radius (1,1,1) when nz > 1. Returns the tap count. */
int ora_distweight(const ora_params* p, int nz, float* w, int max_n);

/* Weights the reference CPU filter actually applies (iternlm_cpu.cpp:97-114):
 * the eight specialised kernels (iternlm_cpu_kernels.cpp) hold the distweight
 * table printed with 6 significant digits ("%g"), p111 holds float(1/7);
 * every other patch shape goes to the generic filterslice with distweight.
 * Returns the tap count; *specialised is set to 1 for the eight shapes. */
int ora_filter_weights(const ora_params* p, int nz, float* w, int max_n, int* specialised);

/* Reflective padding without edge repeat (iternlm_prepare.cpp:6-48). */
void ora_pad_reflective(const float* in, const int shape[3], const int pad[3], float* out);

/* One filter iteration over padded raw/prev, FP32 with the reference's
 * operation order (iternlm_cpu_kernels.cpp:7-99 and iternlm_cpu.cpp:758-843).
 * mult[z] = -1/(sigma[z]^2 beta). out is unpadded. */
void ora_filter_f32(const float* raw_pad, const float* prev_pad, const int shape[3],
                    const ora_params* p, const float* mult, float* out);

/* Same algorithm with every quantity in double (weights from the same table,
 * Pade[3/3] with the same cutoff). */
void ora_filter_f64(const double* raw_pad, const double* prev_pad, const int shape[3],
                    const ora_params* p, const double* mult, double* out);

/* n_iter iterations (IterativeNLM_CPU::Run_GaussianNoise, iternlm_cpu.cpp:8):
 * iteration k uses sigmas[(k-1)*nz ...]. out_all (nullable) gets every iterate. */
void ora_denoise_f32(const float* raw, const int shape[3], const ora_params* p,
                     const float* sigmas, int n_iter, float* out_last, float* out_all);
void ora_denoise_f64(const float* raw, const int shape[3], const ora_params* p,
                     const float* sigmas, int n_iter, double* out_last);

/* ora_denoise_f64 with the search restricted per tile (tile[0] x tile[1] x
 * tile[2] voxels, x-fastest tile index) to offsets with keep[tile*S + s] set.
 * Iteration k reads keep + (k-1)*keep_iter_stride (0: one table for all). */
void ora_denoise_f64_plan(const float* raw, const int shape[3], const ora_params* p,
                          const float* sigmas, int n_iter, const int tile[3],
                          const unsigned char* keep, long long keep_iter_stride, double* out_last);

/* Weight mass per tile and search offset of one iteration in FP64: each
 * voxel's offset weights (Pade + cutoff on m * patch distance over prev,
 * m = -1/(sigma[z]^2 beta)) divided by their sum, summed over the tile's
 * voxels, each tile row then normalised to sum 1 (rows of all-zero stay 0).
 * out: n_tiles x S. The training target of the learned offset proposal. */
void ora_weight_mass_f64(const float* prev, const int shape[3], const ora_params* p,
                         const float* sigma, const int tile[3], double* out);

/* ora_filter_f32 evaluated only at the given unpadded linear voxel indices
 * (sampled parity checks on full-size volumes). */
void ora_filter_f32_voxels(const float* raw_pad, const float* prev_pad, const int shape[3],
                           const ora_params* p, const float* mult, int64_t n,
                           const int64_t* voxels, float* out);

/* mult[z] = -1/(sigma[z]^2 beta) in float (iternlm_cpu.cpp:94-95). */
void ora_sigma_to_mult(const float* sigma, int nz, float beta, float* mult);

/* ---- noise estimation (Noise/noiselevel.cpp) ---- */

/* glibc random_r TYPE_3 (degree 31, separation 3) restated from its published
 * description: r[0]=seed, r[i]=16807*r[i-1] mod (2^31-1) for i<31,
 * r[i]=r[i-31] for i=31..33, r[i]=r[i-3]+r[i-31] mod 2^32 after, output
 * r[k+344]>>1. */
typedef struct { uint32_t r[34]; int k; } ora_rand_state;
void ora_srand(ora_rand_state* st, unsigned int seed);
int ora_rand(ora_rand_state* st);

/* drawsamples (noiselevel.cpp:192-234) with the sequential rand() order,
 * then sorted ascending. */
void ora_draw_samples(const int shape[3], int64_t n_samples, int patchsize,
                      int circular_mask_diameter, unsigned int seed, int64_t* out);

/* get_patchstd (noiselevel.cpp:235-283). */
void ora_patchstd(const float* stack, const int shape[3], const int64_t* samples, int64_t n,
                  int patchsize, float* out);

/* create2clusters (noiselevel.cpp:366-528), float accumulation exactly as the
 * reference; out = {mean, std}. first/last = -1 select the whole array. */
void ora_create2clusters_f32(const float* values, int n, int first, int last, float out[2]);

/* Same EM with the sums, counts and variances accumulated in double (the
 * device estimator's arithmetic); decisions use the reference formulas. */
void ora_create2clusters_f64acc(const float* values, int n, int first, int last, float out[2]);

/* z windows of create2clusters_zwindow (noiselevel.cpp:529-545):
 * start[z], end[z] inclusive sample ranges. */
void ora_zwindows(const int64_t* samples, int64_t n, const int shape[3], int windowsize,
                  int* start, int* end);

/* Neighbour fill of empty slices (noiselevel.cpp:571-603), in place on
 * mean[nz], sd[nz]. */
void ora_fill_empty_slices(float* mean, float* sd, int nz);

/* Whole get_noiselevel for modes 0 = global, 1 = z-adaptive over given
 * patch stds; f64acc selects the EM arithmetic. sigma: nz floats. */
void ora_noise_from_patchstd(const float* patchstd, const int64_t* samples, int64_t n,
                             const int shape[3], int mode, int zwindow, float stds_from_mean,
                             int f64acc, float* sigma);

/* colour path: the three-channel 2D filter and the Anscombe transforms */
void ora_filter_rgb(const float* const raw[3], const float* const prev[3], int nx, int ny,
                    const ora_params* p2d, const float mult[3], int independent, float* const out[3]);
void ora_anscombe(float* v, int64_t n, int inverse);

#ifdef __cplusplus
}
#endif
#endif
