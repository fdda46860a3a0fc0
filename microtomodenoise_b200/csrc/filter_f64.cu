// FP64 full-search form of the iterNLM filter on sub-blocks of a volume: the
// full-search FP64 result the precision and learned forms are measured
// against, at volume sizes where a CPU restatement cannot finish in time.
//
// Arithmetic: the reference's per-voxel algorithm (Denoiser/iternlm_cpu.cpp:
// 795-834) with every quantity in double, each product, sum and quotient
// rounded separately (__dmul_rn / __dadd_rn / __ddiv_rn) in the reference's
// order: dist += (t*t)*w per tap, dist *= m, Pade[3/3]
// (120 + 60x + 12x*x + x*x*x) / (120 - 60x + 12x*x - x*x*x) above the cutoff
// (double)-3.56648f, acc += w*raw, wsum += w, wmax = max; out = wmax > 0 ?
// (acc + wmax*raw0) / (wsum + wmax) : raw0. Iterates stay in double between
// iterations and m = -1/(sigma*sigma*beta) in double, as the FP64 restatement
// of the oracle does.
//
// Sub-blocks: iteration k of n runs on the block grown by (n - k) x the
// filter's padding per side (clipped to the volume), from iteration k - 1 on
// that box grown by one padding, so the last iteration's block equals the
// whole-volume result there. Positions outside the volume take the
// reference's reflective rule (-i below 0, 2n-i-2 above n-1,
// Denoiser/iternlm_prepare.cpp:6-48).
#include <cmath>
#include <vector>

#include "api_internal.hpp"
#include "geometry.hpp"

using namespace inlm;

namespace {

struct F64Args {
    const double* raw_pad;   // box + padding, [nz + 2 pz][ny + 2 py][nx + 2 px]
    const double* prev_pad;
    int nx, ny, nz;          // box interior
    int px, py, pz;          // padding
    const long long* soff;   // S search offsets as padded-index deltas
    int S;
    const long long* poff;   // P patch taps as padded-index deltas (tap 0 = centre)
    const double* w;         // P weights
    int P;
    const double* mult;      // per interior z
    double* out;             // box interior
};

__device__ __forceinline__ double pade_f64_rn(double x) {
    const double a = __dmul_rn(60.0, x);
    const double b = __dmul_rn(__dmul_rn(12.0, x), x);
    const double c = __dmul_rn(__dmul_rn(x, x), x);
    const double num = __dadd_rn(__dadd_rn(__dadd_rn(120.0, a), b), c);
    const double den = __dsub_rn(__dadd_rn(__dsub_rn(120.0, a), b), c);
    return __ddiv_rn(num, den);
}

__global__ void __launch_bounds__(128) nlm_f64_kernel(const F64Args a) {
    const long long n = (long long)a.nx * a.ny * a.nz;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int x = (int)(i % a.nx);
    const long long r = i / a.nx;
    const int y = (int)(r % a.ny);
    const int z = (int)(r / a.ny);
    const long long sy = a.nx + 2 * a.px, sz = sy * (a.ny + 2 * a.py);
    const long long idx0 = (z + a.pz) * sz + (y + a.py) * sy + (x + a.px);
    const double m = a.mult[z];
    const double raw0 = a.raw_pad[idx0];
    const double cut = (double)-3.56648f;
    double acc = 0.0, wsum = 0.0, wmax = 0.0;
    for (int s = 0; s < a.S; s++) {
        const long long idx1 = idx0 + a.soff[s];
        double dist = 0.0;
        for (int q = 0; q < a.P; q++) {
            const long long po = a.poff[q];
            const double t = __dsub_rn(a.prev_pad[idx1 + po], a.prev_pad[idx0 + po]);
            dist = __dadd_rn(dist, __dmul_rn(__dmul_rn(t, t), a.w[q]));
        }
        dist = __dmul_rn(dist, m);
        const double wt = (dist > cut) ? pade_f64_rn(dist) : 0.0;
        acc = __dadd_rn(acc, __dmul_rn(wt, a.raw_pad[idx1]));
        wsum = __dadd_rn(wsum, wt);
        if (wt > wmax) wmax = wt;
    }
    a.out[i] = (wmax > 0.0) ? __ddiv_rn(__dadd_rn(acc, __dmul_rn(wmax, raw0)), __dadd_rn(wsum, wmax)) : raw0;
}

// dst[z][y][x] = src[iz[z]][iy[y]][ix[x]] (src pitches sy, sz), as double.
template <typename T>
__global__ void __launch_bounds__(256) gather_f64_kernel(const T* __restrict__ src, long long sy, long long sz,
                                                         const int* __restrict__ ix, const int* __restrict__ iy,
                                                         const int* __restrict__ iz, int nx, int ny, int nz,
                                                         double* __restrict__ dst) {
    const long long n = (long long)nx * ny * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const long long r = i / nx;
        const int y = (int)(r % ny);
        const int z = (int)(r / ny);
        dst[i] = (double)src[iz[z] * sz + iy[y] * sy + ix[x]];
    }
}

int mirror(int i, int n) {
    for (int g = 0; g < 64 && (i < 0 || i > n - 1); g++) {
        if (i < 0) i = -i;
        if (i > n - 1) i = 2 * n - i - 2;
    }
    return std::min(std::max(i, 0), n - 1);
}

// Device buffers and the stream of one call, released on every return path.
struct Scratch {
    std::vector<void*> bufs;
    cudaStream_t st = nullptr;
    ~Scratch() {
        cudaStreamSynchronize(st);
        for (void* b : bufs) device_free(b);
        cudaStreamDestroy(st);
    }
    template <typename T>
    cudaError_t get(T** p, size_t n) {
        cudaError_t e = dalloc(p, n);
        if (e == cudaSuccess) bufs.push_back(*p);
        return e;
    }
};

struct Box {
    int lo[3], hi[3];  // x, y, z
    int n(int a) const { return hi[a] - lo[a]; }
};

}  // namespace

extern "C" int inlm_denoise_f64_blocks(const int shape[3], const inlm_params* p, const float* raw,
                                       int on_device, const float* sigmas, int n_iter, const int* corners,
                                       int n_blocks, const int size[3], double* out_host) {
    if (!shape || !p || !raw || !sigmas || !corners || !size || !out_host)
        return fail(INLM_ERR_ARG, "null argument");
    if (n_iter < 1 || n_blocks < 0) return fail(INLM_ERR_ARG, "n_iter must be >= 1, n_blocks >= 0");
    for (int a = 0; a < 3; a++) {
        if (shape[a] < 2 || size[a] < 1 || size[a] > shape[a])
            return fail(INLM_ERR_ARG, "shape and block size must be positive, blocks inside the volume");
        if (p->search_radius[a] < 0 || p->patch_radius[a] < 0) return fail(INLM_ERR_ARG, "radii must be >= 0");
    }
    for (int b = 0; b < n_blocks; b++)
        for (int a = 0; a < 3; a++)
            if (corners[3 * b + a] < 0 || corners[3 * b + a] + size[a] > shape[a])
                return fail(INLM_ERR_ARG, "block %d lies outside the volume", b);
    CUDA_TRY(cudaSetDevice(p->device_id));
    const int nx = shape[0], ny = shape[1], nz = shape[2];
    Geometry g0 = make_geometry(p->search_radius, p->patch_radius, p->nslices, p->z_anisotropy, 0, nz + 2);
    const int pad[3] = {g0.pad[0], g0.pad[1], g0.pad[2]};
    for (int a = 0; a < 3; a++)
        if (pad[a] >= shape[a]) return fail(INLM_ERR_ARG, "the padding exceeds an axis of the volume");
    cudaStream_t st;
    CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    Scratch S;
    S.st = st;
    // largest boxes: iteration 1's, grown by one padding
    auto box_of = [&](const int* c, int k) {  // iteration k (1..n_iter)
        Box b;
        const int grow = n_iter - k;
        for (int a = 0; a < 3; a++) {
            b.lo[a] = std::max(0, c[a] - grow * pad[a]);
            b.hi[a] = std::min(shape[a], c[a] + size[a] + grow * pad[a]);
        }
        return b;
    };
    size_t max_crop = 0, max_box = 0;
    for (int b = 0; b < n_blocks; b++) {
        Box b1 = box_of(corners + 3 * b, 1);
        max_crop = std::max(max_crop, (size_t)(b1.n(0) + 2 * pad[0]) * (b1.n(1) + 2 * pad[1]) * (b1.n(2) + 2 * pad[2]));
        max_box = std::max(max_box, (size_t)b1.n(0) * b1.n(1) * b1.n(2));
    }
    if (n_blocks == 0) return INLM_OK;
    // tables: search and patch deltas depend on the padded pitches of a box
    const int Sn = (int)g0.search.size(), Pn = (int)g0.taps.size();
    std::vector<double> wd(Pn);
    for (int q = 0; q < Pn; q++) wd[q] = (double)g0.weights[q];
    long long *d_soff, *d_poff;
    double *d_w, *d_mult, *d_rawpad, *d_prevpad, *d_res0, *d_res1, *d_crop1;
    int* d_idx;
    float* d_rawcrop = nullptr;
    const int maxdim = std::max(nx, std::max(ny, nz)) + 2 * std::max(pad[0], std::max(pad[1], pad[2]));
    CUDA_TRY(S.get(&d_soff, Sn));
    CUDA_TRY(S.get(&d_poff, Pn));
    CUDA_TRY(S.get(&d_w, Pn));
    CUDA_TRY(S.get(&d_mult, nz));
    CUDA_TRY(S.get(&d_rawpad, max_crop));
    CUDA_TRY(S.get(&d_prevpad, max_crop));
    CUDA_TRY(S.get(&d_crop1, max_crop));
    CUDA_TRY(S.get(&d_res0, max_box));
    CUDA_TRY(S.get(&d_res1, max_box));
    CUDA_TRY(S.get(&d_idx, 3 * (size_t)maxdim));
    if (!on_device) CUDA_TRY(S.get(&d_rawcrop, max_crop));
    CUDA_TRY(cudaMemcpyAsync(d_w, wd.data(), Pn * 8, cudaMemcpyHostToDevice, st));
    std::vector<float> hcrop(on_device ? 0 : max_crop);
    std::vector<int> hidx(3 * (size_t)maxdim);
    std::vector<long long> soff(Sn), poff(Pn);
    std::vector<double> mult(nz);
    std::vector<double> hout;
    const double beta = (double)p->beta;
    auto upload_idx = [&](const int* lo, const int* n, const int* base, bool mirrored) -> int {
        // index arrays of a crop: position i of axis a maps to
        // mirror(lo + i) - base (mirrored) or lo + i - base
        for (int a = 0; a < 3; a++)
            for (int i = 0; i < n[a]; i++) {
                const int c = lo[a] + i;
                hidx[a * maxdim + i] = (mirrored ? mirror(c, shape[a]) : c) - base[a];
            }
        CUDA_TRY(cudaMemcpyAsync(d_idx, hidx.data(), 3 * (size_t)maxdim * 4, cudaMemcpyHostToDevice, st));
        return INLM_OK;
    };
    for (int b = 0; b < n_blocks; b++) {
        const int* c = corners + 3 * b;
        const Box b1 = box_of(c, 1);
        const int clo[3] = {b1.lo[0] - pad[0], b1.lo[1] - pad[1], b1.lo[2] - pad[2]};
        const int cn[3] = {b1.n(0) + 2 * pad[0], b1.n(1) + 2 * pad[1], b1.n(2) + 2 * pad[2]};
        const size_t ncrop = (size_t)cn[0] * cn[1] * cn[2];
        // raw over iteration 1's box + padding, mirrored at the volume's faces
        const int zero[3] = {0, 0, 0};
        int rc;
        if (on_device) {
            rc = upload_idx(clo, cn, zero, true);
            if (rc) return rc;
            gather_f64_kernel<float><<<148 * 8, 256, 0, st>>>(raw, nx, (long long)nx * ny, d_idx, d_idx + maxdim,
                                                              d_idx + 2 * maxdim, cn[0], cn[1], cn[2], d_crop1);
            CUDA_TRY(cudaGetLastError());
        } else {
            CUDA_TRY(cudaStreamSynchronize(st));  // hcrop is reused
            for (int z = 0; z < cn[2]; z++)
                for (int y = 0; y < cn[1]; y++) {
                    const float* row = raw + ((long long)mirror(clo[2] + z, nz) * ny + mirror(clo[1] + y, ny)) * nx;
                    float* d = hcrop.data() + ((size_t)z * cn[1] + y) * cn[0];
                    for (int x = 0; x < cn[0]; x++) d[x] = row[mirror(clo[0] + x, nx)];
                }
            CUDA_TRY(cudaMemcpyAsync(d_rawcrop, hcrop.data(), ncrop * 4, cudaMemcpyHostToDevice, st));
            for (int a = 0; a < 3; a++)
                for (int i = 0; i < cn[a]; i++) hidx[a * maxdim + i] = i;
            CUDA_TRY(cudaMemcpyAsync(d_idx, hidx.data(), 3 * (size_t)maxdim * 4, cudaMemcpyHostToDevice, st));
            gather_f64_kernel<float><<<148 * 8, 256, 0, st>>>(d_rawcrop, cn[0], (long long)cn[0] * cn[1], d_idx,
                                                              d_idx + maxdim, d_idx + 2 * maxdim, cn[0], cn[1],
                                                              cn[2], d_crop1);
            CUDA_TRY(cudaGetLastError());
        }
        double* res_prev = d_res0;
        double* res_cur = d_res1;
        Box prev_box = b1;
        for (int k = 1; k <= n_iter; k++) {
            const Box bk = box_of(c, k);
            const int n3[3] = {bk.n(0), bk.n(1), bk.n(2)};
            const int lo[3] = {bk.lo[0] - pad[0], bk.lo[1] - pad[1], bk.lo[2] - pad[2]};
            const int pn[3] = {n3[0] + 2 * pad[0], n3[1] + 2 * pad[1], n3[2] + 2 * pad[2]};
            // raw: the sub-box of iteration 1's crop (the same mirrored positions)
            rc = upload_idx(lo, pn, clo, false);
            if (rc) return rc;
            gather_f64_kernel<double><<<148 * 8, 256, 0, st>>>(d_crop1, cn[0], (long long)cn[0] * cn[1], d_idx,
                                                               d_idx + maxdim, d_idx + 2 * maxdim, pn[0], pn[1],
                                                               pn[2], d_rawpad);
            CUDA_TRY(cudaGetLastError());
            const double* prevpad = d_rawpad;
            if (k > 1) {
                // the previous iterate over this box + padding, mirrored into the volume
                rc = upload_idx(lo, pn, prev_box.lo, true);
                if (rc) return rc;
                gather_f64_kernel<double><<<148 * 8, 256, 0, st>>>(res_prev, prev_box.n(0),
                                                                   (long long)prev_box.n(0) * prev_box.n(1), d_idx,
                                                                   d_idx + maxdim, d_idx + 2 * maxdim, pn[0], pn[1],
                                                                   pn[2], d_prevpad);
                CUDA_TRY(cudaGetLastError());
                prevpad = d_prevpad;
            }
            // padded-index deltas for this box's pitches
            const long long sy = pn[0], sz = (long long)pn[0] * pn[1];
            for (int s = 0; s < Sn; s++) soff[s] = g0.search[s].z * sz + g0.search[s].y * sy + g0.search[s].x;
            for (int q = 0; q < Pn; q++) poff[q] = g0.taps[q].z * sz + g0.taps[q].y * sy + g0.taps[q].x;
            for (int z = 0; z < n3[2]; z++) {
                const double s = (double)sigmas[(size_t)(k - 1) * nz + bk.lo[2] + z];
                mult[z] = -1.0 / (s * s * beta);
            }
            CUDA_TRY(cudaStreamSynchronize(st));  // the host tables are rewritten below
            CUDA_TRY(cudaMemcpyAsync(d_soff, soff.data(), Sn * 8, cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaMemcpyAsync(d_poff, poff.data(), Pn * 8, cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaMemcpyAsync(d_mult, mult.data(), n3[2] * 8, cudaMemcpyHostToDevice, st));
            F64Args a{d_rawpad, prevpad, n3[0], n3[1], n3[2], pad[0], pad[1], pad[2], d_soff, Sn,
                      d_poff, d_w, Pn, d_mult, res_cur};
            const long long nv = (long long)n3[0] * n3[1] * n3[2];
            nlm_f64_kernel<<<(unsigned)((nv + 127) / 128), 128, 0, st>>>(a);
            CUDA_TRY(cudaGetLastError());
            std::swap(res_prev, res_cur);
            prev_box = bk;
        }
        // the block out of the last box (which is the block itself)
        const Box bn = prev_box;
        hout.resize((size_t)bn.n(0) * bn.n(1) * bn.n(2));
        CUDA_TRY(cudaMemcpyAsync(hout.data(), res_prev, hout.size() * 8, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        double* o = out_host + (size_t)b * size[0] * size[1] * size[2];
        for (int z = 0; z < size[2]; z++)
            for (int y = 0; y < size[1]; y++)
                for (int x = 0; x < size[0]; x++)
                    o[((size_t)z * size[1] + y) * size[0] + x] =
                        hout[((size_t)(c[2] - bn.lo[2] + z) * bn.n(1) + (c[1] - bn.lo[1] + y)) * bn.n(0) +
                             (c[0] - bn.lo[0] + x)];
    }
    return INLM_OK;
}
