// Noise-level estimators on the device (Noise/noiselevel.cpp).
//
//  * patch std: one thread per sample, the 15x15 sums accumulated in the
//    reference's order in float (noiselevel.cpp:235-283), so every per-sample
//    std equals the reference's bit for bit.
//  * two-cluster hard EM (noiselevel.cpp:366-528): one CTA per z window
//    (z-adaptive) or one CTA over all samples (global). The per-sample
//    decisions use the reference's formulas; the cluster sums, counts and
//    variances are block reductions accumulated in FP64 (warp shuffles, then
//    shared memory). Assignments persist in a global int8 scratch array.
//  * neighbour fill of empty windows (noiselevel.cpp:571-603) and
//    sigma = mean + shift*std, sequential in one thread (nz is small).
#include <mutex>

#include "common.cuh"
#include "noise_kernels.cuh"

namespace inlm {

__global__ void __launch_bounds__(256) noise_patchstd_kernel(const float* __restrict__ stack,
                                                             long long pitch_y, long long pitch_z,
                                                             int nx, long long nslice,
                                                             const long long* __restrict__ samples,
                                                             long long n, int patchsize,
                                                             float* __restrict__ out, int z_base) {
    long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= n) return;
    long long idx = samples[s];
    // stack holds slices z_base.. (a z-slab of the volume, or all of it)
    int z0 = (int)(idx / nslice);
    idx -= (long long)z_base * nslice;
    z0 -= z_base;
    int y0 = (int)((idx - z0 * nslice) / nx);
    int x0 = (int)(idx - z0 * nslice - (long long)y0 * nx);
    const int patchlength = patchsize * patchsize;
    float sum = 0.0f;
    for (int y = y0; y < y0 + patchsize; y++) {
        const float* row = stack + z0 * pitch_z + (long long)y * pitch_y + x0;
        for (int x = 0; x < patchsize; x++) sum = __fadd_rn(sum, row[x]);
    }
    float mean = __fdiv_rn(sum, (float)patchlength);
    float sq = 0.0f;
    for (int y = y0; y < y0 + patchsize; y++) {
        const float* row = stack + z0 * pitch_z + (long long)y * pitch_y + x0;
        for (int x = 0; x < patchsize; x++) {
            float d = __fsub_rn(row[x], mean);
            sq = __fadd_rn(sq, __fmul_rn(d, d));
        }
    }
    out[s] = __fsqrt_rn(__fdiv_rn(sq, (float)patchlength));
}

// Gaussian membership as written at noiselevel.cpp:456-457: 1./sqrtf(...) is a
// double division and the product is rounded to float.
__device__ __forceinline__ float cluster_prob(float v, float mean, float var) {
    const float PI = 3.141592654f;
    float d = __fsub_rn(v, mean);
    float q = __fdiv_rn(__fmul_rn(d, d), __fmul_rn(2.f, var));
    float e = expf(-q);
    double inv = __ddiv_rn(1.0, (double)__fsqrt_rn(__fmul_rn(__fmul_rn(var, 2.f), PI)));
    return __double2float_rn(__dmul_rn(inv, (double)e));
}

constexpr int kEmThreads = 256;

struct EmRed {
    double s1, s2;
    long long n1, n2;
};

// Block-wide sum of (s1, s2, n1, n2) and OR of flag; result broadcast to all
// NT threads.
template <int NT>
__device__ __forceinline__ void block_reduce(EmRed& r, int& flag, EmRed* sh, int* shflag) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        r.s1 += __shfl_down_sync(0xffffffffu, r.s1, o);
        r.s2 += __shfl_down_sync(0xffffffffu, r.s2, o);
        r.n1 += __shfl_down_sync(0xffffffffu, r.n1, o);
        r.n2 += __shfl_down_sync(0xffffffffu, r.n2, o);
    }
    int any = __any_sync(0xffffffffu, flag);
    __syncthreads();
    if (lane == 0) {
        sh[warp] = r;
        shflag[warp] = any;
    }
    __syncthreads();
    if (warp == 0) {
        constexpr int NW = NT / 32;
        EmRed t = (lane < NW) ? sh[lane] : EmRed{0.0, 0.0, 0, 0};
        int f = (lane < NW) ? shflag[lane] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            t.s1 += __shfl_down_sync(0xffffffffu, t.s1, o);
            t.s2 += __shfl_down_sync(0xffffffffu, t.s2, o);
            t.n1 += __shfl_down_sync(0xffffffffu, t.n1, o);
            t.n2 += __shfl_down_sync(0xffffffffu, t.n2, o);
        }
        f = __any_sync(0xffffffffu, f);
        if (lane == 0) {
            sh[0] = t;
            shflag[0] = f;
        }
    }
    __syncthreads();
    r = sh[0];
    flag = shflag[0];
    __syncthreads();
}

// Two-cluster EM over values[fs..ls] by one CTA of NT threads; asg[i] holds
// sample i's cluster (-1 excluded, 0, 1). Writes out_mean[w], out_sd[w].
template <int NT>
__device__ __forceinline__ void em_window(const float* __restrict__ values, int fs, int ls,
                                          signed char* __restrict__ asg, int w,
                                          float* __restrict__ out_mean,
                                          float* __restrict__ out_sd) {
    __shared__ EmRed sh[NT / 32];
    __shared__ int shflag[NT / 32];
    __shared__ float shmin[NT / 32], shmax[NT / 32];
    // assignments indexed by sample id
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // min / max (noiselevel.cpp:384-390)
    float mn = 1e20f, mx = -1e20f;
    for (int i = fs + tid; i <= ls; i += NT) {
        float v = values[i];
        mn = fminf(mn, v);
        mx = fmaxf(mx, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_down_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_down_sync(0xffffffffu, mx, o));
    }
    if (lane == 0) {
        shmin[warp] = mn;
        shmax[warp] = mx;
    }
    __syncthreads();
    mn = 1e20f;
    mx = -1e20f;
    for (int q = 0; q < NT / 32; q++) {
        mn = fminf(mn, shmin[q]);
        mx = fmaxf(mx, shmax[q]);
    }
    float range = __fsub_rn(mx, mn);
    float mean1 = __double2float_rn(__dadd_rn((double)mn, __dmul_rn(0.25, (double)range)));
    float mean2 = __double2float_rn(__dsub_rn((double)mx, __dmul_rn(0.25, (double)range)));

    // initial assignment, zero values excluded (noiselevel.cpp:398-423)
    EmRed r{0.0, 0.0, 0, 0};
    int flag = 0;
    for (int i = fs + tid; i <= ls; i += NT) {
        float v = values[i];
        signed char a;
        if (v == 0.0f) {
            a = -1;
        } else if (fabsf(__fsub_rn(v, mean1)) < fabsf(__fsub_rn(v, mean2))) {
            a = 0;
            r.s1 += (double)v;
            r.n1++;
        } else {
            a = 1;
            r.s2 += (double)v;
            r.n2++;
        }
        asg[i] = a;
    }
    block_reduce<NT>(r, flag, sh, shflag);
    if (r.n1 > 0) mean1 = __double2float_rn(r.s1 / (double)r.n1);
    if (r.n2 > 0) mean2 = __double2float_rn(r.s2 / (double)r.n2);
    if (r.n1 == 0 && r.n2 == 0) {
        if (tid == 0) {
            out_mean[w] = 0.0f;
            out_sd[w] = 0.0f;
        }
        return;
    }
    long long n1 = r.n1, n2 = r.n2;

    // cluster variances (noiselevel.cpp:428-443)
    auto variances = [&](float m1, float m2, float& v1, float& v2) {
        EmRed q{0.0, 0.0, 0, 0};
        int f = 0;
        for (int i = fs + tid; i <= ls; i += NT) {
            float v = values[i];
            signed char a = asg[i];
            if (a == 0) {
                float d = __fsub_rn(v, m1);
                q.s1 += (double)__fmul_rn(d, d);
            } else if (a == 1) {
                float d = __fsub_rn(v, m2);
                q.s2 += (double)__fmul_rn(d, d);
            }
        }
        block_reduce<NT>(q, f, sh, shflag);
        v1 = __double2float_rn(q.s1 / (double)(n1 > 1 ? n1 : 1));
        v2 = __double2float_rn(q.s2 / (double)(n2 > 1 ? n2 : 1));
    };
    __syncthreads();  // assignments visible to all threads
    float var1, var2;
    variances(mean1, mean2, var1, var2);

    // hard EM, at most 1000 passes (noiselevel.cpp:445-521)
    int change = 1;
    int iters = 0;
    while (change && var1 > 0.0f && var2 > 0.0f) {
        change = 0;
        iters++;
        EmRed q{0.0, 0.0, 0, 0};
        int f = 0;
        for (int i = fs + tid; i <= ls; i += NT) {
            float v = values[i];
            if (v == 0.0f) continue;
            float p1 = cluster_prob(v, mean1, var1);
            float p2 = cluster_prob(v, mean2, var2);
            signed char a = asg[i];
            if (p2 > p1) {
                if (a != 1) {
                    f = 1;
                    asg[i] = 1;
                }
                q.s2 += (double)v;
                q.n2++;
            } else {
                if (a != 0) {
                    f = 1;
                    asg[i] = 0;
                }
                q.s1 += (double)v;
                q.n1++;
            }
        }
        block_reduce<NT>(q, f, sh, shflag);
        change = f;
        n1 = q.n1;
        n2 = q.n2;
        if (n1 > 0) mean1 = __double2float_rn(q.s1 / (double)n1);
        if (n2 > 0) mean2 = __double2float_rn(q.s2 / (double)n2);
        variances(mean1, mean2, var1, var2);
        if (iters == 1000) break;
    }
    if (tid == 0) {
        if (mean1 <= mean2 || var2 <= 0.0f) {
            out_mean[w] = mean1;
            out_sd[w] = __fsqrt_rn(var1);
        } else {
            out_mean[w] = mean2;
            out_sd[w] = __fsqrt_rn(var2);
        }
    }
}

template <int NT>
__global__ void __launch_bounds__(NT) noise_em_kernel(const float* __restrict__ values,
                                                      const int2* __restrict__ windows,
                                                      const long long* __restrict__ scratch_off,
                                                      signed char* __restrict__ assign_scratch,
                                                      float* __restrict__ out_mean,
                                                      float* __restrict__ out_sd) {
    const int w = blockIdx.x;
    const int fs = windows[w].x, ls = windows[w].y;
    em_window<NT>(values, fs, ls, assign_scratch + scratch_off[w] - fs, w, out_mean, out_sd);
}

// ---- allocation-free EM: scratch in file-scope device arrays ----
//
// For callers that cannot allocate device memory. The cluster-assignment
// scratch (one byte per sample per window) and the window table live in
// static device arrays that every GPU loading this library holds until the
// process exits: 16 MiB + 256 KiB. Every call on a device shares them and
// leaves the last call's contents behind; calls whose work overlaps on the
// GPU (different streams, or different host threads) race on them.
// Nothing needs clearing between calls: the EM writes every assignment of a
// window (its initial pass) before it reads any, and every call rewrites the
// window-table entries it uses.
// The window table reaches the device inside kernel launch parameters (a
// small copy kernel per 1024 windows), so a call enqueues kernels only: no
// host-to-device copy from pageable memory and no wait on the host.
struct NoAllocWindow {
    int first, last;     // inclusive sample range (last < first: empty)
    long long offset;    // byte offset of the window's assignments in the scratch
};

static __device__ __align__(256) signed char g_noalloc_assign[kNoAllocAssignBytes];
static __device__ __align__(256) NoAllocWindow g_noalloc_windows[kNoAllocMaxWindows];

constexpr int kNoAllocChunk = 1024;  // windows per launch-parameter block (16 KiB)
struct NoAllocTableChunk {
    int base, count;
    NoAllocWindow win[kNoAllocChunk];
};

__global__ void __launch_bounds__(256) noalloc_table_kernel(const __grid_constant__ NoAllocTableChunk c,
                                                            NoAllocWindow* __restrict__ table) {
    for (int i = threadIdx.x; i < c.count; i += blockDim.x) table[c.base + i] = c.win[i];
}

__global__ void __launch_bounds__(kEmThreads) noise_em_noalloc_kernel(
    const float* __restrict__ values, const NoAllocWindow* __restrict__ windows,
    signed char* __restrict__ assign_scratch, float* __restrict__ out_mean,
    float* __restrict__ out_sd) {
    const int w = blockIdx.x;
    const NoAllocWindow win = windows[w];
    em_window<kEmThreads>(values, win.first, win.last, assign_scratch + win.offset - win.first, w,
                          out_mean, out_sd);
}

// Device addresses of the two arrays, looked up once per device with that
// device current (host code must not use the symbols themselves: they are
// host-side stand-ins, not device addresses).
struct NoAllocPtrs {
    bool ready = false;
    signed char* assign = nullptr;
    NoAllocWindow* windows = nullptr;
};
static NoAllocPtrs g_noalloc_ptrs[kNoAllocMaxDevices];
static std::mutex g_noalloc_mutex;

static cudaError_t noalloc_setup(int device, NoAllocPtrs* out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoAllocPtrs& p = g_noalloc_ptrs[device];
    if (!p.ready) {
        int cur = -1;
        cudaError_t e = cudaGetDevice(&cur);
        if (e != cudaSuccess) return e;
        if (cur != device) return cudaErrorInvalidDevice;
        e = cudaGetSymbolAddress((void**)&p.assign, g_noalloc_assign);
        if (e != cudaSuccess) return e;
        e = cudaGetSymbolAddress((void**)&p.windows, g_noalloc_windows);
        if (e != cudaSuccess) return e;
        p.ready = true;
    }
    *out = p;
    return cudaSuccess;
}

cudaError_t launch_noise_em_noalloc(int device, const float* values, const long long* windows_host,
                                    int n_windows, float* out_mean, float* out_sd,
                                    cudaStream_t st) {
    if (n_windows <= 0) return cudaSuccess;
    if (device < 0 || device >= kNoAllocMaxDevices || n_windows > kNoAllocMaxWindows)
        return cudaErrorInvalidValue;
    NoAllocPtrs ptrs;
    cudaError_t e = noalloc_setup(device, &ptrs);
    if (e != cudaSuccess) return e;
    // the chunk is copied into the launch parameters when the kernel is enqueued
    static thread_local NoAllocTableChunk chunk;
    long long offset = 0;
    for (int base = 0; base < n_windows; base += kNoAllocChunk) {
        const int cnt = n_windows - base < kNoAllocChunk ? n_windows - base : kNoAllocChunk;
        chunk.base = base;
        chunk.count = cnt;
        for (int i = 0; i < cnt; i++) {
            const long long f = windows_host[2 * (base + i)], l = windows_host[2 * (base + i) + 1];
            NoAllocWindow& w = chunk.win[i];
            if (l < f) {  // empty: stored as 0..-1 whatever the caller's values
                w.first = 0;
                w.last = -1;
            } else {
                w.first = (int)f;
                w.last = (int)l;
            }
            w.offset = offset;
            offset += (long long)w.last - w.first + 1;
        }
        noalloc_table_kernel<<<1, 256, 0, st>>>(chunk, ptrs.windows);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    noise_em_noalloc_kernel<<<n_windows, kEmThreads, 0, st>>>(values, ptrs.windows, ptrs.assign,
                                                              out_mean, out_sd);
    return cudaGetLastError();
}

// Neighbour fill (z-adaptive) and sigma = mean + shift*sd, single thread.
__global__ void noise_finalize_kernel(float* __restrict__ mean, float* __restrict__ sd, int nz,
                                      int zadaptive, float shift, float* __restrict__ sigma) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (!zadaptive) {
        float s = __fadd_rn(mean[0], __fmul_rn(shift, sd[0]));
        for (int z = 0; z < nz; z++) sigma[z] = s;
        return;
    }
    float max_std = -1.f;
    int zero = 0;
    for (int i = 0; i < nz; i++) {
        if (mean[i] > max_std) max_std = mean[i];
        if (mean[i] == 0.0f) zero = 1;
    }
    if (zero && max_std > 0.0f) {
        // every sweep fills at least one more slice next to a filled one
        for (int sweep = 0; zero && sweep <= nz; sweep++) {
            zero = 0;
            for (int i = 0; i < nz; i++) {
                float this_var = mean[i];
                if (this_var == 0.0f) {
                    float nv = 0.0f, nvs = 0.0f;
                    int count = 0;
                    if (i > 0 && mean[i - 1] > 0.0f) {
                        nv = __fadd_rn(nv, mean[i - 1]);
                        nvs = __fadd_rn(nvs, sd[i - 1]);
                        count++;
                    }
                    if (i < nz - 1 && mean[i + 1] > 0.0f) {
                        nv = __fadd_rn(nv, mean[i + 1]);
                        nvs = __fadd_rn(nvs, sd[i + 1]);
                        count++;
                    }
                    if (count > 0) {
                        this_var = __fdiv_rn(nv, (float)count);
                        mean[i] = this_var;
                        sd[i] = __fdiv_rn(nvs, (float)count);
                    }
                }
                if (this_var == 0.0f) zero = 1;
            }
        }
    }
    for (int z = 0; z < nz; z++) sigma[z] = __fadd_rn(mean[z], __fmul_rn(shift, sd[z]));
}

cudaError_t launch_noise_patchstd(const float* stack, long long pitch_y, long long pitch_z, int nx,
                                  long long nslice, const long long* samples, long long n,
                                  int patchsize, float* out, cudaStream_t st, int z_base) {
    if (n <= 0) return cudaSuccess;
    if (n <= 0) return cudaSuccess;
    noise_patchstd_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
        stack, pitch_y, pitch_z, nx, nslice, samples, n, patchsize, out, z_base);
    return cudaGetLastError();
}

cudaError_t launch_noise_em(const float* values, const int2* windows, int n_windows,
                            const long long* scratch_off, signed char* scratch, float* out_mean,
                            float* out_sd, cudaStream_t st, long long mean_window) {
    if (n_windows <= 0) return cudaSuccess;
    // long windows (few of them, e.g. a global estimate or a short stack) get
    // 1024 threads each so one CTA per window still keeps an SM busy
    if (mean_window >= kEmWideWindow)
        noise_em_kernel<1024><<<n_windows, 1024, 0, st>>>(values, windows, scratch_off, scratch,
                                                          out_mean, out_sd);
    else
        noise_em_kernel<kEmThreads><<<n_windows, kEmThreads, 0, st>>>(values, windows, scratch_off,
                                                                      scratch, out_mean, out_sd);
    return cudaGetLastError();
}

cudaError_t launch_noise_finalize(float* mean, float* sd, int nz, int zadaptive, float shift,
                                  float* sigma, cudaStream_t st) {
    noise_finalize_kernel<<<1, 32, 0, st>>>(mean, sd, nz, zadaptive, shift, sigma);
    return cudaGetLastError();
}

}  // namespace inlm
