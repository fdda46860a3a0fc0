// Shared device helpers: TMA / mbarrier inline PTX, exact-rounding float ops,
// bounded waits, error flag.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace inlm {

// Device error codes written to the per-handle error word.
enum DeviceError : int {
    DEV_OK = 0,
    DEV_TMA_TIMEOUT = 1,
    DEV_QUEUE_TIMEOUT = 2,
    DEV_BAD_ITEM = 3,
};

// Cycles a bounded wait may spin before it gives up (~1 s at 1.9 GHz).
constexpr long long kWaitCycles = 2000000000LL;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Plain arrival (release semantics for the thread's prior shared-memory
// writes; a waiter's completed try_wait acquires them).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Spins on the mbarrier phase with a cycle budget; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  long long budget = kWaitCycles) {
    long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > budget) return false;
    }
    return true;
}

// 3D tiled TMA load (no multicast), completion signalled on bar.
// x must be a multiple of 4 for 32-bit elements (16-byte rule).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* tm, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* tm) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tm)) : "memory");
}

__device__ __forceinline__ void set_error(int* flag, int code) {
    if (flag) atomicCAS(flag, 0, code);
}

// 3rd-order Pade approximation of exp(x) with the reference's hard cutoff
// (Denoiser/iternlm_cpu.h:125-126), with each operation rounded exactly as the
// C++ expression (120 + 60x + 12x*x + x*x*x) / (120 - 60x + 12x*x - x*x*x)
// rounds under IEEE single precision without contraction.
__device__ __forceinline__ float pade_weight_exact(float x) {
    float a = __fmul_rn(60.f, x);
    float b = __fmul_rn(__fmul_rn(12.f, x), x);
    float c = __fmul_rn(__fmul_rn(x, x), x);
    float num = __fadd_rn(__fadd_rn(__fadd_rn(120.f, a), b), c);
    float den = __fsub_rn(__fadd_rn(__fsub_rn(120.f, a), b), c);
    float w = __fdiv_rn(num, den);
    return (x > -3.56648f) ? w : 0.0f;
}

}  // namespace inlm
