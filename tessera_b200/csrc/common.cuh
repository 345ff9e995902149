// common.cuh -- shared device types and helpers for the sm_100a MPS-TEBD engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tq {

// Every device allocation of the library goes through here (engine.cu): cudaMalloc, except
// that tessera_qa_debug_fail_allocations(after, count) makes chosen calls fail with
// cudaErrorMemoryAllocation, so the out-of-memory paths can be tested without exhausting a GPU.
cudaError_t device_alloc(void** p, size_t bytes);

// ---------------------------------------------------------------------------------
// Complex arithmetic on interleaved (re, im) pairs.  T = double (complex128 mode) or
// float (complex64 mode).  Storage uses the CUDA vector types so loads are 16 / 8 byte
// vectorised.
// ---------------------------------------------------------------------------------
template <typename T> struct CT;
template <> struct CT<double> { using type = double2; };
template <> struct CT<float> { using type = float2; };
template <typename T> using cplx_t = typename CT<T>::type;

template <typename V> __host__ __device__ __forceinline__ V mk(decltype(V::x) re, decltype(V::x) im) {
    V v; v.x = re; v.y = im; return v;
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// acc += a * b
template <typename V> __device__ __forceinline__ void cfma(V& acc, V a, V b) {
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}
// acc += conj(a) * b
template <typename V> __device__ __forceinline__ void cfma_conj(V& acc, V a, V b) {
    acc.x = fma(a.x, b.x, fma(a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(-a.y, b.x, acc.y));
}
template <typename V> __host__ __device__ __forceinline__ V cscale(V a, decltype(V::x) s) {
    V r; r.x = a.x * s; r.y = a.y * s; return r;
}
template <typename V> __host__ __device__ __forceinline__ V czero() { V r; r.x = 0; r.y = 0; return r; }

// ---------------------------------------------------------------------------------
// Status bits shared by kernels and the host (tessera_qa_result.status).
// ---------------------------------------------------------------------------------
enum : int {
    ST_OK = 0,
    ST_JACOBI_NOT_CONVERGED = 1,   // sweep cap reached with rotations still above tol
    ST_BARRIER_TIMEOUT = 2,        // a bounded grid barrier gave up (should never happen)
    ST_BAD_DIMS = 4,               // a kernel saw bond dimensions outside capacity
    ST_NONFINITE = 8,              // NaN/Inf met in a reduction
};

// ---------------------------------------------------------------------------------
// Bounded grid barrier for cooperative launches.  Sense is carried by a generation
// counter; a waiting CTA gives up after `budget_ns` of %globaltimer, raises
// ST_BARRIER_TIMEOUT in *status and returns false.  Callers leave the kernel when it
// returns false (every CTA checks the flag after each barrier).
// ---------------------------------------------------------------------------------
struct GridBar {
    unsigned int count;
    unsigned int gen;
};

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool grid_sync(GridBar* bar, int* status, unsigned int nblocks,
                                          uint64_t budget_ns = 2000000000ull) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned int g = ld_acquire_u32(&bar->gen);
        __threadfence();
        const unsigned int arrived = atomicAdd(&bar->count, 1u);
        if (arrived == nblocks - 1) {
            bar->count = 0;
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            const uint64_t t0 = globaltimer_ns();
            unsigned int spins = 0;
            while (ld_acquire_u32(&bar->gen) == g) {
                if ((++spins & 255u) == 0 && globaltimer_ns() - t0 > budget_ns) {
                    atomicOr(status, ST_BARRIER_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (ok && (*(volatile int*)status & ST_BARRIER_TIMEOUT)) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ---------------------------------------------------------------------------------
// mbarrier + 1-D TMA bulk copies (cp.async.bulk, sm_90+; no tensor map, no multicast).
// ---------------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// global -> shared bulk copy completing on `bar`; dst/src 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for phase `parity` of `bar`; returns false after budget_ns.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, uint64_t budget_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    uint64_t t0 = 0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        uint64_t t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > budget_ns) return false;
    }
}
// Makes this thread's generic-proxy view of global memory consistent with async-proxy
// (TMA) accesses issued after it.
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

// Orders this thread's generic-proxy shared-memory accesses before async-proxy (TMA) writes
// into the same buffer that it issues after the fence.
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Warp-level sum with shuffles.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace tq
