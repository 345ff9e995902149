// common.cuh -- shared device types and helpers for the sm_100a MPS-TEBD engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tq {

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

__device__ __forceinline__ bool grid_sync(GridBar* bar, int* status, unsigned int nblocks,
                                          uint64_t budget_ns = 2000000000ull) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned int* vgen = &bar->gen;
        const unsigned int g = *vgen;
        __threadfence();
        const unsigned int arrived = atomicAdd(&bar->count, 1u);
        if (arrived == nblocks - 1) {
            bar->count = 0;
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            const uint64_t t0 = globaltimer_ns();
            unsigned int spins = 0;
            while (*vgen == g) {
                if ((++spins & 63u) == 0 && globaltimer_ns() - t0 > budget_ns) {
                    atomicOr(status, ST_BARRIER_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        if (ok && (*(volatile int*)status & ST_BARRIER_TIMEOUT)) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Warp-level sum with shuffles.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace tq
