// theta_tc.cu -- K1t: the complex64 bond contraction on the 5th-generation tensor cores.
//
//   T_{s1 s2}[a, b] = sum_c A[(2a+s1), c] C[(2c+s2), b]        (cuda/src/mps.cpp:46-70)
//   theta[(2a+r1), (r2 dr + b)] = sum_{s1 s2} G[r1 r2][s1 s2] T_{s1 s2}[a, b]
//
// as real GEMMs on tcgen05.mma (kind::tf32) with FP32 accumulators in tensor memory, in
// split-TF32: every FP32 operand x is split into hi = tf32(x) and lo = tf32(x - hi), and
// D = A_hi B_hi + A_hi B_lo + A_lo B_hi (three passes), which keeps about FP32 accuracy.
// Complex arithmetic by stacking the real and imaginary parts along K:
//   A'[m][k'] = (Re A | Im A)[m][c],  B_re[n][k'] = (Re C | -Im C),  B_im[n][k'] = (Im C | Re C)
//   D_re = A' B_re^T = Re(A C),  D_im = A' B_im^T = Im(A C).
// A CTA owns 64 a x 64 b: M = 128 rows m = 2(a - a0) + s1, N = 128 columns n = 64 s2 + (b - b0);
// D_re and D_im take 2 x 128 of the 512 tensor-memory columns.  K runs over mid in chunks of 16
// complex (K' = 32 real = 4 MMAs of K = 8 per pass).  Operands are staged by the CTA's 256
// threads into shared memory in the canonical K-major layout without swizzle (8-row x 16-byte
// core matrices: rows 16 B apart, 8-row groups 128 B apart (SBO), 16-byte K chunks 2 KiB apart
// (LBO)), in two buffers: one elected thread issues a chunk's MMAs and commits them to that
// buffer's mbarrier, and the threads go on to stage the next chunk into the other buffer while
// the tensor cores work; a buffer is restaged only after its previous MMAs completed.  The gate
// epilogue reads D row by row from tensor memory (warp w owns lanes 32 (w % 4) .. + 31; the two
// warp groups take the two halves of the columns), swaps the s1 partner row with a lane
// shuffle, applies the 4x4 gate and writes theta and its Jacobi copy W.  Rows, columns and K beyond the bond dimensions are zero-padded, so any bond works.
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "engine.cuh"

namespace tq {

#define TC_CHECK(x)                                                                              \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess)                                                                   \
            throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_) + " at " +   \
                                     __FILE__ + ":" + std::to_string(__LINE__));                 \
    } while (0)

constexpr int TC_BM = 64;    // a per CTA (M = 2 TC_BM rows)
constexpr int TC_BN = 64;    // b per CTA (N = 2 TC_BN columns)
constexpr int TC_KC = 16;    // complex K per chunk
constexpr int TC_M = 2 * TC_BM;
constexpr int TC_N = 2 * TC_BN;
constexpr int TC_KR = 2 * TC_KC;            // real K per chunk
constexpr int TC_NT = 256;                     // two warp groups: both stage, each reads half the columns
constexpr int TC_OP_BYTES = TC_M * TC_KR * 4;  // one operand tile (128 rows x 32 floats) = 16 KiB
constexpr int TC_LBO = (TC_M / 8) * 128;       // bytes between 16-byte K chunks
constexpr int TC_SBO = 128;                    // bytes between 8-row groups
constexpr int TC_STAGE = 6 * TC_OP_BYTES;      // one buffer: A hi/lo, B_re hi/lo, B_im hi/lo
constexpr int TC_SMEM = 2 * TC_STAGE;          // two buffers: chunk k+1 is staged under chunk k's MMAs
constexpr int TC_TMEM_COLS = 2 * TC_N;         // D_re, D_im

static_assert(TC_M == 128 && TC_N % 16 == 0 && TC_N <= 256, "tcgen05 kind::tf32 shape");

// byte offset of element (row, k) of an operand tile in the canonical K-major layout
__device__ __forceinline__ uint32_t tc_off(int row, int k) {
    return (uint32_t)((k >> 2) * TC_LBO + (row >> 3) * TC_SBO + (row & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// shared-memory matrix descriptor: start, LBO, SBO (16-byte units), version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((TC_LBO >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((TC_SBO >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor: D F32, A and B TF32, both K-major, N = TC_N, M = TC_M
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
    const uint32_t z = 0;  // disable-output-lane mask: every lane written
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(TC_IDESC), "r"(acc), "r"(z)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <typename V>
__device__ __forceinline__ void tc_gate(const GateOp& op, const ScheduleView& sch, V g[16]) {
    for (int q = 0; q < 16; ++q) g[q] = make_float2(0.f, 0.f);
    if (op.kind == GATE_SWAP) {
        g[0] = make_float2(1.f, 0.f); g[1 * 4 + 2] = make_float2(1.f, 0.f);
        g[2 * 4 + 1] = make_float2(1.f, 0.f); g[15] = make_float2(1.f, 0.f);
    } else {
        const double th = -sch.sb[*sch.step] * sch.w[op.edge] * sch.sub;
        const double c = cos(th), s = sin(th);
        g[0] = make_float2((float)c, (float)-s); g[15] = g[0];
        g[5] = make_float2((float)c, (float)s); g[10] = g[5];
    }
}

// One 64 a x 64 b tile of theta for bond op.bond.  Returns without touching tensor memory when
// the tile lies outside the bond dimensions.
__device__ void theta_tc_tile(const MpsView<float>& mps, const ScheduleView& sch, const GateOp& op,
                              const SvdWork<float>& wk, int tile_a, int tile_b, unsigned char* smem) {
    using V = float2;
    __shared__ __align__(8) uint64_t s_bar[2];  // MMAs of the chunk staged in buffer 0 / 1 done
    __shared__ uint32_t s_taddr;
    __shared__ int s_ok;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int i = op.bond;
    const int dl = mps.dims[i], mid = mps.dims[i + 1], dr = mps.dims[i + 2];
    const int a0 = tile_a * TC_BM, b0 = tile_b * TC_BN;
    if (a0 >= dl || b0 >= dr) return;  // uniform: before any tensor-memory allocation
    const int cap = mps.cap;
    const V* A = mps.site(i);
    const V* Cm = mps.site(i + 1);
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_taddr)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_taddr;
    const uint32_t d_re = tmem, d_im = tmem + TC_N;
    unsigned phase = 0u;    // bit b: the parity to wait for on s_bar[b]
    unsigned pending = 0u;  // bit b: a commit on buffer b not yet waited for
    // one CTA-wide outcome per wait (thread 0 waits with a bound, the others re-check the phase)
    auto wait_buf = [&](int b) -> bool {
        const unsigned par = (phase >> b) & 1u;
        if (tid == 0) s_ok = mbar_wait(&s_bar[b], par, 1000000000ull) ? 1 : 0;
        __syncthreads();
        const bool good = s_ok != 0;
        if (good) {
            if (tid != 0) mbar_wait(&s_bar[b], par, 1000000000ull);
            phase ^= 1u << b;
            pending &= ~(1u << b);
        }
        __syncthreads();  // s_ok free again
        return good;
    };
    bool ok = true;
    const int nchunk = (mid + TC_KC - 1) / TC_KC;
    for (int kc = 0; kc < nchunk && ok; ++kc) {
        const int buf = kc & 1;
        // the MMAs of chunk kc - 2 read this buffer: wait for them before restaging it
        if (((pending >> buf) & 1u) && !wait_buf(buf)) { ok = false; break; }
        unsigned char* opA_hi = smem + buf * TC_STAGE;
        unsigned char* opA_lo = opA_hi + TC_OP_BYTES;
        unsigned char* opR_hi = opA_hi + 2 * TC_OP_BYTES;
        unsigned char* opR_lo = opA_hi + 3 * TC_OP_BYTES;
        unsigned char* opI_hi = opA_hi + 4 * TC_OP_BYTES;
        unsigned char* opI_lo = opA_hi + 5 * TC_OP_BYTES;
        const int c0 = kc * TC_KC;
        // Each task converts 4 consecutive k of one operand row and writes them as 16-byte
        // vectors; a warp's 32 tasks are 32 consecutive rows (8-row groups of 128 contiguous
        // bytes in the canonical layout), so the stores are free of bank conflicts.
        // A' rows m = 2(a - a0) + s1 = site row 2 a0 + m: real parts at k' = k, imaginary at TC_KC + k.
        // Lane l of a warp task takes row 8 task + (l & 7) and k = 4 (l >> 3) .. + 3: the four lanes
        // of a row read its 128 contiguous bytes (two 16-byte loads each when the row pitch keeps
        // them aligned), and lanes 0-7 of each store phase write eight different rows.
        for (int t = tid; t < TC_M * (TC_KC / 4); t += TC_NT) {
            const int lane = t & 31, m = 8 * (t >> 5) + (lane & 7), kq = lane >> 3;
            const int a = a0 + (m >> 1), c = c0 + 4 * kq;
            float2 xv[4];
            const V* src = A + (long long)(2 * a0 + m) * cap + c;
            if (a < dl && c + 3 < mid && (cap & 1) == 0) {
                const float4 v0 = *reinterpret_cast<const float4*>(src);
                const float4 v1 = *reinterpret_cast<const float4*>(src + 2);
                xv[0] = make_float2(v0.x, v0.y); xv[1] = make_float2(v0.z, v0.w);
                xv[2] = make_float2(v1.x, v1.y); xv[3] = make_float2(v1.z, v1.w);
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j) xv[j] = (a < dl && c + j < mid) ? src[j] : make_float2(0.f, 0.f);
            }
            uint4 hr, hi, lr, li;
            uint32_t* phr = &hr.x; uint32_t* phi = &hi.x; uint32_t* plr = &lr.x; uint32_t* pli = &li.x;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                phr[j] = to_tf32(xv[j].x);
                phi[j] = to_tf32(xv[j].y);
                plr[j] = to_tf32(xv[j].x - __uint_as_float(phr[j]));
                pli[j] = to_tf32(xv[j].y - __uint_as_float(phi[j]));
            }
            *reinterpret_cast<uint4*>(opA_hi + tc_off(m, 4 * kq)) = hr;
            *reinterpret_cast<uint4*>(opA_hi + tc_off(m, TC_KC + 4 * kq)) = hi;
            *reinterpret_cast<uint4*>(opA_lo + tc_off(m, 4 * kq)) = lr;
            *reinterpret_cast<uint4*>(opA_lo + tc_off(m, TC_KC + 4 * kq)) = li;
        }
        // B rows n = TC_BN s2 + (b - b0): B_re = (Re C | -Im C), B_im = (Im C | Re C) along k'
        for (int t = tid; t < TC_N * (TC_KC / 4); t += TC_NT) {
            const int n = t & (TC_N - 1), kq = t / TC_N;
            const int s2 = n / TC_BN, b = b0 + (n - s2 * TC_BN), c = c0 + 4 * kq;
            uint4 hr, hi, lr, li;
            uint32_t* phr = &hr.x; uint32_t* phi = &hi.x; uint32_t* plr = &lr.x; uint32_t* pli = &li.x;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const V y = (b < dr && c + j < mid) ? Cm[(long long)(2 * (c + j) + s2) * cap + b] : make_float2(0.f, 0.f);
                phr[j] = to_tf32(y.x);
                phi[j] = to_tf32(y.y);
                plr[j] = to_tf32(y.x - __uint_as_float(phr[j]));
                pli[j] = to_tf32(y.y - __uint_as_float(phi[j]));
            }
            const uint4 nhi = make_uint4(hi.x ^ 0x80000000u, hi.y ^ 0x80000000u, hi.z ^ 0x80000000u, hi.w ^ 0x80000000u);
            const uint4 nli = make_uint4(li.x ^ 0x80000000u, li.y ^ 0x80000000u, li.z ^ 0x80000000u, li.w ^ 0x80000000u);
            *reinterpret_cast<uint4*>(opR_hi + tc_off(n, 4 * kq)) = hr;
            *reinterpret_cast<uint4*>(opR_hi + tc_off(n, TC_KC + 4 * kq)) = nhi;
            *reinterpret_cast<uint4*>(opR_lo + tc_off(n, 4 * kq)) = lr;
            *reinterpret_cast<uint4*>(opR_lo + tc_off(n, TC_KC + 4 * kq)) = nli;
            *reinterpret_cast<uint4*>(opI_hi + tc_off(n, 4 * kq)) = hi;
            *reinterpret_cast<uint4*>(opI_hi + tc_off(n, TC_KC + 4 * kq)) = hr;
            *reinterpret_cast<uint4*>(opI_lo + tc_off(n, 4 * kq)) = li;
            *reinterpret_cast<uint4*>(opI_lo + tc_off(n, TC_KC + 4 * kq)) = lr;
        }
        // the tensor cores read shared memory through the async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa[2] = {smem_u32(opA_hi), smem_u32(opA_lo)};
            const uint32_t sr[2] = {smem_u32(opR_hi), smem_u32(opR_lo)};
            const uint32_t si[2] = {smem_u32(opI_hi), smem_u32(opI_lo)};
            const int pa[3] = {0, 0, 1}, pb[3] = {0, 1, 0};  // hi.hi, hi.lo, lo.hi
            for (int p = 0; p < 3; ++p)
                for (int ks = 0; ks < TC_KR / 8; ++ks) {
                    const uint32_t koff = (uint32_t)(ks * 2 * TC_LBO);
                    const uint32_t acc = (kc > 0 || p > 0 || ks > 0) ? 1u : 0u;
                    const uint64_t da = tc_desc(sa[pa[p]] + koff);
                    tc_mma(d_re, da, tc_desc(sr[pb[p]] + koff), acc);
                    tc_mma(d_im, da, tc_desc(si[pb[p]] + koff), acc);
                }
            tc_commit(&s_bar[buf]);
        }
        pending |= 1u << buf;  // the next chunk stages the other buffer without waiting
    }
    // drain: the last commit covers every MMA issued before it; both barriers are consumed
    for (int q = 0; q < 2 && ok; ++q) {
        const int b = (nchunk - 2 + q) & 1;  // the older pending chunk first
        if (((pending >> b) & 1u) && !wait_buf(b)) ok = false;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
        V g[16];
        tc_gate(op, sch, g);
        // row m (TMEM lane) of this thread: warp w reads lanes 32 (w % 4) .. + 31; the two warp
        // groups take the two halves of the b columns
        const int m = tid & (TC_M - 1), s1 = m & 1, a = a0 + (m >> 1);
        const int half = tid / TC_M;
        const uint32_t lane_off = (uint32_t)(32 * (warp & 3)) << 16;
        const int ld = wk.ld;
        for (int j0 = half * (TC_BN / 2); j0 < (half + 1) * (TC_BN / 2); j0 += 16) {
            float r0[16], i0[16], r1[16], i1[16];  // s2 = 0 and 1 columns
            tc_ld16(d_re + lane_off + j0, r0);
            tc_ld16(d_im + lane_off + j0, i0);
            tc_ld16(d_re + lane_off + TC_BN + j0, r1);
            tc_ld16(d_im + lane_off + TC_BN + j0, i1);
#pragma unroll
            for (int jj = 0; jj < 16; ++jj) {
                V t[2][2];  // t[s1'][s2]
                const V own0 = make_float2(r0[jj], i0[jj]), own1 = make_float2(r1[jj], i1[jj]);
                const V oth0 = make_float2(__shfl_xor_sync(0xffffffffu, own0.x, 1), __shfl_xor_sync(0xffffffffu, own0.y, 1));
                const V oth1 = make_float2(__shfl_xor_sync(0xffffffffu, own1.x, 1), __shfl_xor_sync(0xffffffffu, own1.y, 1));
                t[s1][0] = own0; t[s1][1] = own1;
                t[s1 ^ 1][0] = oth0; t[s1 ^ 1][1] = oth1;
                const int b = b0 + j0 + jj;
                if (a >= dl || b >= dr) continue;
#pragma unroll
                for (int r2 = 0; r2 < 2; ++r2) {
                    V o = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q1 = 0; q1 < 2; ++q1)
#pragma unroll
                        for (int q2 = 0; q2 < 2; ++q2) cfma(o, g[(s1 * 2 + r2) * 4 + q1 * 2 + q2], t[q1][q2]);
                    const long long idx = (long long)(2 * a + s1) + (long long)(r2 * dr + b) * ld;
                    wk.theta[idx] = o;
                    wk.W[idx] = o;
                }
            }
        }
    } else if (tid == 0) {
        atomicOr(&wk.stats->status, ST_BARRIER_TIMEOUT);
        for (int b = 0; b < 2; ++b)  // let the MMAs in flight finish (bounded)
            if ((pending >> b) & 1u) mbar_wait(&s_bar[b], (phase >> b) & 1u, 1000000000ull);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS)
                     : "memory");
}

__global__ void __launch_bounds__(TC_NT, 1) k_theta_tc(MpsView<float> mps, ScheduleView sch, GateOp op,
                                                       SvdWork<float> wk) {
    extern __shared__ __align__(1024) unsigned char smem[];
    theta_tc_tile(mps, sch, op, wk, blockIdx.x, blockIdx.y, smem);
}

__global__ void __launch_bounds__(TC_NT, 1) k_theta_tc_batch(const InstTask<float>* insts, const UpdRef* refs) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const UpdRef rf = refs[blockIdx.z];
    const InstTask<float>& it = insts[rf.inst];
    theta_tc_tile(it.mps, it.sch, rf.op, it.wk, blockIdx.x, blockIdx.y, smem);
}

bool theta_tc_supported(const GateOp& op) { return op.kind == GATE_SWAP || op.kind == GATE_ZZ; }

void launch_theta_tc(const MpsView<float>& mps, const ScheduleView& sch, GateOp op, SvdWork<float> wk, int dl_ub,
                     int dr_ub, cudaStream_t s) {
    TC_CHECK(cudaFuncSetAttribute(k_theta_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
    dim3 grid((dl_ub + TC_BM - 1) / TC_BM, (dr_ub + TC_BN - 1) / TC_BN);
    k_theta_tc<<<grid, TC_NT, TC_SMEM, s>>>(mps, sch, op, wk);
    TC_CHECK(cudaGetLastError());
}

void launch_theta_tc_batch(const InstTask<float>* insts, const UpdRef* refs, int nref, int d_ub, cudaStream_t s) {
    TC_CHECK(cudaFuncSetAttribute(k_theta_tc_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
    const int t = (d_ub + TC_BM - 1) / TC_BM;
    k_theta_tc_batch<<<dim3(t, t, nref), TC_NT, TC_SMEM, s>>>(insts, refs);
    TC_CHECK(cudaGetLastError());
}

}  // namespace tq
