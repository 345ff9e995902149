// kernels.cu -- sm_100a kernels of the MPS-TEBD anneal.
//
//   K5 k_single_site : all n single-site half-step gates exp(-i dt/2 (-A X - B h Z)) in one
//                      launch, built in closed form cos(phi) I - i sin(phi) n.sigma
//                      (replaces cuda/src/mps.cpp:313-322,344-353 + linalg.cpp:174-197).
//   K1 k_theta       : theta = G . (A_i A_{i+1}) -- the bond contraction as a tiled GEMM
//                      whose register tile holds whole (s1,s2) quads, so the 4x4 gate is an
//                      epilogue (cuda/src/mps.cpp:46-70).
//   K2 k_svd         : cooperative one-sided (Hestenes) Jacobi on theta's columns, block
//                      tournament ordering, column pairs reduced with warp shuffles;
//                      ends with the sigma sort, keep rule and discarded weight (K3)
//                      (replaces cuda/src/linalg.cpp:7-172 and mps.cpp:76-85).
//   K4 k_absorb_*    : A <- U[:, :keep], C <- U[:, :keep]^dagger theta (= S Vh[:keep])
//                      (cuda/src/mps.cpp:87-99).
//   K6 k_chain       : environment transfers (right env for the qubit-0 entropy, left and
//                      right envs and Z insertions for the final observables), O(n chi^3).
//   K7 k_pair_dots, k_amplitude, k_entropy : closing contractions, in FP64.
#include <cstdio>
#include <stdexcept>
#include <string>

#include "engine.cuh"

namespace tq {

#define TQ_CHECK(x)                                                                            \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_) + " at " + \
                                     __FILE__ + ":" + std::to_string(__LINE__));               \
    } while (0)

static int g_num_sms = 0;
static int num_sms() {
    if (!g_num_sms) {
        int dev = 0;
        TQ_CHECK(cudaGetDevice(&dev));
        TQ_CHECK(cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    return g_num_sms;
}

// ------------------------------------------------------------------------------------
// initial state |+>^n (cuda/src/mps.cpp:9-17)
// ------------------------------------------------------------------------------------
template <typename T>
__global__ void k_init_plus(MpsView<T> mps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= mps.n) mps.dims[i] = 1;
    if (i < mps.n) {
        const T a = (T)0.70710678118654752440;
        cplx_t<T>* s = mps.site(i);
        s[0] = mk<cplx_t<T>>(a, 0);          // (0, 0, 0)
        s[mps.cap] = mk<cplx_t<T>>(a, 0);    // (0, 1, 0)
    }
}

template <typename T>
void launch_init_plus(const MpsView<T>& mps, cudaStream_t s) {
    k_init_plus<T><<<(mps.n + 1 + 127) / 128, 128, 0, s>>>(mps);
    TQ_CHECK(cudaGetLastError());
}

__global__ void k_step_inc(int* step) { *step += 1; }
void launch_step_inc(int* step, cudaStream_t s) {
    k_step_inc<<<1, 1, 0, s>>>(step);
    TQ_CHECK(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// K5: single-site half step.  g = -A X - (B h + C b) Z = nx X + nz Z (C b: optional warm-start
// bias field, zero when unused); exp(-i (dt/2) g) =
// cos(phi) I - i sin(phi) (nx X + nz Z)/r with r = |(nx, nz)|, phi = r dt/2.
// ------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void single_site_body(const MpsView<T>& mps, const ScheduleView& sch, const int i,
                                                 const int bx, const int nbx) {
    using V = cplx_t<T>;
    if (i >= mps.n) return;
    const int k = *sch.step;
    const double A = sch.sa[k], B = sch.sb[k];
    const double nx = -A, nz = -(B * sch.h[i] + sch.sc[k] * sch.bias[i]);
    const double r = sqrt(nx * nx + nz * nz);
    double c = 1.0, sn = 0.0;
    if (r > 0) {
        const double phi = 0.5 * sch.dt * r;
        c = cos(phi);
        sn = sin(phi) / r;
    }
    // U = [[c - i sn nz, -i sn nx], [-i sn nx, c + i sn nz]]
    const V u00 = mk<V>((T)c, (T)(-sn * nz)), u01 = mk<V>((T)0, (T)(-sn * nx));
    const V u11 = mk<V>((T)c, (T)(sn * nz));
    const int dl = mps.dims[i], dr = mps.dims[i + 1];
    V* S = mps.site(i);
    const int tot = dl * dr;
    for (int t = bx * blockDim.x + threadIdx.x; t < tot; t += nbx * blockDim.x) {
        const int a = t / dr, b = t - a * dr;
        V* p0 = S + (long long)(2 * a) * mps.cap + b;
        V* p1 = p0 + mps.cap;
        const V x0 = *p0, x1 = *p1;
        V y0 = czero<V>(), y1 = czero<V>();
        cfma(y0, u00, x0); cfma(y0, u01, x1);
        cfma(y1, u01, x0); cfma(y1, u11, x1);
        *p0 = y0;
        *p1 = y1;
    }
}

template <typename T>
__global__ void k_single_site(MpsView<T> mps, ScheduleView sch) {
    single_site_body<T>(mps, sch, blockIdx.y, blockIdx.x, gridDim.x);
}

template <typename T>
void launch_single_site(const MpsView<T>& mps, const ScheduleView& sch, int d2_ub_max, cudaStream_t s) {
    int bx = (d2_ub_max + 255) / 256;
    if (bx < 1) bx = 1;
    if (bx > 64) bx = 64;
    dim3 grid(bx, mps.n);
    k_single_site<T><<<grid, 256, 0, s>>>(mps, sch);
    TQ_CHECK(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// K1: theta contraction with the gate as an epilogue.
// T_{s1 s2}[a, b] = sum_c A[(2a+s1), c] C[c, (s2, b)]; out[(2a+r1), (r2*Dr+b)] =
// sum_{s1 s2} G[r1 r2][s1 s2] T_{s1 s2}[a, b].  A CTA owns 32 a x 32 b quads; thread
// (tx, ty) owns a in {tx, tx+16}, b in {ty, ty+16}, i.e. 16 complex accumulators.
// ------------------------------------------------------------------------------------
constexpr int TH_KC = 8;

template <typename V>
__device__ __forceinline__ void gate_of(const GateOp& op, const ScheduleView& sch, const double* gen, V g[16]) {
    using T = decltype(V::x);
    for (int q = 0; q < 16; ++q) g[q] = czero<V>();
    if (op.kind == GATE_SWAP) {
        g[0] = mk<V>(1, 0); g[1 * 4 + 2] = mk<V>(1, 0); g[2 * 4 + 1] = mk<V>(1, 0); g[15] = mk<V>(1, 0);
    } else if (op.kind == GATE_ZZ) {
        const double th = -sch.sb[*sch.step] * sch.w[op.edge] * sch.sub;
        const double c = cos(th), s = sin(th);
        g[0] = mk<V>((T)c, (T)(-s)); g[15] = g[0];       // exp(-i th) on |00>, |11>
        g[5] = mk<V>((T)c, (T)s); g[10] = g[5];          // exp(+i th) on |01>, |10>
    } else {
        for (int q = 0; q < 16; ++q) g[q] = mk<V>((T)gen[2 * q], (T)gen[2 * q + 1]);
    }
}

template <typename T>
__device__ __forceinline__ void theta_tile(const MpsView<T>& mps, const ScheduleView& sch, const GateOp& op,
                                           const double* gen, const SvdWork<T>& wk, const int tile_a, const int tile_b) {
    using V = cplx_t<T>;
    __shared__ V As[TH_KC][2][32];
    __shared__ V Cs[TH_KC][2][32];
    const int i = op.bond;
    const int dl = mps.dims[i], mid = mps.dims[i + 1], dr = mps.dims[i + 2];
    const int a0 = tile_a * 32, b0 = tile_b * 32;
    if (a0 >= dl || b0 >= dr) return;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const V* A = mps.site(i);
    const V* Cm = mps.site(i + 1);
    const int cap = mps.cap;
    V acc[2][2][2][2];  // [ia][ib][s1][s2]
#pragma unroll
    for (int x = 0; x < 16; ++x) (&acc[0][0][0][0])[x] = czero<V>();
    for (int c0 = 0; c0 < mid; c0 += TH_KC) {
        // A tile: 64 rows (a, s1) x KC; C tile: KC x (s2, 32 b)
        for (int e = tid; e < 64 * TH_KC; e += 256) {
            const int kk = e % TH_KC, rr = e / TH_KC;
            const int a = a0 + (rr >> 1), s1 = rr & 1, c = c0 + kk;
            As[kk][s1][rr >> 1] = (a < dl && c < mid) ? A[(long long)(2 * a + s1) * cap + c] : czero<V>();
        }
        for (int e = tid; e < 64 * TH_KC; e += 256) {
            const int bb = e & 31, rest = e >> 5;
            const int kk = rest >> 1, s2 = rest & 1, c = c0 + kk, b = b0 + bb;
            Cs[kk][s2][bb] = (b < dr && c < mid) ? Cm[(long long)(2 * c + s2) * cap + b] : czero<V>();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TH_KC; ++kk) {
            V av[2][2], cv[2][2];
#pragma unroll
            for (int u = 0; u < 2; ++u)
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    av[u][s] = As[kk][s][tx + 16 * u];
                    cv[u][s] = Cs[kk][s][ty + 16 * u];
                }
#pragma unroll
            for (int ia = 0; ia < 2; ++ia)
#pragma unroll
                for (int ib = 0; ib < 2; ++ib)
#pragma unroll
                    for (int s1 = 0; s1 < 2; ++s1)
#pragma unroll
                        for (int s2 = 0; s2 < 2; ++s2) cfma(acc[ia][ib][s1][s2], av[ia][s1], cv[ib][s2]);
        }
        __syncthreads();
    }
    V g[16];
    gate_of(op, sch, gen, g);
    const int ld = wk.ld;
#pragma unroll
    for (int ia = 0; ia < 2; ++ia)
#pragma unroll
        for (int ib = 0; ib < 2; ++ib) {
            const int a = a0 + tx + 16 * ia, b = b0 + ty + 16 * ib;
            if (a >= dl || b >= dr) continue;
#pragma unroll
            for (int r1 = 0; r1 < 2; ++r1)
#pragma unroll
                for (int r2 = 0; r2 < 2; ++r2) {
                    V o = czero<V>();
#pragma unroll
                    for (int s1 = 0; s1 < 2; ++s1)
#pragma unroll
                        for (int s2 = 0; s2 < 2; ++s2) cfma(o, g[(r1 * 2 + r2) * 4 + s1 * 2 + s2], acc[ia][ib][s1][s2]);
                    const long long idx = (long long)(2 * a + r1) + (long long)(r2 * dr + b) * ld;
                    wk.theta[idx] = o;
                    wk.W[idx] = o;
                }
        }
}

template <typename T>
__global__ void __launch_bounds__(256) k_theta(MpsView<T> mps, ScheduleView sch, GateOp op, const double* gen,
                                               SvdWork<T> wk) {
    theta_tile<T>(mps, sch, op, gen, wk, blockIdx.x, blockIdx.y);
}

template <typename T>
void launch_theta(const MpsView<T>& mps, const ScheduleView& sch, GateOp op, const double* gen_gate,
                  SvdWork<T> wk, int dl_ub, int dr_ub, cudaStream_t s) {
    dim3 grid((dl_ub + 31) / 32, (dr_ub + 31) / 32);
    k_theta<T><<<grid, 256, 0, s>>>(mps, sch, op, gen_gate, wk);
    TQ_CHECK(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// K2 + K3: cooperative one-sided Jacobi SVD of W (R x N, column-major).
//
// Columns are cut into blocks of BW; a round-robin tournament over the P (even) blocks
// gives P-1 rounds per sweep, each with P/2 disjoint block pairs, one pair per CTA at a
// time.  A CTA stages its 2*BW columns in shared memory and, on round 0 of a sweep,
// first rotates the pairs inside each block; then it rotates the BW*BW cross pairs in BW
// inner rounds of BW disjoint pairs.  Each pair (p, q) is owned by G = 256/BW threads:
// alpha = |w_p|^2, beta = |w_q|^2, gamma = w_p^dagger w_q are reduced with warp
// shuffles (and shared memory across the group's warps) in FP64, and the pair is
// rotated when |gamma| > tol sqrt(alpha beta):
//   zeta = (beta - alpha) / (2|gamma|), t = sign(zeta)/(|zeta| + sqrt(1 + zeta^2)),
//   c = 1/sqrt(1+t^2), s = c t, e = gamma/|gamma|,
//   w_p <- c w_p - s conj(e) w_q,   w_q <- s e w_p + c w_q.
// A sweep with no rotation ends the iteration.  Column norms then give sigma; CTA 0
// sorts them (bitonic, descending), applies the keep rule of cuda/src/mps.cpp:76-85
// (keep = min(chi, k), then drop trailing sigma < 1e-14) and records the discarded
// weight ratio.
// ------------------------------------------------------------------------------------

template <int G>
__device__ __forceinline__ void group_reduce4(double v[4], double* red, int tid) {
    // G threads per group; groups are aligned to G.
    if (G <= 32) {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1)
#pragma unroll
            for (int q = 0; q < 4; ++q) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = warp_sum(v[q]);
        const int warp = tid >> 5, lane = tid & 31;
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < 4; ++q) red[warp * 4 + q] = v[q];
        __syncthreads();
        constexpr int WG = G / 32;
        const int w0 = (tid / G) * WG;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < WG; ++w) s += red[(w0 + w) * 4 + q];
            v[q] = s;
        }
    }
}

// Freeze rule for columns under the noise floor `tiny` (on |w|^2).  In the early phase of an
// SVD ("mixed": the previous sweep still rotated at least 10% of the N(N-1)/2 pairs) a pair is
// live when one column is above the floor and the other holds more than 1e-6 of it; after
// that, only when both columns are above the floor.  A column whose norm dips under the floor
// mid-sweep is thereby still orthogonalised against the resolved columns, so values a few
// times the floor come back right, while noise columns (rank-deficient or wide theta) are
// dropped as soon as the sweeps settle.  The 1e-6 margin also bounds the ratio of the two
// norms, so the rotation below cannot overflow.
__device__ __forceinline__ bool pair_live(const double v0, const double v1, const double tiny, const bool mixed) {
    const double lo = fmin(v0, v1);
    return mixed ? (fmax(v0, v1) > tiny && lo > 1e-6 * tiny) : lo > tiny;
}

// Whether the next sweep stays in the mixed phase: this sweep rotated at least 10% of the pairs,
// and the phase has not yet lasted 8 + 3 log2(N) sweeps.  The cap bounds the phase on the rare
// theta where a few mixed pairs keep rotating by rounding (seen on small exact-chi theta: the
// count then stays above 10% of a handful of pairs and the sweeps never settle); the late rule
// converges from there.  It leaves room for the slower tournament order of the cooperative
// kernel on 1024 columns (cap 38).
__device__ __forceinline__ bool still_mixed(const bool mixed, const double rotated, const int N, const int sweep) {
    int lg = 0;
    while ((1 << lg) < N) ++lg;
    return mixed && rotated >= 0.05 * (double)N * (double)(N - 1) && sweep + 1 < 8 + 3 * lg;
}

// Rotation of a column pair from alpha = |w_p|^2 (v0), beta = |w_q|^2 (v1) and
// gamma = w_p^H w_q (v2 + i v3), all accumulated in FP64.  Returns false for a converged
// pair (|gamma|^2 <= tol^2 alpha beta, the FP64 convergence test) or a pair that the freeze
// rule (pair_live) leaves alone; else c, s and the phase e = gamma/|gamma| of
//   w_p <- c w_p - s conj(e) w_q,   w_q <- s e w_p + c w_q,
//   zeta = (beta - alpha) / (2|gamma|), t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)),
//   c = 1/sqrt(1 + t^2), s = c t.
// 1/|gamma| comes from one FP64 rsqrt; in complex64 the tangent and cosine are formed in FP32
// (the precision they are applied in).
template <typename T>
__device__ __forceinline__ bool jacobi_rotation(const double v0, const double v1, const double v2, const double v3,
                                                const double tol, const double tiny, const bool mixed, T& c, T& s,
                                                T& er, T& ei) {
    const double g2 = v2 * v2 + v3 * v3;
    if (!(pair_live(v0, v1, tiny, mixed) && g2 > tol * tol * (v0 * v1))) return false;
    const double rg = rsqrt(g2);
    const double zeta = 0.5 * (v1 - v0) * rg;
    er = (T)(v2 * rg);
    ei = (T)(v3 * rg);
    if constexpr (sizeof(T) == 8) {
        // t = sgn(zeta) / u with u = |zeta| + sqrt(1 + zeta^2) = (|d| + sqrt(d^2 + 4 g2)) / (2 |gamma|),
        // d = v1 - v0; then c = 1 / sqrt(1 + t^2) = u w and s = c t = sgn(zeta) w for
        // w = 1 / sqrt(u^2 + 1).  No division, and the square root runs beside rsqrt(g2).
        const double d = v1 - v0;
        const double u = 0.5 * rg * (fabs(d) + sqrt(fma(d, d, 4.0 * g2)));
        const double w = rsqrt(fma(u, u, 1.0));
        c = u * w;
        s = zeta >= 0 ? w : -w;
    } else {
        const float z = (float)zeta, az = fabsf(z);
        // for |zeta| >= 1e18 1 + zeta^2 overflows float; t = 1/(2 zeta) to float precision there
        const float ta = az < 1e18f ? 1.f / (az + sqrtf(1.f + az * az)) : 0.5f / az;
        const float t = z >= 0.f ? ta : -ta;
        const float cs = rsqrtf(1.f + t * t);
        c = cs;
        s = cs * t;
    }
    return true;
}

// Per-lane partial sums of alpha = |x|^2, beta = |y|^2 and gamma = x^H y over the rows a lane
// holds, for complex64: FP32 products summed in FP32 over the lane's rows (at most 16 in every
// kernel here, relative error about 1e-6, under the complex64 convergence tolerance
// 8 sqrt(R) eps_f32), so they run on the FP32 pipe; the lane sums are widened to FP64 before
// the cross-lane sum, the noise-floor test and the FP64 convergence test.  complex128 keeps FP64
// products and sums.
struct LaneDotsF32 {
    float a = 0.f, b = 0.f, gr = 0.f, gi = 0.f;
    __device__ __forceinline__ void add(const float2 x, const float2 y) {
        a = fmaf(x.x, x.x, fmaf(x.y, x.y, a));
        b = fmaf(y.x, y.x, fmaf(y.y, y.y, b));
        gr = fmaf(x.x, y.x, fmaf(x.y, y.y, gr));
        gi = fmaf(x.x, y.y, fmaf(-x.y, y.x, gi));
    }
};

// The rotation w_p <- c w_p - s conj(e) w_q, w_q <- s e w_p + c w_q as x' = c x + b y,
// y' = d x + c y with the complex coefficients b = -s conj(e) and d = s e formed once per pair:
// 12 real multiply-adds per row instead of 16.
template <typename T>
struct PairRot {
    T c, br, bi, dr, di;
    __device__ __forceinline__ PairRot(T c_, T s, T er, T ei) : c(c_), br(-s * er), bi(s * ei), dr(s * er), di(s * ei) {}
    __device__ __forceinline__ void apply(cplx_t<T>& x, cplx_t<T>& y) const {
        const cplx_t<T> xo = x, yo = y;
        x.x = fma(-bi, yo.y, fma(br, yo.x, c * xo.x));
        x.y = fma(bi, yo.x, fma(br, yo.y, c * xo.y));
        y.x = fma(-di, xo.y, fma(dr, xo.x, c * yo.x));
        y.y = fma(di, xo.x, fma(dr, xo.y, c * yo.y));
    }
};

// Rotate local columns p, q (shared memory) of a group; returns 1 if rotated.
template <typename T, int G>
__device__ __forceinline__ int rotate_pair(cplx_t<T>* cp, cplx_t<T>* cq, bool valid, int R, double tol,
                                           double tiny, bool mixed, double* red, int tid) {
    using V = cplx_t<T>;
    const int lg = tid % G;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (valid) {
        if constexpr (sizeof(T) == 4) {
            LaneDotsF32 d;
            for (int r = lg; r < R; r += G) d.add(cp[r], cq[r]);
            v[0] = d.a; v[1] = d.b; v[2] = d.gr; v[3] = d.gi;
        } else {
            for (int r = lg; r < R; r += G) {
                const V x = cp[r], y = cq[r];
                v[0] += (double)x.x * x.x + (double)x.y * x.y;
                v[1] += (double)y.x * y.x + (double)y.y * y.y;
                v[2] += (double)x.x * y.x + (double)x.y * y.y;   // Re conj(x) y
                v[3] += (double)x.x * y.y - (double)x.y * y.x;   // Im conj(x) y
            }
        }
    }
    group_reduce4<G>(v, red, tid);
    if (!valid) return 0;
    T cc, ss, er, ei;
    if (!jacobi_rotation<T>(v[0], v[1], v[2], v[3], tol, tiny, mixed, cc, ss, er, ei)) return 0;
    const PairRot<T> rt(cc, ss, er, ei);
    for (int r = lg; r < R; r += G) {
        V x = cp[r], y = cq[r];
        rt.apply(x, y);
        cp[r] = x;
        cq[r] = y;
    }
    return 1;
}

// Barrier across the CTAs that share one SVD: the grid barrier when several cooperate,
// a plain CTA barrier when one CTA does it all.
__device__ __forceinline__ bool cta_sync(GridBar* bar, int* status, unsigned int nblk) {
    if (nblk == 1) {
        __syncthreads();
        return true;
    }
    return grid_sync(bar, status, nblk);
}

__device__ __forceinline__ void tournament(int P, int r, int pr, int& I, int& J) {
    const int Q = P - 1;
    if (pr == 0) {
        I = Q;
        J = r;
    } else {
        I = (r + pr) % Q;
        J = (r - pr + Q) % Q;
    }
}

constexpr int SVD_THREADS = 512;

// RPL = 0: shared-memory rotations, SVD_THREADS threads, G = SVD_THREADS/BW threads per pair.
// RPL > 0: register-resident cross rounds, one warp per pair (NT = 32 BW threads): warp w keeps
//          column w of block I in registers (RPL complex rows per lane, R <= 32 RPL) for all BW
//          inner rounds and streams the J columns through shared memory, so a cross rotation
//          reads and writes one column of shared memory instead of two, and reduces with warp
//          shuffles only.
template <int BW, int RPL>
struct SvdShape {
    static constexpr int NT = RPL > 0 ? 32 * BW : SVD_THREADS;
};

// ---- K3: sort + keep rule + discarded weight, by one CTA once wk.sig2 holds the column
// norms.  Shared by the block-tournament and the resident Jacobi; `bytes` is the global
// traffic the caller's Jacobi moved (run statistics).  red holds >= 4 (blockDim.x / 32) doubles.
template <typename T>
__device__ void svd_finish(const MpsView<T>& mps, const SvdWork<T>& wk, const SvdParams& pp, const int R, const int N,
                           const double keep_floor, const int sweep, const bool converged, const double bytes,
                           unsigned char* smraw, double* red, const double flops = 0.0) {
    const int tid = threadIdx.x;
    const int NT = blockDim.x, NW = NT >> 5;
    int P2 = 1;
    while (P2 < N) P2 <<= 1;
    double* key = reinterpret_cast<double*>(smraw);  // [P2] then idx [P2]: 12 P2 bytes
    int* idx = reinterpret_cast<int*>(key + P2);
    for (int e = tid; e < P2; e += NT) {
        key[e] = e < N ? wk.sig2[e] : -1.0;
        idx[e] = e;
    }
    __syncthreads();
    for (int k = 2; k <= P2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int e = tid; e < P2; e += NT) {
                const int o = e ^ j;
                if (o > e) {
                    const bool desc = ((e & k) == 0);
                    const double ke = key[e], ko = key[o];
                    const int ie = idx[e], io = idx[o];
                    // "e before o" in descending order with ascending-index tie break
                    const bool e_first = (ke > ko) || (ke == ko && ie < io);
                    if (desc ? !e_first : e_first) {
                        key[e] = ko; key[o] = ke; idx[e] = io; idx[o] = ie;
                    }
                }
            }
            __syncthreads();
        }
    const int kk = R < N ? R : N;
    const int keep0 = pp.chi < kk ? pp.chi : kk;
    double tot = 0.0, big = 0.0;
    for (int e = tid; e < kk; e += NT) {
        const double v = key[e] > 0 ? key[e] : 0.0;
        tot += v;
        if (e < keep0 && v >= keep_floor) big += 1.0;
    }
    tot = warp_sum(tot);
    big = warp_sum(big);
    if ((tid & 31) == 0) { red[(tid >> 5) * 4] = tot; red[(tid >> 5) * 4 + 1] = big; }
    __syncthreads();
    __shared__ int s_keep;
    __shared__ double s_tot;
    if (tid == 0) {
        double t2 = 0.0, b2 = 0.0;
        for (int w = 0; w < NW; ++w) { t2 += red[w * 4]; b2 += red[w * 4 + 1]; }
        int keep = pp.no_trunc ? kk : (int)b2;
        if (keep < 1) keep = 1;
        s_keep = keep;
        s_tot = t2;
    }
    __syncthreads();
    const int keep = s_keep;
    double disc = 0.0;
    for (int e = keep + tid; e < kk; e += NT) disc += key[e] > 0 ? key[e] : 0.0;
    disc = warp_sum(disc);
    __syncthreads();
    if ((tid & 31) == 0) red[(tid >> 5) * 4 + 2] = disc;
    for (int e = tid; e < keep; e += NT) {
        wk.perm[e] = idx[e];
        wk.sig[e] = sqrt(key[e] > 0 ? key[e] : 0.0);
    }
    __syncthreads();
    if (tid == 0 && !pp.no_trunc) {
        double d2 = 0.0;
        for (int w = 0; w < NW; ++w) d2 += red[w * 4 + 2];
        RunStats* st = wk.stats;
        if (s_tot > 0) {
            const double ratio = d2 / s_tot;
            if (ratio > st->max_trunc) st->max_trunc = ratio;
        }
        if (!isfinite(s_tot)) st->status |= ST_NONFINITE;
        if (keep < kk && key[0] > 0) {
            const double s0 = sqrt(key[0]), a = sqrt(fmax(key[keep - 1], 0.0)), b = sqrt(fmax(key[keep], 0.0));
            const double deficit = 1.0 - (a - b) / s0;
            if (deficit > st->gap_deficit) st->gap_deficit = deficit;
        }
        if (!converged) st->status |= ST_JACOBI_NOT_CONVERGED;
        if (sweep > st->max_sweeps) st->max_sweeps = sweep;
        st->svd_sweeps += sweep;
        st->svd_bytes += bytes;
        st->svd_flops += flops;
        if (keep > st->max_bond) st->max_bond = keep;
        st->updates += 1;
        mps.dims[pp.bond + 1] = keep;
    }
}

// Whole SVD of one theta by `ncta` cooperating CTAs (this one is number `cta`); with
// ncta == 1 a single CTA runs every block pair itself and needs no grid barrier.
template <typename T, int BW, int RPL>
__device__ __forceinline__ void svd_body(const MpsView<T>& mps, const SvdWork<T>& wk, const SvdParams& pp,
                                         const int cta, const int ncta, unsigned char* smraw) {
    using V = cplx_t<T>;
    constexpr int NT = SvdShape<BW, RPL>::NT;
    constexpr int NW = NT / 32;
    constexpr int G = NT / BW;
    V* col = reinterpret_cast<V*>(smraw);  // [2*BW][rows_cap]
    __shared__ double red[4 * NW];         // [warps][4]
    __shared__ int s_rot;
    __shared__ __align__(8) uint64_t s_mbar;
    unsigned phase = 0;
    if (threadIdx.x == 0) mbar_init(&s_mbar, 1);
    __syncthreads();
    const int tid = threadIdx.x;
    const int R = pp.R > 0 ? pp.R : 2 * mps.dims[pp.bond];
    const int N0 = pp.N > 0 ? pp.N : 2 * mps.dims[pp.bond + 2];
    const int N = pp.lq && N0 > R ? R : N0;
    const int ld = wk.ld;
    V* W = wk.W;
    const int nb = (N + BW - 1) / BW;
    const int P = nb + (nb & 1);
    const unsigned int nblk = (unsigned)ncta;
    int* status = &wk.stats->status;
    if (R > pp.rows_cap) {  // host sizing bug guard: never index past shared memory
        if (cta == 0 && tid == 0) atomicOr(status, ST_BAD_DIMS);
        return;
    }
    const int grp = tid / G;
    if (ncta == 1) {  // a lone CTA owns its counters (cooperative launches zero them on the host)
        for (int e = tid; e < pp.max_sweeps; e += NT) wk.counters[e] = 0;
        if (tid == 0) wk.scal[0] = 0.0;
        __syncthreads();
    }
    // ||W||_F^2 first: columns whose squared norm is below the noise floor of the matrix
    // (tiny) are left alone once the sweeps settle (pair_live), and the keep rule drops them.
    {
        const int warp = tid >> 5, lane = tid & 31;
        double part = 0.0;
        for (int j = cta * NW + warp; j < N; j += ncta * NW) {
            double sj = 0.0;
            const V* w = W + (long long)j * ld;
            for (int row = lane; row < R; row += 32) sj += (double)w[row].x * w[row].x + (double)w[row].y * w[row].y;
            part += warp_sum(sj);
        }
        if (lane == 0) red[warp] = part;
        __syncthreads();
        if (tid == 0) {
            double b = 0.0;
            for (int w = 0; w < NW; ++w) b += red[w];
            if (b != 0.0) atomicAdd(&wk.scal[0], b);
        }
    }
    if (!cta_sync(wk.bar, status, nblk)) return;
    const double fro2 = *(volatile double*)&wk.scal[0];
    // Noise floor: a column whose norm is below 8 sqrt(R) ulps of ||W||_F carries only rounding
    // noise and is dropped by the keep rule; pairs of such columns are never rotated (that never
    // converges and costs many sweeps on rank-deficient theta), and pairs with one of them only
    // in the early sweeps (pair_live).
    const double ulp = sizeof(T) == 8 ? 2.220446049250313e-16 : 1.1920928955078125e-07;
    const double floor_rel = 8.0 * sqrt((double)R) * ulp;
    const double tiny = fmax(pp.tiny, floor_rel * floor_rel * fro2);
    const double keep_floor = fmax(1e-28, tiny);  // on sigma^2: the reference's 1e-14, or the noise floor
    int sweep = 0;
    bool converged = false;
    bool mixed = true;
    for (; sweep < pp.max_sweeps; ++sweep) {
        for (int r = 0; r < P - 1; ++r) {
            for (int pr = cta; pr < P / 2; pr += ncta) {
                int I, J;
                tournament(P, r, pr, I, J);
                // stage columns with 1-D TMA bulk copies: local c < BW -> block I, c >= BW -> block J
                if (tid == 0) {
                    s_rot = 0;
                    unsigned bytes = 0;
                    for (int c = 0; c < 2 * BW; ++c) {
                        const int gc = (c < BW) ? I * BW + c : J * BW + (c - BW);
                        if (gc < N) bytes += (unsigned)(R * sizeof(V));
                    }
                    fence_proxy_async_global();
                    mbar_expect_tx(&s_mbar, bytes);
                    for (int c = 0; c < 2 * BW; ++c) {
                        const int gc = (c < BW) ? I * BW + c : J * BW + (c - BW);
                        if (gc < N)
                            tma_load_1d(col + c * pp.rows_cap, W + (long long)gc * ld, (unsigned)(R * sizeof(V)),
                                        &s_mbar);
                    }
                }
                if (!mbar_wait(&s_mbar, phase, 1000000000ull)) {
                    atomicOr(status, ST_BARRIER_TIMEOUT);
                    // keep waiting (bounded) for the copies in flight before leaving
                    mbar_wait(&s_mbar, phase, 1000000000ull);
                    return;
                }
                phase ^= 1u;
                int rot = 0;
                if constexpr (BW >= 2) if (r == 0) {
                    // intra-block pairs: circle method over BW columns, both blocks at once
                    const int half = BW / 2;
                    const int blk = grp < half ? 0 : 1;
                    const int ip = grp < half ? grp : grp - half;
                    for (int t = 0; t < BW - 1; ++t) {
                        int x, y;
                        if (ip == 0) { x = BW - 1; y = t; }
                        else { x = (t + ip) % (BW - 1); y = (t - ip + (BW - 1)) % (BW - 1); }
                        const int base = blk ? J * BW : I * BW;
                        const bool ok = (base + x < N) && (base + y < N);
                        rot += rotate_pair<T, G>(col + (blk * BW + x) * pp.rows_cap, col + (blk * BW + y) * pp.rows_cap,
                                                 ok, R, pp.tol, tiny, mixed, red, tid);
                        __syncthreads();
                    }
                }
                if constexpr (RPL == 0) {
                    for (int t = 0; t < BW; ++t) {
                        const int p = grp, q = (grp + t) % BW;
                        const bool ok = (I * BW + p < N) && (J * BW + q < N);
                        rot += rotate_pair<T, G>(col + p * pp.rows_cap, col + (BW + q) * pp.rows_cap, ok, R, pp.tol,
                                                 tiny, mixed, red, tid);
                        __syncthreads();
                    }
                } else {
                    static_assert(G == 32, "register path: one warp per pair");
                    const int lane = tid & 31;
                    const bool vi = I * BW + grp < N;
                    V* ci = col + grp * pp.rows_cap;
                    V xi[RPL];
#pragma unroll
                    for (int k = 0; k < RPL; ++k) {
                        const int row = lane + 32 * k;
                        xi[k] = (row < R) ? ci[row] : czero<V>();
                    }
                    for (int t = 0; t < BW; ++t) {
                        const int q = (grp + t) % BW;
                        const bool ok = vi && (J * BW + q < N);
                        V* cq = col + (BW + q) * pp.rows_cap;
                        V yj[RPL];
#pragma unroll
                        for (int k = 0; k < RPL; ++k) {
                            const int row = lane + 32 * k;
                            yj[k] = (row < R) ? cq[row] : czero<V>();
                        }
                        double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
                        if constexpr (sizeof(T) == 4) {
                            LaneDotsF32 d;
#pragma unroll
                            for (int k = 0; k < RPL; ++k) d.add(xi[k], yj[k]);
                            v0 = d.a; v1 = d.b; v2 = d.gr; v3 = d.gi;
                        } else {
#pragma unroll
                            for (int k = 0; k < RPL; ++k) {
                                const V x = xi[k], y = yj[k];
                                v0 += (double)x.x * x.x + (double)x.y * x.y;
                                v1 += (double)y.x * y.x + (double)y.y * y.y;
                                v2 += (double)x.x * y.x + (double)x.y * y.y;
                                v3 += (double)x.x * y.y - (double)x.y * y.x;
                            }
                        }
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) {
                            v0 += __shfl_xor_sync(0xffffffffu, v0, o);
                            v1 += __shfl_xor_sync(0xffffffffu, v1, o);
                            v2 += __shfl_xor_sync(0xffffffffu, v2, o);
                            v3 += __shfl_xor_sync(0xffffffffu, v3, o);
                        }
                        T c, sn, er, ei;
                        if (ok && jacobi_rotation<T>(v0, v1, v2, v3, pp.tol, tiny, mixed, c, sn, er, ei)) {
                            const PairRot<T> rt(c, sn, er, ei);
#pragma unroll
                            for (int k = 0; k < RPL; ++k) rt.apply(xi[k], yj[k]);
#pragma unroll
                            for (int k = 0; k < RPL; ++k) {
                                const int row = lane + 32 * k;
                                if (row < R) cq[row] = yj[k];
                            }
                            if (lane == 0) ++rot;
                        }
                        __syncthreads();
                    }
#pragma unroll
                    for (int k = 0; k < RPL; ++k) {
                        const int row = lane + 32 * k;
                        if (row < R) ci[row] = xi[k];
                    }
                    __syncthreads();
                }
                if (rot && (tid % G) == 0) atomicAdd(&s_rot, rot);
                __syncthreads();
                for (int c = 0; c < 2 * BW; ++c) {
                    const int gc = (c < BW) ? I * BW + c : J * BW + (c - BW);
                    if (gc >= N) continue;
                    V* dst = W + (long long)gc * ld;
                    const V* src = col + c * pp.rows_cap;
                    for (int row = tid; row < R; row += NT) dst[row] = src[row];
                }
                if (tid == 0 && s_rot) atomicAdd(&wk.counters[sweep], s_rot);
                __syncthreads();
            }
            if (!cta_sync(wk.bar, status, nblk)) return;
        }
        const int done = *(volatile int*)&wk.counters[sweep];
        if (done == 0) {
            converged = true;
            ++sweep;
            break;
        }
        mixed = still_mixed(mixed, done, N, sweep);
    }
    // column norms -> sig2 (FP64)
    {
        const int warp = tid >> 5, lane = tid & 31;
        for (int j = cta * NW + warp; j < N; j += ncta * NW) {
            double s = 0.0;
            const V* w = W + (long long)j * ld;
            for (int row = lane; row < R; row += 32) s += (double)w[row].x * w[row].x + (double)w[row].y * w[row].y;
            s = warp_sum(s);
            if (lane == 0) wk.sig2[j] = s;
        }
    }
    if (!cta_sync(wk.bar, status, nblk)) return;
    if (cta != 0) return;
    // pairs evaluated (16 flops per row: four FP64 dot products) and rotated (32 per row)
    double rots = 0.0;
    for (int e = 0; e < sweep && e < pp.max_sweeps; ++e) rots += (double)(*(volatile int*)&wk.counters[e]);
    const double flops = (double)sweep * 0.5 * N * (N - 1) * R * 16.0 + rots * R * 32.0;
    svd_finish<T>(mps, wk, pp, R, N, keep_floor, sweep, converged,
                  ((double)sweep * (P - 1) * 2.0 + 2.0) * (double)R * N * sizeof(V), smraw, red, flops);
}

// ------------------------------------------------------------------------------------
// K2r: resident one-sided Jacobi for small theta.  The whole R x N matrix stays in shared
// memory (column c at col + c * rows_cap) for the entire SVD, so there is no staging and
// no block structure: every round of the circle method over all N columns rotates N/2
// disjoint pairs.  A pair is owned by LPP lanes (RPL complex rows per lane, R <= LPP RPL),
// so a warp rotates 32/LPP pairs at once and the reduction is log2(LPP) shuffle levels;
// alpha, beta, gamma are accumulated and reduced in FP64 and the rotation is
// jacobi_rotation's.  A sweep is N-1 rounds; a sweep without a rotation ends the
// iteration.  Up to 8 register rows per lane (fewer in use for small R) and LPP by size
// class: 8 up to R = 64, 16 up to 128, 32 up to 256.  One instantiation serves a whole class,
// so a theta is rotated by the same instructions whatever batch it runs in.
// ------------------------------------------------------------------------------------
constexpr int RES_MAXT = 512;
constexpr int RES_RPL = 8;  // register rows per lane; R <= LPP * RES_RPL

template <typename T, int LPP>
__device__ void jacobi_core(cplx_t<T>* col, const int rc, const int R, const int N, const double tol,
                            const double tiny, const int max_sweeps, int* s_rot, int& sweeps, bool& converged,
                            double& rotations) {
    using V = cplx_t<T>;
    constexpr int PPW = 32 / LPP;
    constexpr int RPL = RES_RPL;
    const int rpl = (R + LPP - 1) / LPP;  // rows per lane in use (<= RPL)
    const int tid = threadIdx.x, NW = blockDim.x >> 5, warp = tid >> 5, lane = tid & 31;
    const int sub = lane / LPP, sl = lane % LPP;
    const int Nc = N + (N & 1);
    const int npairs = Nc / 2;
    if (tid == 0) {
        s_rot[0] = 0;
        s_rot[1] = 0;
    }
    __syncthreads();
    int sweep = 0;
    converged = false;
    rotations = 0.0;
    bool mixed = true;
    for (; sweep < max_sweeps; ++sweep) {
        int rot = 0;
        for (int r = 0; r < Nc - 1; ++r) {
            for (int base = warp * PPW; base < npairs; base += NW * PPW) {  // warp-uniform
                const int pr = base + sub;
                int p = N, q = N;
                if (pr < npairs) tournament(Nc, r, pr, p, q);
                const bool ok = p < N && q < N;
                V* cp = col + (ok ? p : 0) * rc;
                V* cq = col + (ok ? q : 0) * rc;
                V x[RPL], y[RPL];
#pragma unroll
                for (int k = 0; k < RPL; ++k) {
                    const int row = sl + LPP * k;
                    const bool in = ok && k < rpl && row < R;
                    x[k] = in ? cp[row] : czero<V>();
                    y[k] = in ? cq[row] : czero<V>();
                }
                double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
                if constexpr (sizeof(T) == 4) {
                    LaneDotsF32 d;
#pragma unroll
                    for (int k = 0; k < RPL; ++k) {
                        if (k >= rpl) break;
                        d.add(x[k], y[k]);
                    }
                    v0 = d.a; v1 = d.b; v2 = d.gr; v3 = d.gi;
                } else {
#pragma unroll
                    for (int k = 0; k < RPL; ++k) {
                        if (k >= rpl) break;
                        v0 += (double)x[k].x * x[k].x + (double)x[k].y * x[k].y;
                        v1 += (double)y[k].x * y[k].x + (double)y[k].y * y[k].y;
                        v2 += (double)x[k].x * y[k].x + (double)x[k].y * y[k].y;
                        v3 += (double)x[k].x * y[k].y - (double)x[k].y * y[k].x;
                    }
                }
#pragma unroll
                for (int o = LPP / 2; o > 0; o >>= 1) {
                    v0 += __shfl_xor_sync(0xffffffffu, v0, o);
                    v1 += __shfl_xor_sync(0xffffffffu, v1, o);
                    v2 += __shfl_xor_sync(0xffffffffu, v2, o);
                    v3 += __shfl_xor_sync(0xffffffffu, v3, o);
                }
                T c, sn, er, ei;
                if (ok && jacobi_rotation<T>(v0, v1, v2, v3, tol, tiny, mixed, c, sn, er, ei)) {
                    const PairRot<T> rt(c, sn, er, ei);
#pragma unroll
                    for (int k = 0; k < RPL; ++k) {
                        if (k >= rpl) break;
                        const int row = sl + LPP * k;
                        V xv = x[k], yv = y[k];
                        rt.apply(xv, yv);
                        if (row < R) {
                            cp[row] = xv;
                            cq[row] = yv;
                        }
                    }
                    if (sl == 0) ++rot;
                }
            }
            __syncthreads();
        }
        // per-sweep rotation count in alternating slots: the slot read here is reset only
        // after the barrier that ends the next sweep's first round
        if (rot) atomicAdd(&s_rot[sweep & 1], rot);
        __syncthreads();
        const int done = s_rot[sweep & 1];
        if (tid == 0) s_rot[(sweep + 1) & 1] = 0;
        rotations += done;
        if (done == 0) {
            converged = true;
            ++sweep;
            break;
        }
        mixed = still_mixed(mixed, done, N, sweep);
    }
    sweeps = sweep;
    __syncthreads();
}

// sum of |w|^2 over an R x N shared-memory matrix, returned to every thread
template <typename T>
__device__ double block_fro2(const cplx_t<T>* col, const int rc, const int R, const int N, double* red) {
    using V = cplx_t<T>;
    __shared__ double s_sum;
    const int tid = threadIdx.x, NW = blockDim.x >> 5, warp = tid >> 5, lane = tid & 31;
    double part = 0.0;
    for (int c = warp; c < N; c += NW) {
        const V* w = col + c * rc;
        double sj = 0.0;
        for (int r = lane; r < R; r += 32) sj += (double)w[r].x * w[r].x + (double)w[r].y * w[r].y;
        part += warp_sum(sj);
    }
    if (lane == 0) red[warp] = part;
    __syncthreads();
    if (tid == 0) {
        double b = 0.0;
        for (int w = 0; w < NW; ++w) b += red[w];
        s_sum = b;
    }
    __syncthreads();
    return s_sum;
}

// column norms of the shared-memory matrix into wk.sig2 (optionally writing the columns to W)
template <typename T>
__device__ void resident_norms(const cplx_t<T>* col, const int rc, const int R, const int N, cplx_t<T>* W,
                               const int ld, double* sig2) {
    using V = cplx_t<T>;
    const int NW = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = warp; c < N; c += NW) {
        const V* src = col + c * rc;
        double sj = 0.0;
        for (int r = lane; r < R; r += 32) {
            const V w = src[r];
            if (W) W[(long long)c * ld + r] = w;
            sj += (double)w.x * w.x + (double)w.y * w.y;
        }
        sj = warp_sum(sj);
        if (lane == 0) sig2[c] = sj;
    }
    __syncthreads();
}

__device__ __forceinline__ double noise_tiny(double pp_tiny, int R, double fro2, bool single) {
    const double ulp = single ? 1.1920928955078125e-07 : 2.220446049250313e-16;
    const double floor_rel = 8.0 * sqrt((double)R) * ulp;
    return fmax(pp_tiny, floor_rel * floor_rel * fro2);
}

template <typename T, int LPP>
__device__ void svd_resident_body(const MpsView<T>& mps, const SvdWork<T>& wk, const SvdParams& pp,
                                  unsigned char* smraw) {
    using V = cplx_t<T>;
    const int NW = blockDim.x >> 5;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    __shared__ double red[4 * 32];
    __shared__ int s_rot[2];
    const int R = pp.R > 0 ? pp.R : 2 * mps.dims[pp.bond];
    const int N0 = pp.N > 0 ? pp.N : 2 * mps.dims[pp.bond + 2];
    const int N = pp.lq && N0 > R ? R : N0;
    const int rc = pp.rows_cap;
    V* col = reinterpret_cast<V*>(smraw);  // [cols_cap][rows_cap]
    if (R > rc || R > LPP * RES_RPL || N > pp.cols_cap) {  // host sizing bug guard
        if (tid == 0) atomicOr(&wk.stats->status, ST_BAD_DIMS);
        return;
    }
    const int ld = wk.ld;
    for (int c = warp; c < N; c += NW) {
        const V* src = wk.W + (long long)c * ld;
        V* dst = col + c * rc;
        for (int r = lane; r < R; r += 32) dst[r] = src[r];
    }
    __syncthreads();
    const double tiny = noise_tiny(pp.tiny, R, block_fro2<T>(col, rc, R, N, red), sizeof(T) == 4);
    int sweep = 0;
    bool converged = false;
    double rots = 0.0;
    jacobi_core<T, LPP>(col, rc, R, N, pp.tol, tiny, pp.max_sweeps, s_rot, sweep, converged, rots);
    resident_norms<T>(col, rc, R, N, wk.W, ld, wk.sig2);
    const double flops = (double)sweep * 0.5 * N * (N - 1) * R * 16.0 + rots * R * 32.0;
    svd_finish<T>(mps, wk, pp, R, N, fmax(1e-28, tiny), sweep, converged, 2.0 * (double)R * N * sizeof(V), smraw,
                  red, flops);
}

template <typename T, int LPP>
__global__ void __launch_bounds__(RES_MAXT, 1) k_svd_res(MpsView<T> mps, SvdWork<T> wk, SvdParams pp) {
    extern __shared__ __align__(16) unsigned char smraw[];
    svd_resident_body<T, LPP>(mps, wk, pp, smraw);
}

template <typename T, int LPP>
__global__ void __launch_bounds__(RES_MAXT, 1) k_svd_res_batch(const InstTask<T>* insts, const UpdRef* refs,
                                                              int nref) {
    extern __shared__ __align__(16) unsigned char smraw[];
    for (int t = blockIdx.x; t < nref; t += gridDim.x) {
        const UpdRef rf = refs[t];
        const InstTask<T>& it = insts[rf.inst];
        SvdParams pp = it.pp;
        pp.bond = rf.op.bond;
        svd_resident_body<T, LPP>(it.mps, it.wk, pp, smraw);
        __syncthreads();
    }
}

template <typename T>
__device__ void chain_body(const MpsView<T>& mps, int right, const ChainStep* steps, int nsteps, cplx_t<T>* envs,
                           cplx_t<T>* X, GridBar* bar, RunStats* stats, int cta, int ncta);
template <typename T>
__device__ void entropy_body(const MpsView<T>& mps, const cplx_t<T>* r1, double* out, const int* step);

// ------------------------------------------------------------------------------------
// K8: the whole anneal of small-bond instances, one CTA per instance at a time.  A CTA
// takes the next instance (longest first) from a work counter and runs every Trotter step
// of it: single-site half step, every two-site update of the ZZ block in order (theta
// quads formed straight into shared memory, resident Jacobi, keep rule, absorption from
// shared memory), single-site half step, qubit-0 entropy.  Nothing waits on another CTA,
// so instances never wait for the slowest SVD of a gate slot and the whole run is one
// launch.  256 threads (the environment GEMMs of the entropy step use 256).
// ------------------------------------------------------------------------------------
template <typename T, int LPP>
__device__ void resident_update(const MpsView<T>& mps, const ScheduleView& sch, const GateOp& op,
                                const SvdWork<T>& wk, const SvdParams& pp0, cplx_t<T>* col, unsigned char* sortbuf,
                                double* red, int* s_rot) {
    using V = cplx_t<T>;
    const int tid = threadIdx.x, NT = blockDim.x;
    const int i = op.bond;
    const int dl = mps.dims[i], mid = mps.dims[i + 1], dr = mps.dims[i + 2];
    const int R = 2 * dl, N = 2 * dr, rc = pp0.rows_cap, ld = wk.ld, cap = mps.cap;
    if (R > rc || R > LPP * RES_RPL || N > pp0.cols_cap) {
        if (tid == 0) atomicOr(&wk.stats->status, ST_BAD_DIMS);
        return;
    }
    // theta[(2a + r1), (r2 dr + b)] = sum_{s1 s2} G[r1 r2][s1 s2] sum_c A[(2a+s1), c] C[(2c+s2), b]
    {
        V g[16];
        gate_of(op, sch, nullptr, g);
        const V* A = mps.site(i);
        const V* Cm = mps.site(i + 1);
        for (int e = tid; e < dl * dr; e += NT) {
            const int a = e / dr, b = e - a * dr;
            V acc[2][2];
#pragma unroll
            for (int q = 0; q < 4; ++q) (&acc[0][0])[q] = czero<V>();
            const V* a0 = A + (long long)(2 * a) * cap;
            const V* a1 = a0 + cap;
            for (int c = 0; c < mid; ++c) {
                const V x0 = a0[c], x1 = a1[c];
                const V y0 = Cm[(long long)(2 * c) * cap + b], y1 = Cm[(long long)(2 * c + 1) * cap + b];
                cfma(acc[0][0], x0, y0); cfma(acc[0][1], x0, y1);
                cfma(acc[1][0], x1, y0); cfma(acc[1][1], x1, y1);
            }
#pragma unroll
            for (int r1 = 0; r1 < 2; ++r1)
#pragma unroll
                for (int r2 = 0; r2 < 2; ++r2) {
                    V o = czero<V>();
#pragma unroll
                    for (int s1 = 0; s1 < 2; ++s1)
#pragma unroll
                        for (int s2 = 0; s2 < 2; ++s2) cfma(o, g[(r1 * 2 + r2) * 4 + s1 * 2 + s2], acc[s1][s2]);
                    const int row = 2 * a + r1, cc = r2 * dr + b;
                    col[cc * rc + row] = o;
                    wk.theta[(long long)cc * ld + row] = o;
                }
        }
    }
    __syncthreads();
    const double tiny = noise_tiny(pp0.tiny, R, block_fro2<T>(col, rc, R, N, red), sizeof(T) == 4);
    int sweep = 0;
    bool converged = false;
    double rots = 0.0;
    jacobi_core<T, LPP>(col, rc, R, N, pp0.tol, tiny, pp0.max_sweeps, s_rot, sweep, converged, rots);
    resident_norms<T>(col, rc, R, N, nullptr, ld, wk.sig2);
    SvdParams pp = pp0;
    pp.bond = i;
    // global traffic of the update: A and C read, theta written and read back, A' and C' written
    const double bytes = (double)sizeof(V) * (2.0 * dl * mid + 2.0 * mid * dr + 3.0 * R * N);
    const double flops = (double)sweep * 0.5 * N * (N - 1) * R * 16.0 + rots * R * 32.0;
    svd_finish<T>(mps, wk, pp, R, N, fmax(1e-28, tiny), sweep, converged, bytes, sortbuf, red, flops);
    __syncthreads();
    const int keep = mps.dims[i + 1];
    // A' (a, s1, k) = W[(2a+s1), perm k] / sigma_k
    V* An = mps.site(i);
    for (int e = tid; e < R * keep; e += NT) {
        const int row = e / keep, k = e - row * keep;
        const double inv = 1.0 / wk.sig[k];
        const V w = col[wk.perm[k] * rc + row];
        An[(long long)row * cap + k] = mk<V>((T)(w.x * inv), (T)(w.y * inv));
    }
    // C' (k, s2, b) = (1/sigma_k) sum_row conj(W[row, perm k]) theta[row, s2 dr + b]
    V* Cn = mps.site(i + 1);
    for (int e = tid; e < keep * N; e += NT) {
        const int k = e / N, j = e - k * N;
        const V* u = col + wk.perm[k] * rc;
        const V* t = wk.theta + (long long)j * ld;
        double re = 0.0, im = 0.0;
        for (int row = 0; row < R; ++row) {
            const V uu = u[row], tt = t[row];
            re += (double)uu.x * tt.x + (double)uu.y * tt.y;
            im += (double)uu.x * tt.y - (double)uu.y * tt.x;
        }
        const double inv = 1.0 / wk.sig[k];
        const int s2 = j >= dr ? 1 : 0, b = j - s2 * dr;
        Cn[(long long)(2 * k + s2) * cap + b] = mk<V>((T)(re * inv), (T)(im * inv));
    }
    __syncthreads();
}

template <typename T, int LPP>
__global__ void __launch_bounds__(256) k_anneal_res(const InstTask<T>* insts, const GateOp* ops, const int* op_off,
                                                    const int* order, int ninst, int k0, int k1, int* work,
                                                    size_t col_bytes) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double red[4 * 32];
    __shared__ int s_rot[2];
    __shared__ int s_step;
    __shared__ int s_idx;
    const int tid = threadIdx.x;
    cplx_t<T>* col = reinterpret_cast<cplx_t<T>*>(smraw);
    unsigned char* sortbuf = smraw + col_bytes;
    for (;;) {
        if (tid == 0) s_idx = atomicAdd(work, 1);
        __syncthreads();
        const int idx = s_idx;
        __syncthreads();
        if (idx >= ninst) break;
        const int b = order[idx];
        const InstTask<T>& it = insts[b];
        const MpsView<T> mps = it.mps;
        ScheduleView sch = it.sch;
        sch.step = &s_step;
        const int q0 = op_off[b], q1 = op_off[b + 1];
        for (int k = k0; k < k1; ++k) {
            if (tid == 0) s_step = k;
            __syncthreads();
            for (int i = 0; i < mps.n; ++i) single_site_body<T>(mps, sch, i, 0, 1);
            __syncthreads();
            for (int q = q0; q < q1; ++q)
                resident_update<T, LPP>(mps, sch, ops[q], it.wk, it.pp, col, sortbuf, red, s_rot);
            for (int i = 0; i < mps.n; ++i) single_site_body<T>(mps, sch, i, 0, 1);
            __syncthreads();
            if (mps.n >= 2) {
                chain_body<T>(mps, 1, it.ent_steps, it.n_ent, it.envs, it.X, nullptr, it.wk.stats, 0, 1);
                __syncthreads();
                entropy_body<T>(mps, it.envs + it.r1_off, it.entropy, &s_step);
            } else {
                entropy_body<T>(mps, nullptr, it.entropy, &s_step);
            }
            __syncthreads();
        }
    }
}

// Shared memory of the resident kernels for a rows_cap x cols_cap theta (0: does not fit).
// with_cols: the sort buffer follows the matrix instead of overlaying it.
template <typename T>
static size_t resident_smem(int rows_cap, int cols_cap, bool with_cols = false) {
    int P2 = 1;
    while (P2 < cols_cap) P2 <<= 1;
    const size_t m = sizeof(cplx_t<T>) * (size_t)rows_cap * cols_cap;
    const size_t sort = (size_t)P2 * (sizeof(double) + sizeof(int));
    const size_t b = with_cols ? ((m + 15) & ~(size_t)15) + sort : (m < sort ? sort : m);
    return (rows_cap <= 256 && b <= 200 * 1024) ? b : 0;
}

// lanes per pair for a row count: the size class (8 lanes up to 64 rows, 16 up to 128, 32 up to 256)
static int resident_lpp(int rows_cap) {
    if (rows_cap <= 8 * RES_RPL) return 8;
    if (rows_cap <= 16 * RES_RPL) return 16;
    if (rows_cap <= 32 * RES_RPL) return 32;
    return 0;
}

#define TQ_RES_SHAPES(F)                     \
    switch (resident_lpp(pp.rows_cap)) {     \
        case 8: F(8); break;                 \
        case 16: F(16); break;               \
        case 32: F(32); break;               \
        default: return false;               \
    }

// Launch one resident-Jacobi kernel (single theta when insts == nullptr, else a batch).
template <typename T, int LPP>
static void res_launch(const MpsView<T>* mps, const SvdWork<T>* wk, const SvdParams& pp, const InstTask<T>* insts,
                       const UpdRef* refs, int nref, cudaStream_t s) {
    const size_t smem = resident_smem<T>(pp.rows_cap, pp.cols_cap);
    const int pairs = pp.cols_cap / 2;
    const int warps = (pairs + (32 / LPP) - 1) / (32 / LPP);
    int nt = 32 * (warps < 1 ? 1 : warps);
    if (nt > RES_MAXT) nt = RES_MAXT;
    if (insts) {
        auto fn = k_svd_res_batch<T, LPP>;
        TQ_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        TQ_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, nt, smem));
        if (per_sm < 1) throw std::runtime_error("k_svd_res_batch does not fit on an SM");
        int grid = per_sm * num_sms();
        if (grid > nref) grid = nref;
        fn<<<grid, nt, smem, s>>>(insts, refs, nref);
    } else {
        auto fn = k_svd_res<T, LPP>;
        TQ_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        fn<<<1, nt, smem, s>>>(*mps, *wk, pp);
    }
    TQ_CHECK(cudaGetLastError());
}

template <typename T>
static bool res_dispatch(const MpsView<T>* mps, const SvdWork<T>* wk, const SvdParams& pp, const InstTask<T>* insts,
                         const UpdRef* refs, int nref, cudaStream_t s) {
    if (!resident_smem<T>(pp.rows_cap, pp.cols_cap)) return false;
#define TQ_F(L) res_launch<T, L>(mps, wk, pp, insts, refs, nref, s)
    TQ_RES_SHAPES(TQ_F)
#undef TQ_F
    return true;
}

template <typename T, int LPP>
static void anneal_res_launch(const InstTask<T>* insts, const GateOp* ops, const int* op_off, const int* order,
                              int ninst, int k0, int k1, int* work, int rows_cap, cudaStream_t s) {
    const size_t smem = resident_smem<T>(rows_cap, rows_cap, true);
    const size_t col_bytes = (sizeof(cplx_t<T>) * (size_t)rows_cap * rows_cap + 15) & ~(size_t)15;
    auto fn = k_anneal_res<T, LPP>;
    TQ_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    TQ_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, smem));
    if (per_sm < 1) throw std::runtime_error("k_anneal_res does not fit on an SM");
    int grid = per_sm * num_sms();
    if (grid > ninst) grid = ninst;
    TQ_CHECK(cudaMemsetAsync(work, 0, sizeof(int), s));
    fn<<<grid, 256, smem, s>>>(insts, ops, op_off, order, ninst, k0, k1, work, col_bytes);
    TQ_CHECK(cudaGetLastError());
}

template <typename T>
bool launch_anneal_resident(const InstTask<T>* insts, const GateOp* ops, const int* op_off, const int* order,
                            int ninst, int k0, int k1, int* work, int rows_cap, cudaStream_t s) {
    if (!resident_smem<T>(rows_cap, rows_cap, true)) return false;
    SvdParams pp{};
    pp.rows_cap = rows_cap;
#define TQ_F(L) anneal_res_launch<T, L>(insts, ops, op_off, order, ninst, k0, k1, work, rows_cap, s)
    TQ_RES_SHAPES(TQ_F)
#undef TQ_F
    return true;
}

// ------------------------------------------------------------------------------------
// K2g: block-Gram one-sided Jacobi for large theta, one CTA per theta (the batched path).
// Columns are cut into blocks of BG_B = 32; a round-robin tournament over the P blocks gives
// P-1 rounds of P/2 block pairs per sweep, all taken by the one CTA in turn.  For a block
// pair (64 columns Wp) the CTA
//   1. forms the 64 x 64 Gram matrix G = Wp^H Wp in FP64 from row chunks of the 64 columns,
//      streamed into shared memory by 1-D TMA bulk copies (two buffers: the copy of chunk
//      k+1 runs under the arithmetic on chunk k);
//   2. runs one cyclic sweep of two-sided Jacobi on G (circle method, 32 disjoint rotations
//      per round, each from jacobi_rotation on (G_pp, G_qq, G_pq): the rotation the
//      column-pair kernel would compute from the same dot products), accumulating the
//      64 x 64 unitary V;
//   3. applies Wp <- Wp V over the row chunks (a GEMM) -- skipped when nothing rotated.
// The convergence test is FP64 on every pair of a freshly formed Gram matrix; a sweep in
// which no block pair rotates ends the iteration.  Per sweep the columns are read twice and
// written once per block pair: (P-1) (2 + 1) column passes for P = N/32 blocks, against
// 2 (P-1) passes of 8-column blocks (P = N/8) in the column-pair kernel, and the arithmetic
// is two GEMMs per block pair instead of one shuffle reduction and one barrier per pair.
// ------------------------------------------------------------------------------------
constexpr int BG_B = 32;
constexpr int BG_W = 2 * BG_B;  // columns of a block pair
constexpr int BG_RC = 32;       // rows per streamed chunk
constexpr int BG_NT = 256;
constexpr int BG_GS = BG_W + 1;  // padded row stride of G and V (double2 elements)

template <typename T>
struct BgShape {
    // padded column stride of a chunk (elements): odd for 16-byte elements (bank spread),
    // even for 8-byte ones (16-byte aligned TMA destinations)
    static constexpr int CS = sizeof(T) == 8 ? BG_RC + 1 : BG_RC + 2;
    static constexpr size_t g_bytes = sizeof(double2) * BG_W * BG_GS;
    static constexpr size_t chunk_bytes = ((sizeof(cplx_t<T>) * BG_W * CS + 127) / 128) * 128;
    static constexpr size_t smem = 2 * g_bytes + 2 * chunk_bytes;
};

struct BgRot {
    double c, s, er, ei;
    int p, q, act, pad;
};

template <typename T>
__device__ __forceinline__ int bg_col(int c, int I, int J, int N) {
    const int g = c < BG_B ? I * BG_B + c : J * BG_B + (c - BG_B);
    return g < N ? g : -1;
}

// Stage rows [r0, r0 + BG_RC) of the pair's 64 columns into `ch` (column c at c * CS):
// thread 0 issues one bulk copy per valid column; all threads zero the rest.
template <typename T>
__device__ __forceinline__ void bg_stage(cplx_t<T>* ch, const cplx_t<T>* W, int ld, int R, int N, int I, int J,
                                         int r0, uint64_t* bar) {
    using V = cplx_t<T>;
    constexpr int CS = BgShape<T>::CS;
    const int rows = R - r0 < BG_RC ? R - r0 : BG_RC;
    const int tid = threadIdx.x;
    for (int e = tid; e < BG_W * BG_RC; e += BG_NT) {
        const int c = e / BG_RC, r = e - c * BG_RC;
        if (bg_col<T>(c, I, J, N) < 0 || r >= rows) ch[c * CS + r] = czero<V>();
    }
    if (tid == 0) {
        unsigned nv = 0;
        for (int c = 0; c < BG_W; ++c) nv += bg_col<T>(c, I, J, N) >= 0;
        const unsigned bytes = (unsigned)(rows * sizeof(V));
        fence_proxy_async_shared();
        mbar_expect_tx(bar, nv * bytes);
        for (int c = 0; c < BG_W; ++c) {
            const int g = bg_col<T>(c, I, J, N);
            if (g >= 0) tma_load_1d(ch + c * CS, W + (long long)g * ld + r0, bytes, bar);
        }
    }
}

// Wait for a staged chunk with one CTA-wide decision: thread 0 waits (bounded) and
// publishes the outcome, every thread then re-checks the completed phase (bounded, returns
// at once) so that its own reads of the buffer are ordered after the copies.
__device__ __forceinline__ bool bg_wait(uint64_t* bar, unsigned& ph, int* s_ok) {
    if (threadIdx.x == 0) *s_ok = mbar_wait(bar, ph, 1000000000ull) ? 1 : 0;
    __syncthreads();
    const bool ok = *s_ok != 0;
    if (ok && threadIdx.x != 0) mbar_wait(bar, ph, 1000000000ull);
    if (ok) ph ^= 1u;
    return ok;
}

// One block pair: Gram, one Jacobi sweep on it, apply.  Returns false (on every thread) when
// a copy did not complete within its time budget.
template <typename T>
__device__ bool bg_pair(const SvdWork<T>& wk, int R, int N, int I, int J, double tol, double tiny, bool mixed,
                        double2* G,
                        double2* Vm, cplx_t<T>* ch0, cplx_t<T>* ch1, uint64_t* bars, unsigned* phase, BgRot* prm,
                        int* s_rot, double* bytes, double* flops) {
    using V = cplx_t<T>;
    constexpr int CS = BgShape<T>::CS;
    const int tid = threadIdx.x;
    const int ld = wk.ld;
    V* W = wk.W;
    V* ch[2] = {ch0, ch1};
    const int nchunk = (R + BG_RC - 1) / BG_RC;
    int nvalid = 0;
    for (int c = 0; c < BG_W; ++c) nvalid += bg_col<T>(c, I, J, N) >= 0;
    // ---- 1. Gram: thread (ti, tj) owns G[ti + 16k][tj + 16l], k, l < 4 ----
    const int ti = tid >> 4, tj = tid & 15;
    double2 acc[4][4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int l = 0; l < 4; ++l) acc[k][l] = make_double2(0.0, 0.0);
    bg_stage<T>(ch[0], W, ld, R, N, I, J, 0, &bars[0]);
    for (int kc = 0; kc < nchunk; ++kc) {
        const int b = kc & 1;
        if (kc + 1 < nchunk) bg_stage<T>(ch[b ^ 1], W, ld, R, N, I, J, (kc + 1) * BG_RC, &bars[b ^ 1]);
        if (!bg_wait(&bars[b], phase[b], &s_rot[2])) return false;  // (its barrier also publishes the zero fills)
        const V* cb = ch[b];
#pragma unroll 2
        for (int r = 0; r < BG_RC; ++r) {
            V a[4], y[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                a[k] = cb[(ti + 16 * k) * CS + r];
                y[k] = cb[(tj + 16 * k) * CS + r];
            }
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int l = 0; l < 4; ++l) {
                    const double ax = a[k].x, ay = a[k].y, bx = y[l].x, by = y[l].y;
                    acc[k][l].x = fma(ax, bx, fma(ay, by, acc[k][l].x));
                    acc[k][l].y = fma(ax, by, fma(-ay, bx, acc[k][l].y));
                }
        }
        __syncthreads();  // buffer b free for the copy after next
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int l = 0; l < 4; ++l) G[(ti + 16 * k) * BG_GS + tj + 16 * l] = acc[k][l];
    for (int e = tid; e < BG_W * BG_W; e += BG_NT) {
        const int i = e / BG_W, j = e - i * BG_W;
        Vm[i * BG_GS + j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    }
    if (tid == 0) s_rot[1] = 0;
    __syncthreads();
    *bytes += (double)nvalid * R * sizeof(V);
    *flops += 8.0 * nvalid * nvalid * R;  // Gram: one complex multiply-add per entry and row
    // ---- 2. one cyclic two-sided Jacobi sweep on G, V accumulated ----
    for (int rd = 0; rd < BG_W - 1; ++rd) {
        if (tid < BG_W / 2) {
            int p, q;
            tournament(BG_W, rd, tid, p, q);
            BgRot t;
            t.p = p;
            t.q = q;
            const double2 gpq = G[p * BG_GS + q];
            t.act = jacobi_rotation<double>(G[p * BG_GS + p].x, G[q * BG_GS + q].x, gpq.x, gpq.y, tol, tiny, mixed,
                                            t.c, t.s, t.er, t.ei)
                        ? 1
                        : 0;
            prm[tid] = t;
            if (t.act) atomicAdd(&s_rot[1], 1);
        }
        __syncthreads();
        // columns p, q of G and V:  x' = c x - s conj(e) y,  y' = s e x + c y
        for (int e = tid; e < 2 * BG_W * (BG_W / 2); e += BG_NT) {
            const int m = e / (BG_W * (BG_W / 2));
            const int rem = e - m * (BG_W * (BG_W / 2));
            const int k = rem / BG_W, row = rem - k * BG_W;
            const BgRot t = prm[k];
            if (!t.act) continue;
            double2* M = m ? Vm : G;
            const double2 x = M[row * BG_GS + t.p], y = M[row * BG_GS + t.q];
            const double ey_re = t.er * y.x + t.ei * y.y, ey_im = t.er * y.y - t.ei * y.x;
            const double ex_re = t.er * x.x - t.ei * x.y, ex_im = t.er * x.y + t.ei * x.x;
            M[row * BG_GS + t.p] = make_double2(t.c * x.x - t.s * ey_re, t.c * x.y - t.s * ey_im);
            M[row * BG_GS + t.q] = make_double2(t.s * ex_re + t.c * y.x, t.s * ex_im + t.c * y.y);
        }
        __syncthreads();
        // rows p, q of G:  x' = c x - s e y,  y' = s conj(e) x + c y
        for (int e = tid; e < BG_W * (BG_W / 2); e += BG_NT) {
            const int k = e / BG_W, col = e - k * BG_W;
            const BgRot t = prm[k];
            if (!t.act) continue;
            const double2 x = G[t.p * BG_GS + col], y = G[t.q * BG_GS + col];
            const double ey_re = t.er * y.x - t.ei * y.y, ey_im = t.er * y.y + t.ei * y.x;
            const double ex_re = t.er * x.x + t.ei * x.y, ex_im = t.er * x.y - t.ei * x.x;
            G[t.p * BG_GS + col] = make_double2(t.c * x.x - t.s * ey_re, t.c * x.y - t.s * ey_im);
            G[t.q * BG_GS + col] = make_double2(t.s * ex_re + t.c * y.x, t.s * ex_im + t.c * y.y);
        }
        __syncthreads();
    }
    const int nrot = s_rot[1];
    // a two-sided rotation updates two columns of G and V and two rows of G: 3 x 64 x 2 complex
    // entries at 16 flops each
    *flops += (double)nrot * 3.0 * BG_W * 2.0 * 16.0;
    if (nrot == 0) return true;
    if (tid == 0) s_rot[0] += nrot;
    // ---- 3. Wp <- Wp V: thread (tr, tc) owns chunk row tr, columns tc + 8m ----
    const int tr = tid & 31, tc = tid >> 5;
    bg_stage<T>(ch[0], W, ld, R, N, I, J, 0, &bars[0]);
    for (int kc = 0; kc < nchunk; ++kc) {
        const int b = kc & 1;
        if (kc + 1 < nchunk) bg_stage<T>(ch[b ^ 1], W, ld, R, N, I, J, (kc + 1) * BG_RC, &bars[b ^ 1]);
        if (!bg_wait(&bars[b], phase[b], &s_rot[2])) return false;
        const V* cb = ch[b];
        double2 o[8];
#pragma unroll
        for (int m = 0; m < 8; ++m) o[m] = make_double2(0.0, 0.0);
        for (int k = 0; k < BG_W; ++k) {
            const V w = cb[k * CS + tr];
            const double wx = w.x, wy = w.y;
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                const double2 v = Vm[k * BG_GS + tc + 8 * m];
                o[m].x = fma(wx, v.x, fma(-wy, v.y, o[m].x));
                o[m].y = fma(wx, v.y, fma(wy, v.x, o[m].y));
            }
        }
        const int row = kc * BG_RC + tr;
        if (row < R)
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                const int g = bg_col<T>(tc + 8 * m, I, J, N);
                if (g >= 0) W[(long long)g * ld + row] = mk<V>((T)o[m].x, (T)o[m].y);
            }
        __syncthreads();
    }
    // the next block pair's bulk copies read what these stores wrote
    fence_proxy_async_global();
    __syncthreads();
    *bytes += 2.0 * (double)nvalid * R * sizeof(V);
    *flops += 8.0 * BG_W * nvalid * R;  // apply: 64 complex multiply-adds per output element
    return true;
}

template <typename T>
__device__ void svd_bgj_body(const MpsView<T>& mps, const SvdWork<T>& wk, const SvdParams& pp, unsigned char* smraw) {
    using V = cplx_t<T>;
    __shared__ double red[4 * (BG_NT / 32)];
    __shared__ int s_rot[3];  // [0] rotations this sweep, [1] this block pair, [2] copy-wait outcome
    __shared__ BgRot prm[BG_W / 2];
    __shared__ __align__(8) uint64_t bars[2];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int NW = BG_NT / 32;
    const int R = pp.R > 0 ? pp.R : 2 * mps.dims[pp.bond];
    const int N = pp.N > 0 ? pp.N : 2 * mps.dims[pp.bond + 2];
    int* status = &wk.stats->status;
    double2* G = reinterpret_cast<double2*>(smraw);
    double2* Vm = G + BG_W * BG_GS;
    V* ch0 = reinterpret_cast<V*>(smraw + 2 * BgShape<T>::g_bytes);
    V* ch1 = reinterpret_cast<V*>(smraw + 2 * BgShape<T>::g_bytes + BgShape<T>::chunk_bytes);
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
    }
    unsigned phase[2] = {0u, 0u};
    // ||W||_F^2 for the noise floor
    double part = 0.0;
    for (int j = warp; j < N; j += NW) {
        const V* w = wk.W + (long long)j * wk.ld;
        double sj = 0.0;
        for (int row = lane; row < R; row += 32) sj += (double)w[row].x * w[row].x + (double)w[row].y * w[row].y;
        part += warp_sum(sj);
    }
    if (lane == 0) red[warp] = part;
    __syncthreads();
    double fro2 = 0.0;
    for (int w = 0; w < NW; ++w) fro2 += red[w];
    const double tiny = noise_tiny(pp.tiny, R, fro2, sizeof(T) == 4);
    __syncthreads();
    const int nb = (N + BG_B - 1) / BG_B;
    const int P = nb + (nb & 1);
    double bytes = (double)R * N * sizeof(V);
    double flops = 0.0;
    int sweep = 0;
    bool converged = false;
    bool mixed = true;
    for (; sweep < pp.max_sweeps; ++sweep) {
        if (tid == 0) s_rot[0] = 0;
        __syncthreads();
        for (int r = 0; r < P - 1; ++r)
            for (int pr = 0; pr < P / 2; ++pr) {
                int I, J;
                tournament(P, r, pr, I, J);
                if (!bg_pair<T>(wk, R, N, I, J, pp.tol, tiny, mixed, G, Vm, ch0, ch1, bars, phase, prm, s_rot, &bytes,
                                &flops)) {
                    // every thread leaves here together; wait (bounded) for the copies still in
                    // flight so that none lands in shared memory after the CTA has moved on
                    if (tid == 0) {
                        atomicOr(status, ST_BARRIER_TIMEOUT);
                        mbar_wait(&bars[0], phase[0], 1000000000ull);
                        mbar_wait(&bars[1], phase[1], 1000000000ull);
                    }
                    __syncthreads();
                    return;
                }
            }
        __syncthreads();
        const int done = s_rot[0];
        __syncthreads();
        if (done == 0) {
            converged = true;
            ++sweep;
            break;
        }
        mixed = still_mixed(mixed, done, N, sweep);
    }
    // column norms -> sig2 (FP64)
    for (int j = warp; j < N; j += NW) {
        const V* w = wk.W + (long long)j * wk.ld;
        double sj = 0.0;
        for (int row = lane; row < R; row += 32) sj += (double)w[row].x * w[row].x + (double)w[row].y * w[row].y;
        sj = warp_sum(sj);
        if (lane == 0) wk.sig2[j] = sj;
    }
    __syncthreads();
    bytes += (double)R * N * sizeof(V);
    svd_finish<T>(mps, wk, pp, R, N, fmax(1e-28, tiny), sweep, converged, bytes, smraw, red, flops);
}

template <typename T>
__global__ void __launch_bounds__(BG_NT, 1) k_svd_bgj_batch(const InstTask<T>* insts, const UpdRef* refs, int nref) {
    extern __shared__ __align__(16) unsigned char smraw[];
    for (int t = blockIdx.x; t < nref; t += gridDim.x) {
        const UpdRef rf = refs[t];
        const InstTask<T>& it = insts[rf.inst];
        SvdParams pp = it.pp;
        pp.bond = rf.op.bond;
        svd_bgj_body<T>(it.mps, it.wk, pp, smraw);
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(BG_NT, 1) k_svd_bgj(MpsView<T> mps, SvdWork<T> wk, SvdParams pp) {
    extern __shared__ __align__(16) unsigned char smraw[];
    svd_bgj_body<T>(mps, wk, pp, smraw);
}

// Block-Gram Jacobi for one theta (insts == nullptr) or a batch, one CTA per theta.
template <typename T>
static void bgj_launch(const MpsView<T>* mps, const SvdWork<T>* wk, const SvdParams* pp, const InstTask<T>* insts,
                       const UpdRef* refs, int nref, cudaStream_t s) {
    size_t smem = BgShape<T>::smem;
    const size_t sort_smem = 4096 * (sizeof(double) + sizeof(int));
    if (smem < sort_smem) smem = sort_smem;
    if (insts) {
        auto fn = k_svd_bgj_batch<T>;
        TQ_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int grid = num_sms();
        if (grid > nref) grid = nref;
        fn<<<grid, BG_NT, smem, s>>>(insts, refs, nref);
    } else {
        auto fn = k_svd_bgj<T>;
        TQ_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        fn<<<1, BG_NT, smem, s>>>(*mps, *wk, *pp);
    }
    TQ_CHECK(cudaGetLastError());
}

template <typename T, int BW, int RPL>
__global__ void __launch_bounds__(SvdShape<BW, RPL>::NT, 1) k_svd(MpsView<T> mps, SvdWork<T> wk, SvdParams pp) {
    extern __shared__ __align__(16) unsigned char smraw[];
    svd_body<T, BW, RPL>(mps, wk, pp, blockIdx.x, gridDim.x, smraw);
}

// ------------------------------------------------------------------------------------
// K2b: the batched column-pair Jacobi (one CTA per theta), block-row-cyclic.  With one CTA
// per theta the block pairs need not be disjoint within a round, so the sweep runs them in
// row-cyclic order: for each block I, first its BW(BW-1)/2 inner pairs (staged in shared
// memory), then block I stays in registers (warp w holds column w, RPL rows per lane) while
// the blocks J > I stream past it, two shared-memory buffers deep: the 1-D TMA bulk copy of
// block J+1 runs under the BW cross rounds of block J, and only J is written back after
// them.  Per sweep the columns move (nb + nb(nb-1)/2) times in each direction instead of
// 2 (P-1) P/2 times, and no copy waits in the open.  Every pair is visited once per sweep
// (a cyclic ordering), with the rotation of jacobi_rotation.
// ------------------------------------------------------------------------------------
constexpr int RC_MAXN = 1024;  // columns of one theta in the block-row-cyclic kernel

template <typename T>
__device__ __forceinline__ void rc_stage(cplx_t<T>* dst, const cplx_t<T>* W, int ld, int rc, int R, int N, int blk,
                                         int BW, uint64_t* bar, const int* perm) {
    using V = cplx_t<T>;
    unsigned nv = 0;
    for (int c = 0; c < BW; ++c) nv += blk * BW + c < N;
    const unsigned bytes = (unsigned)(R * sizeof(V));
    fence_proxy_async_shared();
    mbar_expect_tx(bar, nv * bytes);
    for (int c = 0; c < BW; ++c)
        if (blk * BW + c < N) tma_load_1d(dst + c * rc, W + (long long)perm[blk * BW + c] * ld, bytes, bar);
}

// descending bitonic sort of key[0..P2) carrying idx (ties: ascending idx); P2 a power of two
__device__ void bitonic_desc(double* key, int* idx, int P2) {
    const int tid = threadIdx.x, NT = blockDim.x;
    for (int k = 2; k <= P2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int e = tid; e < P2; e += NT) {
                const int o = e ^ j;
                if (o > e) {
                    const bool desc = ((e & k) == 0);
                    const double ke = key[e], ko = key[o];
                    const int ie = idx[e], io = idx[o];
                    const bool e_first = (ke > ko) || (ke == ko && ie < io);
                    if (desc ? !e_first : e_first) {
                        key[e] = ko; key[o] = ke; idx[e] = io; idx[o] = ie;
                    }
                }
            }
            __syncthreads();
        }
}

template <typename T, int BW, int RPL>
__device__ void svd_body_rc(const MpsView<T>& mps, const SvdWork<T>& wk, const SvdParams& pp, unsigned char* smraw) {
    using V = cplx_t<T>;
    constexpr int NT = 32 * BW;
    constexpr int NW = BW;
    constexpr int G2 = 2 * NT / BW;  // threads per pair of the inner rounds (BW/2 pairs)
    static_assert(RPL > 0, "register-resident rows");
    __shared__ double red[4 * NW];
    __shared__ int s_rot;
    __shared__ int s_ok;
    __shared__ __align__(8) uint64_t bars[3];  // [0] block I, [1], [2] the two J buffers
    // columns modified in the previous sweep and so far in this one: a block pair whose columns
    // are all unchanged since they were last found orthogonal is not checked again
    __shared__ unsigned char cprev[RC_MAXN], ccur[RC_MAXN];
    // this sweep's column order: descending norm (block position p holds column perm[p])
    __shared__ int perm[RC_MAXN];
    __shared__ int s_irot, s_jrot;
    // cross rounds: column q of the J buffer has been through s_ver[q] rounds since the SVD
    // began; warp w takes column (w + t) % BW in round t once its neighbour w + 1 has released
    // it from round t - 1, so warps are not held in step by a CTA barrier per round
    __shared__ int s_ver[BW];
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int R = pp.R > 0 ? pp.R : 2 * mps.dims[pp.bond];
    const int N0 = pp.N > 0 ? pp.N : 2 * mps.dims[pp.bond + 2];
    const int N = pp.lq && N0 > R ? R : N0;
    const int rc = pp.rows_cap;
    const int ld = wk.ld;
    V* W = wk.W;
    int* status = &wk.stats->status;
    if (R > rc || R > 32 * RPL) {  // host sizing bug guard
        if (tid == 0) atomicOr(status, ST_BAD_DIMS);
        return;
    }
    V* ci = reinterpret_cast<V*>(smraw);  // [BW][rc]
    V* cj[2] = {ci + BW * rc, ci + 2 * BW * rc};
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1);
    }
    unsigned ph[3] = {0u, 0u, 0u};
    // one CTA-wide outcome per copy wait (thread 0 waits, the others re-check the phase)
    auto wait = [&](int k) -> bool {
        if (tid == 0) s_ok = mbar_wait(&bars[k], ph[k], 1000000000ull) ? 1 : 0;
        __syncthreads();
        const bool ok = s_ok != 0;
        if (ok && tid != 0) mbar_wait(&bars[k], ph[k], 1000000000ull);
        if (ok) ph[k] ^= 1u;
        return ok;
    };
    // ||W||_F^2 for the noise floor
    double part = 0.0;
    for (int j = warp; j < N; j += NW) {
        const V* w = W + (long long)j * ld;
        double sj = 0.0;
        for (int row = lane; row < R; row += 32) sj += (double)w[row].x * w[row].x + (double)w[row].y * w[row].y;
        part += warp_sum(sj);
    }
    if (lane == 0) red[warp] = part;
    __syncthreads();
    double fro2 = 0.0;
    for (int w = 0; w < NW; ++w) fro2 += red[w];
    const double tiny = noise_tiny(pp.tiny, R, fro2, sizeof(T) == 4);
    __syncthreads();
    const int nb = (N + BW - 1) / BW;
    if (N > RC_MAXN) {  // host sizing bug guard
        if (tid == 0) atomicOr(status, ST_BAD_DIMS);
        return;
    }
    for (int e = tid; e < N; e += NT) { cprev[e] = 1; ccur[e] = 1; }
    if (tid < BW) s_ver[tid] = 0;
    if (tid == 0) s_fail = 0;
    int vbase = 0;  // rounds each J column has been through before the current J block
    double rots_total = 0.0;
    double pairs_checked = 0.0;
    double moved = 2.0 * nb;  // column blocks read or written (the norm passes: one read each)
    auto blk_dirty = [&](int B) {
        bool d = false;
        for (int c = 0; c < BW; ++c) {
            const int q = B * BW + c;
            if (q < N) d = d || cprev[perm[q]] || ccur[perm[q]];
        }
        return d;
    };
    // first block J >= j0 whose pair with I needs a check (nb: none)
    auto next_needed = [&](int j0, bool iflag) {
        int j = j0;
        while (j < nb && !(iflag || blk_dirty(j))) ++j;
        return j;
    };
    int P2 = 1;
    while (P2 < N) P2 <<= 1;
    int sweep = 0;
    bool converged = false;
    bool fail = false;
    bool mixed = true;
    for (; sweep < pp.max_sweeps && !fail; ++sweep) {
        if (tid == 0) s_rot = 0;
        __syncthreads();
        // order the columns by descending norm for this sweep (fewer sweeps in block-row-cyclic
        // order); the staging buffer is free between sweeps and holds the sort keys
        {
            double* key = reinterpret_cast<double*>(smraw);
            int* idx = reinterpret_cast<int*>(key + P2);
            for (int c = warp; c < P2; c += NW) {
                double sj = -1.0;
                if (c < N) {
                    const V* w = W + (long long)c * ld;
                    sj = 0.0;
                    for (int row = lane; row < R; row += 32)
                        sj += (double)w[row].x * w[row].x + (double)w[row].y * w[row].y;
                    sj = warp_sum(sj);
                }
                if (lane == 0) { key[c] = sj; idx[c] = c; }
            }
            __syncthreads();
            bitonic_desc(key, idx, P2);
            for (int e = tid; e < N; e += NT) {
                perm[e] = idx[e];
                cprev[e] = ccur[e];
                ccur[e] = 0;
            }
            moved += (double)N / BW;
            __syncthreads();
        }
        int rot = 0;
        for (int I = 0; I < nb && !fail; ++I) {
            const bool iflag = blk_dirty(I);
            int jn = next_needed(I + 1, iflag);
            if (!iflag && jn >= nb) continue;  // every pair of block I is unchanged and orthogonal
            if (tid == 0) { s_irot = 0; rc_stage<T>(ci, W, ld, rc, R, N, I, BW, &bars[0], perm); }
            moved += 1.0;
            if (!wait(0)) { fail = true; break; }
            // inner pairs of block I: circle method, BW/2 pairs per round, G2 threads each
            if (iflag) {
                pairs_checked += 0.5 * BW * (BW - 1);
                const int ip = tid / G2;
                for (int t = 0; t < BW - 1; ++t) {
                    int x, y;
                    if (ip == 0) { x = BW - 1; y = t; }
                    else { x = (t + ip) % (BW - 1); y = (t - ip + (BW - 1)) % (BW - 1); }
                    const bool ok = (I * BW + x < N) && (I * BW + y < N);
                    const int r1 = rotate_pair<T, G2>(ci + x * rc, ci + y * rc, ok, R, pp.tol, tiny, mixed, red, tid);
                    if (r1 && (tid % G2) == 0) { ++rot; s_irot = 1; }
                    __syncthreads();
                }
            }
            const bool vi = I * BW + warp < N;
            V xi[RPL];
#pragma unroll
            for (int k = 0; k < RPL; ++k) {
                const int row = lane + 32 * k;
                xi[k] = row < R ? ci[warp * rc + row] : czero<V>();
            }
            __syncthreads();  // ci free for the next block I
            if (jn < nb && tid == 0) rc_stage<T>(cj[0], W, ld, rc, R, N, jn, BW, &bars[1], perm);
            int b = 0;
            for (int J = jn; J < nb; J = jn, b ^= 1) {
                jn = next_needed(J + 1, iflag);
                if (jn < nb && tid == 0) rc_stage<T>(cj[b ^ 1], W, ld, rc, R, N, jn, BW, &bars[1 + (b ^ 1)], perm);
                if (tid == 0) s_jrot = 0;
                if (!wait(1 + b)) { fail = true; break; }
                pairs_checked += (double)BW * BW;
                moved += 1.0;
                V* cb = cj[b];
                for (int t = 0; t < BW; ++t) {
                    const int q = (warp + t) % BW;
                    const bool ok = vi && (J * BW + q < N);
                    V* cq = cb + q * rc;
                    if (t > 0) {  // bounded wait for warp w + 1 to release column q from round t - 1
                        if (lane == 0) {
                            const volatile int* vq = &s_ver[q];
                            unsigned spin = 0;
                            while (*vq < vbase + t && !*(volatile int*)&s_fail)
                                if (++spin > (1u << 24)) { s_fail = 1; break; }
                        }
                        __syncwarp();
                        __threadfence_block();
                    }
                    V yj[RPL];
#pragma unroll
                    for (int k = 0; k < RPL; ++k) {
                        const int row = lane + 32 * k;
                        yj[k] = (ok && row < R) ? cq[row] : czero<V>();
                    }
                    double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
                    if constexpr (sizeof(T) == 4) {
                        LaneDotsF32 d;
#pragma unroll
                        for (int k = 0; k < RPL; ++k) d.add(xi[k], yj[k]);
                        v0 = d.a; v1 = d.b; v2 = d.gr; v3 = d.gi;
                    } else {
#pragma unroll
                        for (int k = 0; k < RPL; ++k) {
                            const V x = xi[k], y = yj[k];
                            v0 += (double)x.x * x.x + (double)x.y * x.y;
                            v1 += (double)y.x * y.x + (double)y.y * y.y;
                            v2 += (double)x.x * y.x + (double)x.y * y.y;
                            v3 += (double)x.x * y.y - (double)x.y * y.x;
                        }
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        v0 += __shfl_xor_sync(0xffffffffu, v0, o);
                        v1 += __shfl_xor_sync(0xffffffffu, v1, o);
                        v2 += __shfl_xor_sync(0xffffffffu, v2, o);
                        v3 += __shfl_xor_sync(0xffffffffu, v3, o);
                    }
                    T c, sn, er, ei;
                    if (ok && jacobi_rotation<T>(v0, v1, v2, v3, pp.tol, tiny, mixed, c, sn, er, ei)) {
                        const PairRot<T> rt(c, sn, er, ei);
#pragma unroll
                        for (int k = 0; k < RPL; ++k) rt.apply(xi[k], yj[k]);
#pragma unroll
                        for (int k = 0; k < RPL; ++k) {
                            const int row = lane + 32 * k;
                            if (row < R) cq[row] = yj[k];
                        }
                        if (lane == 0) { ++rot; s_jrot = 1; s_irot = 1; }
                    }
                    // release column q to warp w - 1 for round t + 1
                    __syncwarp();
                    __threadfence_block();
                    if (lane == 0) *(volatile int*)&s_ver[q] = vbase + t + 1;
                }
                vbase += BW;
                __syncthreads();
                if (s_fail) { fail = true; break; }
                // block J back to global memory when it changed; later bulk copies read it
                if (s_jrot) {
                    moved += 1.0;
                    for (int c = warp; c < BW; c += NW) {
                        if (J * BW + c >= N) continue;
                        if (lane == 0) ccur[perm[J * BW + c]] = 1;
                        V* dst = W + (long long)perm[J * BW + c] * ld;
                        const V* src = cb + c * rc;
                        for (int row = lane; row < R; row += 32) dst[row] = src[row];
                    }
                    fence_proxy_async_global();
                }
                __syncthreads();
            }
            if (fail) break;
            const bool i_changed = s_irot != 0;
            if (i_changed && vi && lane == 0) ccur[perm[I * BW + warp]] = 1;
            if (i_changed) moved += 1.0;
            if (vi && i_changed) {
                V* dst = W + (long long)perm[I * BW + warp] * ld;
#pragma unroll
                for (int k = 0; k < RPL; ++k) {
                    const int row = lane + 32 * k;
                    if (row < R) dst[row] = xi[k];
                }
            }
            fence_proxy_async_global();
            __syncthreads();
        }
        if (fail) break;
        if (rot) atomicAdd(&s_rot, rot);
        __syncthreads();
        const int done = s_rot;
        __syncthreads();
        rots_total += done;
        if (done == 0) {
            converged = true;
            ++sweep;
            break;
        }
        mixed = still_mixed(mixed, done, N, sweep);
    }
    if (fail) {
        // every thread leaves together; wait (bounded) for copies still in flight
        if (tid == 0) {
            atomicOr(status, ST_BARRIER_TIMEOUT);
            for (int k = 0; k < 3; ++k) mbar_wait(&bars[k], ph[k], 1000000000ull);
        }
        __syncthreads();
        return;
    }
    // column norms -> sig2 (FP64)
    for (int j = warp; j < N; j += NW) {
        const V* w = W + (long long)j * ld;
        double sj = 0.0;
        for (int row = lane; row < R; row += 32) sj += (double)w[row].x * w[row].x + (double)w[row].y * w[row].y;
        sj = warp_sum(sj);
        if (lane == 0) wk.sig2[j] = sj;
    }
    __syncthreads();
    const double flops = pairs_checked * R * 16.0 + rots_total * R * 32.0;
    svd_finish<T>(mps, wk, pp, R, N, fmax(1e-28, tiny), sweep, converged, moved * (double)BW * R * sizeof(V), smraw,
                  red, flops);
}

// Batched: each CTA takes whole SVD tasks (one theta each) in turn; no inter-CTA waits.
// lq: W holds the pivoted LQ factor P L of theta (lq.cu), whose columns beyond min(R, N) are zero.
template <typename T, int BW, int RPL>
__global__ void __launch_bounds__(SvdShape<BW, RPL>::NT, 1) k_svd_batch(const InstTask<T>* insts, const UpdRef* refs,
                                                                       int nref, int lq) {
    extern __shared__ __align__(16) unsigned char smraw[];
    for (int t = blockIdx.x; t < nref; t += gridDim.x) {
        const UpdRef rf = refs[t];
        const InstTask<T>& it = insts[rf.inst];
        SvdParams pp = it.pp;
        pp.bond = rf.op.bond;
        pp.lq = lq;
        if constexpr (RPL > 0) svd_body_rc<T, BW, RPL>(it.mps, it.wk, pp, smraw);
        else svd_body<T, BW, RPL>(it.mps, it.wk, pp, 0, 1, smraw);
        __syncthreads();
    }
}

template <typename T, int BW, int RPL>
static int svd_launch_bw(const MpsView<T>& mps, const SvdParams& pp, SvdWork<T> wk, int cols_ub,
                         cudaStream_t s) {
    using V = cplx_t<T>;
    constexpr int NT = SvdShape<BW, RPL>::NT;
    size_t smem = sizeof(V) * 2 * BW * (size_t)pp.rows_cap;
    const size_t sort_smem = 4096 * (sizeof(double) + sizeof(int));
    if (smem < sort_smem) smem = sort_smem;
    auto fn = k_svd<T, BW, RPL>;
    TQ_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    TQ_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, NT, smem));
    if (per_sm < 1) throw std::runtime_error("k_svd does not fit on an SM");
    const int nb = (cols_ub + BW - 1) / BW;
    const int pairs = (nb + (nb & 1)) / 2;
    int grid = pairs < 1 ? 1 : pairs;
    const int maxg = per_sm * num_sms();
    if (grid > maxg) grid = maxg;
    MpsView<T> m = mps;
    SvdParams p = pp;
    void* args[] = {&m, &wk, &p};
    TQ_CHECK(cudaLaunchCooperativeKernel((const void*)fn, dim3(grid), dim3(NT), args, smem, s));
    return grid;
}

template <typename T>
int launch_svd(const MpsView<T>& mps, int bond, int chi, double tol, int max_sweeps, SvdWork<T> wk,
               int rows_ub, int cols_ub, int block_w, cudaStream_t s, int R, int N, int lq) {
    SvdParams pp{};
    pp.lq = lq;
    pp.bond = bond;
    pp.R = R;
    pp.N = N;
    pp.no_trunc = R > 0 ? 1 : 0;
    pp.chi = chi;
    pp.tol = tol;
    pp.tiny = sizeof(T) == 8 ? 1e-200 : 1e-60;
    pp.max_sweeps = max_sweeps;
    pp.rows_cap = (rows_ub + 7) & ~7;
    if (pp.rows_cap < 8) pp.rows_cap = 8;
    pp.cols_cap = (cols_ub + 1) & ~1;
    if (pp.cols_cap < 2) pp.cols_cap = 2;
    // small theta: the whole matrix stays in one CTA's shared memory
    if (res_dispatch<T>(&mps, &wk, pp, nullptr, nullptr, 0, s)) return 1;
    TQ_CHECK(cudaMemsetAsync(wk.counters, 0, sizeof(int) * max_sweeps, s));
    TQ_CHECK(cudaMemsetAsync(wk.scal, 0, sizeof(double) * 2, s));
    // register-resident path for rows <= 512: rows per lane = next power of two >= rows/32
    int rpl = 1;
    while (32 * rpl < pp.rows_cap) rpl <<= 1;
    if (rpl <= 16) {
        int bw = block_w < 4 ? 4 : block_w;
        if (rpl == 16 && bw > 8) bw = 8;  // registers: 2 columns x 16 rows per lane
#define TQ_RR(B, RP) \
    if (bw == B && rpl == RP) return svd_launch_bw<T, B, RP>(mps, pp, wk, cols_ub, s);
        TQ_RR(4, 1) TQ_RR(4, 2) TQ_RR(4, 4) TQ_RR(4, 8) TQ_RR(4, 16)
        TQ_RR(8, 1) TQ_RR(8, 2) TQ_RR(8, 4) TQ_RR(8, 8) TQ_RR(8, 16)
        TQ_RR(16, 1) TQ_RR(16, 2) TQ_RR(16, 4) TQ_RR(16, 8)
#undef TQ_RR
        throw std::runtime_error("unsupported Jacobi block width");
    }
    switch (block_w) {
        case 1:
        case 2: return svd_launch_bw<T, 2, 0>(mps, pp, wk, cols_ub, s);
        default: return svd_launch_bw<T, 4, 0>(mps, pp, wk, cols_ub, s);
    }
}

// ------------------------------------------------------------------------------------
// K4: absorption.  A_new(a, s1, k) = W[(2a+s1), perm[k]] / sigma_k ;
// C_new(k, s2, b) = (1/sigma_k) sum_row conj(W[row, perm[k]]) theta[row, s2*Dr + b].
// ------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void absorb_u_tile(const MpsView<T>& mps, int bond, const SvdWork<T>& wk, int tk, int tr) {
    using V = cplx_t<T>;
    const int R = 2 * mps.dims[bond];
    const int keep = mps.dims[bond + 1];
    const int k = tk * 32 + threadIdx.x;
    const int row = tr * 8 + threadIdx.y;
    if (k >= keep || row >= R) return;
    const double inv = 1.0 / wk.sig[k];
    const V w = wk.W[(long long)wk.perm[k] * wk.ld + row];
    mps.site(bond)[(long long)row * mps.cap + k] = mk<V>((T)(w.x * inv), (T)(w.y * inv));
}

template <typename T>
__global__ void k_absorb_u(MpsView<T> mps, int bond, SvdWork<T> wk) {
    absorb_u_tile<T>(mps, bond, wk, blockIdx.x, blockIdx.y);
}

template <typename T>
__device__ __forceinline__ void absorb_c_tile(const MpsView<T>& mps, int bond, const SvdWork<T>& wk, int tc, int tk) {
    using V = cplx_t<T>;
    constexpr int KC = 8;
    __shared__ V Us[KC][32];
    __shared__ V Ts[KC][32];
    __shared__ int pk[32];
    const int R = 2 * mps.dims[bond];
    const int keep = mps.dims[bond + 1];
    const int dr = mps.dims[bond + 2];
    const int N = 2 * dr;
    const int k0 = tk * 32, c0 = tc * 32;
    if (k0 >= keep || c0 >= N) return;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    if (tid < 32) pk[tid] = (k0 + tid < keep) ? wk.perm[k0 + tid] : -1;
    __syncthreads();
    const int ld = wk.ld;
    V acc[2][2];
    for (int q = 0; q < 4; ++q) (&acc[0][0])[q] = czero<V>();
    for (int r0 = 0; r0 < R; r0 += KC) {
        {
            const int kk = tid % KC, q = tid / KC;  // 256 = 8 x 32
            const int row = r0 + kk;
            const int pc = pk[q];
            V u = czero<V>();
            if (pc >= 0 && row < R) { u = wk.W[(long long)pc * ld + row]; u.y = -u.y; }
            Us[kk][q] = u;
            const int col = c0 + q;
            Ts[kk][q] = (col < N && row < R) ? wk.theta[(long long)col * ld + row] : czero<V>();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) {
            const V u0 = Us[kk][ty], u1 = Us[kk][ty + 16];
            const V t0 = Ts[kk][tx], t1 = Ts[kk][tx + 16];
            cfma(acc[0][0], u0, t0); cfma(acc[0][1], u0, t1);
            cfma(acc[1][0], u1, t0); cfma(acc[1][1], u1, t1);
        }
        __syncthreads();
    }
    V* Cn = mps.site(bond + 1);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int k = k0 + ty + 16 * i, col = c0 + tx + 16 * j;
            if (k >= keep || col >= N) continue;
            const int s2 = col >= dr ? 1 : 0, b = col - s2 * dr;
            const double inv = 1.0 / wk.sig[k];
            const V v = acc[i][j];
            Cn[(long long)(2 * k + s2) * mps.cap + b] = mk<V>((T)(v.x * inv), (T)(v.y * inv));
        }
}

template <typename T>
__global__ void __launch_bounds__(256) k_absorb_c(MpsView<T> mps, int bond, SvdWork<T> wk) {
    absorb_c_tile<T>(mps, bond, wk, blockIdx.x, blockIdx.y);
}

template <typename T>
void launch_absorb(const MpsView<T>& mps, int bond, SvdWork<T> wk, int rows_ub, int cols_ub, int keep_ub,
                   cudaStream_t s) {
    k_absorb_u<T><<<dim3((keep_ub + 31) / 32, (rows_ub + 7) / 8), dim3(32, 8), 0, s>>>(mps, bond, wk);
    TQ_CHECK(cudaGetLastError());
    k_absorb_c<T><<<dim3((cols_ub + 31) / 32, (keep_ub + 31) / 32), 256, 0, s>>>(mps, bond, wk);
    TQ_CHECK(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// K6: environment transfer chain (cooperative; two GEMM phases per step).
// ------------------------------------------------------------------------------------
template <typename V, class LA, class LB, class ST>
__device__ void gemm_phase(int M, int N, int K, LA la, LB lb, ST st, V (*As)[32], V (*Bs)[32], int cta, int ncta) {
    constexpr int KC = 8;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int tm = (M + 31) / 32, tn = (N + 31) / 32;
    for (int t = cta; t < tm * tn; t += ncta) {
        const int i0 = (t / tn) * 32, j0 = (t % tn) * 32;
        V acc[2][2];
        for (int q = 0; q < 4; ++q) (&acc[0][0])[q] = czero<V>();
        for (int k0 = 0; k0 < K; k0 += KC) {
            {
                const int kk = tid % KC, q = tid / KC;
                const int k = k0 + kk;
                As[kk][q] = (i0 + q < M && k < K) ? la(i0 + q, k) : czero<V>();
                Bs[kk][q] = (j0 + q < N && k < K) ? lb(k, j0 + q) : czero<V>();
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < KC; ++kk) {
                const V a0 = As[kk][ty], a1 = As[kk][ty + 16];
                const V b0 = Bs[kk][tx], b1 = Bs[kk][tx + 16];
                cfma(acc[0][0], a0, b0); cfma(acc[0][1], a0, b1);
                cfma(acc[1][0], a1, b0); cfma(acc[1][1], a1, b1);
            }
            __syncthreads();
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int ii = i0 + ty + 16 * i, jj = j0 + tx + 16 * j;
                if (ii < M && jj < N) st(ii, jj, acc[i][j]);
            }
    }
}

template <typename T>
__device__ void chain_body(const MpsView<T>& mps, int right, const ChainStep* steps, int nsteps, cplx_t<T>* envs,
                           cplx_t<T>* X, GridBar* bar, RunStats* stats, int cta, int ncta) {
    using V = cplx_t<T>;
    __shared__ V As[8][32];
    __shared__ V Bs[8][32];
    const int cap = mps.cap;
    const int ldx = 2 * cap;
    const unsigned int nblk = (unsigned)ncta;
    for (int q = 0; q < nsteps; ++q) {
        const ChainStep cs = steps[q];
        const int dl = mps.dims[cs.site], dr = mps.dims[cs.site + 1];
        const V* A = mps.site(cs.site);
        const V* E = envs + cs.in_off;
        V* O = envs + cs.out_off;
        const bool z = cs.zflag != 0;
        if (!right) {
            // Y[a', s*dr + b] = sum_a E[a, a'] A[(2a+s), b] z_s
            gemm_phase<V>(dl, 2 * dr, dl,
                [&](int i, int k) { return E[(long long)k * cap + i]; },
                [&](int k, int j) {
                    const int s = j >= dr ? 1 : 0, b = j - s * dr;
                    V v = A[(long long)(2 * k + s) * cap + b];
                    if (z && s) { v.x = -v.x; v.y = -v.y; }
                    return v;
                },
                [&](int i, int j, V v) { X[(long long)i * ldx + j] = v; }, As, Bs, cta, ncta);
            if (!cta_sync(bar, &stats->status, nblk)) return;
            // O[b, b'] = sum_{a', s} Y[a', s*dr + b] conj(A[(2a'+s), b'])
            gemm_phase<V>(dr, dr, 2 * dl,
                [&](int i, int k) { return X[(long long)(k >> 1) * ldx + (k & 1) * dr + i]; },
                [&](int k, int j) { V v = A[(long long)k * cap + j]; v.y = -v.y; return v; },
                [&](int i, int j, V v) { O[(long long)i * cap + j] = v; }, As, Bs, cta, ncta);
        } else {
            // X[(2a+s), b'] = sum_b A[(2a+s), b] E[b, b'] z_s
            gemm_phase<V>(2 * dl, dr, dr,
                [&](int i, int k) {
                    V v = A[(long long)i * cap + k];
                    if (z && (i & 1)) { v.x = -v.x; v.y = -v.y; }
                    return v;
                },
                [&](int k, int j) { return E[(long long)k * cap + j]; },
                [&](int i, int j, V v) { X[(long long)i * ldx + j] = v; }, As, Bs, cta, ncta);
            if (!cta_sync(bar, &stats->status, nblk)) return;
            // O[a, a'] = sum_{s, b'} X[(2a+s), b'] conj(A[(2a'+s), b'])   (k = s*dr + b')
            gemm_phase<V>(dl, dl, 2 * dr,
                [&](int i, int k) {
                    const int s = k >= dr ? 1 : 0, b = k - s * dr;
                    return X[(long long)(2 * i + s) * ldx + b];
                },
                [&](int k, int j) {
                    const int s = k >= dr ? 1 : 0, b = k - s * dr;
                    V v = A[(long long)(2 * j + s) * cap + b];
                    v.y = -v.y;
                    return v;
                },
                [&](int i, int j, V v) { O[(long long)i * cap + j] = v; }, As, Bs, cta, ncta);
        }
        if (!cta_sync(bar, &stats->status, nblk)) return;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_chain(MpsView<T> mps, int right, const ChainStep* steps, int nsteps,
                                               cplx_t<T>* envs, cplx_t<T>* X, GridBar* bar, RunStats* stats) {
    chain_body<T>(mps, right, steps, nsteps, envs, X, bar, stats, blockIdx.x, gridDim.x);
}

template <typename T>
void launch_chain(const MpsView<T>& mps, int right, const ChainStep* d_steps, int nsteps, cplx_t<T>* envs,
                  cplx_t<T>* scratch, GridBar* bar, RunStats* stats, int d_ub, cudaStream_t s) {
    if (nsteps <= 0) return;
    auto fn = k_chain<T>;
    int per_sm = 0;
    TQ_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0));
    const int tiles = ((2 * d_ub + 31) / 32) * ((d_ub + 31) / 32);
    int grid = tiles < 1 ? 1 : tiles;
    const int maxg = per_sm * num_sms();
    if (grid > maxg) grid = maxg;
    MpsView<T> m = mps;
    int r = right;
    int ns = nsteps;
    void* args[] = {&m, &r, (void*)&d_steps, &ns, &envs, &scratch, &bar, &stats};
    TQ_CHECK(cudaLaunchCooperativeKernel((const void*)fn, dim3(grid), dim3(256), args, 0, s));
}

// rho_0[s, s'] = sum_{b, b'} A0[s, b] R1[b, b'] conj(A0[s', b']), entropy in bits of rho/tr
// with eigenvalues clamped to [0, 1] and terms lambda <= 1e-12 dropped
// (cuda/src/mps.cpp:218-291).
template <typename T>
__device__ void entropy_body(const MpsView<T>& mps, const cplx_t<T>* r1, double* out, const int* step) {
    using V = cplx_t<T>;
    __shared__ double red[8][8];
    const int tid = threadIdx.x;
    const int d = mps.dims[1];
    const V* A = mps.site(0);
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // rho00, rho11 (re), rho01 (re, im)
    for (int bp = tid; bp < d; bp += blockDim.x) {
        double v0r = 0, v0i = 0, v1r = 0, v1i = 0;
        for (int b = 0; b < d; ++b) {
            const V rr = r1 ? r1[(long long)b * mps.cap + bp] : mk<V>(1, 0);
            const V x0 = A[b], x1 = A[mps.cap + b];
            v0r += (double)x0.x * rr.x - (double)x0.y * rr.y;
            v0i += (double)x0.x * rr.y + (double)x0.y * rr.x;
            v1r += (double)x1.x * rr.x - (double)x1.y * rr.y;
            v1i += (double)x1.x * rr.y + (double)x1.y * rr.x;
        }
        const V y0 = A[bp], y1 = A[mps.cap + bp];
        // v_s[bp] * conj(A0[s', bp])
        acc[0] += v0r * y0.x + v0i * y0.y;
        acc[1] += v1r * y1.x + v1i * y1.y;
        acc[2] += v0r * y1.x + v0i * y1.y;
        acc[3] += v0i * y1.x - v0r * y1.y;
    }
    for (int q = 0; q < 4; ++q) acc[q] = warp_sum(acc[q]);
    if ((tid & 31) == 0)
        for (int q = 0; q < 4; ++q) red[tid >> 5][q] = acc[q];
    __syncthreads();
    if (tid == 0) {
        double r00 = 0, r11 = 0, r01r = 0, r01i = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            r00 += red[w][0]; r11 += red[w][1]; r01r += red[w][2]; r01i += red[w][3];
        }
        const double tr = r00 + r11;
        double S = 0.0;
        if (tr > 0) {
            const double p = r00 / tr, q = r11 / tr;
            const double off2 = (r01r * r01r + r01i * r01i) / (tr * tr);
            const double mid = 0.5 * (p + q);
            const double rad = sqrt(fmax(0.0, 0.25 * (p - q) * (p - q) + off2));
            const double l1 = fmin(1.0, fmax(0.0, mid + rad)), l2 = fmin(1.0, fmax(0.0, mid - rad));
            if (l1 > 1e-12) S -= l1 * log2(l1);
            if (l2 > 1e-12) S -= l2 * log2(l2);
        }
        out[*step] = S;
    }
}

template <typename T>
__global__ void k_entropy(MpsView<T> mps, const cplx_t<T>* r1, double* out, const int* step) {
    entropy_body<T>(mps, r1, out, step);
}

template <typename T>
void launch_entropy(const MpsView<T>& mps, const cplx_t<T>* r1, double* out_entropy, const int* step,
                    cudaStream_t s) {
    k_entropy<T><<<1, 256, 0, s>>>(mps, r1, out_entropy, step);
    TQ_CHECK(cudaGetLastError());
}

template <typename T>
__global__ void k_pair_dots(MpsView<T> mps, const cplx_t<T>* envs, const PairDot* jobs, double* out) {
    using V = cplx_t<T>;
    __shared__ double red[8];
    const PairDot jb = jobs[blockIdx.x];
    const int d = mps.dims[jb.bond];
    const V* X = envs + jb.x_off;
    const V* Y = envs + jb.y_off;
    double acc = 0.0;
    for (int e = threadIdx.x; e < d * d; e += blockDim.x) {
        const int b = e / d, bp = e - b * d;
        const V x = X[(long long)b * mps.cap + bp], y = Y[(long long)b * mps.cap + bp];
        acc += (double)x.x * y.x - (double)x.y * y.y;
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        out[blockIdx.x] = s;
    }
}

template <typename T>
void launch_pair_dots(const MpsView<T>& mps, const cplx_t<T>* envs, const PairDot* d_jobs, int njobs, double* out,
                      cudaStream_t s) {
    if (njobs <= 0) return;
    k_pair_dots<T><<<njobs, 256, 0, s>>>(mps, envs, d_jobs, out);
    TQ_CHECK(cudaGetLastError());
}

// |<x|psi>|^2 for one spin pattern (+1 <-> physical 0), cuda/src/mps.cpp:197-216.
template <typename T>
__global__ void k_amplitude(MpsView<T> mps, const int8_t* spins, cplx_t<T>* vbuf, double* out) {
    using V = cplx_t<T>;
    V* v = vbuf;
    V* w = vbuf + mps.cap;
    if (threadIdx.x == 0) v[0] = mk<V>(1, 0);
    __syncthreads();
    for (int i = 0; i < mps.n; ++i) {
        const int dl = mps.dims[i], dr = mps.dims[i + 1];
        const int s = spins[i] > 0 ? 0 : 1;
        const V* A = mps.site(i);
        for (int b = threadIdx.x; b < dr; b += blockDim.x) {
            double re = 0, im = 0;
            for (int a = 0; a < dl; ++a) {
                const V x = v[a], y = A[(long long)(2 * a + s) * mps.cap + b];
                re += (double)x.x * y.x - (double)x.y * y.y;
                im += (double)x.x * y.y + (double)x.y * y.x;
            }
            w[b] = mk<V>((T)re, (T)im);
        }
        __syncthreads();
        V* t = v; v = w; w = t;
    }
    if (threadIdx.x == 0) out[0] = (double)v[0].x * v[0].x + (double)v[0].y * v[0].y;
}

template <typename T>
void launch_amplitude(const MpsView<T>& mps, const int8_t* spins, cplx_t<T>* scratch, double* out_amp2,
                      cudaStream_t s) {
    k_amplitude<T><<<1, 256, 0, s>>>(mps, spins, scratch, out_amp2);
    TQ_CHECK(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// K9: perfect sampling of basis patterns x with probability |<x|psi>|^2 / <psi|psi> from the
// MPS, site by site: with the left vector v = A_0^{s_0} ... A_{i-1}^{s_{i-1}} (rescaled) and
// the right environment R_{i+1} (the observables' chain), w_s = v A_i^s and
// p(s_i = s | s_<i) ~ w_s R_{i+1} w_s^dagger.  One CTA per sample, FP64 sums, a counter-based
// splitmix64 stream per (seed, sample, site).  Replaces the sign<Z> readout where it is
// undefined (Z2-symmetric instances, <Z_i> = 0).
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double sample_uniform(unsigned long long seed, int smp, int site) {
    unsigned long long x = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(smp + 1) +
                           0xD1B54A32D192ED03ull * (unsigned long long)(site + 1);
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x ^= x >> 31;
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

template <typename T>
__global__ void __launch_bounds__(256) k_sample(MpsView<T> mps, const cplx_t<T>* envs, int count,
                                                unsigned long long seed, int8_t* out) {
    using V = cplx_t<T>;
    extern __shared__ double2 sbuf[];  // v, w0, w1: cap complex each
    __shared__ double red[2][8];
    __shared__ double s_scale;
    __shared__ int s_pick;
    const int tid = threadIdx.x, NT = blockDim.x;
    const int n = mps.n, cap = mps.cap;
    double2* v = sbuf;
    double2* w0 = v + cap;
    double2* w1 = w0 + cap;
    const long long U = (long long)cap * cap;
    for (int smp = blockIdx.x; smp < count; smp += gridDim.x) {
        if (tid == 0) v[0] = make_double2(1.0, 0.0);
        __syncthreads();
        for (int i = 0; i < n; ++i) {
            const int dl = mps.dims[i], dr = mps.dims[i + 1];
            const V* A = mps.site(i);
            for (int b = tid; b < dr; b += NT) {
                double2 a0 = make_double2(0, 0), a1 = make_double2(0, 0);
                for (int a = 0; a < dl; ++a) {
                    const double2 va = v[a];
                    const V x0 = A[(long long)(2 * a) * cap + b], x1 = A[(long long)(2 * a + 1) * cap + b];
                    a0.x += va.x * x0.x - va.y * x0.y; a0.y += va.x * x0.y + va.y * x0.x;
                    a1.x += va.x * x1.x - va.y * x1.y; a1.y += va.x * x1.y + va.y * x1.x;
                }
                w0[b] = a0;
                w1[b] = a1;
            }
            __syncthreads();
            const V* Rm = envs + (i + 1 == n ? 0LL : (1LL + n + i + 1) * U);  // R_{i+1}; R_n = 1
            double p0 = 0.0, p1 = 0.0;
            for (int b = tid; b < dr; b += NT) {
                double2 t0 = make_double2(0, 0), t1 = make_double2(0, 0);  // sum_b' R[b, b'] conj(w[b'])
                for (int bp = 0; bp < dr; ++bp) {
                    const V r = Rm[(long long)b * cap + bp];
                    const double2 c0 = w0[bp], c1 = w1[bp];
                    t0.x += r.x * c0.x + r.y * c0.y; t0.y += r.y * c0.x - r.x * c0.y;
                    t1.x += r.x * c1.x + r.y * c1.y; t1.y += r.y * c1.x - r.x * c1.y;
                }
                p0 += w0[b].x * t0.x - w0[b].y * t0.y;
                p1 += w1[b].x * t1.x - w1[b].y * t1.y;
            }
            p0 = warp_sum(p0);
            p1 = warp_sum(p1);
            if ((tid & 31) == 0) { red[0][tid >> 5] = p0; red[1][tid >> 5] = p1; }
            __syncthreads();
            if (tid == 0) {
                double q0 = 0, q1 = 0;
                for (int w = 0; w < (NT >> 5); ++w) { q0 += red[0][w]; q1 += red[1][w]; }
                q0 = fmax(q0, 0.0);
                q1 = fmax(q1, 0.0);
                const double tot = q0 + q1;
                const int pick = (tot > 0 && sample_uniform(seed, smp, i) * tot >= q0) ? 1 : 0;
                s_pick = pick;
                const double pp = pick ? q1 : q0;
                s_scale = pp > 0 ? 1.0 / sqrt(pp) : 1.0;
                out[(long long)smp * n + i] = pick ? -1 : 1;  // physical 0 <-> spin +1
            }
            __syncthreads();
            const double2* wc = s_pick ? w1 : w0;
            const double sc = s_scale;
            for (int b = tid; b < dr; b += NT) v[b] = make_double2(wc[b].x * sc, wc[b].y * sc);
            __syncthreads();
        }
    }
}

template <typename T>
void launch_sample(const MpsView<T>& mps, const cplx_t<T>* envs, int count, unsigned long long seed, int8_t* out,
                   cudaStream_t s) {
    const size_t smem = sizeof(double2) * 3 * (size_t)mps.cap;
    auto fn = k_sample<T>;
    if (smem > 48 * 1024) TQ_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int grid = 4 * num_sms();
    if (grid > count) grid = count;
    fn<<<grid, 256, smem, s>>>(mps, envs, count, seed, out);
    TQ_CHECK(cudaGetLastError());
}

// ------------------------------------------------------------------------------------
// Batched kernels: many instances (each with its own MPS, workspace and statistics) in
// one launch.  Every instance keeps its own gate order; a launch runs gate q of every
// instance that has one.
// ------------------------------------------------------------------------------------
template <typename T>
__global__ void k_single_site_batch(const InstTask<T>* insts, int ninst) {
    const InstTask<T>& it = insts[blockIdx.z];
    single_site_body<T>(it.mps, it.sch, blockIdx.y, blockIdx.x, gridDim.x);
}

template <typename T>
void launch_single_site_batch(const InstTask<T>* insts, int ninst, int n_max, int d2_ub_max, cudaStream_t s) {
    int bx = (d2_ub_max + 255) / 256;
    bx = bx < 1 ? 1 : (bx > 16 ? 16 : bx);
    k_single_site_batch<T><<<dim3(bx, n_max, ninst), 256, 0, s>>>(insts, ninst);
    TQ_CHECK(cudaGetLastError());
}

template <typename T>
__global__ void __launch_bounds__(256) k_theta_batch(const InstTask<T>* insts, const UpdRef* refs) {
    const UpdRef rf = refs[blockIdx.z];
    const InstTask<T>& it = insts[rf.inst];
    theta_tile<T>(it.mps, it.sch, rf.op, nullptr, it.wk, blockIdx.x, blockIdx.y);
}

template <typename T>
__global__ void k_absorb_u_batch(const InstTask<T>* insts, const UpdRef* refs) {
    const UpdRef rf = refs[blockIdx.z];
    const InstTask<T>& it = insts[rf.inst];
    absorb_u_tile<T>(it.mps, rf.op.bond, it.wk, blockIdx.x, blockIdx.y);
}

template <typename T>
__global__ void __launch_bounds__(256) k_absorb_c_batch(const InstTask<T>* insts, const UpdRef* refs) {
    const UpdRef rf = refs[blockIdx.z];
    const InstTask<T>& it = insts[rf.inst];
    absorb_c_tile<T>(it.mps, rf.op.bond, it.wk, blockIdx.x, blockIdx.y);
}

template <typename T, int BW, int RPL>
static void svd_batch_bw(const InstTask<T>* insts, const UpdRef* refs, int nref, int rows_cap, cudaStream_t s,
                         int lq = 0) {
    using V = cplx_t<T>;
    constexpr int NT = SvdShape<BW, RPL>::NT;
    // block-row-cyclic (RPL > 0): block I plus two J buffers; else one staged block pair
    size_t smem = sizeof(V) * (RPL > 0 ? 3 : 2) * BW * (size_t)rows_cap;
    const size_t sort_smem = 4096 * (sizeof(double) + sizeof(int));
    if (smem < sort_smem) smem = sort_smem;
    auto fn = k_svd_batch<T, BW, RPL>;
    TQ_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    TQ_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, NT, smem));
    if (per_sm < 1) throw std::runtime_error("k_svd_batch does not fit on an SM");
    int grid = per_sm * num_sms();
    if (grid > nref) grid = nref;
    fn<<<grid, NT, smem, s>>>(insts, refs, nref, lq);
    TQ_CHECK(cudaGetLastError());
}

// complex64 at 512 rows: blocks of 16 columns (512 threads, 16 warps); a complex128 column pair
// of 512 rows does not fit in the registers that 16 warps leave each thread
template <typename T>
static bool svd_batch_wide(const InstTask<T>* insts, const UpdRef* refs, int nref, int rows_cap, cudaStream_t s,
                           int lq) {
    if constexpr (sizeof(T) == 4) {
        svd_batch_bw<T, 16, 16>(insts, refs, nref, rows_cap, s, lq);
        return true;
    }
    return false;
}

template <typename T>
int launch_update_batch(const InstTask<T>* insts, const UpdRef* refs, int nref, int d_ub, int rows_ub,
                        int block_w, cudaStream_t s, cudaEvent_t svd_begin, cudaEvent_t svd_end, bool theta_tc,
                        bool precond, cudaEvent_t lq_begin, cudaEvent_t lq_end) {
    if (nref <= 0) return 0;
    int launches = 4;
    if constexpr (sizeof(T) == 4) {
        if (theta_tc) {
            launch_theta_tc_batch(reinterpret_cast<const InstTask<float>*>(insts), refs, nref, d_ub, s);
        } else {
            const int tiles = (d_ub + 31) / 32;
            k_theta_batch<T><<<dim3(tiles, tiles, nref), 256, 0, s>>>(insts, refs);
        }
    } else {
        const int tiles = (d_ub + 31) / 32;
        k_theta_batch<T><<<dim3(tiles, tiles, nref), 256, 0, s>>>(insts, refs);
    }
    TQ_CHECK(cudaGetLastError());
    const int rows_cap = ((rows_ub + 7) & ~7) < 8 ? 8 : ((rows_ub + 7) & ~7);
    int rpl = 1;
    while (32 * rpl < rows_cap) rpl <<= 1;
    if (rpl > 16 && block_w != BG_B) throw std::runtime_error("the column-pair batched SVD supports at most 512 rows");
    int bw = block_w < 4 ? 4 : block_w;
    if (rpl == 16 && bw > 8 && !(sizeof(T) == 4 && bw == 16)) bw = 8;
    SvdParams rp{};
    rp.rows_cap = rows_cap;
    rp.cols_cap = rows_cap;  // every instance's theta is at most rows_ub x rows_ub
    // small theta: resident Jacobi; large theta: the column-pair kernel (block width 8, or the
    // one asked for; complex64 at 257..512 rows: 16), or the block-Gram kernel when block width
    // 32 is asked for
    if (block_w == 0) bw = (sizeof(T) == 4 && rpl == 16) ? 16 : 8;
    // the pivoted LQ preconditioner for the column-pair kernel at 257..512 rows (outside the
    // svd_begin/svd_end window, so that window times the Jacobi alone)
    const int lq = (precond && block_w != BG_B && rpl == 16 && resident_smem<T>(rows_cap, rows_cap) == 0) ? 1 : 0;
    if (lq) {  // lq_begin/lq_end are recorded only here: a return of 5 launches says they were
        if (lq_begin) TQ_CHECK(cudaEventRecord(lq_begin, s));
        launch_lq_batch<T>(insts, refs, nref, s);
        if (lq_end) TQ_CHECK(cudaEventRecord(lq_end, s));
        ++launches;
    }
    if (svd_begin) TQ_CHECK(cudaEventRecord(svd_begin, s));
    if (res_dispatch<T>(nullptr, nullptr, rp, insts, refs, nref, s)) {
    } else if (block_w == BG_B) {
        bgj_launch<T>(nullptr, nullptr, nullptr, insts, refs, nref, s);
    } else if (bw == 16 && rpl == 16 && svd_batch_wide<T>(insts, refs, nref, rows_cap, s, lq)) {
    } else {
#define TQ_RB(B, RP) \
    if (bw == B && rpl == RP) { svd_batch_bw<T, B, RP>(insts, refs, nref, rows_cap, s, lq); } else
        TQ_RB(4, 1) TQ_RB(4, 2) TQ_RB(4, 4) TQ_RB(4, 8) TQ_RB(4, 16)
        TQ_RB(8, 1) TQ_RB(8, 2) TQ_RB(8, 4) TQ_RB(8, 8) TQ_RB(8, 16)
        TQ_RB(16, 1) TQ_RB(16, 2) TQ_RB(16, 4) TQ_RB(16, 8)
        throw std::runtime_error("unsupported Jacobi block width");
#undef TQ_RB
    }
    if (svd_end) TQ_CHECK(cudaEventRecord(svd_end, s));
    const int keep_tiles = (d_ub + 31) / 32;
    k_absorb_u_batch<T><<<dim3(keep_tiles, (2 * d_ub + 7) / 8, nref), dim3(32, 8), 0, s>>>(insts, refs);
    TQ_CHECK(cudaGetLastError());
    k_absorb_c_batch<T><<<dim3((2 * d_ub + 31) / 32, keep_tiles, nref), 256, 0, s>>>(insts, refs);
    TQ_CHECK(cudaGetLastError());
    return launches;
}

// One CTA per instance: right-environment chain to bond 1, then the qubit-0 entropy.
template <typename T>
__device__ void entropy_body(const MpsView<T>& mps, const cplx_t<T>* r1, double* out, const int* step);

template <typename T>
__global__ void __launch_bounds__(256) k_entropy_batch(const InstTask<T>* insts) {
    const InstTask<T>& it = insts[blockIdx.x];
    if (it.mps.n >= 2) {
        chain_body<T>(it.mps, 1, it.ent_steps, it.n_ent, it.envs, it.X, nullptr, it.wk.stats, 0, 1);
        __syncthreads();
        entropy_body<T>(it.mps, it.envs + it.r1_off, it.entropy, it.sch.step);
    } else {
        entropy_body<T>(it.mps, nullptr, it.entropy, it.sch.step);
    }
}

template <typename T>
void launch_entropy_batch(const InstTask<T>* insts, int ninst, cudaStream_t s) {
    k_entropy_batch<T><<<ninst, 256, 0, s>>>(insts);
    TQ_CHECK(cudaGetLastError());
}

// explicit instantiations
#define TQ_INST(T)                                                                                          \
    template void launch_init_plus<T>(const MpsView<T>&, cudaStream_t);                                     \
    template void launch_single_site<T>(const MpsView<T>&, const ScheduleView&, int, cudaStream_t);         \
    template void launch_theta<T>(const MpsView<T>&, const ScheduleView&, GateOp, const double*, SvdWork<T>, \
                                  int, int, cudaStream_t);                                                  \
    template int launch_svd<T>(const MpsView<T>&, int, int, double, int, SvdWork<T>, int, int, int,         \
                               cudaStream_t, int, int, int);                                                \
    template void launch_absorb<T>(const MpsView<T>&, int, SvdWork<T>, int, int, int, cudaStream_t);        \
    template void launch_chain<T>(const MpsView<T>&, int, const ChainStep*, int, cplx_t<T>*, cplx_t<T>*,   \
                                  GridBar*, RunStats*, int, cudaStream_t);                                  \
    template void launch_entropy<T>(const MpsView<T>&, const cplx_t<T>*, double*, const int*, cudaStream_t); \
    template void launch_pair_dots<T>(const MpsView<T>&, const cplx_t<T>*, const PairDot*, int, double*,    \
                                      cudaStream_t);                                                        \
    template void launch_amplitude<T>(const MpsView<T>&, const int8_t*, cplx_t<T>*, double*, cudaStream_t);   \
    template void launch_single_site_batch<T>(const InstTask<T>*, int, int, int, cudaStream_t);                \
    template int launch_update_batch<T>(const InstTask<T>*, const UpdRef*, int, int, int, int, cudaStream_t,   \
                                        cudaEvent_t, cudaEvent_t, bool, bool, cudaEvent_t, cudaEvent_t);     \
    template void launch_entropy_batch<T>(const InstTask<T>*, int, cudaStream_t);                               \
    template void launch_sample<T>(const MpsView<T>&, const cplx_t<T>*, int, unsigned long long, int8_t*,       \
                                   cudaStream_t);                                                              \
    template bool launch_anneal_resident<T>(const InstTask<T>*, const GateOp*, const int*, const int*, int, int, \
                                            int, int*, int, cudaStream_t);
TQ_INST(double)
TQ_INST(float)

}  // namespace tq
