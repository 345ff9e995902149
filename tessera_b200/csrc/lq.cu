// lq.cu -- K2q: row-pivoted Householder LQ of theta, the preconditioner of the one-sided Jacobi:
// k_lq_batch (one CTA per theta) before the batched kernel, k_lq_coop (one theta over many CTAs)
// before the single-instance cooperative kernel.
//
// The one-sided Jacobi (K2b) converges in far fewer sweeps on the lower-triangular factor L of
// a row-pivoted LQ decomposition  P^T theta = L Q^H  than on theta itself: this is the
// preconditioning of Drmac and Veselic ("New fast and accurate Jacobi SVD algorithm I",
// SIAM J. Matrix Anal. Appl. 29, 2008): a column-pivoted QR  theta^H P = Q R  followed by the
// Jacobi on X = R^H.  In a model of the batched kernel's ordering a 512 x 512 theta with graded
// spectrum (Schmidt values falling by orders of magnitude, as in a TEBD state) takes ~10 sweeps
// instead of ~26; on the GPU the chi=256 bench's random input went 13.5 -> 10.9 sweeps and its
// graded input 14.5 -> 10.2.
//
// Nothing downstream changes.  The Jacobi is blind to the order of the rows, so the factor is
// left in W in theta's own row order, as P L (row piv[k] of theta holds row k of L).  The Jacobi
// then turns P L into P L V = U Sigma, so U = W / sigma are theta's left singular vectors in
// theta's row order (theta = P L Q^H = U Sigma (Q V)^H), and C = U^H theta = Sigma (Q V)^H is
// formed from theta by the unchanged absorption.  Q is never formed.  L has min(R, N) columns:
// for a wide theta the columns beyond R are exactly zero and the Jacobi leaves them out.
//
// One CTA per theta, one thread per row (R <= 512).  Step k picks the unpivoted row p with the
// largest remaining norm ||X[p, k:]||, builds the Householder reflector of that row,
//     x = X[p, k:],  alpha = ||x||,  e = x_0 / |x_0|,
//     u = x with u_0 = e (|x_0| + alpha),  tau = 1 / (alpha (alpha + |x_0|)),
//     x (I - tau u^H u) = -e alpha e_0      (row vectors; I - tau u^H u is Hermitian unitary),
// and applies it to every other unpivoted row z:  z <- z - tau (z . conj(u)) u.  The updates
// are delayed over panels of LQ_B steps (the blocking of LAPACK's pivoted QR): a step reads the
// trailing block once for the products w_i = X[i, k:] . conj(u), corrects them for the panel's
// pending updates, and writes only column k; the panel's updates reach memory in one pass at its
// end.  Per step that moves (1 + 2/LQ_B) instead of 2 trailing blocks.  Row norms are downdated
// by the new column-k entry before each pivot search and recomputed exactly at panel ends.  All
// sums (w, norms, alpha) are FP64; complex64 stores in FP32.
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

constexpr int LQ_NT = 512;     // threads per CTA: one per row of theta
constexpr int LQ_MAXN = 1024;  // columns of theta
constexpr int LQ_U = 4;        // columns per chunk of the per-row walk
constexpr int LQ_B = 8;        // reflectors per panel (delayed updates)

__device__ __forceinline__ double2 to_d2(const double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(const float2 v) { return make_double2(v.x, v.y); }
template <typename V> __device__ __forceinline__ V from_d2(const double2 v);
template <> __device__ __forceinline__ double2 from_d2<double2>(const double2 v) { return v; }
template <> __device__ __forceinline__ float2 from_d2<float2>(const double2 v) {
    return make_float2((float)v.x, (float)v.y);
}

// block argmax of key over the threads (ties: lowest index); key < 0 never wins unless all are
__device__ __forceinline__ int block_argmax(double key, double* rv, int* ri) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int idx = tid;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double k2 = __shfl_xor_sync(0xffffffffu, key, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, idx, o);
        if (k2 > key || (k2 == key && i2 < idx)) { key = k2; idx = i2; }
    }
    if (lane == 0) { rv[warp] = key; ri[warp] = idx; }
    __syncthreads();
    double bk = rv[0];
    int bi = ri[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
        if (rv[w] > bk || (rv[w] == bk && ri[w] < bi)) { bk = rv[w]; bi = ri[w]; }
    __syncthreads();  // rv, ri free again
    return bi;
}

__device__ __forceinline__ double block_sum(double v, double* rv) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    v = warp_sum(v);
    if (lane == 0) rv[warp] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += rv[w];
    __syncthreads();
    return s;
}

// sum of up to LQ_RED doubles v[0..n) over the CTA into out[0..n) (every thread may read out after)
constexpr int LQ_RED = 2 * LQ_B;
__device__ __forceinline__ void block_sum_n(double* v, int n, double (*red)[LQ_RED], double* out) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    for (int q = 0; q < n; ++q) {
        const double s = warp_sum(v[q]);
        if (lane == 0) red[warp][q] = s;
    }
    __syncthreads();
    if (tid < n) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += red[w][tid];
        out[tid] = s;
    }
    __syncthreads();
}

__device__ __forceinline__ double2 cm(const double2 a, const double2 b) {  // a * b
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmc(const double2 a, const double2 b) {  // a * conj(b)
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// In-place pivoted LQ of W (R x N, column-major, ld): W <- P L (see the file comment).  Panels
// of LQ_B steps: within a panel the trailing block in memory is not updated; row i's current
// values are X[i, c] - sum_j tw_j[i] u_j[c] over the panel's reflectors so far (tw_j[i] =
// tau_j w_j[i]), so each step reads the trailing block once (its products with the new
// reflector, corrected by g_j = u_j . conj(u)), writes only column k, and the panel's updates
// are written in one pass at its end, where the row norms are also recomputed exactly.
template <typename T>
__device__ void lq_body(cplx_t<T>* W, const int ld, const int R, const int N, int* status, unsigned char* smraw) {
    using V = cplx_t<T>;
    __shared__ double rv[LQ_NT / 32];
    __shared__ int ri[LQ_NT / 32];
    __shared__ double red[LQ_NT / 32][LQ_RED];
    __shared__ double s_red[LQ_RED];
    __shared__ double s_tau;
    __shared__ double2 s_d;
    const int tid = threadIdx.x;
    if (R > (int)blockDim.x || N > LQ_MAXN || R < 1 || N < 1) {  // host sizing bug guard
        if (tid == 0) atomicOr(status, ST_BAD_DIMS);
        return;
    }
    double2* U = reinterpret_cast<double2*>(smraw);  // [LQ_B][LQ_MAXN] the panel's reflectors
    double2* TW = U + LQ_B * LQ_MAXN;                 // [LQ_B][LQ_NT] tau_j w_j of every row
    const int kmax = R < N ? R : N;
    const bool mine = tid < R;
    bool pivoted = !mine;
    V* row = W + tid;
    // exact row norms
    double nrm = 0.0;
    if (mine)
        for (int c = 0; c < N; ++c) {
            const double2 x = to_d2(row[(long long)c * ld]);
            nrm += x.x * x.x + x.y * x.y;
        }
    int k = 0;
    while (k < kmax) {
        int jn = 0;  // reflectors of this panel so far
        for (; jn < LQ_B && k < kmax; ++jn, ++k) {
            const int p = block_argmax(pivoted ? -1.0 : nrm, rv, ri);
            // reflector from row p's current values, columns >= k
            double2* u = U + jn * LQ_MAXN;
            double part = 0.0;
            for (int c = k + tid; c < N; c += blockDim.x) {
                double2 x = to_d2(W[p + (long long)c * ld]);
                for (int j = 0; j < jn; ++j) {
                    const double2 t = cm(TW[j * LQ_NT + p], U[j * LQ_MAXN + c]);
                    x.x -= t.x;
                    x.y -= t.y;
                }
                u[c] = x;
                part += x.x * x.x + x.y * x.y;
            }
            const double alpha2 = block_sum(part, rv);  // ends with a barrier: u complete
            if (tid == 0) {
                const double alpha = sqrt(alpha2);
                const double2 x0 = u[k];
                const double a0 = sqrt(x0.x * x0.x + x0.y * x0.y);
                const double ex = a0 > 0.0 ? x0.x / a0 : 1.0, ey = a0 > 0.0 ? x0.y / a0 : 0.0;
                if (alpha > 0.0) {
                    s_d = make_double2(-ex * alpha, -ey * alpha);
                    s_tau = 1.0 / (alpha * (alpha + a0));
                    u[k] = make_double2(ex * (a0 + alpha), ey * (a0 + alpha));
                } else {  // the rest of theta is zero: the identity
                    s_d = make_double2(0.0, 0.0);
                    s_tau = 0.0;
                }
            }
            __syncthreads();
            // g_j = u_j . conj(u) over columns >= k, for the panel's earlier reflectors
            if (jn > 0) {
                double gv[LQ_RED];
                for (int q = 0; q < 2 * jn; ++q) gv[q] = 0.0;
                for (int c = k + tid; c < N; c += blockDim.x) {
                    const double2 uc = u[c];
                    for (int j = 0; j < jn; ++j) {
                        const double2 t = cmc(U[j * LQ_MAXN + c], uc);
                        gv[2 * j] += t.x;
                        gv[2 * j + 1] += t.y;
                    }
                }
                block_sum_n(gv, 2 * jn, red, s_red);
            }
            const double tau = s_tau;
            const double2 d = s_d;
            // the pivot row takes its diagonal entry and zeros to its right; every other free row
            // reads its trailing columns once: w = X[i, k:] . conj(u), corrected by the panel's
            // pending updates (- sum_j tw_j[i] g_j), then its final column-k value
            if (tid == p) {
                W[p + (long long)k * ld] = from_d2<V>(d);
                for (int c = k + 1; c < N; ++c) W[p + (long long)c * ld] = czero<V>();
                pivoted = true;
            } else if (!pivoted) {
                double2 acc = make_double2(0.0, 0.0);
                const double2 xk = to_d2(row[(long long)k * ld]);
                {
                    const double2 t = cmc(xk, u[k]);
                    acc.x += t.x;
                    acc.y += t.y;
                }
                int c = k + 1;
                const int nfull = (N - c) / LQ_U;
                if (nfull > 0) {
                    V cur[LQ_U];
#pragma unroll
                    for (int j = 0; j < LQ_U; ++j) cur[j] = row[(long long)(c + j) * ld];
                    for (int it = 0; it < nfull; ++it, c += LQ_U) {
                        V nxt[LQ_U];
                        if (it + 1 < nfull) {
#pragma unroll
                            for (int j = 0; j < LQ_U; ++j) nxt[j] = row[(long long)(c + LQ_U + j) * ld];
                        }
#pragma unroll
                        for (int j = 0; j < LQ_U; ++j) {
                            const double2 t = cmc(to_d2(cur[j]), u[c + j]);
                            acc.x += t.x;
                            acc.y += t.y;
                            cur[j] = nxt[j];
                        }
                    }
                }
                for (; c < N; ++c) {
                    const double2 t = cmc(to_d2(row[(long long)c * ld]), u[c]);
                    acc.x += t.x;
                    acc.y += t.y;
                }
                for (int j = 0; j < jn; ++j) {
                    const double2 t = cm(TW[j * LQ_NT + tid], make_double2(s_red[2 * j], s_red[2 * j + 1]));
                    acc.x -= t.x;
                    acc.y -= t.y;
                }
                const double2 tw = make_double2(tau * acc.x, tau * acc.y);
                TW[jn * LQ_NT + tid] = tw;
                double2 col = xk;
                for (int j = 0; j <= jn; ++j) {
                    const double2 t = cm(TW[j * LQ_NT + tid], U[j * LQ_MAXN + k]);
                    col.x -= t.x;
                    col.y -= t.y;
                }
                const V cv = from_d2<V>(col);
                row[(long long)k * ld] = cv;
                const double2 cd = to_d2(cv);
                nrm = fmax(0.0, nrm - (cd.x * cd.x + cd.y * cd.y));
            }
            __syncthreads();  // TW[jn] complete; s_red, s_tau, s_d free
        }
        // panel end: the panel's updates into columns >= k of every free row, exact norms
        if (!pivoted && k < N) {
            double2 tw[LQ_B];
#pragma unroll
            for (int j = 0; j < LQ_B; ++j) tw[j] = j < jn ? TW[j * LQ_NT + tid] : make_double2(0.0, 0.0);
            double nz = 0.0;
            for (int c = k; c < N; ++c) {
                double2 x = to_d2(row[(long long)c * ld]);
#pragma unroll
                for (int j = 0; j < LQ_B; ++j) {
                    if (j < jn) {
                        const double2 t = cm(tw[j], U[j * LQ_MAXN + c]);
                        x.x -= t.x;
                        x.y -= t.y;
                    }
                }
                const V z = from_d2<V>(x);
                row[(long long)c * ld] = z;
                const double2 zd = to_d2(z);
                nz += zd.x * zd.x + zd.y * zd.y;
            }
            nrm = nz;
        }
        __syncthreads();  // the next panel rewrites U and TW
    }
}

template <typename T>
__global__ void __launch_bounds__(LQ_NT, 1) k_lq_batch(const InstTask<T>* insts, const UpdRef* refs, int nref) {
    extern __shared__ __align__(16) unsigned char smraw[];
    for (int t = blockIdx.x; t < nref; t += gridDim.x) {
        const UpdRef rf = refs[t];
        const InstTask<T>& it = insts[rf.inst];
        const int R = 2 * it.mps.dims[rf.op.bond], N = 2 * it.mps.dims[rf.op.bond + 2];
        lq_body<T>(it.wk.W, it.wk.ld, R, N, &it.wk.stats->status, smraw);
    }
}

size_t lq_smem_bytes() { return sizeof(double2) * LQ_B * (LQ_MAXN + LQ_NT); }

template <typename T>
void launch_lq_batch(const InstTask<T>* insts, const UpdRef* refs, int nref, cudaStream_t s) {
    if (nref <= 0) return;
    const size_t smem = lq_smem_bytes();
    auto fn = k_lq_batch<T>;
    TQ_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 0;
    TQ_CHECK(cudaGetDevice(&dev));
    TQ_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int per_sm = 0;
    TQ_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, LQ_NT, smem));
    if (per_sm < 1) throw std::runtime_error("k_lq_batch does not fit on an SM");
    int grid = per_sm * sms;
    if (grid > nref) grid = nref;
    fn<<<grid, LQ_NT, smem, s>>>(insts, refs, nref);
    TQ_CHECK(cudaGetLastError());
}

template void launch_lq_batch<double>(const InstTask<double>*, const UpdRef*, int, cudaStream_t);
template void launch_lq_batch<float>(const InstTask<float>*, const UpdRef*, int, cudaStream_t);

// ------------------------------------------------------------------------------------
// The same LQ for the single-instance engine, cooperative over ceil(R / LQC_RB) CTAs: CTA g keeps
// rows [g LQC_RB, (g + 1) LQC_RB) of W in shared memory for the whole factorization.  Per step
// every CTA publishes its best unpivoted row (largest remaining norm) and that row's columns >= k
// to a global candidate slot, one bounded grid barrier follows, and every CTA then picks the same
// winner (largest norm, lowest row on ties), forms the reflector from the winner's row, and
// updates its own rows in shared memory (exact norms recomputed).  The candidate slots alternate
// between two buffers by step parity: a CTA rewrites the buffer of step k only after the barrier
// of step k + 1, which every CTA passes after it has read step k's.  W is written back at the
// end; if a barrier gives up, W keeps theta (the Jacobi then runs unpreconditioned) and the
// status reports the timeout.
// ------------------------------------------------------------------------------------
constexpr int LQC_RB = 8;    // rows per CTA (2 LQC_RB <= LQ_RED values per reduction)
constexpr int LQC_NT = 256;  // threads per CTA

template <typename T>
__global__ void __launch_bounds__(LQC_NT, 1) k_lq_coop(MpsView<T> mps, int bond, SvdWork<T> wk, cplx_t<T>* cand,
                                                       double* keys, int* idxs) {
    using V = cplx_t<T>;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double rv[LQC_NT / 32];
    __shared__ int ri[LQC_NT / 32];
    __shared__ double red[LQC_NT / 32][LQ_RED];
    __shared__ double s_red[LQ_RED];
    __shared__ double nrm[LQC_RB];
    __shared__ int piv[LQC_RB];
    __shared__ double s_tau, s_a2;
    __shared__ double2 s_d;
    __shared__ int s_p, s_gc;
    const int tid = threadIdx.x, cta = blockIdx.x, G = gridDim.x;
    const int R = 2 * mps.dims[bond], N = 2 * mps.dims[bond + 2];
    const int ld = wk.ld;
    int* status = &wk.stats->status;
    if (R > G * LQC_RB || N > LQ_MAXN || G > LQC_NT) {  // host sizing bug guard (uniform over the grid)
        if (cta == 0 && tid == 0) atomicOr(status, ST_BAD_DIMS);
        return;
    }
    V* X = reinterpret_cast<V*>(smraw);               // [LQC_RB][N] this CTA's rows
    double2* u = reinterpret_cast<double2*>(X + LQC_RB * N);  // [N] the step's reflector
    const int r0 = cta * LQC_RB;
    const int nr = R - r0 < LQC_RB ? (R - r0 > 0 ? R - r0 : 0) : LQC_RB;
    for (int e = tid; e < LQC_RB * N; e += LQC_NT) {
        const int r = e % LQC_RB, c = e / LQC_RB;  // 8 consecutive rows of a column: 128 contiguous bytes
        X[r * N + c] = r < nr ? wk.W[(r0 + r) + (long long)c * ld] : czero<V>();
    }
    if (tid < LQC_RB) piv[tid] = tid < nr ? 0 : 1;
    __syncthreads();
    // exact row norms
    {
        double v[LQ_RED];
        for (int r = 0; r < LQC_RB; ++r) v[r] = 0.0;
        for (int c = tid; c < N; c += LQC_NT)
            for (int r = 0; r < LQC_RB; ++r) {
                const double2 x = to_d2(X[r * N + c]);
                v[r] += x.x * x.x + x.y * x.y;
            }
        block_sum_n(v, LQC_RB, red, s_red);
        if (tid < LQC_RB) nrm[tid] = s_red[tid];
        __syncthreads();
    }
    const int kmax = R < N ? R : N;
    for (int k = 0; k < kmax; ++k) {
        const int par = k & 1;
        // this CTA's candidate: its unpivoted row of largest remaining norm
        if (tid == 0) {
            double best = -1.0;
            int br = -1;
            for (int r = 0; r < nr; ++r)
                if (!piv[r] && nrm[r] > best) { best = nrm[r]; br = r; }
            keys[par * G + cta] = best;
            idxs[par * G + cta] = br < 0 ? -1 : r0 + br;
            s_p = br;
        }
        __syncthreads();
        if (s_p >= 0)
            for (int c = k + tid; c < N; c += LQC_NT) cand[((long long)par * G + cta) * ld + c] = X[s_p * N + c];
        if (!grid_sync(wk.bar, status, (unsigned)G)) return;  // W untouched: still theta
        // the winner, the same on every CTA: thread g reads CTA g's candidate, then a block argmax
        // (largest norm; ties to the lowest CTA, which holds the lowest row)
        double kv = -2.0;
        int rr = -1;
        if (tid < G) {
            kv = *(volatile double*)&keys[par * G + tid];
            rr = *(volatile int*)&idxs[par * G + tid];
            if (rr < 0) kv = -2.0;
        }
        const int gw = block_argmax(kv, rv, ri);
        if (tid == gw) {
            s_gc = gw;
            s_p = rr;
            s_a2 = kv;  // the winner's exact remaining norm^2 (summed from the stored values)
        }
        __syncthreads();
        const int gc = s_gc, p = s_p;
        // reflector from the winner's row (published by its owner), columns >= k
        for (int c = k + tid; c < N; c += LQC_NT) {
            const V* src = cand + ((long long)par * G + gc) * ld + c;
            u[c] = to_d2(*(const volatile V*)src);
        }
        __syncthreads();
        if (tid == 0) {
            const double alpha = sqrt(fmax(s_a2, 0.0));
            const double2 x0 = u[k];
            const double a0 = sqrt(x0.x * x0.x + x0.y * x0.y);
            const double ex = a0 > 0.0 ? x0.x / a0 : 1.0, ey = a0 > 0.0 ? x0.y / a0 : 0.0;
            if (alpha > 0.0) {
                s_d = make_double2(-ex * alpha, -ey * alpha);
                s_tau = 1.0 / (alpha * (alpha + a0));
                u[k] = make_double2(ex * (a0 + alpha), ey * (a0 + alpha));
            } else {
                s_d = make_double2(0.0, 0.0);
                s_tau = 0.0;
            }
            if (p >= r0 && p < r0 + nr) piv[p - r0] = 1;
        }
        __syncthreads();
        const double tau = s_tau;
        const double2 d = s_d;
        const int mine_p = (p >= r0 && p < r0 + nr) ? p - r0 : -1;
        // products w_r = X[r, k:] . conj(u) of this CTA's unpivoted rows
        double v[LQ_RED];
        for (int q = 0; q < 2 * LQC_RB; ++q) v[q] = 0.0;
        for (int c = k + tid; c < N; c += LQC_NT) {
            const double2 uc = u[c];
            for (int r = 0; r < LQC_RB; ++r) {
                const double2 t = cmc(to_d2(X[r * N + c]), uc);
                v[2 * r] += t.x;
                v[2 * r + 1] += t.y;
            }
        }
        block_sum_n(v, 2 * LQC_RB, red, s_red);
        double2 tw[LQC_RB];
        bool upd[LQC_RB];
        for (int r = 0; r < LQC_RB; ++r) {
            upd[r] = r < nr && !piv[r];
            tw[r] = make_double2(tau * s_red[2 * r], tau * s_red[2 * r + 1]);
        }
        __syncthreads();  // s_red read by every thread before the norm sums reuse it
        // updates and exact remaining norms; the pivot row takes d and zeros to its right
        for (int q = 0; q < LQC_RB; ++q) v[q] = 0.0;
        for (int c = k + tid; c < N; c += LQC_NT) {
            const double2 uc = u[c];
            for (int r = 0; r < LQC_RB; ++r) {
                if (r == mine_p) {
                    X[r * N + c] = c == k ? from_d2<V>(d) : czero<V>();
                } else if (upd[r]) {
                    const double2 x = to_d2(X[r * N + c]);
                    const double2 t = cm(tw[r], uc);
                    const V z = from_d2<V>(make_double2(x.x - t.x, x.y - t.y));
                    X[r * N + c] = z;
                    if (c > k) {
                        const double2 zd = to_d2(z);
                        v[r] += zd.x * zd.x + zd.y * zd.y;
                    }
                }
            }
        }
        block_sum_n(v, LQC_RB, red, s_red);
        if (tid < LQC_RB && tid < nr && !piv[tid]) nrm[tid] = s_red[tid];
        __syncthreads();
    }
    // this CTA's rows of P L back to W
    for (int e = tid; e < LQC_RB * N; e += LQC_NT) {
        const int r = e % LQC_RB, c = e / LQC_RB;
        if (r < nr) wk.W[(r0 + r) + (long long)c * ld] = X[r * N + c];
    }
}

size_t lq_coop_smem_bytes(int N, int esz) { return (size_t)LQC_RB * N * esz + sizeof(double2) * N; }

// Candidate buffer of the cooperative LQ: two parities of up to `ctas` rows of `ld` elements, plus
// keys and row indices.
size_t lq_coop_scratch_bytes(int ld, int esz, int ctas) {
    return (size_t)2 * ctas * ld * esz + (size_t)2 * ctas * (sizeof(double) + sizeof(int)) + 64;
}

template <typename T>
void launch_lq_coop(const MpsView<T>& mps, int bond, SvdWork<T> wk, void* scratch, int rows_ub, int cols_ub,
                    cudaStream_t s) {
    using V = cplx_t<T>;
    const int G = (rows_ub + LQC_RB - 1) / LQC_RB;
    V* cand = reinterpret_cast<V*>(scratch);
    double* keys = reinterpret_cast<double*>(cand + (size_t)2 * G * wk.ld);
    int* idxs = reinterpret_cast<int*>(keys + 2 * G);
    const size_t smem = lq_coop_smem_bytes(cols_ub, (int)sizeof(V));
    auto fn = k_lq_coop<T>;
    TQ_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MpsView<T> m = mps;
    int b = bond;
    void* args[] = {&m, &b, &wk, &cand, &keys, &idxs};
    TQ_CHECK(cudaLaunchCooperativeKernel((const void*)fn, dim3(G), dim3(LQC_NT), args, smem, s));
}

template void launch_lq_coop<double>(const MpsView<double>&, int, SvdWork<double>, void*, int, int, cudaStream_t);
template void launch_lq_coop<float>(const MpsView<float>&, int, SvdWork<float>, void*, int, int, cudaStream_t);


}  // namespace tq
