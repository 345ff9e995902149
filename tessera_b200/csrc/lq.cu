// lq.cu -- K2q: column-pivoted Householder LQ of theta, the preconditioner of the batched
// one-sided Jacobi.
//
// The one-sided Jacobi (K2b) converges in far fewer sweeps on the lower-triangular factor L of
// a row-pivoted LQ decomposition  P^T theta = L Q^H  than on theta itself: this is the
// preconditioning of Drmac and Veselic ("New fast and accurate Jacobi SVD algorithm I",
// SIAM J. Matrix Anal. Appl. 29, 2008): a column-pivoted QR  theta^H P = Q R  followed by the
// Jacobi on X = R^H.  On graded spectra (Schmidt values falling by orders of magnitude, as in a
// TEBD state) a 512 x 512 theta takes ~10 sweeps instead of ~26.
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
// and applies it to every other unpivoted row z:  z <- z - tau (z . conj(u)) u.  The products
// w_i = X[i, k:] . conj(u) of all rows are accumulated in the same pass that applies the
// previous step's reflector, so each step reads and writes the trailing block once.  Row norms
// are downdated by the new column-k entry before the pivot search and recomputed exactly in
// the next pass.  All sums (w, norms, alpha) are FP64; complex64 stores in FP32.
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

// In-place pivoted LQ of W (R x N, column-major, ld): W <- P L (see the file comment).
template <typename T>
__device__ void lq_body(cplx_t<T>* W, const int ld, const int R, const int N, int* status, unsigned char* smraw) {
    using V = cplx_t<T>;
    __shared__ double rv[LQ_NT / 32];
    __shared__ int ri[LQ_NT / 32];
    __shared__ double s_tau;
    __shared__ double2 s_d, s_tw;
    const int tid = threadIdx.x;
    if (R > (int)blockDim.x || N > LQ_MAXN || R < 1 || N < 1) {  // host sizing bug guard
        if (tid == 0) atomicOr(status, ST_BAD_DIMS);
        return;
    }
    double2* ucur = reinterpret_cast<double2*>(smraw);  // reflector of the current step [LQ_MAXN]
    double2* unext = ucur + LQ_MAXN;                    // reflector of the next step
    const int kmax = R < N ? R : N;
    const bool mine = tid < R;
    bool pivoted = !mine;

    // Reflector of step k from row p into u (columns >= k): x[c] = X[p, c] - tw uprev[c], where
    // tw uprev is the previous step's update of row p, not yet written; sets s_tau and s_d (the
    // diagonal entry of L).
    auto form = [&](const int k, const int p, const double2 tw, const double2* uprev, double2* u) {
        double part = 0.0;
        for (int c = k + tid; c < N; c += blockDim.x) {
            double2 x = to_d2(W[p + (long long)c * ld]);
            if (uprev) {
                const double2 q = uprev[c];
                x.x -= tw.x * q.x - tw.y * q.y;
                x.y -= tw.x * q.y + tw.y * q.x;
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
    };

    // exact row norms, the first pivot and its reflector
    double nrm = 0.0;
    if (mine)
        for (int c = 0; c < N; ++c) {
            const double2 x = to_d2(W[tid + (long long)c * ld]);
            nrm += x.x * x.x + x.y * x.y;
        }
    int p = block_argmax(mine ? nrm : -1.0, rv, ri);
    form(0, p, make_double2(0.0, 0.0), nullptr, ucur);
    double tau = s_tau;
    double2 d = s_d;
    // w_i = X[i, 0:] . conj(u_0)
    double2 w = make_double2(0.0, 0.0);
    if (mine && tid != p)
        for (int c = 0; c < N; ++c) {
            const double2 x = to_d2(W[tid + (long long)c * ld]);
            const double2 q = ucur[c];
            w.x += x.x * q.x + x.y * q.y;
            w.y += x.y * q.x - x.x * q.y;
        }

    for (int k = 0; k < kmax; ++k) {
        // column k: the pivot row takes its diagonal entry of L, every other unpivoted row the
        // update of step k; the norms of columns > k follow by downdating
        if (tid == p) {
            W[p + (long long)k * ld] = from_d2<V>(d);
            pivoted = true;
        } else if (!pivoted) {
            const double2 x = to_d2(W[tid + (long long)k * ld]);
            const double2 q = ucur[k];
            const double twx = tau * w.x, twy = tau * w.y;
            const V a = from_d2<V>(make_double2(x.x - (twx * q.x - twy * q.y), x.y - (twx * q.y + twy * q.x)));
            W[tid + (long long)k * ld] = a;
            const double2 ad = to_d2(a);
            nrm = fmax(0.0, nrm - (ad.x * ad.x + ad.y * ad.y));
        }
        if (k + 1 == kmax) {
            // last step: a wide theta's last pivot row is zero right of the diagonal
            if (tid == p)
                for (int c = k + 1; c < N; ++c) W[p + (long long)c * ld] = czero<V>();
            break;
        }
        __syncthreads();
        const int pn = block_argmax(pivoted ? -1.0 : nrm, rv, ri);
        if (tid == pn) s_tw = make_double2(tau * w.x, tau * w.y);
        __syncthreads();
        // the next pivot row, brought up to date by step k on the fly, gives the next reflector
        form(k + 1, pn, s_tw, ucur, unext);
        // one pass over the columns > k: apply step k's reflector to every unpivoted row but the
        // next pivot (its update is folded into its reflector), accumulating step k+1's
        // products and the exact remaining norms; the row pivoted at step k is zeroed there
        if (tid == p) {
            for (int c = k + 1; c < N; ++c) W[p + (long long)c * ld] = czero<V>();
        } else if (!pivoted && tid != pn) {
            const double twx = tau * w.x, twy = tau * w.y;
            double2 acc = make_double2(0.0, 0.0);
            double nz = 0.0;
            V* row = W + tid;
            auto step = [&](const V xv, const int c) {
                const double2 x = to_d2(xv);
                const double2 q = ucur[c];
                const V z = from_d2<V>(make_double2(x.x - (twx * q.x - twy * q.y), x.y - (twx * q.y + twy * q.x)));
                row[(long long)c * ld] = z;
                const double2 zd = to_d2(z);
                const double2 un = unext[c];
                acc.x += zd.x * un.x + zd.y * un.y;
                acc.y += zd.y * un.x - zd.x * un.y;
                nz += zd.x * zd.x + zd.y * zd.y;
            };
            // columns in chunks of LQ_U, the loads of the next chunk issued before the current one
            // is applied and stored, so two chunks of memory latency overlap per thread
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
                    for (int j = 0; j < LQ_U; ++j) step(cur[j], c + j);
#pragma unroll
                    for (int j = 0; j < LQ_U; ++j) cur[j] = nxt[j];
                }
            }
            for (; c < N; ++c) step(row[(long long)c * ld], c);
            w = acc;
            nrm = nz;
        }
        tau = s_tau;
        d = s_d;
        __syncthreads();  // the pass has read ucur and unext; s_tau, s_d, s_tw free
        double2* t = ucur;
        ucur = unext;
        unext = t;
        p = pn;
    }
    __syncthreads();
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

size_t lq_smem_bytes() { return sizeof(double2) * 2 * LQ_MAXN; }

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

}  // namespace tq
