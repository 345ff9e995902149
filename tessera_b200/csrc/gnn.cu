// gnn.cu -- the learned-schedule layer and the exact ground state, on the GPU.
//
// 1. tessera_qa_exact_ground: brute force over the 2^n spin patterns (n <= 32), bit b set
//    <-> spin +1, first minimum kept: the scorer of rust/src/ising.rs:46-61 as a CUDA
//    reduction.  Used to score anneals (energy gap to the ground state) when labelling
//    schedules and counting solves.
// 2. A message-passing GNN that maps an Ising graph to a K-knot monotone anneal schedule
//    s(u_j), u_j = j/(K-1), and a per-spin warm-start bias p_i = P(s_i = +1).  The
//    reference's python/gnn_guide.py:81-103 (node embedding, edge messages from (x_src, J),
//    sum aggregation, node update, sigmoid readout) is the starting point:
//      x0_i  = relu(We f_i + be),                 f_i = [h_i, sum_j |J_ij|/4, sum_j J_ij/4, 1]
//      layer l = 0..L-1:
//        m_e  = relu(W1 [x_src(e); J_e] + b1)       over both directions of every edge
//        a_i  = sum_{e: dst(e) = i} m_e
//        x_i <- x_i + relu(W2 [x_i; a_i] + b2)
//      p_i   = sigmoid(wn . x_i + bn)
//      g     = mean_i x_i ; z = relu(Wg1 g + bg1) ; o = Wg2 z + bg2 (K-1 values)
//      d_k   = softplus(o_k), c_j = sum_{k<j} d_k, knot_j = c_j / c_{K-1}   (0 = knot_0 <= ... = 1)
//    Loss = lambda_k mean_j (knot_j - t_j)^2 + lambda_n mean BCE(p_i, t_i).
//    Weights are read in BF16 with FP32 accumulation (FP32 master copy for Adam), or in FP32
//    when bf16 is off (gradient checks).  Every forward, backward and optimizer kernel is
//    hand-written here: one thread per output element, no library call.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tessera_qa.h"

namespace tq {

cudaError_t device_alloc(void** p, size_t bytes);  // engine.cu: cudaMalloc with failure injection

void set_last_error(const std::string& msg);

#define GN_CK(x)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (x);                                                                             \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_)); \
    } while (0)

// =====================================================================================
// exact ground state
// =====================================================================================
__global__ void k_ground(const double* h, const int* ei, const int* ej, const double* w, int n, int m,
                         unsigned long long total, double* blk_e, unsigned long long* blk_x) {
    extern __shared__ double sh[];
    double* sh_h = sh;
    double* sh_w = sh + n;
    int* sh_i = reinterpret_cast<int*>(sh_w + m);
    int* sh_j = sh_i + m;
    for (int t = threadIdx.x; t < n; t += blockDim.x) sh_h[t] = h[t];
    for (int t = threadIdx.x; t < m; t += blockDim.x) {
        sh_w[t] = w[t];
        sh_i[t] = ei[t];
        sh_j[t] = ej[t];
    }
    __syncthreads();
    double best = INFINITY;
    unsigned long long bx = ~0ull;
    for (unsigned long long x = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; x < total;
         x += (unsigned long long)gridDim.x * blockDim.x) {
        double e = 0.0;
        for (int q = 0; q < m; ++q) {
            const int si = ((x >> sh_i[q]) & 1ull) ? 1 : -1, sj = ((x >> sh_j[q]) & 1ull) ? 1 : -1;
            e -= sh_w[q] * (double)(si * sj);
        }
        for (int i = 0; i < n; ++i) e -= sh_h[i] * (((x >> i) & 1ull) ? 1.0 : -1.0);
        if (e < best || (e == best && x < bx)) {
            best = e;
            bx = x;
        }
    }
    __shared__ double re[256];
    __shared__ unsigned long long rx[256];
    re[threadIdx.x] = best;
    rx[threadIdx.x] = bx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            const double e2 = re[threadIdx.x + o];
            const unsigned long long x2 = rx[threadIdx.x + o];
            if (e2 < re[threadIdx.x] || (e2 == re[threadIdx.x] && x2 < rx[threadIdx.x])) {
                re[threadIdx.x] = e2;
                rx[threadIdx.x] = x2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        blk_e[blockIdx.x] = re[0];
        blk_x[blockIdx.x] = rx[0];
    }
}

// =====================================================================================
// GNN
// =====================================================================================
struct GnnLayout {
    int H, L, K, F;
    size_t We, be, W1[8], b1[8], W2[8], b2[8], wn, bn, Wg1, bg1, Wg2, bg2, total;
    void build() {
        size_t o = 0;
        auto take = [&](size_t n) {
            size_t r = o;
            o += n;
            return r;
        };
        We = take((size_t)H * F);
        be = take(H);
        for (int l = 0; l < L; ++l) {
            W1[l] = take((size_t)H * (H + 1));
            b1[l] = take(H);
            W2[l] = take((size_t)H * 2 * H);
            b2[l] = take(H);
        }
        wn = take(H);
        bn = take(1);
        Wg1 = take((size_t)H * H);
        bg1 = take(H);
        Wg2 = take((size_t)(K - 1) * H);
        bg2 = take(K - 1);
        total = o;
    }
};

// weights as read by the forward/backward: the BF16 copy, or the FP32 master
struct Wt {
    const float* f;
    const __nv_bfloat16* b;
    __device__ __forceinline__ float operator[](size_t i) const { return b ? __bfloat162float(b[i]) : f[i]; }
};

__device__ __forceinline__ float relu(float x) { return x > 0.f ? x : 0.f; }
__device__ __forceinline__ float softplus_f(float x) { return x > 20.f ? x : log1pf(expf(x)); }

__global__ void k_embed(Wt W, size_t oW, size_t ob, const float* feat, int Nn, int H, int F, float* pre, float* x) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Nn * H) return;
    const int i = t / H, o = t - i * H;
    float acc = W[ob + o];
    for (int f = 0; f < F; ++f) acc += W[oW + (size_t)o * F + f] * feat[i * F + f];
    pre[t] = acc;
    x[t] = relu(acc);
}

__global__ void k_msg(Wt W, size_t oW1, size_t ob1, const float* x, const int* src, const float* ew, int E, int H,
                      float* mpre, float* mout) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= E * H) return;
    const int e = t / H, o = t - e * H;
    const float* xs = x + (size_t)src[e] * H;
    const size_t row = oW1 + (size_t)o * (H + 1);
    float acc = W[ob1 + o] + W[row + H] * ew[e];
    for (int k = 0; k < H; ++k) acc += W[row + k] * xs[k];
    mpre[t] = acc;
    mout[t] = relu(acc);
}

__global__ void k_scatter_add(const float* m, const int* dst, int E, int H, float* a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= E * H) return;
    const int e = t / H, o = t - e * H;
    atomicAdd(&a[(size_t)dst[e] * H + o], m[t]);
}

__global__ void k_update(Wt W, size_t oW2, size_t ob2, const float* x, const float* a, int Nn, int H, float* upre,
                         float* xn) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Nn * H) return;
    const int i = t / H, o = t - i * H;
    const size_t row = oW2 + (size_t)o * 2 * H;
    float acc = W[ob2 + o];
    for (int k = 0; k < H; ++k) acc += W[row + k] * x[(size_t)i * H + k] + W[row + H + k] * a[(size_t)i * H + k];
    upre[t] = acc;
    xn[t] = x[t] + relu(acc);
}

__global__ void k_node_head(Wt W, size_t own, size_t obn, const float* x, int Nn, int H, float* p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Nn) return;
    float acc = W[obn];
    for (int k = 0; k < H; ++k) acc += W[own + k] * x[(size_t)i * H + k];
    p[i] = 1.f / (1.f + expf(-acc));
}

// one CTA per graph: mean pool, MLP, monotone knots
__global__ void k_graph_head(Wt W, GnnLayout Ly, const float* x, const int* goff, float* gmean, float* zpre,
                             float* o, float* knots) {
    const int g = blockIdx.x, H = Ly.H, K = Ly.K;
    const int t = threadIdx.x;
    extern __shared__ float sm[];
    float* gm = sm;          // H
    float* z = sm + H;       // H
    float* ob = sm + 2 * H;  // K-1
    const int n0 = goff[g], n1 = goff[g + 1];
    if (t < H) {
        float s = 0.f;
        for (int i = n0; i < n1; ++i) s += x[(size_t)i * H + t];
        s /= (float)(n1 - n0 > 0 ? n1 - n0 : 1);
        gm[t] = s;
        gmean[(size_t)g * H + t] = s;
    }
    __syncthreads();
    if (t < H) {
        float acc = W[Ly.bg1 + t];
        for (int k = 0; k < H; ++k) acc += W[Ly.Wg1 + (size_t)t * H + k] * gm[k];
        zpre[(size_t)g * H + t] = acc;
        z[t] = relu(acc);
    }
    __syncthreads();
    if (t < K - 1) {
        float acc = W[Ly.bg2 + t];
        for (int k = 0; k < H; ++k) acc += W[Ly.Wg2 + (size_t)t * H + k] * z[k];
        ob[t] = acc;
        o[(size_t)g * (K - 1) + t] = acc;
    }
    __syncthreads();
    if (t == 0) {
        float c = 0.f, tot = 0.f;
        for (int k = 0; k < K - 1; ++k) tot += softplus_f(ob[k]);
        knots[(size_t)g * K] = 0.f;
        for (int j = 1; j < K; ++j) {
            c += softplus_f(ob[j - 1]);
            knots[(size_t)g * K + j] = c / tot;
        }
    }
}

// ---------------- backward ----------------
// graph head, one CTA per graph.  dL/dknot_j = lk * 2 (knot_j - t_j) / (G K).
__global__ void k_graph_head_bwd(Wt W, GnnLayout Ly, int G, const float* gmean, const float* zpre, const float* o,
                                 const float* knots, const float* tk, float lk, const int* goff, float* grad,
                                 float* dx) {
    const int g = blockIdx.x, H = Ly.H, K = Ly.K;
    const int t = threadIdx.x;
    extern __shared__ float sm[];
    float* dknot = sm;            // K
    float* dd = sm + K;           // K-1
    float* dz = sm + 2 * K;       // H
    float* dgm = sm + 2 * K + H;  // H
    if (t < K) dknot[t] = lk * 2.f * (knots[(size_t)g * K + t] - tk[(size_t)g * K + t]) / (float)(G * K);
    __syncthreads();
    if (t < K - 1) {
        // knot_j = c_j / S, c_j = sum_{k < j} d_k, S = c_{K-1}: d(knot_j)/d(d_t) = ([t < j] S - c_j) / S^2
        float S = 0.f;
        for (int k = 0; k < K - 1; ++k) S += softplus_f(o[(size_t)g * (K - 1) + k]);
        float acc = 0.f, c = 0.f;
        for (int j = 1; j < K; ++j) {
            c += softplus_f(o[(size_t)g * (K - 1) + j - 1]);
            acc += dknot[j] * (((t < j) ? S : 0.f) - c) / (S * S);
        }
        const float ot = o[(size_t)g * (K - 1) + t];
        dd[t] = acc / (1.f + expf(-ot));  // softplus' = sigmoid
    }
    __syncthreads();
    for (int e = t; e < (K - 1) * H; e += blockDim.x) {
        const int r = e / H, k = e - r * H;
        atomicAdd(&grad[Ly.Wg2 + e], dd[r] * relu(zpre[(size_t)g * H + k]));
    }
    if (t < K - 1) atomicAdd(&grad[Ly.bg2 + t], dd[t]);
    if (t < H) {
        float acc = 0.f;
        for (int r = 0; r < K - 1; ++r) acc += W[Ly.Wg2 + (size_t)r * H + t] * dd[r];
        dz[t] = zpre[(size_t)g * H + t] > 0.f ? acc : 0.f;
    }
    __syncthreads();
    for (int e = t; e < H * H; e += blockDim.x) {
        const int r = e / H, k = e - r * H;
        atomicAdd(&grad[Ly.Wg1 + e], dz[r] * gmean[(size_t)g * H + k]);
    }
    if (t < H) atomicAdd(&grad[Ly.bg1 + t], dz[t]);
    if (t < H) {
        float acc = 0.f;
        for (int r = 0; r < H; ++r) acc += W[Ly.Wg1 + (size_t)r * H + t] * dz[r];
        dgm[t] = acc;
    }
    __syncthreads();
    const int n0 = goff[g], n1 = goff[g + 1];
    const float inv = 1.f / (float)(n1 - n0 > 0 ? n1 - n0 : 1);
    for (int e = t; e < (n1 - n0) * H; e += blockDim.x) {
        const int i = n0 + e / H, k = e % H;
        dx[(size_t)i * H + k] += dgm[k] * inv;
    }
}

// node head: BCE over labelled nodes (t in {0, 1}; t < 0 = unlabelled)
__global__ void k_node_head_bwd(Wt W, size_t own, const float* p, const float* tn, int Nn, int H, float ln,
                                float inv_nlab, float* dz, float* dx) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Nn * H) return;
    const int i = t / H, k = t - i * H;
    const float g = tn[i] >= 0.f ? ln * (p[i] - tn[i]) * inv_nlab : 0.f;
    if (k == 0) dz[i] = g;
    dx[t] += g * W[own + k];
}

// weight gradient of a linear map: dW[o][k] += sum_r d[r][o] in(r, k), db[o] += sum_r d[r][o], where
// input row r = [in0[idx0 ? idx0[r] : r][0..K0), in1[idx1 ? idx1[r] : r][0..K1), in2[r] (if in2)]
__global__ void k_wgrad_lin(const float* d, int rows, int H_out, const float* in0, const int* idx0, int K0,
                            const float* in1, const int* idx1, int K1, const float* in2, float* gW, float* gb) {
    const int Kt = K0 + K1 + (in2 ? 1 : 0);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= H_out * (Kt + 1)) return;
    const int o = t / (Kt + 1), k = t - o * (Kt + 1);
    float acc = 0.f;
    if (k == Kt) {
        for (int r = 0; r < rows; ++r) acc += d[(size_t)r * H_out + o];
        atomicAdd(&gb[o], acc);
        return;
    }
    for (int r = 0; r < rows; ++r) {
        float v;
        if (k < K0) v = in0[(size_t)(idx0 ? idx0[r] : r) * K0 + k];
        else if (k < K0 + K1) v = in1[(size_t)(idx1 ? idx1[r] : r) * K1 + (k - K0)];
        else v = in2[r];
        acc += d[(size_t)r * H_out + o] * v;
    }
    atomicAdd(&gW[(size_t)o * Kt + k], acc);
}

__global__ void k_relu_mask(const float* g, const float* pre, int n, float* out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = pre[t] > 0.f ? g[t] : 0.f;
}

// update backward: dx_l = dx_{l+1} + W2[:, :H]^T du ; da = W2[:, H:]^T du
__global__ void k_update_bwd_x(Wt W, size_t oW2, const float* du, int Nn, int H, float* dx, float* da) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Nn * H) return;
    const int i = t / H, k = t - i * H;
    float ax = 0.f, aa = 0.f;
    for (int o = 0; o < H; ++o) {
        const float g = du[(size_t)i * H + o];
        ax += W[oW2 + (size_t)o * 2 * H + k] * g;
        aa += W[oW2 + (size_t)o * 2 * H + H + k] * g;
    }
    dx[t] += ax;
    da[t] = aa;
}

// message backward: dm_e = da[dst(e)] * [mpre > 0]
__global__ void k_msg_bwd(const float* da, const int* dst, const float* mpre, int E, int H, float* dm) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= E * H) return;
    const int e = t / H, o = t - e * H;
    dm[t] = mpre[t] > 0.f ? da[(size_t)dst[e] * H + o] : 0.f;
}

// dx_src += W1[:, :H]^T dm_e
__global__ void k_msg_bwd_x(Wt W, size_t oW1, const float* dm, const int* src, int E, int H, float* dx) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= E * H) return;
    const int e = t / H, k = t - e * H;
    float acc = 0.f;
    for (int o = 0; o < H; ++o) acc += W[oW1 + (size_t)o * (H + 1) + k] * dm[(size_t)e * H + o];
    atomicAdd(&dx[(size_t)src[e] * H + k], acc);
}

__global__ void k_adam(float* w, const float* g, float* m1, float* m2, size_t n, float lr, float b1, float b2,
                       float eps, float c1, float c2, __nv_bfloat16* wb) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float gt = g[t];
    const float a = b1 * m1[t] + (1.f - b1) * gt;
    const float b = b2 * m2[t] + (1.f - b2) * gt * gt;
    m1[t] = a;
    m2[t] = b;
    w[t] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
    wb[t] = __float2bfloat16(w[t]);
}

__global__ void k_to_bf16(const float* w, size_t n, __nv_bfloat16* wb) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t < n) wb[t] = __float2bfloat16(w[t]);
}

__global__ void k_loss(const float* p, const float* tn, int Nn, const float* knots, const float* tk, int GK,
                       float ln, float lk, float inv_nlab, float* out) {
    __shared__ float red[256];
    float acc = 0.f;
    for (int i = threadIdx.x; i < Nn; i += blockDim.x)
        if (tn[i] >= 0.f) {
            const float q = fminf(fmaxf(p[i], 1e-7f), 1.f - 1e-7f);
            acc -= ln * inv_nlab * (tn[i] * logf(q) + (1.f - tn[i]) * logf(1.f - q));
        }
    for (int j = threadIdx.x; j < GK; j += blockDim.x) {
        const float d = knots[j] - tk[j];
        acc += lk * d * d / (float)GK;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0];
}

// ------------------------------------------------------------------------------------
// host model
// ------------------------------------------------------------------------------------
static inline unsigned grid_of(size_t n, unsigned b = 256) { return (unsigned)((n + b - 1) / b); }

struct GnnBatchHost {
    int G = 0, Nn = 0, E = 0;
    std::vector<int> goff, src, dst;
    std::vector<float> feat, ew;
};

class Gnn {
public:
    GnnLayout Ly;
    bool bf16;
    int step = 0;
    Gnn(int H, int L, int K, unsigned long long seed, bool use_bf16) : bf16(use_bf16) {
        if (H < 8 || H > 256 || L < 1 || L > 8 || K < 2 || K > 64 || K - 1 > H)
            throw std::invalid_argument("gnn: need 8 <= hidden <= 256, 1 <= layers <= 8, 2 <= knots <= min(64, hidden+1)");
        Ly.H = H;
        Ly.L = L;
        Ly.K = K;
        Ly.F = 4;
        Ly.build();
        try {  // a failed allocation or CUDA call releases what was made before it
            init(seed);
        } catch (...) {
            release();
            throw;
        }
    }
    ~Gnn() { release(); }
    void release() noexcept {
        if (st) cudaStreamSynchronize(st);
        if (arena) cudaFree(arena);
        if (w) cudaFree(w);
        if (wb) cudaFree(wb);
        if (st) cudaStreamDestroy(st);
        arena = nullptr;
        w = nullptr;
        wb = nullptr;
        st = nullptr;
    }
    void init(unsigned long long seed) {
        const int H = Ly.H, L = Ly.L, K = Ly.K;
        GN_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        GN_CK(device_alloc((void**)&w, sizeof(float) * Ly.total * 4));
        g = w + Ly.total;
        m1 = g + Ly.total;
        m2 = m1 + Ly.total;
        GN_CK(device_alloc((void**)&wb, sizeof(__nv_bfloat16) * Ly.total));
        // uniform fan-in initialisation from a seeded splitmix64 stream; biases zero
        std::vector<float> hw(Ly.total, 0.f);
        unsigned long long z = seed * 0x9E3779B97F4A7C15ull + 1;
        auto uni = [&]() {
            z += 0x9E3779B97F4A7C15ull;
            unsigned long long x = z;
            x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
            x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
            x ^= x >> 31;
            return ((x >> 11) + 0.5) * (1.0 / 9007199254740992.0);
        };
        auto fill = [&](size_t off, size_t n, int fan_in, double scale) {
            const double a = scale * std::sqrt(6.0 / fan_in);
            for (size_t i = 0; i < n; ++i) hw[off + i] = (float)((2.0 * uni() - 1.0) * a);
        };
        fill(Ly.We, (size_t)H * 4, 4, 1.0);
        for (int l = 0; l < L; ++l) {
            fill(Ly.W1[l], (size_t)H * (H + 1), H + 1, 1.0);
            fill(Ly.W2[l], (size_t)H * 2 * H, 2 * H, 0.5);
        }
        fill(Ly.wn, H, H, 1.0);
        fill(Ly.Wg1, (size_t)H * H, H, 1.0);
        fill(Ly.Wg2, (size_t)(K - 1) * H, H, 0.1);
        set_params(hw.data());
        GN_CK(cudaMemset(m1, 0, sizeof(float) * Ly.total * 2));
    }
    void set_params(const float* host) {
        GN_CK(cudaMemcpy(w, host, sizeof(float) * Ly.total, cudaMemcpyHostToDevice));
        k_to_bf16<<<grid_of(Ly.total), 256, 0, st>>>(w, Ly.total, wb);
        GN_CK(cudaGetLastError());
        GN_CK(cudaStreamSynchronize(st));
    }
    void get_params(float* host) {
        GN_CK(cudaStreamSynchronize(st));
        GN_CK(cudaMemcpy(host, w, sizeof(float) * Ly.total, cudaMemcpyDeviceToHost));
    }
    Wt weights() const { return Wt{w, bf16 ? wb : nullptr}; }
    // the graph-head kernels index one thread per hidden unit and per knot
    unsigned head_threads() const { return (unsigned)((std::max(64, std::max(Ly.H, Ly.K)) + 31) / 32 * 32); }

    void upload(const GnnBatchHost& B) {
        ensure(B.G, B.Nn, B.E);
        G = B.G;
        Nn = B.Nn;
        E = B.E;
        GN_CK(cudaMemcpyAsync(d_goff, B.goff.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
        GN_CK(cudaMemcpyAsync(d_feat, B.feat.data(), sizeof(float) * Nn * Ly.F, cudaMemcpyHostToDevice, st));
        if (E) {
            GN_CK(cudaMemcpyAsync(d_src, B.src.data(), sizeof(int) * E, cudaMemcpyHostToDevice, st));
            GN_CK(cudaMemcpyAsync(d_dst, B.dst.data(), sizeof(int) * E, cudaMemcpyHostToDevice, st));
            GN_CK(cudaMemcpyAsync(d_ew, B.ew.data(), sizeof(float) * E, cudaMemcpyHostToDevice, st));
        }
    }

    void forward() {
        const int H = Ly.H, L = Ly.L, K = Ly.K;
        const Wt W = weights();
        k_embed<<<grid_of((size_t)Nn * H), 256, 0, st>>>(W, Ly.We, Ly.be, d_feat, Nn, H, Ly.F, e_pre, X(0));
        for (int l = 0; l < L; ++l) {
            if (E)
                k_msg<<<grid_of((size_t)E * H), 256, 0, st>>>(W, Ly.W1[l], Ly.b1[l], X(l), d_src, d_ew, E, H, MP(l),
                                                              MO(l));
            GN_CK(cudaMemsetAsync(A(l), 0, sizeof(float) * Nn * H, st));
            if (E) k_scatter_add<<<grid_of((size_t)E * H), 256, 0, st>>>(MO(l), d_dst, E, H, A(l));
            k_update<<<grid_of((size_t)Nn * H), 256, 0, st>>>(W, Ly.W2[l], Ly.b2[l], X(l), A(l), Nn, H, UP(l),
                                                              X(l + 1));
        }
        k_node_head<<<grid_of(Nn), 256, 0, st>>>(W, Ly.wn, Ly.bn, X(L), Nn, H, p);
        k_graph_head<<<G, head_threads(), sizeof(float) * (2 * H + K), st>>>(W, Ly, X(L), d_goff, gmean, zpre, o,
                                                                              knots);
        GN_CK(cudaGetLastError());
    }

    // gradient of the loss into g (zeroed first); returns the loss
    float backward(const float* tn_host, const float* tk_host, float ln, float lk) {
        const int H = Ly.H, L = Ly.L, K = Ly.K;
        const Wt W = weights();
        GN_CK(cudaMemcpyAsync(d_tn, tn_host, sizeof(float) * Nn, cudaMemcpyHostToDevice, st));
        GN_CK(cudaMemcpyAsync(d_tk, tk_host, sizeof(float) * G * K, cudaMemcpyHostToDevice, st));
        int nlab = 0;
        for (int i = 0; i < Nn; ++i) nlab += tn_host[i] >= 0.f;
        const float inv_nlab = nlab ? 1.f / nlab : 0.f;
        k_loss<<<1, 256, 0, st>>>(p, d_tn, Nn, knots, d_tk, G * K, ln, lk, inv_nlab, d_loss);
        GN_CK(cudaMemsetAsync(g, 0, sizeof(float) * Ly.total, st));
        GN_CK(cudaMemsetAsync(dx, 0, sizeof(float) * Nn * H, st));
        k_graph_head_bwd<<<G, head_threads(), sizeof(float) * (2 * K + 2 * H), st>>>(W, Ly, G, gmean, zpre, o, knots,
                                                                                     d_tk, lk, d_goff, g, dx);
        k_node_head_bwd<<<grid_of((size_t)Nn * H), 256, 0, st>>>(W, Ly.wn, p, d_tn, Nn, H, ln, inv_nlab, dz, dx);
        k_wgrad_lin<<<grid_of(H + 1), 256, 0, st>>>(dz, Nn, 1, X(L), nullptr, H, nullptr, nullptr, 0, nullptr,
                                                    g + Ly.wn, g + Ly.bn);
        for (int l = L - 1; l >= 0; --l) {
            // x_{l+1} = x_l + relu(u):  du = dx [u > 0]; dx carries through the residual
            k_relu_mask<<<grid_of((size_t)Nn * H), 256, 0, st>>>(dx, UP(l), Nn * H, du);
            k_wgrad_lin<<<grid_of((size_t)H * (2 * H + 1)), 256, 0, st>>>(du, Nn, H, X(l), nullptr, H, A(l), nullptr,
                                                                         H, nullptr, g + Ly.W2[l], g + Ly.b2[l]);
            k_update_bwd_x<<<grid_of((size_t)Nn * H), 256, 0, st>>>(W, Ly.W2[l], du, Nn, H, dx, da);
            if (E) {
                k_msg_bwd<<<grid_of((size_t)E * H), 256, 0, st>>>(da, d_dst, MP(l), E, H, dm);
                k_wgrad_lin<<<grid_of((size_t)H * (H + 2)), 256, 0, st>>>(dm, E, H, X(l), d_src, H, nullptr, nullptr,
                                                                         0, d_ew, g + Ly.W1[l], g + Ly.b1[l]);
                k_msg_bwd_x<<<grid_of((size_t)E * H), 256, 0, st>>>(W, Ly.W1[l], dm, d_src, E, H, dx);
            }
        }
        k_relu_mask<<<grid_of((size_t)Nn * H), 256, 0, st>>>(dx, e_pre, Nn * H, du);
        k_wgrad_lin<<<grid_of((size_t)H * (Ly.F + 1)), 256, 0, st>>>(du, Nn, H, d_feat, nullptr, Ly.F, nullptr,
                                                                    nullptr, 0, nullptr, g + Ly.We, g + Ly.be);
        GN_CK(cudaGetLastError());
        float loss = 0.f;
        GN_CK(cudaMemcpyAsync(&loss, d_loss, sizeof(float), cudaMemcpyDeviceToHost, st));
        GN_CK(cudaStreamSynchronize(st));
        return loss;
    }

    void adam(float lr) {
        ++step;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
        k_adam<<<grid_of(Ly.total), 256, 0, st>>>(w, g, m1, m2, Ly.total, lr, b1, b2, 1e-8f, c1, c2, wb);
        GN_CK(cudaGetLastError());
    }

    void read_outputs(float* out_knots, float* out_p) {
        if (out_knots) GN_CK(cudaMemcpyAsync(out_knots, knots, sizeof(float) * G * Ly.K, cudaMemcpyDeviceToHost, st));
        if (out_p) GN_CK(cudaMemcpyAsync(out_p, p, sizeof(float) * Nn, cudaMemcpyDeviceToHost, st));
        GN_CK(cudaStreamSynchronize(st));
    }
    // an externally reduced gradient (data-parallel training) into the gradient buffer
    void write_grads(const float* in) {
        GN_CK(cudaStreamSynchronize(st));
        GN_CK(cudaMemcpy(g, in, sizeof(float) * Ly.total, cudaMemcpyHostToDevice));
    }
    void read_grads(float* out) {
        GN_CK(cudaStreamSynchronize(st));
        GN_CK(cudaMemcpy(out, g, sizeof(float) * Ly.total, cudaMemcpyDeviceToHost));
    }

private:
    cudaStream_t st = nullptr;
    float *w = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    __nv_bfloat16* wb = nullptr;
    int G = 0, Nn = 0, E = 0, capG = 0, capN = 0, capE = 0;
    void* arena = nullptr;
    int *d_goff = nullptr, *d_src = nullptr, *d_dst = nullptr;
    float *d_feat = nullptr, *d_ew = nullptr, *d_tn = nullptr, *d_tk = nullptr, *d_loss = nullptr;
    float *xs = nullptr, *e_pre = nullptr, *mp = nullptr, *mo = nullptr, *as = nullptr, *up = nullptr;
    float *p = nullptr, *gmean = nullptr, *zpre = nullptr, *o = nullptr, *knots = nullptr;
    float *dx = nullptr, *du = nullptr, *da = nullptr, *dm = nullptr, *dz = nullptr;
    float* X(int l) { return xs + (size_t)l * capN * Ly.H; }
    float* MP(int l) { return mp + (size_t)l * capE * Ly.H; }
    float* MO(int l) { return mo + (size_t)l * capE * Ly.H; }
    float* A(int l) { return as + (size_t)l * capN * Ly.H; }
    float* UP(int l) { return up + (size_t)l * capN * Ly.H; }
    void ensure(int nG, int nN, int nE) {
        if (nG <= capG && nN <= capN && nE <= capE) return;
        if (arena) {
            GN_CK(cudaStreamSynchronize(st));
            cudaFree(arena);
        }
        arena = nullptr;
        capG = std::max(nG, 1);
        capN = std::max(nN, 1);
        capE = std::max(nE, 1);
        const int H = Ly.H, L = Ly.L, K = Ly.K;
        size_t off = 0;
        std::vector<std::pair<size_t, void**>> plan;
        auto add = [&](void** ptr, size_t bytes) {
            plan.push_back({off, ptr});
            off += (bytes + 255) & ~(size_t)255;
        };
        add((void**)&d_goff, sizeof(int) * (capG + 1));
        add((void**)&d_src, sizeof(int) * capE);
        add((void**)&d_dst, sizeof(int) * capE);
        add((void**)&d_feat, sizeof(float) * capN * Ly.F);
        add((void**)&d_ew, sizeof(float) * capE);
        add((void**)&d_tn, sizeof(float) * capN);
        add((void**)&d_tk, sizeof(float) * capG * K);
        add((void**)&d_loss, sizeof(float));
        add((void**)&xs, sizeof(float) * (size_t)(L + 1) * capN * H);
        add((void**)&e_pre, sizeof(float) * (size_t)capN * H);
        add((void**)&mp, sizeof(float) * (size_t)L * capE * H);
        add((void**)&mo, sizeof(float) * (size_t)L * capE * H);
        add((void**)&as, sizeof(float) * (size_t)L * capN * H);
        add((void**)&up, sizeof(float) * (size_t)L * capN * H);
        add((void**)&p, sizeof(float) * capN);
        add((void**)&gmean, sizeof(float) * (size_t)capG * H);
        add((void**)&zpre, sizeof(float) * (size_t)capG * H);
        add((void**)&o, sizeof(float) * (size_t)capG * K);
        add((void**)&knots, sizeof(float) * (size_t)capG * K);
        add((void**)&dx, sizeof(float) * (size_t)capN * H);
        add((void**)&du, sizeof(float) * (size_t)capN * H);
        add((void**)&da, sizeof(float) * (size_t)capN * H);
        add((void**)&dm, sizeof(float) * (size_t)capE * H);
        add((void**)&dz, sizeof(float) * capN);
        GN_CK(device_alloc((void**)&arena, off));
        for (auto& it : plan) *it.second = static_cast<char*>(arena) + it.first;
    }
};

// Graph batch from tessera_qa_problem instances: node features [h_i, sum|J|/4, sum J/4, 1] and both
// directions of every edge (self-loops skipped).
static GnnBatchHost batch_of(const tessera_qa_problem* probs, size_t count) {
    GnnBatchHost B;
    B.G = (int)count;
    B.goff.push_back(0);
    for (size_t b = 0; b < count; ++b) {
        const tessera_qa_problem& P = probs[b];
        if (!P.h || P.n == 0) throw std::invalid_argument("gnn: every problem needs n >= 1 and h");
        if (P.m && (!P.ei || !P.ej || !P.ew)) throw std::invalid_argument("gnn: edge arrays are NULL");
        const int base = B.Nn;
        std::vector<float> sa(P.n, 0.f), ss(P.n, 0.f);
        for (size_t e = 0; e < P.m; ++e) {
            if (P.ei[e] >= P.n || P.ej[e] >= P.n) throw std::invalid_argument("gnn: edge index out of range");
            if (P.ei[e] == P.ej[e]) continue;
            const float wv = (float)P.ew[e];
            sa[P.ei[e]] += std::fabs(wv);
            sa[P.ej[e]] += std::fabs(wv);
            ss[P.ei[e]] += wv;
            ss[P.ej[e]] += wv;
            B.src.push_back(base + (int)P.ei[e]);
            B.dst.push_back(base + (int)P.ej[e]);
            B.ew.push_back(wv);
            B.src.push_back(base + (int)P.ej[e]);
            B.dst.push_back(base + (int)P.ei[e]);
            B.ew.push_back(wv);
        }
        for (size_t i = 0; i < P.n; ++i) {
            B.feat.push_back((float)P.h[i]);
            B.feat.push_back(sa[i] / 4.f);
            B.feat.push_back(ss[i] / 4.f);
            B.feat.push_back(1.f);
        }
        B.Nn += (int)P.n;
        B.goff.push_back(B.Nn);
    }
    B.E = (int)B.src.size();
    return B;
}

template <typename F>
static int gn_guard(F&& f) {
    try {
        return f();
    } catch (const std::invalid_argument& e) {
        set_last_error(e.what());
        return TESSERA_QA_EINVAL;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return TESSERA_QA_ECUDA;
    }
}

}  // namespace tq

using namespace tq;

struct tessera_qa_gnn {
    std::unique_ptr<Gnn> net;
};

extern "C" {

double tessera_qa_exact_ground(const double* h, size_t n, const size_t* ei, const size_t* ej, const double* ew,
                               size_t m, int8_t* out_spins) {
    double result = std::nan("");
    const int rc = gn_guard([&]() -> int {
        if (!h || n == 0 || n > 32) throw std::invalid_argument("exact ground state needs 1 <= n <= 32 and h");
        if (m && (!ei || !ej || !ew)) throw std::invalid_argument("edge arrays are NULL");
        std::vector<int> a(m), b(m);
        for (size_t e = 0; e < m; ++e) {
            if (ei[e] >= n || ej[e] >= n) throw std::invalid_argument("edge index out of range");
            a[e] = (int)ei[e];
            b[e] = (int)ej[e];
        }
        const size_t smem = sizeof(double) * (n + m) + sizeof(int) * 2 * m;
        if (smem > 200 * 1024) throw std::invalid_argument("too many edges for the exact ground state kernel");
        const unsigned long long total = 1ull << n;
        int nsm = 0, dev = 0;
        GN_CK(cudaGetDevice(&dev));
        GN_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        unsigned long long blocks = (total + 255) / 256;
        if (blocks > (unsigned long long)nsm * 8) blocks = (unsigned long long)nsm * 8;
        char* arena = nullptr;
        const size_t mm = std::max<size_t>(m, 1);
        const size_t bytes = 64 * 8 + 8 * n + 8 * mm + 8 * mm + 16 * blocks;
        GN_CK(device_alloc((void**)&arena, bytes));
        size_t off = 0;
        auto take = [&](size_t sz) {
            void* r = arena + off;
            off += (sz + 63) & ~(size_t)63;
            return r;
        };
        double* dh = (double*)take(8 * n);
        double* dw = (double*)take(8 * mm);
        int* di = (int*)take(4 * mm);
        int* dj = (int*)take(4 * mm);
        double* be = (double*)take(8 * blocks);
        unsigned long long* bx = (unsigned long long*)take(8 * blocks);
        cudaError_t err = cudaMemcpy(dh, h, 8 * n, cudaMemcpyHostToDevice);
        if (err == cudaSuccess && m) err = cudaMemcpy(dw, ew, 8 * m, cudaMemcpyHostToDevice);
        if (err == cudaSuccess && m) err = cudaMemcpy(di, a.data(), 4 * m, cudaMemcpyHostToDevice);
        if (err == cudaSuccess && m) err = cudaMemcpy(dj, b.data(), 4 * m, cudaMemcpyHostToDevice);
        if (err == cudaSuccess && smem > 48 * 1024)
            err = cudaFuncSetAttribute(k_ground, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err == cudaSuccess) {
            k_ground<<<(unsigned)blocks, 256, smem>>>(dh, di, dj, dw, (int)n, (int)m, total, be, bx);
            err = cudaGetLastError();
        }
        std::vector<double> he(blocks);
        std::vector<unsigned long long> hx(blocks);
        if (err == cudaSuccess) err = cudaMemcpy(he.data(), be, 8 * blocks, cudaMemcpyDeviceToHost);
        if (err == cudaSuccess) err = cudaMemcpy(hx.data(), bx, 8 * blocks, cudaMemcpyDeviceToHost);
        cudaFree(arena);
        GN_CK(err);
        double best = INFINITY;
        unsigned long long x = 0;
        for (unsigned long long k = 0; k < blocks; ++k)
            if (he[k] < best || (he[k] == best && hx[k] < x)) {
                best = he[k];
                x = hx[k];
            }
        if (out_spins)
            for (size_t i = 0; i < n; ++i) out_spins[i] = ((x >> i) & 1ull) ? 1 : -1;
        result = best;
        return 0;
    });
    return rc == 0 ? result : std::nan("");
}

tessera_qa_gnn* tessera_qa_gnn_create(int hidden, int layers, int knots, uint64_t seed, int bf16_weights) {
    tessera_qa_gnn* out = nullptr;
    gn_guard([&]() -> int {
        std::unique_ptr<tessera_qa_gnn> g(new tessera_qa_gnn);
        g->net.reset(new Gnn(hidden, layers, knots, seed, bf16_weights != 0));
        out = g.release();
        return 0;
    });
    return out;
}

void tessera_qa_gnn_destroy(tessera_qa_gnn* g) { delete g; }

size_t tessera_qa_gnn_param_count(const tessera_qa_gnn* g) { return g ? g->net->Ly.total : 0; }

int tessera_qa_gnn_get_params(tessera_qa_gnn* g, float* out, size_t count) {
    return gn_guard([&]() -> int {
        if (!g || !out || count < g->net->Ly.total) throw std::invalid_argument("gnn get_params: bad buffer");
        g->net->get_params(out);
        return 0;
    });
}

int tessera_qa_gnn_set_params(tessera_qa_gnn* g, const float* in, size_t count) {
    return gn_guard([&]() -> int {
        if (!g || !in || count < g->net->Ly.total) throw std::invalid_argument("gnn set_params: bad buffer");
        g->net->set_params(in);
        return 0;
    });
}

int tessera_qa_gnn_forward(tessera_qa_gnn* g, const tessera_qa_problem* problems, size_t count, float* out_knots,
                           float* out_p) {
    return gn_guard([&]() -> int {
        if (!g || !problems || count == 0) throw std::invalid_argument("gnn forward: bad arguments");
        GnnBatchHost B = batch_of(problems, count);
        g->net->upload(B);
        g->net->forward();
        g->net->read_outputs(out_knots, out_p);
        return 0;
    });
}

int tessera_qa_gnn_train_step(tessera_qa_gnn* g, const tessera_qa_problem* problems, size_t count,
                              const float* target_knots, const float* target_spins, float lr, float lambda_knots,
                              float lambda_spins, float* out_loss, float* out_grads, size_t grads_count) {
    return gn_guard([&]() -> int {
        if (!g || !problems || count == 0 || !target_knots || !target_spins)
            throw std::invalid_argument("gnn train_step: bad arguments");
        GnnBatchHost B = batch_of(problems, count);
        g->net->upload(B);
        g->net->forward();
        const float loss = g->net->backward(target_spins, target_knots, lambda_spins, lambda_knots);
        if (out_loss) *out_loss = loss;
        if (out_grads) {
            if (grads_count < g->net->Ly.total) throw std::invalid_argument("gnn train_step: grads buffer too small");
            g->net->read_grads(out_grads);
        }
        if (lr > 0.f) g->net->adam(lr);
        return 0;
    });
}

int tessera_qa_gnn_apply_grads(tessera_qa_gnn* g, const float* grads, size_t count, float lr) {
    return gn_guard([&]() -> int {
        if (!g || !grads || count < g->net->Ly.total || !(lr > 0.f))
            throw std::invalid_argument("gnn apply_grads: bad arguments");
        g->net->write_grads(grads);
        g->net->adam(lr);
        GN_CK(cudaDeviceSynchronize());
        return 0;
    });
}

int tessera_qa_schedule_predict(tessera_qa_gnn* g, const tessera_qa_problem* problems, size_t count,
                                double* out_knots, double* out_bias) {
    return gn_guard([&]() -> int {
        if (!g || !problems || count == 0 || !out_knots) throw std::invalid_argument("schedule_predict: bad arguments");
        GnnBatchHost B = batch_of(problems, count);
        std::vector<float> kn((size_t)B.G * g->net->Ly.K), pp(B.Nn);
        g->net->upload(B);
        g->net->forward();
        g->net->read_outputs(kn.data(), pp.data());
        for (size_t i = 0; i < kn.size(); ++i) out_knots[i] = kn[i];
        if (out_bias)
            for (int i = 0; i < B.Nn; ++i) out_bias[i] = 2.0 * pp[i] - 1.0;  // in [-1, 1], + favours spin +1
        return 0;
    });
}

}  // extern "C"
