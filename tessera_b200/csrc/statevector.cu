// statevector.cu -- K10: the exact 2^n state-vector anneal on the GPU (1 <= n <= 30).
//
// The FP64 oracle of the reference, rust/src/quantum.rs:63-112 (anneal_statevector), as CUDA:
//   mode 0 (quantum.rs:82-84): psi <- P(B dt/2) X(A dt) P(B dt/2) psi per step, with
//          P(t) = exp(-i t E(x)) the problem phase (E the Ising energy) and X(t) = prod_i exp(+i t X_i);
//   mode 1 (the MPS engine's splitting, cuda/src/mps.cpp:313-353): single-site half steps
//          exp(-i dt/2 (-A X - B h_i Z)) (plus the warm-start field -C b_i Z when the problem
//          carries one), the exact ZZ block exp(-i dt B E_zz(x)), single-site half steps again.
// Basis: bit i of x is the physical index of spin i (bit 0 <-> spin +1), as the engine's MPS.
// Per step: qubit-0 entanglement entropy (quantum.rs:138-175).  Readout: the most probable
// pattern (quantum.rs:94-103) and the sign<Z> pattern, with energies and probabilities.
//
// Layout: psi is 2^n complex128 in HBM (16 GiB at n = 30), diag_full and diag_zz 2^n doubles.
// Single-qubit gates are applied in tiles: a CTA loads the 2^(5+K) amplitudes that share all
// bits outside {0..4} and K target qubits (the low five bits keep the loads coalesced), applies
// the gates of every target in shared memory, and writes the tile back -- one HBM round trip per
// pass instead of one per qubit.  Passes cover qubits 0..11, then the rest in even groups of at
// most seven (n = 24: three passes per half step).  The diagonal phases ride on the first pass's
// load and the last pass's store, and the last pass of a step also sums the qubit-0 reduced
// density matrix over its tile, so a mode-0 step is exactly one sweep of passes (three round
// trips of psi at n = 24).  In mode 1 the closing single-qubit half step of one step and the
// opening one of the next are merged into one gate per qubit, so that mode too costs one sweep
// per step (plus one).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tessera_qa.h"
#include "common.cuh"

namespace tq {

void set_last_error(const std::string& msg);

#define SV_CK(x)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (x);                                                                             \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_)); \
    } while (0)

constexpr int SV_LOW = 5;         // low bits always in a tile
constexpr int SV_TGT = 7;         // at most this many target qubits per tile above the low bits
constexpr int SV_NT = 256;
constexpr int SV_MAXN = 30;

struct SvPass {
    int nt;            // tile bits (low + targets)
    int nlow;          // tile bits 0..nlow-1 are x bits 0..nlow-1
    int pos[12];       // bit position in x of tile bit t
    int ngate;         // gates applied in this pass
    int gq[12];        // tile bit index of each gated qubit
    int qubit[12];     // its qubit number (row of the gate table)
    int nrest;         // bits outside the tile
    int rpos[SV_MAXN]; // their positions in x, ascending
};

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Ising energy E(x) = -sum w s_i s_j - sum h s_i and its ZZ part, s = +1 for bit 0.
__global__ void k_sv_diag(const double* h, const int* ei, const int* ej, const double* w, int n, int m,
                          unsigned long long dim, double* dfull, double* dzz, double2* psi) {
    const double amp = rsqrt((double)dim);
    for (unsigned long long x = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; x < dim;
         x += (unsigned long long)gridDim.x * blockDim.x) {
        double ez = 0.0, eh = 0.0;
        for (int q = 0; q < m; ++q) {
            const int si = ((x >> ei[q]) & 1ull) ? -1 : 1, sj = ((x >> ej[q]) & 1ull) ? -1 : 1;
            ez -= w[q] * (double)(si * sj);
        }
        for (int i = 0; i < n; ++i) eh -= h[i] * (((x >> i) & 1ull) ? -1.0 : 1.0);
        dzz[x] = ez;
        dfull[x] = ez + eh;
        psi[x] = make_double2(amp, 0.0);
    }
}

// 2x2 single-qubit gate of qubit i at step k (row-major u00 u01 u10 u11).
__device__ void sv_gate(const double* h, const double* sa, const double* sb, const double* bias, const double* sc,
                        int i, int k, double dt, int mode, double2 g[4]) {
    const double A = sa[k], B = sb[k];
    if (mode == 0) {  // exp(+i A dt X)
        const double c = cos(A * dt), s = sin(A * dt);
        g[0] = make_double2(c, 0.0); g[1] = make_double2(0.0, s);
        g[2] = make_double2(0.0, s); g[3] = make_double2(c, 0.0);
    } else {  // exp(-i dt/2 (nx X + nz Z)), nx = -A, nz = -(B h_i + C b_i)
        const double nx = -A, nz = -(B * h[i] + (bias ? sc[k] * bias[i] : 0.0));
        const double r = sqrt(nx * nx + nz * nz);
        double c = 1.0, sn = 0.0;
        if (r > 0) {
            c = cos(0.5 * dt * r);
            sn = sin(0.5 * dt * r) / r;
        }
        g[0] = make_double2(c, -sn * nz); g[1] = make_double2(0.0, -sn * nx);
        g[2] = make_double2(0.0, -sn * nx); g[3] = make_double2(c, sn * nz);
    }
}

// Gate of every qubit for step k, or, with k2 >= 0, the product G(k2) G(k) (G(k) applied first).
__global__ void k_sv_gates(const double* h, const double* sa, const double* sb, const double* bias, const double* sc,
                           int n, int k, int k2, double dt, int mode, double2* gates) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double2 g[4];
    sv_gate(h, sa, sb, bias, sc, i, k, dt, mode, g);
    if (k2 >= 0) {
        double2 f[4];
        sv_gate(h, sa, sb, bias, sc, i, k2, dt, mode, f);
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 2; ++c) {
                const double2 x = zmul(f[2 * r], g[c]), y = zmul(f[2 * r + 1], g[2 + c]);
                gates[4 * i + 2 * r + c] = make_double2(x.x + y.x, x.y + y.y);
            }
    } else {
        for (int q = 0; q < 4; ++q) gates[4 * i + q] = g[q];
    }
}

// Diagonal phase fused into a pass: psi[x] *= exp(-i scale d[x]).
struct SvPhase {
    const double* d;  // NULL: none
    double scale;
};

__device__ __forceinline__ double2 sv_phase(double2 v, const SvPhase& ph, unsigned long long x) {
    double sn, cs;
    sincos(-ph.scale * ph.d[x], &sn, &cs);
    return zmul(v, make_double2(cs, sn));
}

// One tiled pass of single-qubit gates, with an optional diagonal phase applied on load (pre)
// and before the store (post), and optional partial sums of the qubit-0 reduced density matrix
// (r00, r11, Re r01, Im r01 per CTA into rho) of the gated tile: after the post phase, or
// before it when rho_first is set.
__global__ void __launch_bounds__(SV_NT) k_sv_pass(double2* psi, SvPass ps, const double2* gates, SvPhase pre,
                                                   SvPhase post, double* rho, int rho_first) {
    extern __shared__ double2 tile[];
    __shared__ double red[4][SV_NT / 32];
    const int T = 1 << ps.nt;
    // base index of this CTA: blockIdx spread over the rest bits
    unsigned long long base = 0, r = blockIdx.x;
    for (int b = 0; b < ps.nrest; ++b, r >>= 1)
        if (r & 1ull) base |= 1ull << ps.rpos[b];
    const int lowmask = (1 << ps.nlow) - 1;
    for (int t = threadIdx.x; t < T; t += SV_NT) {
        unsigned long long x = base | (unsigned long long)(t & lowmask);
        for (int b = ps.nlow; b < ps.nt; ++b)
            if ((t >> b) & 1) x |= 1ull << ps.pos[b];
        const double2 v = psi[x];
        tile[t] = pre.d ? sv_phase(v, pre, x) : v;
    }
    __syncthreads();
    for (int gI = 0; gI < ps.ngate; ++gI) {
        const int tb = ps.gq[gI];
        const double2* g = gates + 4 * ps.qubit[gI];
        const double2 u00 = g[0], u01 = g[1], u10 = g[2], u11 = g[3];
        for (int p = threadIdx.x; p < T / 2; p += SV_NT) {
            // insert a 0 at tile bit tb
            const int lo = p & ((1 << tb) - 1);
            const int t0 = ((p >> tb) << (tb + 1)) | lo, t1 = t0 | (1 << tb);
            const double2 a = tile[t0], b = tile[t1];
            const double2 x0 = zmul(u00, a), x1 = zmul(u01, b), y0 = zmul(u10, a), y1 = zmul(u11, b);
            tile[t0] = make_double2(x0.x + x1.x, x0.y + x1.y);
            tile[t1] = make_double2(y0.x + y1.x, y0.y + y1.y);
        }
        __syncthreads();
    }
    // the post phase goes into the tile first only when the reduction must see it
    const bool post_in_tile = post.d && rho && !rho_first;
    if (post_in_tile) {
        for (int t = threadIdx.x; t < T; t += SV_NT) {
            unsigned long long x = base | (unsigned long long)(t & lowmask);
            for (int b = ps.nlow; b < ps.nt; ++b)
                if ((t >> b) & 1) x |= 1ull << ps.pos[b];
            tile[t] = sv_phase(tile[t], post, x);
        }
        __syncthreads();
    }
    if (rho) {  // tile bit 0 is x bit 0: pairs (2y, 2y + 1) differ in qubit 0 only
        double a = 0, bb = 0, cr = 0, ci = 0;
        for (int y = threadIdx.x; y < T / 2; y += SV_NT) {
            const double2 u = tile[2 * y], v = tile[2 * y + 1];
            a += u.x * u.x + u.y * u.y;
            bb += v.x * v.x + v.y * v.y;
            cr += u.x * v.x + u.y * v.y;  // u conj(v)
            ci += u.y * v.x - u.x * v.y;
        }
        a = warp_sum(a); bb = warp_sum(bb); cr = warp_sum(cr); ci = warp_sum(ci);
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) { red[0][w] = a; red[1][w] = bb; red[2][w] = cr; red[3][w] = ci; }
        __syncthreads();
        if (threadIdx.x < 4) {
            double sum = 0;
            for (int q = 0; q < SV_NT / 32; ++q) sum += red[threadIdx.x][q];
            rho[4 * (size_t)blockIdx.x + threadIdx.x] = sum;
        }
    }
    const bool post_on_store = post.d && !post_in_tile;
    for (int t = threadIdx.x; t < T; t += SV_NT) {
        unsigned long long x = base | (unsigned long long)(t & lowmask);
        for (int b = ps.nlow; b < ps.nt; ++b)
            if ((t >> b) & 1) x |= 1ull << ps.pos[b];
        psi[x] = post_on_store ? sv_phase(tile[t], post, x) : tile[t];
    }
}

__global__ void k_sv_entropy(const double* part, int nblk, double* out, int k) {
    __shared__ double red[4][SV_NT / 32];
    double r[4] = {0, 0, 0, 0};
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
        for (int q = 0; q < 4; ++q) r[q] += part[4 * (size_t)b + q];
    for (int q = 0; q < 4; ++q) r[q] = warp_sum(r[q]);
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < 4; ++q) red[q][threadIdx.x >> 5] = r[q];
    __syncthreads();
    if (threadIdx.x != 0) return;
    double r00 = 0, r11 = 0, rr = 0, ri = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { r00 += red[0][w]; r11 += red[1][w]; rr += red[2][w]; ri += red[3][w]; }
    const double tot = r00 + r11;
    double S = 0.0;
    if (tot > 0) {
        const double p = r00 / tot, q = r11 / tot, off2 = (rr * rr + ri * ri) / (tot * tot);
        const double mid = 0.5 * (p + q), rad = sqrt(fmax(0.0, 0.25 * (p - q) * (p - q) + off2));
        const double l1 = fmin(1.0, fmax(0.0, mid + rad)), l2 = fmin(1.0, fmax(0.0, mid - rad));
        if (l1 > 1e-12) S -= l1 * log2(l1);
        if (l2 > 1e-12) S -= l2 * log2(l2);
    }
    out[k] = S;
}

// per-block: total probability, sum p E(x), best p and its (smallest) index, sum p z_i
__global__ void k_sv_final(const double2* psi, const double* dfull, unsigned long long dim, int n, double* part,
                           unsigned long long* bestx) {
    __shared__ double sp[SV_NT], se[SV_NT], sb[SV_NT];
    __shared__ unsigned long long sx[SV_NT];
    __shared__ double sz[SV_MAXN][SV_NT / 32];
    double tot = 0, ee = 0, bp = -1.0;
    unsigned long long bx = ~0ull;
    double ez[SV_MAXN];
    for (int i = 0; i < n; ++i) ez[i] = 0.0;
    for (unsigned long long x = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; x < dim;
         x += (unsigned long long)gridDim.x * blockDim.x) {
        const double2 v = psi[x];
        const double p = v.x * v.x + v.y * v.y;
        tot += p;
        ee += p * dfull[x];
        if (p > bp) { bp = p; bx = x; }  // strided visits ascend in x: first maximum kept
        for (int i = 0; i < n; ++i) ez[i] += ((x >> i) & 1ull) ? -p : p;
    }
    sp[threadIdx.x] = tot; se[threadIdx.x] = ee; sb[threadIdx.x] = bp; sx[threadIdx.x] = bx;
    for (int i = 0; i < n; ++i) {
        const double v = warp_sum(ez[i]);
        if ((threadIdx.x & 31) == 0) sz[i][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    for (int o = SV_NT / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sp[threadIdx.x] += sp[threadIdx.x + o];
            se[threadIdx.x] += se[threadIdx.x + o];
            const double p2 = sb[threadIdx.x + o];
            const unsigned long long x2 = sx[threadIdx.x + o];
            if (p2 > sb[threadIdx.x] || (p2 == sb[threadIdx.x] && x2 < sx[threadIdx.x])) {
                sb[threadIdx.x] = p2;
                sx[threadIdx.x] = x2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double* q = part + (size_t)blockIdx.x * (3 + SV_MAXN);
        q[0] = sp[0]; q[1] = se[0]; q[2] = sb[0];
        for (int i = 0; i < n; ++i) {
            double s = 0;
            for (int w = 0; w < SV_NT / 32; ++w) s += sz[i][w];
            q[3 + i] = s;
        }
        bestx[blockIdx.x] = sx[0];
    }
}

// Passes of one half step: the first gates the low bits and the next SV_TGT qubits; the rest
// are spread evenly over as few passes as hold at most SV_TGT targets each (no small last pass).
static std::vector<SvPass> plan_passes(int n) {
    std::vector<SvPass> out;
    const int low = n < SV_LOW ? n : SV_LOW;
    std::vector<std::vector<int>> groups;
    std::vector<int> first;
    for (int q = low; q < n && (int)first.size() < SV_TGT; ++q) first.push_back(q);
    groups.push_back(first);
    const int start = low + (int)first.size(), rem = n - start;
    if (rem > 0) {
        const int np = (rem + SV_TGT - 1) / SV_TGT;
        int q = start;
        for (int k = 0; k < np; ++k) {
            const int cnt = rem / np + (k < rem % np ? 1 : 0);
            std::vector<int> g;
            for (int c = 0; c < cnt; ++c) g.push_back(q++);
            groups.push_back(g);
        }
    }
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        SvPass p{};
        p.nt = 0;
        p.nlow = low;
        for (int b = 0; b < low; ++b) p.pos[p.nt++] = b;  // low bits always in the tile
        p.ngate = 0;
        if (gi == 0)
            for (int b = 0; b < low; ++b) { p.gq[p.ngate] = b; p.qubit[p.ngate] = b; ++p.ngate; }
        for (int q : groups[gi]) {
            p.gq[p.ngate] = p.nt;
            p.qubit[p.ngate] = q;
            ++p.ngate;
            p.pos[p.nt++] = q;
        }
        p.nrest = 0;
        for (int b = 0; b < n; ++b) {
            bool in = false;
            for (int t = 0; t < p.nt; ++t) in = in || p.pos[t] == b;
            if (!in) p.rpos[p.nrest++] = b;
        }
        out.push_back(p);
    }
    return out;
}

}  // namespace tq

using namespace tq;

extern "C" int tessera_qa_sv_anneal(const tessera_qa_problem* P, double dt, int mode, tessera_qa_sv_result* out) {
    try {
        if (!P || !out) throw std::invalid_argument("problem and result are required");
        if (!P->h || P->n < 1 || P->n > SV_MAXN) throw std::invalid_argument("state-vector anneal needs 1 <= n <= 30");
        if (P->m && (!P->ei || !P->ej || !P->ew)) throw std::invalid_argument("edge arrays are NULL");
        if (!P->schedule_a || !P->schedule_b || P->steps < 2) throw std::invalid_argument("schedule needs >= 2 steps");
        if (!(dt > 0) || !std::isfinite(dt)) throw std::invalid_argument("dt must be a finite positive number");
        if (mode != 0 && mode != 1) throw std::invalid_argument("mode must be 0 (quantum.rs) or 1 (engine splitting)");
        if (P->bias && (!P->schedule_c || mode != 1))
            throw std::invalid_argument("the warm-start field needs schedule_c and mode 1");
        if (!out->spins) throw std::invalid_argument("result.spins is NULL");
        const int n = (int)P->n, m = (int)P->m, steps = (int)P->steps;
        std::vector<int> a(m), b(m);
        for (int e = 0; e < m; ++e) {
            if (P->ei[e] >= P->n || P->ej[e] >= P->n) throw std::invalid_argument("edge index out of range");
            a[e] = (int)P->ei[e];
            b[e] = (int)P->ej[e];
        }
        for (size_t i = 0; i < P->n; ++i)
            if (!std::isfinite(P->h[i])) throw std::invalid_argument("non-finite h");
        const unsigned long long dim = 1ull << n;
        size_t freeb = 0, totb = 0;
        SV_CK(cudaMemGetInfo(&freeb, &totb));
        const size_t need = dim * (16 + 8 + 8) + (1 << 20);
        if (need > freeb) throw std::invalid_argument("not enough device memory for the 2^n state");
        cudaStream_t st;
        SV_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        int nsm = 148, dev = 0;
        SV_CK(cudaGetDevice(&dev));
        SV_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const int grid = nsm * 8;
        char* arena = nullptr;
        auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
        const size_t o_psi = 0, o_df = o_psi + al(dim * 16), o_dz = o_df + al(dim * 8);
        const size_t o_h = o_dz + al(dim * 8), o_w = o_h + al(8 * n), o_i = o_w + al(8 * (m + 1));
        const size_t o_j = o_i + al(4 * (m + 1)), o_sa = o_j + al(4 * (m + 1)), o_sb = o_sa + al(8 * steps);
        const size_t o_bias = o_sb + al(8 * steps), o_sc = o_bias + al(8 * n), o_g = o_sc + al(8 * steps);
        const size_t o_part = o_g + al(64 * n), o_ent = o_part + al(8 * (size_t)grid * (3 + SV_MAXN));
        const std::vector<SvPass> passes = plan_passes(n);
        const size_t rho_blocks = 1ull << passes.back().nrest;  // qubit-0 partials: one set per last-pass CTA
        const size_t o_bx = o_ent + al(8 * steps), o_rho = o_bx + al(8 * (size_t)grid);
        const size_t total = o_rho + al(32 * rho_blocks);
        SV_CK(device_alloc((void**)&arena, total));
        auto at = [&](size_t o) { return arena + o; };
        double2* psi = (double2*)at(o_psi);
        double *df = (double*)at(o_df), *dz = (double*)at(o_dz), *dh = (double*)at(o_h), *dw = (double*)at(o_w);
        int *di = (int*)at(o_i), *dj = (int*)at(o_j);
        double *dsa = (double*)at(o_sa), *dsb = (double*)at(o_sb), *dbias = (double*)at(o_bias), *dsc = (double*)at(o_sc);
        double2* dg = (double2*)at(o_g);
        double *part = (double*)at(o_part), *dent = (double*)at(o_ent);
        unsigned long long* dbx = (unsigned long long*)at(o_bx);
        double* drho = (double*)at(o_rho);
        cudaError_t err = cudaSuccess;
        auto cp = [&](void* d, const void* h, size_t bytes) {
            if (err == cudaSuccess && bytes) err = cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st);
        };
        cp(dh, P->h, 8 * n);
        cp(dw, P->ew, 8 * m);
        cp(di, a.data(), 4 * m);
        cp(dj, b.data(), 4 * m);
        cp(dsa, P->schedule_a, 8 * steps);
        cp(dsb, P->schedule_b, 8 * steps);
        if (P->bias) {
            cp(dbias, P->bias, 8 * n);
            cp(dsc, P->schedule_c, 8 * steps);
        }
        cudaEvent_t e0, e1;
        if (err == cudaSuccess) err = cudaEventCreate(&e0);
        if (err == cudaSuccess) err = cudaEventCreate(&e1);
        int maxnt = 0;
        for (const SvPass& p : passes) maxnt = p.nt > maxnt ? p.nt : maxnt;
        const size_t tile_bytes = sizeof(double2) << maxnt;
        if (err == cudaSuccess && tile_bytes > 48 * 1024)
            err = cudaFuncSetAttribute(k_sv_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_bytes);
        if (err == cudaSuccess) err = cudaMemsetAsync(dent, 0, 8 * (size_t)steps, st);  // n = 1: no entanglement
        if (err == cudaSuccess) {
            cudaEventRecord(e0, st);
            k_sv_diag<<<grid, SV_NT, 0, st>>>(dh, di, dj, dw, n, m, dim, df, dz, psi);
            const SvPhase none{nullptr, 0.0};
            const double* hsb = P->schedule_b;
            auto gates = [&](int k, int k2) {
                k_sv_gates<<<(n + 63) / 64, 64, 0, st>>>(dh, dsa, dsb, P->bias ? dbias : nullptr, dsc, n, k, k2, dt,
                                                        mode, dg);
            };
            // One sweep of the gate passes; `pre` rides on the first pass's load, `post` and the
            // qubit-0 partial sums on the last pass.
            auto sweep = [&](SvPhase pre, SvPhase post, double* rho, int rho_first) {
                for (size_t i = 0; i < passes.size(); ++i) {
                    const SvPass& p = passes[i];
                    const bool last = i + 1 == passes.size();
                    const unsigned long long blocks = 1ull << p.nrest;
                    k_sv_pass<<<(unsigned)blocks, SV_NT, sizeof(double2) << p.nt, st>>>(
                        psi, p, dg, i == 0 ? pre : none, last ? post : none, last ? rho : nullptr, rho_first);
                }
            };
            double* rho = n >= 2 ? drho : nullptr;
            if (mode == 0) {  // P X P per step: one sweep, both phases fused into it
                for (int k = 0; k < steps; ++k) {
                    const SvPhase ph{df, 0.5 * hsb[k] * dt};
                    gates(k, -1);
                    sweep(ph, ph, rho, 0);
                    if (rho) k_sv_entropy<<<1, SV_NT, 0, st>>>(rho, (int)rho_blocks, dent, k);
                }
            } else {
                // G(k) Z(k) G(k) per step.  The closing half step of step k and the opening one of
                // step k+1 are single-qubit gates on every qubit, so they run as one sweep of
                // the products G(k+1) G(k).  The qubit-0 entropy of step k is read from that
                // sweep before the next ZZ phase: G(k+1) is a product of one-qubit unitaries,
                // which leaves the Schmidt spectrum across the qubit-0 cut unchanged.
                gates(0, -1);
                sweep(none, SvPhase{dz, 1.0 * hsb[0] * dt}, nullptr, 0);
                for (int k = 0; k < steps; ++k) {
                    const bool more = k + 1 < steps;
                    gates(k, more ? k + 1 : -1);
                    sweep(none, more ? SvPhase{dz, 1.0 * hsb[k + 1] * dt} : none, rho, 1);
                    if (rho) k_sv_entropy<<<1, SV_NT, 0, st>>>(rho, (int)rho_blocks, dent, k);
                }
            }
            k_sv_final<<<grid, SV_NT, 0, st>>>(psi, df, dim, n, part, dbx);
            cudaEventRecord(e1, st);
            err = cudaGetLastError();
        }
        std::vector<double> hp((size_t)grid * (3 + SV_MAXN));
        std::vector<unsigned long long> hbx(grid);
        std::vector<double> ent(steps);
        if (err == cudaSuccess) err = cudaMemcpyAsync(hp.data(), part, 8 * hp.size(), cudaMemcpyDeviceToHost, st);
        if (err == cudaSuccess) err = cudaMemcpyAsync(hbx.data(), dbx, 8 * hbx.size(), cudaMemcpyDeviceToHost, st);
        if (err == cudaSuccess) err = cudaMemcpyAsync(ent.data(), dent, 8 * steps, cudaMemcpyDeviceToHost, st);
        if (err == cudaSuccess && out->state)
            err = cudaMemcpyAsync(out->state, psi, dim * 16, cudaMemcpyDeviceToHost, st);
        if (err == cudaSuccess) err = cudaStreamSynchronize(st);
        float ms = 0;
        if (err == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(arena);
        cudaStreamDestroy(st);
        SV_CK(err);
        double tot = 0, ee = 0, bp = -1;
        unsigned long long bx = 0;
        std::vector<double> ez(n, 0.0);
        for (int g = 0; g < grid; ++g) {
            const double* q = hp.data() + (size_t)g * (3 + SV_MAXN);
            tot += q[0];
            ee += q[1];
            if (q[2] > bp || (q[2] == bp && hbx[g] < bx)) { bp = q[2]; bx = hbx[g]; }
            for (int i = 0; i < n; ++i) ez[i] += q[3 + i];
        }
        auto energy = [&](unsigned long long x) {
            double e = 0;
            for (int q = 0; q < m; ++q) {
                const int si = ((x >> a[q]) & 1ull) ? -1 : 1, sj = ((x >> b[q]) & 1ull) ? -1 : 1;
                e -= P->ew[q] * si * sj;
            }
            for (int i = 0; i < n; ++i) e -= P->h[i] * (((x >> i) & 1ull) ? -1.0 : 1.0);
            return e;
        };
        for (int i = 0; i < n; ++i) out->spins[i] = ((bx >> i) & 1ull) ? -1 : 1;
        unsigned long long xs = 0;
        for (int i = 0; i < n; ++i) {
            const int8_t s = (ez[i] / tot >= 0.0) ? 1 : -1;
            if (out->sign_spins) out->sign_spins[i] = s;
            if (s < 0) xs |= 1ull << i;
        }
        out->energy = energy(bx);
        out->expected_energy = ee / tot;
        out->prob = bp / tot;
        out->sign_energy = energy(xs);
        out->sign_prob = -1.0;  // filled below when the state was read back
        if (out->state) {
            const double* s = out->state;
            out->sign_prob = (s[2 * xs] * s[2 * xs] + s[2 * xs + 1] * s[2 * xs + 1]) / tot;
        }
        out->norm2 = tot;
        out->device_ms = ms;
        if (out->entropy) std::memcpy(out->entropy, ent.data(), 8 * steps);
        return 0;
    } catch (const std::invalid_argument& e) {
        set_last_error(e.what());
        return TESSERA_QA_EINVAL;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return TESSERA_QA_ECUDA;
    }
}
