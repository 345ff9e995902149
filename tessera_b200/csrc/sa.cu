// sa.cu -- best-of-restarts simulated annealing on the GPU (tessera_qa_sa_solve): the
// best-known-energy scorer for instances beyond brute force.
//
// Restates the reference's classical solver (rust/src/ising.rs:64-136, sa_run and sa_solve):
// each restart starts from a random spin pattern; sweep k runs at temperature
// t_k = t0 (t_end / t0)^(k / (max(sweeps, 2) - 1)) and visits spins 0..n-1 in order, flipping
// spin i when dE = 2 s_i (h_i + sum_j J_ij s_j) < 0 or u < exp(-dE / t_k); a run's result is
// the energy of its final pattern, and the solver keeps the lowest (the first restart on ties).
// The reference draws from rand's StdRng; here every uniform comes from a counter-based
// splitmix64 stream keyed by (seed, instance, restart, sweep, spin), so a run is reproducible
// and the CPU oracle restates it draw for draw.
//
// Layout: one CTA per instance, one thread per restart chain (chunks of SA_THREADS restarts).
// The coupling graph sits in shared memory as adjacency lists (offsets, neighbour, weight);
// a chain's spins are a bit mask of SA_MAXN bits in registers (bit i set <-> s_i = -1).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tessera_qa.h"
#include "common.cuh"

namespace tq {

constexpr int SA_MAXN = 128;
constexpr int SA_WORDS = SA_MAXN / 64;
constexpr int SA_THREADS = 128;

#define SA_CK(x)                                                                                          \
    do {                                                                                                  \
        cudaError_t e_ = (x);                                                                             \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_)); \
    } while (0)

// uniform in [0, 1) from a 64-bit counter: splitmix64's finaliser (Steele, Lea and Flood 2014)
__host__ __device__ inline double sa_uniform(uint64_t seed, uint64_t inst, uint64_t restart, uint64_t sweep,
                                             uint64_t spin, uint64_t sweeps, uint64_t n) {
    uint64_t x = seed + 0x9E3779B97F4A7C15ull * ((((inst * 0x100000001B3ull + restart) * (sweeps + 1) + sweep) * n +
                                                  spin) + 1);
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x ^= x >> 31;
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

struct SaTask {
    int n;
    int hoff;  // first field / spin of this instance
    int eoff;  // first edge of this instance
    int m;     // its edges (self-loops included: they enter the energy)
};

__global__ void __launch_bounds__(SA_THREADS) k_sa(const SaTask* tasks, const int* adj_off, const int* adj_nbr,
                                                   const double* adj_w, const double* h, const int* ei, const int* ej,
                                                   const double* ew, int restarts, int sweeps, double t0,
                                                   double t_end, unsigned long long seed, double* out_e,
                                                   int8_t* out_s) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const SaTask tk = tasks[blockIdx.x];
    const int n = tk.n, a0 = adj_off[tk.hoff], deg_tot = adj_off[tk.hoff + n] - a0;
    double* sw = reinterpret_cast<double*>(smraw);     // [deg_tot] weights
    double* sh = sw + deg_tot;                         // [n] fields
    int* so = reinterpret_cast<int*>(sh + n);          // [n + 1] offsets
    short* sn = reinterpret_cast<short*>(so + n + 1);  // [deg_tot] neighbours
    __shared__ double s_best[SA_THREADS];
    __shared__ int s_arg[SA_THREADS];
    __shared__ unsigned long long s_bits[SA_THREADS][SA_WORDS];
    for (int e = threadIdx.x; e < deg_tot; e += blockDim.x) {
        sw[e] = adj_w[a0 + e];
        sn[e] = (short)adj_nbr[a0 + e];
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) sh[i] = h[tk.hoff + i];
    for (int i = threadIdx.x; i <= n; i += blockDim.x) so[i] = adj_off[tk.hoff + i] - a0;
    __syncthreads();
    const double ratio = t_end / t0;
    const double den = (double)((sweeps < 2 ? 2 : sweeps) - 1);
    double best = INFINITY;
    int best_r = -1;
    unsigned long long best_bits[SA_WORDS] = {};
    for (int r0 = 0; r0 < restarts; r0 += blockDim.x) {
        const int r = r0 + threadIdx.x;
        if (r >= restarts) break;
        unsigned long long bits[SA_WORDS] = {};
        for (int i = 0; i < n; ++i)  // random start: s_i = -1 with probability 1/2
            if (sa_uniform(seed, blockIdx.x, r, sweeps, i, sweeps, n) < 0.5) bits[i >> 6] |= 1ull << (i & 63);
        for (int k = 0; k < sweeps; ++k) {
            const double t = t0 * pow(ratio, (double)k / den);
            for (int i = 0; i < n; ++i) {
                double f = sh[i];
                for (int e = so[i]; e < so[i + 1]; ++e) {
                    const int j = sn[e];
                    f += ((bits[j >> 6] >> (j & 63)) & 1ull) ? -sw[e] : sw[e];
                }
                const bool neg = (bits[i >> 6] >> (i & 63)) & 1ull;
                const double de = 2.0 * (neg ? -f : f);
                if (de < 0.0 || sa_uniform(seed, blockIdx.x, r, k, i, sweeps, n) < exp(-de / t))
                    bits[i >> 6] ^= 1ull << (i & 63);
            }
        }
        double en = 0.0;  // E = -sum w s_i s_j - sum h s_i, in the order of the edge list
        for (int e = 0; e < tk.m; ++e) {
            const int i = ei[tk.eoff + e], j = ej[tk.eoff + e];
            const bool si = (bits[i >> 6] >> (i & 63)) & 1ull, sj = (bits[j >> 6] >> (j & 63)) & 1ull;
            en -= (si == sj) ? ew[tk.eoff + e] : -ew[tk.eoff + e];
        }
        for (int i = 0; i < n; ++i) en -= ((bits[i >> 6] >> (i & 63)) & 1ull) ? -sh[i] : sh[i];
        if (en < best) {
            best = en;
            best_r = r;
            for (int w = 0; w < SA_WORDS; ++w) best_bits[w] = bits[w];
        }
    }
    s_best[threadIdx.x] = best;
    s_arg[threadIdx.x] = best_r;
    for (int w = 0; w < SA_WORDS; ++w) s_bits[threadIdx.x][w] = best_bits[w];
    __syncthreads();
    if (threadIdx.x == 0) {
        int bt = 0;
        for (int t = 1; t < (int)blockDim.x; ++t) {
            if (s_arg[t] < 0) continue;
            if (s_best[t] < s_best[bt] || (s_best[t] == s_best[bt] && s_arg[t] < s_arg[bt])) bt = t;
        }
        out_e[blockIdx.x] = s_best[bt];
        for (int i = 0; i < n; ++i) out_s[tk.hoff + i] = ((s_bits[bt][i >> 6] >> (i & 63)) & 1ull) ? -1 : 1;
    }
}

void set_last_error(const std::string& msg);  // engine.cu: the message tessera_qa_last_error() returns

}  // namespace tq

using namespace tq;

extern "C" int tessera_qa_sa_solve(const tessera_qa_problem* problems, size_t count, size_t restarts,
                                   size_t sweeps, double t0, double t_end, uint64_t seed, int8_t* out_spins,
                                   double* out_energy) {
    char* arena = nullptr;
    cudaStream_t st = nullptr;
    auto release = [&]() {
        if (st) cudaStreamSynchronize(st);
        if (arena) cudaFree(arena);
        if (st) cudaStreamDestroy(st);
        arena = nullptr;
        st = nullptr;
    };
    try {
        if (!problems || count == 0 || !out_spins || !out_energy)
            throw std::invalid_argument("problems, out_spins and out_energy must be non-NULL, count >= 1");
        if (count > (1u << 20) || restarts < 1 || restarts > (1u << 20) || sweeps < 1 || sweeps > (1u << 24))
            throw std::invalid_argument("count and restarts in 1..2^20, sweeps in 1..2^24");
        if (!(t0 > 0.0) || !(t_end > 0.0) || !std::isfinite(t0) || !std::isfinite(t_end))
            throw std::invalid_argument("temperatures must be positive and finite");
        // every instance's spins are numbered from hoff; adj_off holds one offset per spin into
        // the concatenated neighbour lists, plus a final one.  The energy keeps the edge list as
        // given (self-loops included, as Ising::energy does); the dynamics skip self-loops,
        // which only add a constant.
        std::vector<SaTask> tasks(count);
        std::vector<int> adj_off, nbr, ei, ej;
        std::vector<double> w, h, ew;
        size_t smem = 0;
        for (size_t b = 0; b < count; ++b) {
            const tessera_qa_problem& p = problems[b];
            if (p.n < 1 || p.n > (size_t)SA_MAXN || !p.h || (p.m && (!p.ei || !p.ej || !p.ew)))
                throw std::invalid_argument("instance " + std::to_string(b) + ": need 1 <= n <= " +
                                            std::to_string(SA_MAXN) + " and non-NULL arrays");
            const int n = (int)p.n;
            std::vector<std::vector<std::pair<int, double>>> adj(n);
            for (int i = 0; i < n; ++i)
                if (!std::isfinite(p.h[i])) throw std::invalid_argument("non-finite field");
            SaTask t{n, (int)h.size(), (int)ei.size(), (int)p.m};
            for (size_t e = 0; e < p.m; ++e) {
                const size_t i = p.ei[e], j = p.ej[e];
                if (i >= p.n || j >= p.n || !std::isfinite(p.ew[e]))
                    throw std::invalid_argument("edge index out of range or non-finite coupling");
                ei.push_back((int)i);
                ej.push_back((int)j);
                ew.push_back(p.ew[e]);
                if (i == j) continue;
                adj[i].push_back({(int)j, p.ew[e]});
                adj[j].push_back({(int)i, p.ew[e]});
            }
            size_t deg = 0;
            for (int i = 0; i < n; ++i) {
                h.push_back(p.h[i]);
                adj_off.push_back((int)nbr.size());
                for (auto& pr : adj[i]) {
                    nbr.push_back(pr.first);
                    w.push_back(pr.second);
                }
                deg += adj[i].size();
            }
            tasks[b] = t;
            smem = std::max(smem, deg * (sizeof(double) + sizeof(short)) + n * sizeof(double) +
                                      (n + 1) * sizeof(int) + 64);
        }
        adj_off.push_back((int)nbr.size());
        if (smem > 200 * 1024) throw std::invalid_argument("instance graph too large for shared memory");
        auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
        const size_t b_tasks = al(sizeof(SaTask) * count), b_off = al(sizeof(int) * adj_off.size()),
                     b_nbr = al(sizeof(int) * std::max<size_t>(nbr.size(), 1)),
                     b_w = al(sizeof(double) * std::max<size_t>(w.size(), 1)), b_h = al(sizeof(double) * h.size()),
                     b_ei = al(sizeof(int) * std::max<size_t>(ei.size(), 1)),
                     b_ew = al(sizeof(double) * std::max<size_t>(ew.size(), 1)), b_e = al(sizeof(double) * count),
                     b_s = al(h.size());
        const size_t total = b_tasks + b_off + b_nbr + b_w + b_h + 2 * b_ei + b_ew + b_e + b_s;
        SA_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        SA_CK(device_alloc((void**)&arena, total));
        char* q = arena;
        auto take = [&](size_t bytes) { char* r = q; q += bytes; return r; };
        SaTask* d_tasks = (SaTask*)take(b_tasks);
        int* d_off = (int*)take(b_off);
        int* d_nbr = (int*)take(b_nbr);
        double* d_w = (double*)take(b_w);
        double* d_h = (double*)take(b_h);
        int* d_ei = (int*)take(b_ei);
        int* d_ej = (int*)take(b_ei);
        double* d_ew = (double*)take(b_ew);
        double* d_e = (double*)take(b_e);
        int8_t* d_s = (int8_t*)take(b_s);
        auto up = [&](void* d, const void* hsrc, size_t bytes) {
            if (bytes) SA_CK(cudaMemcpyAsync(d, hsrc, bytes, cudaMemcpyHostToDevice, st));
        };
        up(d_tasks, tasks.data(), sizeof(SaTask) * count);
        up(d_off, adj_off.data(), sizeof(int) * adj_off.size());
        up(d_nbr, nbr.data(), sizeof(int) * nbr.size());
        up(d_w, w.data(), sizeof(double) * w.size());
        up(d_h, h.data(), sizeof(double) * h.size());
        up(d_ei, ei.data(), sizeof(int) * ei.size());
        up(d_ej, ej.data(), sizeof(int) * ej.size());
        up(d_ew, ew.data(), sizeof(double) * ew.size());
        SA_CK(cudaFuncSetAttribute(k_sa, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const int threads = (int)std::min<size_t>(restarts, SA_THREADS);
        k_sa<<<(unsigned)count, threads, smem, st>>>(d_tasks, d_off, d_nbr, d_w, d_h, d_ei, d_ej, d_ew,
                                                     (int)restarts, (int)sweeps, t0, t_end, seed, d_e, d_s);
        SA_CK(cudaGetLastError());
        std::vector<double> e(count);
        std::vector<int8_t> s(h.size());
        SA_CK(cudaMemcpyAsync(e.data(), d_e, sizeof(double) * count, cudaMemcpyDeviceToHost, st));
        SA_CK(cudaMemcpyAsync(s.data(), d_s, h.size(), cudaMemcpyDeviceToHost, st));
        SA_CK(cudaStreamSynchronize(st));
        release();
        for (size_t b = 0; b < count; ++b) out_energy[b] = e[b];
        std::copy(s.begin(), s.end(), out_spins);
        return 0;
    } catch (const std::invalid_argument& ex) {
        set_last_error(ex.what());
        release();
        return TESSERA_QA_EINVAL;
    } catch (const std::exception& ex) {
        set_last_error(ex.what());
        release();
        return TESSERA_QA_ECUDA;
    }
}
