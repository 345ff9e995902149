// engine.cu -- host orchestration of the anneal and the C ABI of libtessera_qa.so.
//
// One Engine<T> owns one instance's device state (a single cudaMalloc arena) and a CUDA
// stream.  A Trotter step (cuda/src/mps.cpp:309-356) is enqueued without any host wait:
//   K5 single-site half step (all sites, one launch)
//   for every ZZ gate of the step, in the reference's order, expanded through the swap
//   network (cuda/src/mps.cpp:126-145, 330-341): K1 theta -> K2/K3 Jacobi SVD + keep rule
//   -> K4 absorb
//   K5 single-site half step
//   K6 right-environment chain to bond 1 + qubit-0 entropy
// Bond dimensions live on the device; the host only tracks upper bounds
// (dim_{i+1} <= min(chi, 2 dim_i, 2 dim_{i+2})) to size the grids.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tessera_qa.h"
#include "engine.cuh"

namespace tq {

#define TQ_CK(x)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            throw CudaError(std::string("CUDA: ") + cudaGetErrorString(e_) + " (" #x ")");      \
    } while (0)

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct ArgError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

static thread_local std::string t_err;

static void set_err(const std::string& s) { t_err = s; }

// Allocation-failure injection (tessera_qa_debug_fail_allocations): allocations that still
// succeed first, then allocations that fail.
static std::mutex g_fail_mu;
static int g_fail_after = 0, g_fail_count = 0;

cudaError_t device_alloc(void** p, size_t bytes) {
    {
        std::lock_guard<std::mutex> lk(g_fail_mu);
        if (g_fail_count > 0) {
            if (g_fail_after > 0) {
                --g_fail_after;
            } else {
                --g_fail_count;
                *p = nullptr;
                return cudaErrorMemoryAllocation;
            }
        }
    }
    return cudaMalloc(p, bytes);
}
void set_last_error(const std::string& msg) { t_err = msg; }

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// ---------------------------------------------------------------------------------
// small kernels local to the orchestrator
// ---------------------------------------------------------------------------------
__global__ void k_set_int(int* p, int v) { *p = v; }

template <typename T>
__global__ void k_random_sites(MpsView<T> mps, unsigned long long seed, double decay) {
    using V = cplx_t<T>;
    const int i = blockIdx.y;
    const int dl = mps.dims[i], dr = mps.dims[i + 1];
    const long long tot = (long long)dl * 2 * dr;
    const double scale = 1.0 / sqrt(2.0 * dl);
    V* S = mps.site(i);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const long long row = t / dr, b = t - row * dr;
        unsigned long long z = seed ^ ((unsigned long long)i << 40) ^ (unsigned long long)t * 0x9E3779B97F4A7C15ull;
        // splitmix64, twice
        unsigned long long u[2];
        for (int q = 0; q < 2; ++q) {
            z += 0x9E3779B97F4A7C15ull;
            unsigned long long x = z;
            x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
            x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
            u[q] = x ^ (x >> 31);
        }
        const double u1 = ((u[0] >> 11) + 0.5) * (1.0 / 9007199254740992.0);
        const double u2 = (u[1] >> 11) * (1.0 / 9007199254740992.0);
        // decay > 0: column b of every site scaled by exp(-b / decay), so that theta's singular
        // values fall off like a TEBD state's Schmidt values instead of staying flat
        const double r = sqrt(-2.0 * log(u1)) * scale * (decay > 0.0 ? exp(-(double)b / decay) : 1.0);
        S[row * mps.cap + b] = mk<V>((T)(r * cos(6.283185307179586 * u2)), (T)(r * sin(6.283185307179586 * u2)));
    }
}

// ---------------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------------
struct ProblemHost {
    int n = 0, m = 0, steps = 0;
    std::vector<double> h, w, sa, sb;
    std::vector<int> ei, ej;
    std::vector<double> bias, sc;  // empty = no warm-start bias
};

static ProblemHost validate_problem(const tessera_qa_problem* p) {
    if (!p) throw ArgError("problem is NULL");
    if (p->n == 0) throw ArgError("n must be >= 1");
    if (p->n > 4096) throw ArgError("n > 4096 is not supported");
    if (!p->h) throw ArgError("h is NULL");
    if (p->m && (!p->ei || !p->ej || !p->ew)) throw ArgError("edge arrays are NULL");
    if (p->steps && (!p->schedule_a || !p->schedule_b)) throw ArgError("schedule arrays are NULL");
    ProblemHost P;
    P.n = (int)p->n;
    P.m = (int)p->m;
    P.steps = (int)p->steps;
    P.h.assign(p->h, p->h + p->n);
    for (double x : P.h)
        if (!std::isfinite(x)) throw ArgError("h contains NaN/Inf");
    for (size_t e = 0; e < p->m; ++e) {
        if (p->ei[e] >= p->n || p->ej[e] >= p->n) throw ArgError("edge index out of range");
        if (!std::isfinite(p->ew[e])) throw ArgError("ew contains NaN/Inf");
        P.ei.push_back((int)p->ei[e]);
        P.ej.push_back((int)p->ej[e]);
        P.w.push_back(p->ew[e]);
    }
    P.sa.assign(p->schedule_a, p->schedule_a + p->steps);
    P.sb.assign(p->schedule_b, p->schedule_b + p->steps);
    for (size_t k = 0; k < p->steps; ++k)
        if (!std::isfinite(P.sa[k]) || !std::isfinite(P.sb[k])) throw ArgError("schedule contains NaN/Inf");
    if ((p->bias == nullptr) != (p->schedule_c == nullptr)) throw ArgError("bias and schedule_c go together");
    if (p->bias) {
        P.bias.assign(p->bias, p->bias + p->n);
        P.sc.assign(p->schedule_c, p->schedule_c + p->steps);
        for (double x : P.bias)
            if (!std::isfinite(x)) throw ArgError("bias contains NaN/Inf");
        for (double x : P.sc)
            if (!std::isfinite(x)) throw ArgError("schedule_c contains NaN/Inf");
    }
    return P;
}

struct Config {
    double dt = 0.1;
    int ns = 1;
    int precision = TESSERA_QA_C128;
    int chi = 32;
    double tol = 0.0;
    int max_sweeps = 60;
    int block = 0;
    int device = -1;
    int min_ld = 0;  // workspace rows/cols at least this (standalone SVD)
    int timing = 0;  // time each SVD launch with CUDA events
    int theta_tc = 0;  // complex64: bond contraction on tcgen05 tensor cores (split-TF32)
    int precond = 0;   // batched column-pair Jacobi: 0 default (on), 1 on, 2 off (pivoted LQ first)
};

static Config validate_config(const tessera_qa_config* c) {
    Config C;
    if (!c) return C;
    if (!(c->dt > 0) || !std::isfinite(c->dt)) throw ArgError("dt must be a finite positive number");
    if (c->chi == 0) throw ArgError("chi must be >= 1");
    if (c->chi > 1024) throw ArgError("chi > 1024 is not supported");
    if (c->precision != TESSERA_QA_C128 && c->precision != TESSERA_QA_C64) throw ArgError("unknown precision");
    if (c->jacobi_block && !(c->jacobi_block == 1 || c->jacobi_block == 2 || c->jacobi_block == 4 ||
                             c->jacobi_block == 8 || c->jacobi_block == 16 || c->jacobi_block == 32))
        throw ArgError("jacobi_block must be 0, 1, 2, 4, 8, 16 or 32 (32: block-Gram Jacobi, batches only)");
    if (c->jacobi_max_sweeps < 0 || c->jacobi_max_sweeps > 1000) throw ArgError("jacobi_max_sweeps out of range");
    if (c->jacobi_precondition < 0 || c->jacobi_precondition > 2) throw ArgError("jacobi_precondition must be 0, 1 or 2");
    C.dt = c->dt;
    C.ns = c->zz_substeps < 1 ? 1 : c->zz_substeps;
    C.precision = c->precision;
    C.chi = (int)c->chi;
    C.tol = c->jacobi_tol;
    C.max_sweeps = c->jacobi_max_sweeps ? c->jacobi_max_sweeps : 60;
    C.block = c->jacobi_block;
    C.device = c->device;
    C.timing = c->kernel_timing;
    C.theta_tc = c->theta_tensor_cores;
    C.precond = c->jacobi_precondition;
    if (C.theta_tc && c->precision != TESSERA_QA_C64)
        throw ArgError("theta_tensor_cores needs complex64 precision");
    return C;
}

class EngineBase {
public:
    virtual ~EngineBase() = default;
    virtual void init_plus() = 0;
    virtual void randomize(unsigned long long seed, double decay) = 0;
    virtual void run(int k0, int k1) = 0;
    // gates [q0, q1) of the ZZ block of step k only (no single-site half steps, no entropy)
    virtual void run_gates(int k, int q0, int q1) = 0;
    // new values of h, J, A(s), B(s) for the same n, edges and number of steps
    virtual void set_values(const ProblemHost& P) = 0;
    virtual void sync_stats(tessera_qa_result* r) = 0;
    virtual void observe(tessera_qa_result* r) = 0;
    virtual void sample(size_t count, unsigned long long seed, int8_t* spins, double* energies) = 0;
    virtual size_t save(void* buf, size_t bytes, unsigned long long step_next) = 0;
    virtual void load(const void* buf, size_t bytes) = 0;
    virtual void copy_entropy(double* out, int k0, int k1) = 0;
    virtual cudaStream_t stream() const = 0;
    virtual double last_ms() const = 0;
};

// checkpoint layout: "TQMPSv1\0", u32 n, u32 0, u64 step_next, u64 0, i32 dims[n+1] (8-byte padded),
// then site tensors (Dl, 2, Dr) as complex128, (a, s, b) row-major.
static const char kMagic[8] = {'T', 'Q', 'M', 'P', 'S', 'v', '1', 0};
static size_t ckpt_header_bytes(int n) { return 32 + ((size_t)4 * (n + 1) + 7) / 8 * 8; }

template <typename T>
class Engine final : public EngineBase {
    using V = cplx_t<T>;

public:
    Engine(const ProblemHost& P, const Config& C) : P_(P), C_(C) {
        n_ = P.n;
        m_ = P.m;
        // bond cap: min(chi, 2^floor(n/2)), the largest bond any n-site chain can need
        long long full = 1;
        for (int q = 0; q < n_ / 2 && full < C.chi; ++q) full <<= 1;
        cap_ = (int)std::min<long long>(C.chi, full);
        if (cap_ < 1) cap_ = 1;
        ld_ = std::max(2 * cap_, (C.min_ld + 7) & ~7);
        try {  // a failed allocation or CUDA call releases what was made before it
            build_ops();
            allocate();
            TQ_CK(cudaEventCreate(&ev0_));
            TQ_CK(cudaEventCreate(&ev1_));
            upload_problem();
            init_plus();
        } catch (...) {
            release();
            throw;
        }
    }
    ~Engine() override { release(); }
    void release() noexcept {
        if (stream_) cudaStreamSynchronize(stream_);
        for (cudaEvent_t e : pool_) cudaEventDestroy(e);
        if (ev0_) cudaEventDestroy(ev0_);
        if (ev1_) cudaEventDestroy(ev1_);
        if (base_) cudaFree(base_);
        if (res_base_) cudaFree(res_base_);
        if (obs_) cudaFree(obs_);
        if (stream_) cudaStreamDestroy(stream_);
        pool_.clear();
        ev0_ = ev1_ = nullptr;
        base_ = res_base_ = nullptr;
        obs_ = nullptr;
        stream_ = nullptr;
    }

    cudaStream_t stream() const override { return stream_; }
    double last_ms() const override { return last_ms_; }

    void init_plus() override {
        launch_init_plus<T>(mps(), stream_);
        TQ_CK(cudaMemsetAsync(stats_, 0, sizeof(RunStats), stream_));
        std::fill(ub_.begin(), ub_.end(), 1);
    }

    void randomize(unsigned long long seed, double decay) override {
        std::vector<int> d(n_ + 1, 1);
        for (int i = 1; i < n_; ++i) {
            long long a = 1, b = 1;
            for (int q = 0; q < i && a < cap_; ++q) a <<= 1;
            for (int q = 0; q < n_ - i && b < cap_; ++q) b <<= 1;
            d[i] = (int)std::min<long long>(cap_, std::min(a, b));
        }
        TQ_CK(cudaMemcpyAsync(dims_, d.data(), sizeof(int) * (n_ + 1), cudaMemcpyHostToDevice, stream_));
        TQ_CK(cudaStreamSynchronize(stream_));
        k_random_sites<T><<<dim3(64, n_), 256, 0, stream_>>>(mps(), seed, decay);
        TQ_CK(cudaGetLastError());
        TQ_CK(cudaMemsetAsync(stats_, 0, sizeof(RunStats), stream_));
        ub_ = d;
    }

    void run(int k0, int k1) override {
        if (k0 < 0 || k1 > P_.steps || k0 > k1) throw ArgError("step range outside the schedule");
        k_set_int<<<1, 1, 0, stream_>>>(step_, k0);
        TQ_CK(cudaGetLastError());
        TQ_CK(cudaEventRecord(ev0_, stream_));
        // small bonds (theta fits one CTA's shared memory): the whole run is one launch of the
        // resident anneal kernel, the same code a batch runs for each of its instances; the
        // per-update path stays for large bonds, explicit Jacobi block widths and SVD timing
        if (k1 > k0 && C_.block == 0 && !C_.timing && !C_.theta_tc && n_ >= 1) {
            const int rc = std::max(8, (2 * cap_ + 7) & ~7);
            ensure_resident(rc);
            if (launch_anneal_resident<T>(res_inst_, res_ops_, res_off_, res_order_, 1, k0, k1, res_work_, rc,
                                          stream_)) {
                k_set_int<<<1, 1, 0, stream_>>>(step_, k1);
                TQ_CK(cudaGetLastError());
                launches_ += 2;
                svd_launches_ += 1;
                TQ_CK(cudaEventRecord(ev1_, stream_));
                ran_ = true;
                return;
            }
        }
        const ScheduleView sch = schedule();
        const MpsView<T> M = mps();
        for (int k = k0; k < k1; ++k) {
            single_site(sch);
            for (const GateOp& op : ops_) two_site(M, sch, op);
            single_site(sch);
            entropy_step(M);
            launch_step_inc(step_, stream_);
            launches_ += 5;  // two single-site, entropy chain, entropy, step counter
        }
        TQ_CK(cudaEventRecord(ev1_, stream_));
        ran_ = true;
    }

    void run_gates(int k, int q0, int q1) override {
        if (k < 0 || k >= P_.steps || q0 < 0 || q1 > (int)ops_.size() || q0 > q1)
            throw ArgError("gate range outside the step");
        k_set_int<<<1, 1, 0, stream_>>>(step_, k);
        TQ_CK(cudaGetLastError());
        TQ_CK(cudaEventRecord(ev0_, stream_));
        const ScheduleView sch = schedule();
        const MpsView<T> M = mps();
        for (int q = q0; q < q1; ++q) two_site(M, sch, ops_[q]);
        TQ_CK(cudaEventRecord(ev1_, stream_));
        ran_ = true;
    }

    void set_values(const ProblemHost& P) override {
        if (P.n != n_ || P.m != m_ || P.steps != P_.steps || P.ei != P_.ei || P.ej != P_.ej)
            throw ArgError("set_values needs the same n, edges and number of steps");
        P_.h = P.h;
        P_.w = P.w;
        P_.sa = P.sa;
        P_.sb = P.sb;
        P_.bias = P.bias;
        P_.sc = P.sc;
        upload_problem();
    }

    void sync_stats(tessera_qa_result* r) override {
        TQ_CK(cudaStreamSynchronize(stream_));
        TQ_CK(cudaGetLastError());
        RunStats st;
        TQ_CK(cudaMemcpy(&st, stats_, sizeof(st), cudaMemcpyDeviceToHost));
        if (ran_) {
            float ms = 0;
            TQ_CK(cudaEventElapsedTime(&ms, ev0_, ev1_));
            last_ms_ = ms;
        }
        for (auto& pr : timed_) {
            float ms = 0;
            TQ_CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
            svd_ms_ += ms;
        }
        timed_.clear();
        for (auto& pr : timed_lq_) {
            float ms = 0;
            TQ_CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
            lq_ms_ += ms;
        }
        timed_lq_.clear();
        pool_next_ = 0;
        if (r) {
            r->svd_ms = svd_ms_;
            r->precond_ms = lq_ms_;
            r->svd_bytes = st.svd_bytes;
            r->svd_flops = st.svd_flops;
            r->svd_launches = svd_launches_;
            r->svd_sweeps = st.svd_sweeps;
            r->kernel_launches = launches_;
            r->max_trunc = st.max_trunc;
            r->two_site_updates = st.updates;
            r->status = st.status;
            r->max_sweeps = st.max_sweeps;
            r->max_bond = std::max(st.max_bond, 1);
            r->device_ms = last_ms_;
            r->min_cut_gap = 1.0 - st.gap_deficit;
        }
    }

    void copy_entropy(double* out, int k0, int k1) override {
        if (!out || k1 <= k0) return;
        TQ_CK(cudaMemcpyAsync(out, entropy_ + k0, sizeof(double) * (k1 - k0), cudaMemcpyDeviceToHost, stream_));
        TQ_CK(cudaStreamSynchronize(stream_));
    }

    // <Z_i>, <Z_i Z_j>, <psi|psi>, readout, prob (cuda/src/mps.cpp:358-380).
    void observe(tessera_qa_result* r) override {
        const MpsView<T> M = mps();
        if (!obs_) {  // environments for the final observables, allocated on first use
            const size_t bytes = sizeof(V) * (size_t)cap_ * cap_ * obs_units_;
            TQ_CK(device_alloc((void**)&obs_, bytes));
            TQ_CK(cudaMemsetAsync(obs_, 0, sizeof(V), stream_));
            V one = mk<V>(1, 0);
            TQ_CK(cudaMemcpyAsync(obs_, &one, sizeof(V), cudaMemcpyHostToDevice, stream_));
        }
        launch_chain<T>(M, 1, obsR_, n_, obs_, xs_, bar_, stats_, cap_, stream_);
        launch_chain<T>(M, 0, obsL_, n_obsL_, obs_, xs_, bar_, stats_, cap_, stream_);
        launch_pair_dots<T>(M, obs_, dots_, 1 + n_ + m_, dotout_, stream_);
        std::vector<double> v(1 + n_ + m_);
        TQ_CK(cudaMemcpyAsync(v.data(), dotout_, sizeof(double) * v.size(), cudaMemcpyDeviceToHost, stream_));
        TQ_CK(cudaStreamSynchronize(stream_));
        const double nrm = v[0];
        std::vector<double> ez(n_), ezz(m_);
        for (int i = 0; i < n_; ++i) ez[i] = nrm > 0 ? v[1 + i] / nrm : 0.0;
        for (int e = 0; e < m_; ++e) ezz[e] = nrm > 0 ? v[1 + n_ + e] / nrm : 0.0;
        double eexp = 0.0;
        for (int e = 0; e < m_; ++e) eexp -= P_.w[e] * ezz[e];
        for (int i = 0; i < n_; ++i) eexp -= P_.h[i] * ez[i];
        std::vector<int8_t> spins(n_);
        for (int i = 0; i < n_; ++i) spins[i] = ez[i] >= 0.0 ? 1 : -1;
        double E = 0.0;
        for (int e = 0; e < m_; ++e) E -= P_.w[e] * spins[P_.ei[e]] * spins[P_.ej[e]];
        for (int i = 0; i < n_; ++i) E -= P_.h[i] * spins[i];
        TQ_CK(cudaMemcpyAsync(spins_d_, spins.data(), n_, cudaMemcpyHostToDevice, stream_));
        launch_amplitude<T>(M, spins_d_, vbuf_, amp2_, stream_);
        double a2 = 0;
        TQ_CK(cudaMemcpyAsync(&a2, amp2_, sizeof(double), cudaMemcpyDeviceToHost, stream_));
        TQ_CK(cudaStreamSynchronize(stream_));
        if (r) {
            r->energy = E;
            r->expected_energy = eexp;
            r->prob = nrm > 0 ? a2 / nrm : 0.0;
            r->norm2 = nrm;
            if (r->spins) std::memcpy(r->spins, spins.data(), n_);
            if (r->z_expect) std::memcpy(r->z_expect, ez.data(), sizeof(double) * n_);
        }
    }

    // `count` basis patterns drawn from |<x|psi>|^2 (K9), their Ising energies on the host
    void sample(size_t count, unsigned long long seed, int8_t* spins, double* energies) override {
        if (count == 0) return;
        if (count > (size_t)1 << 24) throw ArgError("at most 2^24 samples per call");
        const MpsView<T> M = mps();
        if (!obs_) {
            const size_t bytes = sizeof(V) * (size_t)cap_ * cap_ * obs_units_;
            TQ_CK(device_alloc((void**)&obs_, bytes));
            V one = mk<V>(1, 0);
            TQ_CK(cudaMemcpyAsync(obs_, &one, sizeof(V), cudaMemcpyHostToDevice, stream_));
        }
        launch_chain<T>(M, 1, obsR_, n_, obs_, xs_, bar_, stats_, cap_, stream_);
        int8_t* d = nullptr;
        TQ_CK(device_alloc((void**)&d, count * (size_t)n_));
        cudaError_t err = cudaSuccess;
        try {
            launch_sample<T>(M, obs_, (int)count, seed, d, stream_);
        } catch (...) {
            cudaFree(d);
            throw;
        }
        err = cudaMemcpyAsync(spins, d, count * (size_t)n_, cudaMemcpyDeviceToHost, stream_);
        if (err == cudaSuccess) err = cudaStreamSynchronize(stream_);
        cudaFree(d);
        TQ_CK(err);
        if (energies)
            for (size_t c = 0; c < count; ++c) {
                const int8_t* x = spins + c * n_;
                double e = 0.0;
                for (int q = 0; q < m_; ++q) e -= P_.w[q] * x[P_.ei[q]] * x[P_.ej[q]];
                for (int i = 0; i < n_; ++i) e -= P_.h[i] * x[i];
                energies[c] = e;
            }
    }

    size_t save(void* buf, size_t bytes, unsigned long long step_next) override {
        TQ_CK(cudaStreamSynchronize(stream_));
        std::vector<int> d(n_ + 1);
        TQ_CK(cudaMemcpy(d.data(), dims_, sizeof(int) * (n_ + 1), cudaMemcpyDeviceToHost));
        size_t need = ckpt_header_bytes(n_);
        for (int i = 0; i < n_; ++i) need += (size_t)d[i] * 2 * d[i + 1] * 16;
        if (!buf || bytes < need) throw ArgError("checkpoint buffer too small");
        char* p = static_cast<char*>(buf);
        std::memset(p, 0, ckpt_header_bytes(n_));
        std::memcpy(p, kMagic, 8);
        const uint32_t nn = (uint32_t)n_;
        std::memcpy(p + 8, &nn, 4);
        std::memcpy(p + 16, &step_next, 8);
        std::memcpy(p + 32, d.data(), sizeof(int) * (n_ + 1));
        char* q = p + ckpt_header_bytes(n_);
        std::vector<V> tmp;
        for (int i = 0; i < n_; ++i) {
            const size_t rows = (size_t)2 * d[i], cols = d[i + 1];
            tmp.resize(rows * cols);
            TQ_CK(cudaMemcpy2D(tmp.data(), cols * sizeof(V), sites_ + (size_t)i * site_stride(), cap_ * sizeof(V),
                               cols * sizeof(V), rows, cudaMemcpyDeviceToHost));
            double* o = reinterpret_cast<double*>(q);
            for (size_t e = 0; e < rows * cols; ++e) {
                const double re = (double)tmp[e].x, im = (double)tmp[e].y;
                std::memcpy(o + 2 * e, &re, 8);
                std::memcpy(o + 2 * e + 1, &im, 8);
            }
            q += rows * cols * 16;
        }
        return need;
    }

    void load(const void* buf, size_t bytes) override {
        const char* p = static_cast<const char*>(buf);
        if (!p || bytes < 32 || std::memcmp(p, kMagic, 8) != 0) throw ArgError("not a tessera_qa checkpoint");
        uint32_t nn;
        std::memcpy(&nn, p + 8, 4);
        if ((int)nn != n_) throw ArgError("checkpoint has a different number of sites");
        if (bytes < ckpt_header_bytes(n_)) throw ArgError("checkpoint truncated");
        std::vector<int> d(n_ + 1);
        std::memcpy(d.data(), p + 32, sizeof(int) * (n_ + 1));
        if (d[0] != 1 || d[n_] != 1) throw ArgError("checkpoint end bonds must be 1");
        size_t need = ckpt_header_bytes(n_);
        for (int i = 0; i <= n_; ++i)
            if (d[i] < 1 || d[i] > cap_) throw ArgError("checkpoint bond dimension exceeds this run's cap");
        for (int i = 0; i < n_; ++i) need += (size_t)d[i] * 2 * d[i + 1] * 16;
        if (bytes < need) throw ArgError("checkpoint truncated");
        TQ_CK(cudaStreamSynchronize(stream_));
        TQ_CK(cudaMemcpy(dims_, d.data(), sizeof(int) * (n_ + 1), cudaMemcpyHostToDevice));
        const char* q = p + ckpt_header_bytes(n_);
        std::vector<V> tmp;
        for (int i = 0; i < n_; ++i) {
            const size_t rows = (size_t)2 * d[i], cols = d[i + 1];
            tmp.resize(rows * cols);
            const double* src = reinterpret_cast<const double*>(q);
            for (size_t e = 0; e < rows * cols; ++e) {
                double re, im;
                std::memcpy(&re, src + 2 * e, 8);
                std::memcpy(&im, src + 2 * e + 1, 8);
                tmp[e] = mk<V>((T)re, (T)im);
            }
            TQ_CK(cudaMemcpy2D(sites_ + (size_t)i * site_stride(), cap_ * sizeof(V), tmp.data(), cols * sizeof(V),
                               cols * sizeof(V), rows, cudaMemcpyHostToDevice));
            q += rows * cols * 16;
        }
        TQ_CK(cudaMemset(stats_, 0, sizeof(RunStats)));
        ub_ = d;
    }

    // standalone SVD of an R x N matrix (column-major in W) -> perm, sig
    void svd_only(const std::vector<V>& colmajor, int R, int N, std::vector<int>& perm, std::vector<double>& sig,
                  std::vector<V>& Wout) {
        TQ_CK(cudaMemcpy2DAsync(W_, ld_ * sizeof(V), colmajor.data(), R * sizeof(V), R * sizeof(V), N,
                                cudaMemcpyHostToDevice, stream_));
        const int bw = pick_block(R, N);
        launch_svd<T>(mps(), 0, std::min(R, N), tol_for(R), C_.max_sweeps, work(), R, N, bw, stream_, R, N);
        const int k = std::min(R, N);
        perm.resize(k);
        sig.resize(k);
        Wout.resize((size_t)R * N);
        TQ_CK(cudaMemcpyAsync(perm.data(), perm_, sizeof(int) * k, cudaMemcpyDeviceToHost, stream_));
        TQ_CK(cudaMemcpyAsync(sig.data(), sig_, sizeof(double) * k, cudaMemcpyDeviceToHost, stream_));
        TQ_CK(cudaMemcpy2DAsync(Wout.data(), R * sizeof(V), W_, ld_ * sizeof(V), R * sizeof(V), N,
                                cudaMemcpyDeviceToHost, stream_));
        TQ_CK(cudaStreamSynchronize(stream_));
        RunStats st;
        TQ_CK(cudaMemcpy(&st, stats_, sizeof(st), cudaMemcpyDeviceToHost));
        status_ = st.status;
    }
    int status_ = 0;
    int cap() const { return cap_; }
    int n() const { return n_; }
    const std::vector<GateOp>& ops() const { return ops_; }
    // Device views of this instance for the batched kernels; `step` is the batch's shared
    // step counter, `rows_cap` the batch-wide shared-memory column length.
    InstTask<T> inst_task(int* step, int rows_cap) const {
        InstTask<T> t;
        t.mps = mps();
        t.sch = schedule();
        t.sch.step = step;
        t.wk = work();
        t.pp.bond = 0;
        t.pp.R = 0;
        t.pp.N = 0;
        t.pp.no_trunc = 0;
        t.pp.chi = C_.chi;
        t.pp.tol = tol_for(2 * cap_);
        t.pp.tiny = sizeof(T) == 8 ? 1e-200 : 1e-60;
        t.pp.max_sweeps = C_.max_sweeps;
        t.pp.rows_cap = rows_cap;
        t.pp.cols_cap = rows_cap;  // theta is at most 2 cap x 2 cap
        t.pp.lq = 0;
        t.ent_steps = entc_;
        t.n_ent = n_ent_;
        t.pad = 0;
        t.envs = envs_;
        t.X = xs_;
        t.r1_off = r1_off_;
        t.entropy = entropy_;
        return t;
    }
    void reset_counters() { TQ_CK(cudaMemsetAsync(counters_, 0, sizeof(int) * C_.max_sweeps, stream_)); }
    void mark_ran(double ms) { ran_ = false; last_ms_ = ms; }
    int max_sweeps_cfg() const { return C_.max_sweeps; }
    int* counters_ptr() const { return counters_; }
    // device copies of this instance's task, gate list and work counter for the resident
    // anneal kernel (made on first use)
    void ensure_resident(int rows_cap) {
        if (res_base_) return;
        const size_t a1 = align256(sizeof(InstTask<T>));
        const size_t a2 = a1 + align256(sizeof(GateOp) * std::max<size_t>(ops_.size(), 1));
        TQ_CK(device_alloc((void**)&res_base_, a2 + 256));
        res_inst_ = reinterpret_cast<InstTask<T>*>(res_base_);
        res_ops_ = reinterpret_cast<GateOp*>(res_base_ + a1);
        res_off_ = reinterpret_cast<int*>(res_base_ + a2);
        res_order_ = res_off_ + 2;
        res_work_ = res_off_ + 4;
        const InstTask<T> t = inst_task(step_, rows_cap);
        const int hdr[4] = {0, (int)ops_.size(), 0, 0};
        TQ_CK(cudaMemcpyAsync(res_inst_, &t, sizeof(t), cudaMemcpyHostToDevice, stream_));
        if (!ops_.empty())
            TQ_CK(cudaMemcpyAsync(res_ops_, ops_.data(), sizeof(GateOp) * ops_.size(), cudaMemcpyHostToDevice,
                                  stream_));
        TQ_CK(cudaMemcpyAsync(res_off_, hdr, sizeof(hdr), cudaMemcpyHostToDevice, stream_));
        TQ_CK(cudaStreamSynchronize(stream_));
    }
    double* scal_ptr() const { return scal_; }
    cudaStream_t own_stream() const { return stream_; }

private:
    ProblemHost P_;
    Config C_;
    int n_ = 0, m_ = 0, cap_ = 1, ld_ = 2;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    char* base_ = nullptr;
    char* res_base_ = nullptr;
    InstTask<T>* res_inst_ = nullptr;
    GateOp* res_ops_ = nullptr;
    int *res_off_ = nullptr, *res_order_ = nullptr, *res_work_ = nullptr;
    V *sites_ = nullptr, *theta_ = nullptr, *W_ = nullptr, *envs_ = nullptr, *xs_ = nullptr, *vbuf_ = nullptr;
    void* lqc_ = nullptr;  // cooperative LQ candidate rows
    bool lq_ok_ = false;
    int *dims_ = nullptr, *perm_ = nullptr, *counters_ = nullptr, *step_ = nullptr;
    double* scal_ = nullptr;
    double *sig2_ = nullptr, *sig_ = nullptr, *h_ = nullptr, *w_ = nullptr, *sa_ = nullptr, *sb_ = nullptr;
    double *bias_ = nullptr, *sc_ = nullptr;
    double *entropy_ = nullptr, *dotout_ = nullptr, *amp2_ = nullptr;
    int8_t* spins_d_ = nullptr;
    GridBar* bar_ = nullptr;
    RunStats* stats_ = nullptr;
    ChainStep *entc_ = nullptr, *obsR_ = nullptr, *obsL_ = nullptr;
    PairDot* dots_ = nullptr;
    int n_ent_ = 0, n_obsL_ = 0;
    long long r1_off_ = 0;
    long long obs_units_ = 0;
    V* obs_ = nullptr;
    std::vector<GateOp> ops_;
    std::vector<int> ub_;
    bool ran_ = false;
    double last_ms_ = 0.0;
    long long launches_ = 0, svd_launches_ = 0;
    double svd_ms_ = 0.0, lq_ms_ = 0.0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timed_, timed_lq_;
    std::vector<cudaEvent_t> pool_;
    size_t pool_next_ = 0;

    size_t site_stride() const { return (size_t)2 * cap_ * cap_; }
    MpsView<T> mps() const { return MpsView<T>{sites_, dims_, n_, cap_, (long long)site_stride()}; }
    ScheduleView schedule() const {
        return ScheduleView{h_, w_, sa_, sb_, step_, C_.dt, C_.dt / C_.ns, bias_, sc_};
    }
    SvdWork<T> work() const { return SvdWork<T>{theta_, W_, ld_, sig2_, sig_, perm_, counters_, scal_, bar_, stats_}; }

    double tol_for(int R) const {
        if (C_.tol > 0) return C_.tol;
        const double eps = sizeof(T) == 8 ? 2.220446049250313e-16 : 1.1920928955078125e-07;
        // stop rotating a pair once |w_p^H w_q| <= tol |w_p||w_q|: 1e-13 in complex128 (a few
        // hundred ulps above the rounding floor of the FP64 dot products), 8 sqrt(R) ulps of
        // float in complex64 (whose dot products are accumulated in FP64)
        return sizeof(T) == 8 ? std::max(1e-13, 4.0 * std::sqrt((double)R) * eps)
                              : 8.0 * std::sqrt((double)std::max(R, 16)) * eps;
    }

    int pick_block(int R, int N) const {
        int b = std::min(C_.block, 16);  // a single instance has no block-Gram path
        if (!b) {
            // default schedule: wide blocks for small matrices (few grid barriers), narrower
            // ones for large matrices (enough block pairs to fill the SMs)
            if (N <= 64) b = 16;
            else if (N <= 256) b = 8;
            else b = 8;
        }
        const int rows_cap = (R + 7) & ~7;
        while (b > 1 && (size_t)2 * b * rows_cap * sizeof(V) > 200 * 1024) b >>= 1;
        return b;
    }

    void build_ops() {
        // ZZ block of one step (cuda/src/mps.cpp:330-341) expanded through the swap network
        // (cuda/src/mps.cpp:126-145).
        ops_.clear();
        for (int s = 0; s < C_.ns; ++s) {
            for (int q = 0; q < m_; ++q) {
                const int e = (s % 2 == 0) ? q : m_ - 1 - q;
                int i = P_.ei[e], j = P_.ej[e];
                if (i > j) std::swap(i, j);
                if (i == j) continue;
                for (int k = j; k > i + 1; --k) ops_.push_back(GateOp{k - 1, GATE_SWAP, e, 0});
                ops_.push_back(GateOp{i, GATE_ZZ, e, 0});
                for (int k = i + 1; k < j; ++k) ops_.push_back(GateOp{k, GATE_SWAP, e, 0});
            }
        }
        ub_.assign(n_ + 1, 1);
    }

    void allocate() {
        const size_t es = sizeof(V);
        const size_t unit = (size_t)cap_ * cap_;
        obs_units_ = 3 + 3LL * n_ + m_;  // observables: ONE, L_1..L_n, R_0..R_{n-1}, Z_i, ZZ_e, 2 temps
        // observable chain: L (n) + Z (n) + ZZ chains
        n_obsL_ = 2 * n_;
        for (int e = 0; e < m_; ++e) {
            const int i = std::min(P_.ei[e], P_.ej[e]), j = std::max(P_.ei[e], P_.ej[e]);
            if (i != j) n_obsL_ += j - i + 1;
        }
        n_ent_ = std::max(0, n_ - 1);
        struct Item { void** p; size_t bytes; };
        size_t off = 0;
        std::vector<std::pair<size_t, void**>> plan;
        auto add = [&](void** p, size_t bytes) { plan.push_back({off, p}); off += align256(std::max<size_t>(bytes, 8)); };
        add((void**)&sites_, es * site_stride() * n_);
        add((void**)&dims_, sizeof(int) * (n_ + 1));
        add((void**)&theta_, es * (size_t)ld_ * ld_);
        add((void**)&W_, es * (size_t)ld_ * ld_);
        add((void**)&sig2_, sizeof(double) * ld_);
        add((void**)&sig_, sizeof(double) * ld_);
        add((void**)&perm_, sizeof(int) * ld_);
        add((void**)&counters_, sizeof(int) * C_.max_sweeps);
        add((void**)&scal_, sizeof(double) * 2);
        add((void**)&bar_, sizeof(GridBar));
        add((void**)&stats_, sizeof(RunStats));
        add((void**)&h_, sizeof(double) * n_);
        add((void**)&w_, sizeof(double) * std::max(m_, 1));
        add((void**)&sa_, sizeof(double) * std::max(P_.steps, 1));
        add((void**)&sb_, sizeof(double) * std::max(P_.steps, 1));
        add((void**)&bias_, sizeof(double) * n_);
        add((void**)&sc_, sizeof(double) * std::max(P_.steps, 1));
        add((void**)&step_, sizeof(int));
        add((void**)&entropy_, sizeof(double) * std::max(P_.steps, 1));
        add((void**)&envs_, es * unit * 3);  // entropy chain: ONE, two ping-pong buffers
        add((void**)&xs_, es * unit * 4);  // chain phase-1 product, up to (2 cap) x (2 cap)
        add((void**)&vbuf_, es * (size_t)2 * cap_);
        add((void**)&entc_, sizeof(ChainStep) * std::max(n_ent_, 1));
        add((void**)&obsR_, sizeof(ChainStep) * n_);
        add((void**)&obsL_, sizeof(ChainStep) * n_obsL_);
        add((void**)&dots_, sizeof(PairDot) * (1 + n_ + m_));
        add((void**)&dotout_, sizeof(double) * (1 + n_ + m_));
        add((void**)&amp2_, sizeof(double));
        add((void**)&spins_d_, n_);
        // candidate rows of the cooperative LQ (theta of 257..1024 rows): 8 rows per CTA
        lq_ok_ = ld_ > 256 && ld_ <= 1024;
        add((void**)&lqc_, lq_ok_ ? lq_coop_scratch_bytes(ld_, (int)es, (ld_ + 7) / 8) : 8);
        TQ_CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        TQ_CK(device_alloc((void**)&base_, off));
        for (auto& it : plan) *it.second = base_ + it.first;
        TQ_CK(cudaMemsetAsync(bar_, 0, sizeof(GridBar), stream_));
        TQ_CK(cudaMemsetAsync(stats_, 0, sizeof(RunStats), stream_));
        TQ_CK(cudaMemsetAsync(entropy_, 0, sizeof(double) * std::max(P_.steps, 1), stream_));
        TQ_CK(cudaMemsetAsync(envs_, 0, es * unit, stream_));  // the ONE env
        V one = mk<V>(1, 0);
        TQ_CK(cudaMemcpyAsync(envs_, &one, sizeof(V), cudaMemcpyHostToDevice, stream_));
        // chain step lists
        const long long U = (long long)unit;
        auto Loff = [&](int i) { return i == 0 ? 0LL : (1LL + i) * U; };
        auto Roff = [&](int i) { return i == n_ ? 0LL : (1LL + n_ + i) * U; };
        auto Zoff = [&](int i) { return (1LL + 2LL * n_ + i) * U; };
        auto ZZoff = [&](int e) { return (1LL + 3LL * n_ + e) * U; };
        const long long T0 = (1LL + 3LL * n_ + m_) * U, T1 = T0 + U;
        const long long E0 = U, E1 = 2 * U;  // entropy ping-pong inside envs_
        std::vector<ChainStep> ent;
        for (int q = 0; q < n_ent_; ++q) {
            const int site = n_ - 1 - q;
            ent.push_back(ChainStep{site, 0, q == 0 ? 0LL : ((q - 1) & 1 ? E1 : E0), (q & 1) ? E1 : E0});
        }
        r1_off_ = n_ent_ ? (((n_ent_ - 1) & 1) ? E1 : E0) : 0;
        std::vector<ChainStep> R, L;
        for (int q = 0; q < n_; ++q) {
            const int site = n_ - 1 - q;
            R.push_back(ChainStep{site, 0, Roff(site + 1), Roff(site)});
        }
        for (int i = 0; i < n_; ++i) L.push_back(ChainStep{i, 0, Loff(i), Loff(i + 1)});
        for (int i = 0; i < n_; ++i) L.push_back(ChainStep{i, 1, Loff(i), Zoff(i)});
        std::vector<PairDot> D;
        D.push_back(PairDot{Loff(n_), 0, n_, 0});
        for (int i = 0; i < n_; ++i) D.push_back(PairDot{Zoff(i), Roff(i + 1), i + 1, 0});
        for (int e = 0; e < m_; ++e) {
            const int i = std::min(P_.ei[e], P_.ej[e]), j = std::max(P_.ei[e], P_.ej[e]);
            if (i == j) {
                // the reference's expect_zz(i, i) inserts Z once (cuda/src/mps.cpp:156,188-194)
                D.push_back(PairDot{Zoff(i), Roff(i + 1), i + 1, 0});
                continue;
            }
            long long cur = Loff(i);
            int flip = 0;
            for (int s = i; s <= j; ++s) {
                const bool last = (s == j);
                const long long out = last ? ZZoff(e) : (flip ? T1 : T0);
                L.push_back(ChainStep{s, (s == i || s == j) ? 1 : 0, cur, out});
                cur = out;
                flip ^= 1;
            }
            D.push_back(PairDot{ZZoff(e), Roff(j + 1), j + 1, 0});
        }
        if (!ent.empty())
            TQ_CK(cudaMemcpyAsync(entc_, ent.data(), sizeof(ChainStep) * ent.size(), cudaMemcpyHostToDevice, stream_));
        TQ_CK(cudaMemcpyAsync(obsR_, R.data(), sizeof(ChainStep) * R.size(), cudaMemcpyHostToDevice, stream_));
        TQ_CK(cudaMemcpyAsync(obsL_, L.data(), sizeof(ChainStep) * L.size(), cudaMemcpyHostToDevice, stream_));
        TQ_CK(cudaMemcpyAsync(dots_, D.data(), sizeof(PairDot) * D.size(), cudaMemcpyHostToDevice, stream_));
        TQ_CK(cudaStreamSynchronize(stream_));
    }

    void upload_problem() {
        TQ_CK(cudaMemcpyAsync(h_, P_.h.data(), sizeof(double) * n_, cudaMemcpyHostToDevice, stream_));
        if (m_) TQ_CK(cudaMemcpyAsync(w_, P_.w.data(), sizeof(double) * m_, cudaMemcpyHostToDevice, stream_));
        if (P_.steps) {
            TQ_CK(cudaMemcpyAsync(sa_, P_.sa.data(), sizeof(double) * P_.steps, cudaMemcpyHostToDevice, stream_));
            TQ_CK(cudaMemcpyAsync(sb_, P_.sb.data(), sizeof(double) * P_.steps, cudaMemcpyHostToDevice, stream_));
        }
        if (!P_.bias.empty()) {
            TQ_CK(cudaMemcpyAsync(bias_, P_.bias.data(), sizeof(double) * n_, cudaMemcpyHostToDevice, stream_));
            if (P_.steps)
                TQ_CK(cudaMemcpyAsync(sc_, P_.sc.data(), sizeof(double) * P_.steps, cudaMemcpyHostToDevice, stream_));
        } else {
            TQ_CK(cudaMemsetAsync(bias_, 0, sizeof(double) * n_, stream_));
            TQ_CK(cudaMemsetAsync(sc_, 0, sizeof(double) * std::max(P_.steps, 1), stream_));
        }
        TQ_CK(cudaStreamSynchronize(stream_));
    }

    void single_site(const ScheduleView& sch) {
        int mx = 1;
        for (int i = 0; i < n_; ++i) mx = std::max(mx, ub_[i] * ub_[i + 1]);
        launch_single_site<T>(mps(), sch, mx, stream_);
    }

    void two_site(const MpsView<T>& M, const ScheduleView& sch, const GateOp& op) {
        const int i = op.bond;
        const int dl = ub_[i], dr = ub_[i + 2];
        const int keep_ub = std::min(C_.chi, std::min(2 * dl, 2 * dr));
        bool tc_done = false;
        if constexpr (sizeof(T) == 4) {
            if (C_.theta_tc && theta_tc_supported(op)) {
                launch_theta_tc(M, sch, op, work(), dl, dr, stream_);
                tc_done = true;
            }
        }
        if (!tc_done) launch_theta<T>(M, sch, op, nullptr, work(), dl, dr, stream_);
        // theta above 256 rows (the cooperative column-pair Jacobi): the pivoted LQ first, unless
        // switched off or a block width was forced
        const bool lq = lq_ok_ && C_.precond != 2 && C_.block == 0 && 2 * dl > 256 && 2 * dl <= 1024 &&
                        2 * dr <= 1024;
        cudaEvent_t a = nullptr, b = nullptr;
        if (lq) {
            cudaEvent_t c = nullptr, d = nullptr;
            if (C_.timing) {
                c = event();
                d = event();
                TQ_CK(cudaEventRecord(c, stream_));
            }
            launch_lq_coop<T>(M, i, work(), lqc_, 2 * dl, 2 * dr, stream_);
            if (C_.timing) {
                TQ_CK(cudaEventRecord(d, stream_));
                timed_lq_.push_back({c, d});
            }
            ++launches_;
        }
        if (C_.timing) {
            a = event();
            b = event();
            TQ_CK(cudaEventRecord(a, stream_));
        }
        launch_svd<T>(M, i, C_.chi, tol_for(2 * dl), C_.max_sweeps, work(), 2 * dl, 2 * dr, pick_block(2 * dl, 2 * dr),
                      stream_, 0, 0, lq ? 1 : 0);
        if (C_.timing) {
            TQ_CK(cudaEventRecord(b, stream_));
            timed_.push_back({a, b});
        }
        launch_absorb<T>(M, i, work(), 2 * dl, 2 * dr, keep_ub, stream_);
        ub_[i + 1] = keep_ub;
        launches_ += 4;
        ++svd_launches_;
    }

    cudaEvent_t event() {
        if (pool_next_ < pool_.size()) return pool_[pool_next_++];
        cudaEvent_t e;
        TQ_CK(cudaEventCreate(&e));
        pool_.push_back(e);
        ++pool_next_;
        return e;
    }

    void entropy_step(const MpsView<T>& M) {
        if (n_ >= 2) {
            launch_chain<T>(M, 1, entc_, n_ent_, envs_, xs_, bar_, stats_, cap_, stream_);
            launch_entropy<T>(M, envs_ + r1_off_, entropy_, step_, stream_);
        } else {
            launch_entropy<T>(M, nullptr, entropy_, step_, stream_);
        }
    }
};

static std::unique_ptr<EngineBase> make_engine(const ProblemHost& P, const Config& C) {
    if (C.device >= 0) TQ_CK(cudaSetDevice(C.device));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw CudaError("no CUDA device available");
    if (C.precision == TESSERA_QA_C64) return std::unique_ptr<EngineBase>(new Engine<float>(P, C));
    return std::unique_ptr<EngineBase>(new Engine<double>(P, C));
}

// Many independent instances annealed in lock step: gate slot q of every instance that has
// one goes into one launch of each batched kernel (theta, one-CTA-per-task Jacobi SVD,
// absorption), so each instance keeps the reference's gate order while the GPU is filled
// with independent SVDs.
class BatchBase {
public:
    virtual ~BatchBase() = default;
    virtual int size() const = 0;
    virtual void randomize(unsigned long long seed, double decay) = 0;
    virtual void run(int k0, int k1) = 0;
    virtual void run_gates(int k, int q0, int q1) = 0;
    virtual void set_values(const std::vector<ProblemHost>& P) = 0;
    virtual void sync(tessera_qa_result* r) = 0;  // aggregated over the instances
    virtual cudaStream_t stream() const = 0;
    virtual void save(int b, void* buf, size_t bytes) = 0;  // checkpoint of instance b
};

template <typename T>
class BatchEngine final : public BatchBase {
public:
    BatchEngine(const std::vector<ProblemHost>& P, const std::vector<Config>& C) {
        try {  // a failed allocation or CUDA call releases what was made before it
            init(P, C);
        } catch (...) {
            release();
            throw;
        }
    }
    ~BatchEngine() override { release(); }
    void release() noexcept {
        if (st_) cudaStreamSynchronize(st_);
        if (gexec_) cudaGraphExecDestroy(gexec_);
        if (graph_) cudaGraphDestroy(graph_);
        gexec_ = nullptr;
        graph_ = nullptr;
        for (cudaEvent_t e : pool_) cudaEventDestroy(e);
        if (e0_) cudaEventDestroy(e0_);
        if (e1_) cudaEventDestroy(e1_);
        if (base_) cudaFree(base_);
        if (st_) cudaStreamDestroy(st_);
        pool_.clear();
        e0_ = e1_ = nullptr;
        base_ = nullptr;
        st_ = nullptr;
    }

private:
    void init(const std::vector<ProblemHost>& P, const std::vector<Config>& C) {
        const int B = (int)P.size();
        int steps = 0;
        for (int b = 0; b < B; ++b) {
            eng_.emplace_back(new Engine<T>(P[b], C[b]));
            steps = std::max(steps, P[b].steps);
            cap_max_ = std::max(cap_max_, eng_.back()->cap());
            n_max_ = std::max(n_max_, eng_.back()->n());
            q_max_ = std::max(q_max_, (int)eng_.back()->ops().size());
        }
        steps_ = steps;
        block_ = C[0].block;  // 0: by size (resident, else column pairs of width 8); 32: block-Gram
        rows_cap_ = std::max(8, (2 * cap_max_ + 7) & ~7);
        TQ_CK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
        TQ_CK(cudaEventCreate(&e0_));
        TQ_CK(cudaEventCreate(&e1_));
        // device: shared step counter, instance views, per-slot update lists
        size_t nref_tot = 0;
        refs_off_.assign(q_max_ + 1, 0);
        std::vector<UpdRef> refs;
        for (int q = 0; q < q_max_; ++q) {
            refs_off_[q] = refs.size();
            for (int b = 0; b < B; ++b)
                if (q < (int)eng_[b]->ops().size()) refs.push_back(UpdRef{b, eng_[b]->ops()[q]});
        }
        refs_off_[q_max_] = refs.size();
        nref_tot = refs.size();
        // per-instance gate lists for the resident whole-anneal kernel, and the order in which
        // CTAs take instances: most work (gates x bond capacity^3) first
        std::vector<GateOp> ops_all;
        std::vector<int> op_off(B + 1, 0), order(B);
        for (int b = 0; b < B; ++b) {
            op_off[b] = (int)ops_all.size();
            ops_all.insert(ops_all.end(), eng_[b]->ops().begin(), eng_[b]->ops().end());
            order[b] = b;
        }
        op_off[B] = (int)ops_all.size();
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            const double cx = (double)eng_[x]->ops().size() * std::pow((double)eng_[x]->cap(), 3.0);
            const double cy = (double)eng_[y]->ops().size() * std::pow((double)eng_[y]->cap(), 3.0);
            return cx > cy;
        });
        const size_t a0 = 256, a1 = a0 + align256(sizeof(InstTask<T>) * B);
        const size_t a2 = a1 + align256(sizeof(UpdRef) * std::max<size_t>(nref_tot, 1));
        const size_t a3 = a2 + align256(sizeof(GateOp) * std::max<size_t>(ops_all.size(), 1));
        const size_t a4 = a3 + align256(sizeof(int) * (B + 1));
        const size_t bytes = a4 + align256(sizeof(int) * B);
        TQ_CK(device_alloc((void**)&base_, bytes));
        step_ = reinterpret_cast<int*>(base_);
        work_ = reinterpret_cast<int*>(base_ + 64);
        insts_ = reinterpret_cast<InstTask<T>*>(base_ + a0);
        refs_ = reinterpret_cast<UpdRef*>(base_ + a1);
        ops_all_ = reinterpret_cast<GateOp*>(base_ + a2);
        op_off_ = reinterpret_cast<int*>(base_ + a3);
        order_ = reinterpret_cast<int*>(base_ + a4);
        std::vector<InstTask<T>> it;
        for (int b = 0; b < B; ++b) it.push_back(eng_[b]->inst_task(step_, rows_cap_));
        TQ_CK(cudaMemcpy(insts_, it.data(), sizeof(InstTask<T>) * B, cudaMemcpyHostToDevice));
        if (nref_tot) TQ_CK(cudaMemcpy(refs_, refs.data(), sizeof(UpdRef) * nref_tot, cudaMemcpyHostToDevice));
        if (!ops_all.empty())
            TQ_CK(cudaMemcpy(ops_all_, ops_all.data(), sizeof(GateOp) * ops_all.size(), cudaMemcpyHostToDevice));
        TQ_CK(cudaMemcpy(op_off_, op_off.data(), sizeof(int) * (B + 1), cudaMemcpyHostToDevice));
        TQ_CK(cudaMemcpy(order_, order.data(), sizeof(int) * B, cudaMemcpyHostToDevice));
        resident_ = C[0].block == 0 && !C[0].theta_tc;
        theta_tc_ = C[0].theta_tc != 0;
        precond_ = C[0].precond != 2;
        for (auto& e : eng_) TQ_CK(cudaStreamSynchronize(e->own_stream()));
    }

public:
    int size() const override { return (int)eng_.size(); }
    Engine<T>& at(int b) { return *eng_[b]; }
    void save(int b, void* buf, size_t bytes) override {
        if (b < 0 || b >= (int)eng_.size()) throw ArgError("instance index out of range");
        TQ_CK(cudaStreamSynchronize(st_));
        eng_[b]->save(buf, bytes, 0);
    }
    cudaStream_t stream() const override { return st_; }
    void set_timing(bool on) { timing_ = on; }

    void randomize(unsigned long long seed, double decay) override {
        for (size_t b = 0; b < eng_.size(); ++b) eng_[b]->randomize(seed + 7919ull * b, decay);
        for (auto& e : eng_) TQ_CK(cudaStreamSynchronize(e->own_stream()));
    }

    void set_values(const std::vector<ProblemHost>& P) override {
        if (P.size() != eng_.size()) throw ArgError("set_values needs one problem per instance");
        for (size_t b = 0; b < eng_.size(); ++b) eng_[b]->set_values(P[b]);
    }

    void run_gates(int k, int q0, int q1) override {
        if (q0 < 0 || q1 > q_max_ || q0 > q1) throw ArgError("gate range outside the step");
        k_set_int<<<1, 1, 0, st_>>>(step_, k);
        TQ_CK(cudaGetLastError());
        TQ_CK(cudaEventRecord(e0_, st_));
        for (int q = q0; q < q1; ++q) slot(q);
        TQ_CK(cudaEventRecord(e1_, st_));
        ran_ = true;
    }

    void sync(tessera_qa_result* r) override {
        TQ_CK(cudaStreamSynchronize(st_));
        TQ_CK(cudaGetLastError());
        if (ran_) {
            float ms = 0;
            TQ_CK(cudaEventElapsedTime(&ms, e0_, e1_));
            ms_ = ms;
            ran_ = false;
        }
        for (auto& pr : timed_) {
            float ms = 0;
            TQ_CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
            svd_ms_ += ms;
        }
        timed_.clear();
        for (auto& pr : timed_lq_) {
            float ms = 0;
            TQ_CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
            lq_ms_ += ms;
        }
        timed_lq_.clear();
        pool_next_ = 0;
        if (!r) return;
        tessera_qa_result a;
        std::memset(&a, 0, sizeof(a));
        a.min_cut_gap = 1.0;
        for (auto& e : eng_) {
            tessera_qa_result x;
            std::memset(&x, 0, sizeof(x));
            e->sync_stats(&x);
            a.two_site_updates += x.two_site_updates;
            a.max_trunc = std::max(a.max_trunc, x.max_trunc);
            a.status |= x.status;
            a.max_sweeps = std::max(a.max_sweeps, x.max_sweeps);
            a.max_bond = std::max(a.max_bond, x.max_bond);
            a.min_cut_gap = std::min(a.min_cut_gap, x.min_cut_gap);
            a.svd_bytes += x.svd_bytes;
            a.svd_flops += x.svd_flops;
            a.svd_sweeps += x.svd_sweeps;
        }
        r->two_site_updates = a.two_site_updates;
        r->max_trunc = a.max_trunc;
        r->status = a.status;
        r->max_sweeps = a.max_sweeps;
        r->max_bond = a.max_bond;
        r->min_cut_gap = a.min_cut_gap;
        r->svd_bytes = a.svd_bytes;
        r->svd_flops = a.svd_flops;
        r->svd_sweeps = a.svd_sweeps;
        r->svd_ms = svd_ms_;
        r->precond_ms = lq_ms_;
        r->svd_launches = svd_launches_;
        r->kernel_launches = launches_;
        r->device_ms = ms_;
    }

    void run(int k0, int k1) override {
        const int B = (int)eng_.size();
        k_set_int<<<1, 1, 0, st_>>>(step_, k0);
        TQ_CK(cudaGetLastError());
        TQ_CK(cudaEventRecord(e0_, st_));
        // small bonds: every step of every instance in one launch, one CTA per instance
        if (resident_ && k1 > k0 &&
            launch_anneal_resident<T>(insts_, ops_all_, op_off_, order_, B, k0, k1, work_, rows_cap_, st_)) {
            k_set_int<<<1, 1, 0, st_>>>(step_, k1);
            TQ_CK(cudaGetLastError());
            launches_ += 2;
            svd_launches_ += 1;
            TQ_CK(cudaEventRecord(e1_, st_));
            ran_ = true;
            sync(nullptr);
            return;
        }
        // One Trotter step is the same launch sequence for every k (the kernels read the step
        // from the device counter), so without per-launch timing it is captured once into a CUDA
        // graph and replayed: one launch per step instead of 4 per gate slot.
        const bool graph = !timing_ && k1 - k0 >= 2;
        if (graph && !gexec_) {
            cudaGraph_t g = nullptr;
            const long long l0 = launches_, s0 = svd_launches_;  // capturing launches nothing
            TQ_CK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
            try {
                step_body(B);
            } catch (...) {
                cudaStreamEndCapture(st_, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            TQ_CK(cudaStreamEndCapture(st_, &g));
            graph_launches_ = launches_ - l0;  // kernels one replay launches
            graph_svd_launches_ = svd_launches_ - s0;
            launches_ = l0;
            svd_launches_ = s0;
            graph_ = g;
            TQ_CK(cudaGraphInstantiate(&gexec_, graph_, 0));
        }
        for (int k = k0; k < k1; ++k) {
            if (graph) {
                TQ_CK(cudaGraphLaunch(gexec_, st_));
                launches_ += graph_launches_;
                svd_launches_ += graph_svd_launches_;
            } else {
                step_body(B);
            }
        }
        TQ_CK(cudaEventRecord(e1_, st_));
        ran_ = true;
        sync(nullptr);
    }
    double ms() const { return ms_; }
    long long launches() const { return launches_; }

private:
    // one Trotter step of every instance: half single-site gates, every gate slot, half
    // single-site gates, the qubit-0 entropy, the step counter
    void step_body(int B) {
        launch_single_site_batch<T>(insts_, B, n_max_, cap_max_ * cap_max_, st_);
        for (int q = 0; q < q_max_; ++q) slot(q);
        launch_single_site_batch<T>(insts_, B, n_max_, cap_max_ * cap_max_, st_);
        launch_entropy_batch<T>(insts_, B, st_);
        launch_step_inc(step_, st_);
        launches_ += 4;
    }
    // gate slot q of every instance that has one: theta, Jacobi SVD, absorption
    void slot(int q) {
        const int nref = (int)(refs_off_[q + 1] - refs_off_[q]);
        cudaEvent_t a = nullptr, b = nullptr, c = nullptr, d = nullptr;
        if (timing_) {
            a = event();
            b = event();
            c = event();
            d = event();
        }
        const int nl = launch_update_batch<T>(insts_, refs_ + refs_off_[q], nref, cap_max_, 2 * cap_max_, block_,
                                              st_, a, b, theta_tc_, precond_, c, d);
        launches_ += nl;
        if (timing_) timed_.push_back({a, b});
        if (timing_ && nl == 5) timed_lq_.push_back({c, d});  // the preconditioner ran
        ++svd_launches_;
    }
    cudaEvent_t event() {
        if (pool_next_ < pool_.size()) return pool_[pool_next_++];
        cudaEvent_t e;
        TQ_CK(cudaEventCreate(&e));
        pool_.push_back(e);
        ++pool_next_;
        return e;
    }
    bool timing_ = false, ran_ = false;
    double svd_ms_ = 0.0, lq_ms_ = 0.0;
    long long svd_launches_ = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timed_, timed_lq_;
    std::vector<cudaEvent_t> pool_;
    size_t pool_next_ = 0;

public:

private:
    std::vector<std::unique_ptr<Engine<T>>> eng_;
    cudaStream_t st_ = nullptr;
    cudaEvent_t e0_ = nullptr, e1_ = nullptr;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t gexec_ = nullptr;
    long long graph_launches_ = 0, graph_svd_launches_ = 0;
    char* base_ = nullptr;
    int* step_ = nullptr;
    InstTask<T>* insts_ = nullptr;
    UpdRef* refs_ = nullptr;
    GateOp* ops_all_ = nullptr;
    int *op_off_ = nullptr, *order_ = nullptr, *work_ = nullptr;
    bool resident_ = true;
    bool theta_tc_ = false;
    bool precond_ = true;
    std::vector<size_t> refs_off_;
    int cap_max_ = 1, n_max_ = 1, q_max_ = 0, steps_ = 0, block_ = 8, rows_cap_ = 8;
    double ms_ = 0.0;
    long long launches_ = 0;
};

template <typename T>
static void run_batch(const std::vector<ProblemHost>& P, const std::vector<Config>& C,
                      const tessera_qa_config* configs, tessera_qa_result* results) {
    BatchEngine<T> be(P, C);
    int k0 = (int)configs[0].step_begin;
    int k1 = configs[0].step_end ? (int)configs[0].step_end : P[0].steps;
    for (size_t b = 0; b < P.size(); ++b)
        if (P[b].steps != P[0].steps) throw ArgError("batched instances must share the number of schedule steps");
    if (k0 > k1 || k1 > P[0].steps) throw ArgError("step range outside the schedule");
    be.run(k0, k1);
    for (int b = 0; b < be.size(); ++b) {
        Engine<T>& e = be.at(b);
        tessera_qa_result r = results[b];
        e.sync_stats(&r);
        r.device_ms = be.ms();
        r.kernel_launches = be.launches();
        if (!configs[b].skip_observables) e.observe(&r);
        if (r.entropy) e.copy_entropy(r.entropy, k0, k1);
        if (r.final_mps) e.save(r.final_mps, r.final_mps_bytes, (unsigned long long)k1);
        results[b] = r;
    }
}

// Standalone SVD output: the U columns whose singular value lies under the Jacobi's noise floor
// (8 sqrt(R) ulps of ||A||_F) carry rounding noise, not a resolved direction.  Each is replaced,
// in descending order, by its part orthogonal to every column before it (classical Gram-Schmidt,
// two passes), renormalised; a column with nothing left becomes zero.  U (R x k, row-major) is
// then an isometry on its non-zero columns, as the reference's SVD makes its factor by
// Gram-Schmidt (cuda/src/linalg.cpp:56-105).
static void orthonormalise_subfloor(std::vector<double2>& U, int R, int k, const std::vector<double>& sig) {
    double fro2 = 0.0;
    for (int t = 0; t < k; ++t) fro2 += sig[t] * sig[t];
    const double floor = 8.0 * std::sqrt((double)R) * 2.220446049250313e-16 * std::sqrt(fro2);
    std::vector<double2> x(R);
    for (int t = 0; t < k; ++t) {
        if (sig[t] > floor) continue;
        for (int i = 0; i < R; ++i) x[i] = U[(size_t)i * k + t];
        double n0 = 0.0;
        for (int i = 0; i < R; ++i) n0 += x[i].x * x[i].x + x[i].y * x[i].y;
        for (int pass = 0; pass < 2; ++pass)
            for (int q = 0; q < t; ++q) {
                double re = 0.0, im = 0.0;  // u_q^H x
                for (int i = 0; i < R; ++i) {
                    const double2 u = U[(size_t)i * k + q];
                    re += u.x * x[i].x + u.y * x[i].y;
                    im += u.x * x[i].y - u.y * x[i].x;
                }
                for (int i = 0; i < R; ++i) {
                    const double2 u = U[(size_t)i * k + q];
                    x[i].x -= re * u.x - im * u.y;
                    x[i].y -= re * u.y + im * u.x;
                }
            }
        double n2 = 0.0;
        for (int i = 0; i < R; ++i) n2 += x[i].x * x[i].x + x[i].y * x[i].y;
        const double sc = (n0 > 0.0 && n2 > 1e-16 * n0) ? 1.0 / std::sqrt(n2) : 0.0;
        for (int i = 0; i < R; ++i) U[(size_t)i * k + t] = make_double2(x[i].x * sc, x[i].y * sc);
    }
}

}  // namespace tq

using namespace tq;

struct tessera_qa_session {
    std::unique_ptr<EngineBase> eng;     // single instance
    std::unique_ptr<BatchBase> batch;    // or a batch of instances
    ProblemHost P;
    Config C;
    std::vector<ProblemHost> PB;
};

template <typename F>
static int guarded(F&& f) {
    try {
        return f();
    } catch (const ArgError& e) {
        set_err(e.what());
        return TESSERA_QA_EINVAL;
    } catch (const CudaError& e) {
        set_err(e.what());
        return TESSERA_QA_ECUDA;
    } catch (const std::exception& e) {
        set_err(std::string("CUDA: ") + e.what());
        return TESSERA_QA_ECUDA;
    }
}

extern "C" {

void tessera_qa_config_init(tessera_qa_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->dt = 0.1;
    cfg->zz_substeps = 1;
    cfg->precision = TESSERA_QA_C128;
    cfg->chi = 32;
    cfg->device = -1;
}

size_t tessera_qa_checkpoint_bytes(size_t n, size_t chi) {
    return ckpt_header_bytes((int)n) + n * 2 * chi * chi * 16;
}

int tessera_qa_last_error(char* buf, size_t len) {
    if (buf && len) {
        const size_t k = std::min(len - 1, t_err.size());
        std::memcpy(buf, t_err.data(), k);
        buf[k] = 0;
    }
    return (int)t_err.size();
}

int tessera_qa_anneal_ex(const tessera_qa_problem* problem, const tessera_qa_config* config,
                         tessera_qa_result* result) {
    return guarded([&]() -> int {
        if (!result) throw ArgError("result is NULL");
        ProblemHost P = validate_problem(problem);
        Config C = validate_config(config);
        const int k0 = config ? (int)config->step_begin : 0;
        const int k1 = (config && config->step_end) ? (int)config->step_end : P.steps;
        if (k0 > k1 || k1 > P.steps) throw ArgError("step range outside the schedule");
        auto eng = make_engine(P, C);
        if (config && config->initial_mps)
            eng->load(config->initial_mps, (size_t)-1 / 2);
        eng->run(k0, k1);
        tessera_qa_result r = *result;
        eng->sync_stats(&r);
        if (!(config && config->skip_observables)) eng->observe(&r);
        if (r.entropy) eng->copy_entropy(r.entropy, k0, k1);
        if (r.final_mps) eng->save(r.final_mps, r.final_mps_bytes, (unsigned long long)k1);
        *result = r;
        if (r.status) {
            set_err("kernel status bits set: " + std::to_string(r.status));
            return TESSERA_QA_ESTATUS;
        }
        return 0;
    });
}

int tessera_qa_anneal_batch(const tessera_qa_problem* problems, const tessera_qa_config* configs,
                            tessera_qa_result* results, size_t count) {
    return guarded([&]() -> int {
        if (!problems || !configs || !results) throw ArgError("problems, configs and results must be non-NULL");
        if (count == 0) return 0;
        std::vector<ProblemHost> P;
        std::vector<Config> C;
        for (size_t b = 0; b < count; ++b) {
            P.push_back(validate_problem(&problems[b]));
            C.push_back(validate_config(&configs[b]));
            if (C.back().precision != C[0].precision) throw ArgError("batched instances must share the precision");
            if (configs[b].initial_mps) throw ArgError("batched runs start from |+>^n");
        }
        if (C[0].device >= 0) TQ_CK(cudaSetDevice(C[0].device));
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw CudaError("no CUDA device available");
        if (C[0].precision == TESSERA_QA_C64)
            run_batch<float>(P, C, configs, results);
        else
            run_batch<double>(P, C, configs, results);
        int st = 0;
        for (size_t b = 0; b < count; ++b) st |= results[b].status;
        if (st) {
            set_err("kernel status bits set: " + std::to_string(st));
            return TESSERA_QA_ESTATUS;
        }
        return 0;
    });
}

double tessera_qa_anneal(const double* h, size_t n, const size_t* ei, const size_t* ej, const double* ew,
                         size_t m, const double* schedule_a, const double* schedule_b, size_t steps, size_t chi,
                         int8_t* out_s, double* out_entropy) {
    if (!out_s) {
        set_err("out_s is NULL");
        return std::nan("");
    }
    tessera_qa_problem p{n, h, m, ei, ej, ew, steps, schedule_a, schedule_b};
    tessera_qa_config c;
    tessera_qa_config_init(&c);
    c.dt = 0.1;  // cuda/src/ffi.cpp:28
    c.chi = chi;
    tessera_qa_result r;
    std::memset(&r, 0, sizeof(r));
    std::vector<int8_t> spins(n);
    std::vector<double> ent(steps);
    r.spins = spins.data();
    r.entropy = steps ? ent.data() : nullptr;
    const int rc = tessera_qa_anneal_ex(&p, &c, &r);
    if (rc != 0) return std::nan("");
    std::memcpy(out_s, spins.data(), n);
    if (out_entropy && steps) std::memcpy(out_entropy, ent.data(), sizeof(double) * steps);
    return r.energy;
}

int tessera_qa_debug_fail_allocations(int after, int count) {
    std::lock_guard<std::mutex> lk(g_fail_mu);
    const int pending = g_fail_count;
    g_fail_after = after < 0 ? 0 : after;
    g_fail_count = count < 0 ? 0 : count;
    return pending;
}

int tessera_qa_svd(const double* a, size_t rows, size_t cols, double* s, double* u, double* vh) {
    return guarded([&]() -> int {
        if (!a || !s) throw ArgError("a or s is NULL");
        if (rows == 0 || cols == 0 || rows > 2048 || cols > 2048) throw ArgError("matrix shape out of range");
        const int R = (int)rows, N = (int)cols, k = std::min(R, N);
        ProblemHost P;
        P.n = 1;
        P.h.assign(1, 0.0);
        Config C;
        C.chi = 1;
        C.min_ld = std::max(R, N);
        int dev = 0;
        if (cudaGetDeviceCount(&dev) != cudaSuccess || dev == 0) throw CudaError("no CUDA device available");
        Engine<double> eng(P, C);
        std::vector<double2> cm((size_t)R * N);
        for (int i = 0; i < R; ++i)
            for (int j = 0; j < N; ++j) cm[(size_t)j * R + i] = make_double2(a[2 * ((size_t)i * N + j)], a[2 * ((size_t)i * N + j) + 1]);
        std::vector<int> perm;
        std::vector<double> sig;
        std::vector<double2> Wc;
        eng.svd_only(cm, R, N, perm, sig, Wc);
        for (int t = 0; t < k; ++t) s[t] = sig[t];
        if (u || vh) {
            // U[:, t] = W[:, perm[t]] / sigma_t ; Vh[t, :] = U[:, t]^H A
            std::vector<double2> U((size_t)R * k, make_double2(0, 0));
            for (int t = 0; t < k; ++t) {
                if (!(sig[t] > 1e-300)) continue;
                for (int i = 0; i < R; ++i) {
                    const double2 w = Wc[(size_t)perm[t] * R + i];
                    U[(size_t)i * k + t] = make_double2(w.x / sig[t], w.y / sig[t]);
                }
            }
            orthonormalise_subfloor(U, R, k, sig);
            if (u) std::memcpy(u, U.data(), sizeof(double2) * U.size());
            if (vh) {
                for (int t = 0; t < k; ++t)
                    for (int j = 0; j < N; ++j) {
                        double re = 0, im = 0;
                        if (sig[t] > 1e-300)
                            for (int i = 0; i < R; ++i) {
                                const double2 x = U[(size_t)i * k + t];
                                const double ar = a[2 * ((size_t)i * N + j)], ai = a[2 * ((size_t)i * N + j) + 1];
                                re += x.x * ar + x.y * ai;
                                im += x.x * ai - x.y * ar;
                            }
                        vh[2 * ((size_t)t * N + j)] = re / (sig[t] > 1e-300 ? sig[t] : 1.0);
                        vh[2 * ((size_t)t * N + j) + 1] = im / (sig[t] > 1e-300 ? sig[t] : 1.0);
                    }
            }
        }
        if (eng.status_) {
            set_err("kernel status bits set: " + std::to_string(eng.status_));
            return TESSERA_QA_ESTATUS;
        }
        return 0;
    });
}

tessera_qa_session* tessera_qa_session_create(const tessera_qa_problem* problem, const tessera_qa_config* config) {
    tessera_qa_session* out = nullptr;
    const int rc = guarded([&]() -> int {
        std::unique_ptr<tessera_qa_session> s(new tessera_qa_session);
        s->P = validate_problem(problem);
        s->C = validate_config(config);
        s->eng = make_engine(s->P, s->C);
        out = s.release();
        return 0;
    });
    return rc == 0 ? out : nullptr;
}

tessera_qa_session* tessera_qa_session_create_batch(const tessera_qa_problem* problems,
                                                    const tessera_qa_config* configs, size_t count) {
    tessera_qa_session* out = nullptr;
    const int rc = guarded([&]() -> int {
        if (!problems || !configs || count == 0) throw ArgError("problems/configs must be non-NULL, count >= 1");
        std::unique_ptr<tessera_qa_session> s(new tessera_qa_session);
        std::vector<Config> C;
        for (size_t b = 0; b < count; ++b) {
            s->PB.push_back(validate_problem(&problems[b]));
            C.push_back(validate_config(&configs[b]));
            if (C.back().precision != C[0].precision) throw ArgError("batched instances must share the precision");
            if (s->PB.back().steps != s->PB[0].steps) throw ArgError("batched instances must share the step count");
        }
        if (C[0].device >= 0) TQ_CK(cudaSetDevice(C[0].device));
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw CudaError("no CUDA device available");
        s->C = C[0];
        if (C[0].precision == TESSERA_QA_C64) {
            auto* b = new BatchEngine<float>(s->PB, C);
            b->set_timing(C[0].timing);
            s->batch.reset(b);
        } else {
            auto* b = new BatchEngine<double>(s->PB, C);
            b->set_timing(C[0].timing);
            s->batch.reset(b);
        }
        out = s.release();
        return 0;
    });
    return rc == 0 ? out : nullptr;
}

int tessera_qa_session_randomize(tessera_qa_session* s, uint64_t seed) {
    return tessera_qa_session_randomize_graded(s, seed, 0.0);
}

int tessera_qa_session_randomize_graded(tessera_qa_session* s, uint64_t seed, double decay) {
    return guarded([&]() -> int {
        if (!s) throw ArgError("session is NULL");
        if (!(decay >= 0.0) || !std::isfinite(decay)) throw ArgError("decay must be a finite number >= 0");
        if (s->batch) s->batch->randomize(seed, decay);
        else s->eng->randomize(seed, decay);
        return 0;
    });
}

int tessera_qa_session_run(tessera_qa_session* s, size_t step_begin, size_t nsteps) {
    return guarded([&]() -> int {
        if (!s) throw ArgError("session is NULL");
        if (s->batch) s->batch->run((int)step_begin, (int)(step_begin + nsteps));
        else s->eng->run((int)step_begin, (int)(step_begin + nsteps));
        return 0;
    });
}

int tessera_qa_session_run_gates(tessera_qa_session* s, size_t step, size_t gate_begin, size_t gate_end) {
    return guarded([&]() -> int {
        if (!s) throw ArgError("session is NULL");
        if (s->batch) s->batch->run_gates((int)step, (int)gate_begin, (int)gate_end);
        else s->eng->run_gates((int)step, (int)gate_begin, (int)gate_end);
        return 0;
    });
}

int tessera_qa_session_run_host(tessera_qa_session* s, const tessera_qa_problem* problems, size_t count, size_t step,
                                size_t gate_begin, size_t gate_end, tessera_qa_result* result) {
    return guarded([&]() -> int {
        if (!s || !problems) throw ArgError("session and problems must be non-NULL");
        const size_t B = s->batch ? (size_t)s->batch->size() : 1;
        if (count != B) throw ArgError("one problem per session instance is required");
        std::vector<ProblemHost> P;
        for (size_t b = 0; b < count; ++b) P.push_back(validate_problem(&problems[b]));
        if (s->batch) {
            s->batch->set_values(P);
            if (gate_end) s->batch->run_gates((int)step, (int)gate_begin, (int)gate_end);
            else s->batch->run((int)step, (int)step + 1);
            s->batch->sync(result);
        } else {
            s->eng->set_values(P[0]);
            if (gate_end) s->eng->run_gates((int)step, (int)gate_begin, (int)gate_end);
            else s->eng->run((int)step, (int)step + 1);
            s->eng->sync_stats(result);
        }
        return 0;
    });
}

void* tessera_qa_session_stream(tessera_qa_session* s) {
    if (!s) return nullptr;
    return s->batch ? (void*)s->batch->stream() : (void*)s->eng->stream();
}

int tessera_qa_session_sync(tessera_qa_session* s, tessera_qa_result* result) {
    return guarded([&]() -> int {
        if (!s) throw ArgError("session is NULL");
        tessera_qa_result r;
        std::memset(&r, 0, sizeof(r));
        if (s->batch) s->batch->sync(&r);
        else s->eng->sync_stats(&r);
        if (result) {
            result->max_trunc = r.max_trunc;
            result->two_site_updates = r.two_site_updates;
            result->status = r.status;
            result->max_sweeps = r.max_sweeps;
            result->max_bond = r.max_bond;
            result->device_ms = r.device_ms;
            result->min_cut_gap = r.min_cut_gap;
            result->svd_ms = r.svd_ms;
            result->precond_ms = r.precond_ms;
            result->svd_bytes = r.svd_bytes;
            result->svd_flops = r.svd_flops;
            result->svd_launches = r.svd_launches;
            result->svd_sweeps = r.svd_sweeps;
            result->kernel_launches = r.kernel_launches;
        }
        return 0;
    });
}

int tessera_qa_session_observe(tessera_qa_session* s, tessera_qa_result* result) {
    return guarded([&]() -> int {
        if (!s || !result) throw ArgError("session or result is NULL");
        if (s->batch) throw ArgError("observe is per instance: use tessera_qa_anneal_batch for batched results");
        s->eng->sync_stats(result);
        s->eng->observe(result);
        return 0;
    });
}

int tessera_qa_session_save(tessera_qa_session* s, void* buf, size_t bytes) {
    return guarded([&]() -> int {
        if (!s) throw ArgError("session is NULL");
        if (s->batch) throw ArgError("checkpoints are per instance");
        s->eng->save(buf, bytes, 0);
        return 0;
    });
}

int tessera_qa_session_save_instance(tessera_qa_session* s, size_t index, void* buf, size_t bytes) {
    return guarded([&]() -> int {
        if (!s) throw ArgError("session is NULL");
        if (s->batch) {
            s->batch->save((int)std::min<size_t>(index, 1u << 30), buf, bytes);
        } else {
            if (index != 0) throw ArgError("instance index out of range");
            s->eng->save(buf, bytes, 0);
        }
        return 0;
    });
}

int tessera_qa_session_sample(tessera_qa_session* s, size_t count, uint64_t seed, int8_t* out_spins,
                              double* out_energies) {
    return guarded([&]() -> int {
        if (!s) throw ArgError("session is NULL");
        if (s->batch) throw ArgError("sampling is per instance: use a single-instance session");
        if (count && !out_spins) throw ArgError("out_spins is NULL");
        s->eng->sample(count, (unsigned long long)seed, out_spins, out_energies);
        return 0;
    });
}

int tessera_qa_session_load(tessera_qa_session* s, const void* buf, size_t bytes) {
    return guarded([&]() -> int {
        if (!s) throw ArgError("session is NULL");
        if (s->batch) throw ArgError("checkpoints are per instance");
        s->eng->load(buf, bytes);
        return 0;
    });
}

void tessera_qa_session_destroy(tessera_qa_session* s) { delete s; }

}  // extern "C"
