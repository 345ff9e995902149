// noalloc.cu -- tessera_qa_svd_noalloc: the Jacobi SVD kernel with no device allocation.
//
// Some callers cannot call cudaMalloc at all: code running under an allocator owned by a
// host application or framework (the device heap belongs to someone else), real-time or
// certification-constrained services that forbid allocation after start-up, and hooks
// that are handed device buffers by their caller and must not touch the allocator.
// tessera_qa_svd_noalloc serves them: the caller passes device pointers for the input and
// the outputs, and every scratch buffer the SVD needs lives in one file-scope
// `__device__` array of fixed size (kNoAllocMaxDim = 256 rows and columns, about 1 MiB),
// which each GPU that loads this library holds until the process exits.
//
// Set-up: the first call on a device, with that device current, looks up the array's
// device address with cudaGetSymbolAddress and loads the kernels; make that first call
// before any stream capture.  Every call shares the one array and it keeps the previous
// call's contents: each call clears the counters that must start at zero, and calls whose
// work overlaps on the GPU (other streams, other host threads on the same device) race on
// the array -- serialise them.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/tessera_qa.h"
#include "engine.cuh"

namespace tq {

constexpr int kNoAllocMaxDim = 256;
constexpr int kNoAllocSweeps = 60;

struct NoAllocScratch {
    double2 W[kNoAllocMaxDim * kNoAllocMaxDim];  // column-major working copy, ld = kNoAllocMaxDim
    double sig2[kNoAllocMaxDim];
    double sig[kNoAllocMaxDim];
    int perm[kNoAllocMaxDim];
    int counters[kNoAllocSweeps];
    double scal[2];
    GridBar bar;
    RunStats stats;
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// row-major interleaved (rows x cols) -> column-major W
__global__ void k_noalloc_load(const double2* a, int rows, int cols, double2* W) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= rows * cols) return;
    const int i = t / cols, j = t - i * cols;
    W[(long long)j * kNoAllocMaxDim + i] = a[t];
}

// s[t] = sigma_t; u[i, t] = W[i, perm[t]] / sigma_t (row-major rows x k); zero column if sigma_t == 0
__global__ void k_noalloc_store(const double2* W, const int* perm, const double* sig, int rows, int k, double* s,
                                double2* u) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < k && s) s[t] = sig[t];
    if (!u || t >= rows * k) return;
    const int i = t / k, c = t - i * k;
    const double sg = sig[c];
    const double2 w = W[(long long)perm[c] * kNoAllocMaxDim + i];
    u[t] = sg > 1e-300 ? make_double2(w.x / sg, w.y / sg) : make_double2(0.0, 0.0);
}

static std::mutex g_setup_mu;
static NoAllocScratch* g_setup_ptr[64] = {};

// Once per device, with that device current: resolve the array's device address.
static NoAllocScratch* noalloc_setup(int dev) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (dev < 0 || dev >= 64) throw std::runtime_error("device ordinal out of range");
    if (g_setup_ptr[dev]) return g_setup_ptr[dev];
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        throw std::runtime_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, k_noalloc_load);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_noalloc_store);
    if (e != cudaSuccess) throw std::runtime_error(std::string("kernel load: ") + cudaGetErrorString(e));
    g_setup_ptr[dev] = static_cast<NoAllocScratch*>(p);
    return g_setup_ptr[dev];
}

// engine.cu: the per-thread message returned by tessera_qa_last_error()
void set_last_error(const std::string& msg);

}  // namespace tq

using namespace tq;

extern "C" int tessera_qa_svd_noalloc(const double* d_a, size_t rows, size_t cols, double* d_s, double* d_u,
                                      void* stream) {
    try {
        if (!d_a || !d_s) throw std::invalid_argument("d_a and d_s must be device pointers");
        if (rows == 0 || cols == 0 || rows > (size_t)kNoAllocMaxDim || cols > (size_t)kNoAllocMaxDim)
            throw std::invalid_argument("tessera_qa_svd_noalloc: rows and cols must be in 1.." +
                                        std::to_string(kNoAllocMaxDim));
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) throw std::runtime_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        NoAllocScratch* sc = noalloc_setup(dev);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const int R = (int)rows, N = (int)cols, k = R < N ? R : N;
        // an error left pending by the caller's own earlier launches would otherwise be read
        // back after ours and reported as this call's failure
        (void)cudaGetLastError();
        // clear what must start at zero (the array keeps the previous call's contents)
        e = cudaMemsetAsync(&sc->bar, 0, sizeof(GridBar), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(&sc->stats, 0, sizeof(RunStats), s);
        if (e != cudaSuccess) throw std::runtime_error(std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
        // Once work is queued on the shared array, no error path returns before that work has
        // finished: a next call could otherwise overlap it on the array.
        try {
            k_noalloc_load<<<(R * N + 255) / 256, 256, 0, s>>>(reinterpret_cast<const double2*>(d_a), R, N, sc->W);
            e = cudaGetLastError();
            if (e != cudaSuccess) throw std::runtime_error(std::string("launch: ") + cudaGetErrorString(e));
            SvdWork<double> wk{nullptr, sc->W, kNoAllocMaxDim, sc->sig2, sc->sig, sc->perm,
                               sc->counters, sc->scal, &sc->bar, &sc->stats};
            MpsView<double> none{nullptr, nullptr, 0, 1, 0};
            const int bw = N <= 64 ? 16 : 8;
            const double tol = 1e-13;
            launch_svd<double>(none, 0, k, tol, kNoAllocSweeps, wk, R, N, bw, s, R, N);
            k_noalloc_store<<<(R * k + 255) / 256, 256, 0, s>>>(sc->W, sc->perm, sc->sig, R, k, d_s,
                                                               reinterpret_cast<double2*>(d_u));
            e = cudaGetLastError();
            if (e != cudaSuccess) throw std::runtime_error(std::string("launch: ") + cudaGetErrorString(e));
        } catch (...) {
            (void)cudaStreamSynchronize(s);
            throw;
        }
        int status = 0;
        e = cudaMemcpyAsync(&status, &sc->stats.status, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        else (void)cudaStreamSynchronize(s);
        if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e));
        if (status) {
            set_last_error("kernel status bits set: " + std::to_string(status));
            return TESSERA_QA_ESTATUS;
        }
        return 0;
    } catch (const std::invalid_argument& ex) {
        set_last_error(ex.what());
        return TESSERA_QA_EINVAL;
    } catch (const std::exception& ex) {
        set_last_error(ex.what());
        return TESSERA_QA_ECUDA;
    }
}
