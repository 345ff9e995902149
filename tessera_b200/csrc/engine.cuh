// engine.cuh -- device-side views of the MPS state and launch declarations.
//
// HBM layout (one instance):
//   sites   : n site tensors, each a fixed-capacity slab of 2*cap*cap complex elements.
//             Site i element (a, s, b) sits at sites[i*site_stride + (a*2 + s)*cap + b],
//             the reference's (a*2+s)*Dr+b order (cuda/include/mps.hpp:27-35) with the
//             row stride fixed at the capacity, so site i is the row-major matrix
//             [(a,s), b] with leading dimension cap.
//   dims    : n+1 ints, bond dimensions; dims[0] = dims[n] = 1; site i is
//             (dims[i], 2, dims[i+1]).  Kernels read dims on the device, so the host
//             never waits for a truncation result.
//   theta/W : (2cap) x (2cap) column-major complex workspaces; theta[row + col*ld] with
//             row = (a, s1) = 2a + s1, col = (s2, b) = s2*Dr + b (cuda/src/mps.cpp:49).
#pragma once
#include "common.cuh"

namespace tq {

template <typename T>
struct MpsView {
    cplx_t<T>* sites;
    int* dims;
    int n;
    int cap;
    long long site_stride;
    __device__ __forceinline__ cplx_t<T>* site(int i) const { return sites + (long long)i * site_stride; }
};

// A two-site gate: kind 0 = SWAP, 1 = exp(-i theta Z Z) with theta = -B(step)*w[edge]*sub,
// 2 = a general 4x4 given in `g` (row-major, basis |s_i s_{i+1}>).
struct GateOp {
    int bond;
    int kind;
    int edge;
    int pad;
};
enum : int { GATE_SWAP = 0, GATE_ZZ = 1, GATE_GENERAL = 2 };

struct ScheduleView {
    const double* h;    // n longitudinal fields
    const double* w;    // m couplings
    const double* sa;   // steps, transverse weight A(s_k)
    const double* sb;   // steps, problem weight B(s_k)
    const int* step;    // device step counter (index into sa/sb)
    double dt;          // Trotter step
    double sub;         // dt / zz_substeps
    const double* bias; // n warm-start bias b_i (zeros when unused)
    const double* sc;   // steps, its weight C(s_k)
};

struct RunStats {
    double max_trunc;       // max discarded weight ratio over the run
    long long updates;      // two-site updates performed
    int max_sweeps;         // most Jacobi sweeps any update needed
    int status;             // ST_* bits
    int max_bond;           // largest bond dimension seen
    int pad;
    double gap_deficit;     // max over truncating updates of 1 - (s[keep-1] - s[keep]) / s[0]
    double svd_bytes;       // algorithmic bytes moved by the Jacobi-SVD launches
    long long svd_sweeps;   // sweeps summed over launches
    double svd_flops;       // FP64/FP32 flops of the Jacobi arithmetic (dot products, rotations, GEMMs)
};

// Per-update SVD workspace.
template <typename T>
struct SvdWork {
    cplx_t<T>* theta;   // gated theta, column-major, ld
    cplx_t<T>* W;       // Jacobi working copy (theta J), column-major, ld
    int ld;
    double* sig2;       // per-column squared norms [2cap]
    double* sig;        // sorted kept singular values [2cap]
    int* perm;          // sorted column order [2cap]
    int* counters;      // per-sweep rotation counts [max_sweeps]
    double* scal;       // [2] scratch scalars (squared Frobenius norm of W), zeroed per launch
    GridBar* bar;
    RunStats* stats;
};

struct SvdParams {
    int bond;
    int R, N;          // > 0: explicit matrix shape (standalone SVD); else 2*dims[bond], 2*dims[bond+2]
    int no_trunc;      // 1: keep all min(R, N) values, leave dims and run statistics alone
    int chi;
    double tol;
    double tiny;       // absolute lower bound of the noise floor on |w|^2 (pair_live)
    int max_sweeps;
    int rows_cap;      // shared-memory column length
    int cols_cap;      // shared-memory column count of the resident Jacobi (>= N, even)
    int lq;            // 1: W holds the pivoted LQ factor P L of theta (lq.cu): the Jacobi takes
                       //    min(R, N) columns (the rest are zero)
};

struct ChainStep {
    int site;
    int zflag;
    long long in_off;   // element offset of the input env in `envs`
    long long out_off;  // element offset of the output env
};

// Per-instance views used by the batched kernels (one entry per instance).
template <typename T>
struct InstTask {
    MpsView<T> mps;
    ScheduleView sch;
    SvdWork<T> wk;
    SvdParams pp;              // bond is taken from the UpdRef
    const ChainStep* ent_steps;
    int n_ent;
    int pad;
    cplx_t<T>* envs;
    cplx_t<T>* X;
    long long r1_off;
    double* entropy;
};
// One two-site update of one instance in a batched launch.
struct UpdRef {
    int inst;
    GateOp op;
};

// ---- launchers (kernels.cu) ----
template <typename T>
void launch_single_site(const MpsView<T>& mps, const ScheduleView& sch, int dl_ub_max, cudaStream_t s);
template <typename T>
void launch_theta(const MpsView<T>& mps, const ScheduleView& sch, GateOp op, const double* gen_gate,
                  SvdWork<T> wk, int dl_ub, int dr_ub, cudaStream_t s);
// R, N > 0 run a standalone SVD of an explicit R x N matrix in wk.W (no truncation).
template <typename T>
int launch_svd(const MpsView<T>& mps, int bond, int chi, double tol, int max_sweeps, SvdWork<T> wk,
               int rows_ub, int cols_ub, int block_w, cudaStream_t s, int R = 0, int N = 0, int lq = 0);
// cooperative row-pivoted LQ of one theta's working copy, in place (lq.cu); rows_ub <= 1024
template <typename T>
void launch_lq_coop(const MpsView<T>& mps, int bond, SvdWork<T> wk, void* scratch, int rows_ub, int cols_ub,
                    cudaStream_t s);
size_t lq_coop_scratch_bytes(int ld, int esz, int ctas);
template <typename T>
void launch_absorb(const MpsView<T>& mps, int bond, SvdWork<T> wk, int rows_ub, int cols_ub, int keep_ub,
                   cudaStream_t s);

// Environment transfer chain.  Each step maps env E (ket x bra, ld = cap) through one
// site, optionally with Z inserted on that site's physical index:
//   left : E'[b,b'] = sum_{a,a',s} E[a,a'] A(a,s,b) z_s conj(A(a',s,b'))
//   right: E'[a,a'] = sum_{s,b,b'} A(a,s,b) E[b,b'] z_s conj(A(a',s,b'))
template <typename T>
void launch_chain(const MpsView<T>& mps, int right, const ChainStep* d_steps, int nsteps, cplx_t<T>* envs,
                  cplx_t<T>* scratch, GridBar* bar, RunStats* stats, int d_ub, cudaStream_t s);
template <typename T>
void launch_entropy(const MpsView<T>& mps, const cplx_t<T>* r1, double* out_entropy, const int* step,
                    cudaStream_t s);
// values[j] = Re sum_{b,b'} X_j[b,b'] Y_j[b,b'] over the dims of bond bond_j
struct PairDot {
    long long x_off;
    long long y_off;
    int bond;
    int pad;
};
template <typename T>
void launch_pair_dots(const MpsView<T>& mps, const cplx_t<T>* envs, const PairDot* d_jobs, int njobs,
                      double* out, cudaStream_t s);
template <typename T>
void launch_amplitude(const MpsView<T>& mps, const int8_t* spins, cplx_t<T>* scratch, double* out_amp2,
                      cudaStream_t s);
void launch_step_inc(int* step, cudaStream_t s);
// batched launchers: `refs` selects (instance, gate) pairs; ub_* are upper bounds over the batch
template <typename T>
void launch_single_site_batch(const InstTask<T>* insts, int ninst, int n_max, int d2_ub_max, cudaStream_t s);
// returns the number of kernels launched; precond: the pivoted LQ (lq.cu) before a column-pair
// Jacobi of theta above 256 rows
template <typename T>
int launch_update_batch(const InstTask<T>* insts, const UpdRef* refs, int nref, int d_ub, int rows_ub,
                        int block_w, cudaStream_t s, cudaEvent_t svd_begin = nullptr,
                        cudaEvent_t svd_end = nullptr, bool theta_tc = false, bool precond = false,
                        cudaEvent_t lq_begin = nullptr, cudaEvent_t lq_end = nullptr);
// row-pivoted Householder LQ of each task's theta working copy, in place (lq.cu)
template <typename T>
void launch_lq_batch(const InstTask<T>* insts, const UpdRef* refs, int nref, cudaStream_t s);
template <typename T>
void launch_entropy_batch(const InstTask<T>* insts, int ninst, cudaStream_t s);
// Whole anneal of every instance, one CTA per instance at a time (small bonds only); false
// when theta does not fit one CTA's shared memory.
template <typename T>
bool launch_anneal_resident(const InstTask<T>* insts, const GateOp* ops, const int* op_off, const int* order,
                            int ninst, int k0, int k1, int* work, int rows_cap, cudaStream_t s);
// perfect sampling of basis patterns from the MPS with the right environments in `envs`
template <typename T>
void launch_sample(const MpsView<T>& mps, const cplx_t<T>* envs, int count, unsigned long long seed, int8_t* out,
                   cudaStream_t s);
// complex64 bond contraction on tcgen05 tensor cores, split-TF32 (theta_tc.cu)
bool theta_tc_supported(const GateOp& op);
void launch_theta_tc(const MpsView<float>& mps, const ScheduleView& sch, GateOp op, SvdWork<float> wk, int dl_ub,
                     int dr_ub, cudaStream_t s);
void launch_theta_tc_batch(const InstTask<float>* insts, const UpdRef* refs, int nref, int d_ub, cudaStream_t s);
template <typename T>
void launch_init_plus(const MpsView<T>& mps, cudaStream_t s);

}  // namespace tq
