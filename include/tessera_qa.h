/*
 * tessera_qa.h -- C ABI of libtessera_qa.so, the sm_100a MPS-TEBD quantum-annealing engine.
 *
 * Drop-in for the reference's `tessera_qa` shared library (cuda/CMakeLists.txt:28-30),
 * which the Rust crate links under `--features cuda` (rust/build.rs:15-19) and binds in
 * rust/src/ffi.rs:19-35.  All pointers are caller-owned host memory, read or written only
 * during the call; nothing is retained.  Every call is synchronous.  Calls from different
 * host threads are safe: each thread gets its own CUDA stream and device workspace.
 *
 * Errors: functions returning int give 0 on success and a negative TESSERA_QA_E* code on
 * failure; tessera_qa_anneal returns NaN.  On failure outputs are left untouched and a
 * message is kept per thread for tessera_qa_last_error().
 */
#ifndef TESSERA_QA_H
#define TESSERA_QA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define TESSERA_QA_API __attribute__((visibility("default")))
#else
#define TESSERA_QA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define TESSERA_QA_ABI_VERSION 1

/* error codes (negative returns) */
#define TESSERA_QA_EINVAL   (-1)  /* invalid argument: null pointer, n = 0, chi = 0, edge index out of range, NaN input */
#define TESSERA_QA_ECUDA    (-2)  /* CUDA runtime error (no device, launch failure, out of memory) */
#define TESSERA_QA_ESTATUS  (-3)  /* the run finished but a kernel raised a status bit (see result.status) */
#define TESSERA_QA_ESMALL   (-4)  /* a caller buffer is too small */

/* result.status bits */
#define TESSERA_QA_ST_JACOBI_NOT_CONVERGED 1
#define TESSERA_QA_ST_BARRIER_TIMEOUT      2
#define TESSERA_QA_ST_BAD_DIMS             4
#define TESSERA_QA_ST_NONFINITE            8

enum tessera_qa_precision {
    TESSERA_QA_C128 = 0, /* complex128 everywhere */
    TESSERA_QA_C64 = 1   /* complex64 tensors and rotations; FP64 convergence test, discarded weight,
                            entropy and energies */
};

/*
 * Replaces the reference's only entry point, cuda/src/ffi.cpp:10-37 (bound in
 * rust/src/ffi.rs:19-35).  Same semantics: |+>^n start, dt fixed at 0.1, one ZZ slice per
 * step with edges in the given order, complex128, bond cap `chi`.  Writes n spins
 * (sign of <Z_i>, ties -> +1) to out_s and, when out_entropy is not NULL, `steps` values of
 * the qubit-0 entanglement entropy (bits).  Returns the Ising energy of the spins
 * (E = -sum w s_i s_j - sum h s_i), or NaN on error.
 */
TESSERA_QA_API double tessera_qa_anneal(const double* h, size_t n, const size_t* ei, const size_t* ej, const double* ew,
                         size_t m, const double* schedule_a, const double* schedule_b, size_t steps,
                         size_t chi, int8_t* out_s, double* out_entropy);

/* An Ising instance E(s) = -sum_e ew[e] s_ei s_ej - sum_i h_i s_i and its discretised schedule
 * A(s_k) = schedule_a[k], B(s_k) = schedule_b[k] (rust/src/schedule.rs:8-18). */
typedef struct tessera_qa_problem {
    size_t n;
    const double* h;
    size_t m;
    const size_t* ei;
    const size_t* ej;
    const double* ew;
    size_t steps;
    const double* schedule_a;
    const double* schedule_b;
    /* Optional warm-start bias (NULL = none; not in the reference): a longitudinal field
     * -C(s_k) sum_i bias_i Z_i added to H for step k, with C(s_k) = schedule_c[k].  Choosing
     * C = 0 at both ends leaves the initial and final Hamiltonians unchanged. */
    const double* bias;
    const double* schedule_c;
} tessera_qa_problem;

typedef struct tessera_qa_config {
    double dt;              /* Trotter step; the reference's mps_anneal argument (cuda/include/mps.hpp:76-82) */
    int zz_substeps;        /* ZZ block slices, forward/reverse alternating (cuda/src/mps.cpp:330-341) */
    int precision;          /* enum tessera_qa_precision */
    size_t chi;             /* bond-dimension cap */
    double jacobi_tol;      /* rotate a column pair when |w_p^H w_q| > tol |w_p||w_q|; 0 = default */
    int jacobi_max_sweeps;  /* 0 = default (60) */
    int jacobi_block;       /* 0 = chosen by size (resident Jacobi for small theta, else column pairs in blocks
                               of 8); 1,2,4,8,16 = column-pair blocks of that width; 32 = block-Gram Jacobi
                               (batches) */
    int device;             /* CUDA device ordinal; -1 = the calling thread's current device */
    size_t step_begin;      /* run schedule steps [step_begin, step_end) */
    size_t step_end;        /* 0 = problem.steps */
    const void* initial_mps;/* NULL = |+>^n; else a checkpoint written by a previous call */
    int skip_observables;   /* 1 = skip the final <Z>, <ZZ>, readout and prob (checkpoint runs) */
    int kernel_timing;      /* 1 = time every Jacobi-SVD launch with CUDA events (result.svd_ms) */
    int theta_tensor_cores; /* complex64 only: 1 = bond contraction on the tcgen05 tensor cores in split-TF32
                               (three TF32 passes, FP32 accumulators); 0 = CUDA-core FP32 */
    int jacobi_precondition;/* column-pair Jacobi of theta above 256 rows (up to 512 rows in a batch, 1024
                               in a single instance with jacobi_block 0): 0 = default (on), 1 = on, 2 = off.
                               On: a row-pivoted Householder LQ of theta (P^T theta = L Q^H) runs first and
                               the Jacobi works on L, which takes fewer sweeps (Drmac-Veselic
                               preconditioning); the results are the same up to rounding */
    int reserved[4];
} tessera_qa_config;

typedef struct tessera_qa_result {
    /* caller-provided outputs (each may be NULL) */
    int8_t* spins;          /* n: sign(<Z_i>), ties -> +1 (cuda/src/mps.cpp:369-371) */
    double* entropy;        /* step_end - step_begin values, qubit-0 entropy in bits */
    void* final_mps;        /* checkpoint buffer, tessera_qa_checkpoint_bytes() bytes */
    size_t final_mps_bytes;
    double* z_expect;       /* n: <Z_i> of the final state (cuda/src/mps.cpp:182-186) */
    /* filled by the call */
    double energy;          /* Ising energy of `spins` */
    double expected_energy; /* <psi|H_problem|psi>/<psi|psi> from the MPS */
    double prob;            /* |<spins|psi>|^2 / <psi|psi> */
    double max_trunc;       /* largest discarded weight ratio of any two-site update */
    double norm2;           /* <psi|psi> */
    long long two_site_updates;
    int status;             /* TESSERA_QA_ST_* bits */
    int max_sweeps;         /* most Jacobi sweeps any update used */
    int max_bond;           /* largest bond dimension reached */
    int reserved_i;
    double device_ms;       /* GPU time of the Trotter steps (CUDA events) */
    double min_cut_gap;     /* min over truncating updates of (s[keep-1] - s[keep]) / s[0]; 1 if none
                               truncated.  Near 0 the kept subspace is not unique (degenerate cut). */
    double svd_ms;          /* summed duration of the Jacobi-SVD launches (config.kernel_timing) */
    double svd_bytes;       /* bytes the Jacobi-SVD kernels read and wrote in global memory */
    long long svd_launches; /* Jacobi-SVD launches */
    long long svd_sweeps;   /* Jacobi sweeps summed over launches */
    long long kernel_launches; /* all engine kernel launches */
    double svd_flops;       /* flops of the Jacobi arithmetic: dot products, rotations, Gram and apply GEMMs */
    double precond_ms;      /* summed duration of the pivoted-LQ preconditioner launches (config.kernel_timing;
                               config.jacobi_precondition) */
} tessera_qa_result;

/* Fills `cfg` with the legacy defaults: dt 0.1, zz_substeps 1, complex128, chi 32. */
TESSERA_QA_API void tessera_qa_config_init(tessera_qa_config* cfg);

/* Extended anneal: the reference's mps_anneal (cuda/src/mps.cpp:295-381) with every
 * AnnealResult field (cuda/include/mps.hpp:37-44), a caller-chosen dt / precision, and
 * checkpoint resume.  Returns 0 or a TESSERA_QA_E* code. */
TESSERA_QA_API int tessera_qa_anneal_ex(const tessera_qa_problem* problem, const tessera_qa_config* config,
                         tessera_qa_result* result);

/* Batched anneal of `count` independent instances (the batching layer): each
 * instance runs exactly its own tessera_qa_anneal_ex (same gate order, keep rule, results),
 * but gate slot q of every instance goes into one launch of each batched kernel, with one
 * CTA per Jacobi SVD, so many updates run concurrently.  Instances may differ in n, edges,
 * chi and dt; they must share precision and number of schedule steps, and start from |+>^n.
 * No counterpart in the reference, which anneals one instance per call. */
TESSERA_QA_API int tessera_qa_anneal_batch(const tessera_qa_problem* problems, const tessera_qa_config* configs,
                                           tessera_qa_result* results, size_t count);

/* Bytes of a checkpoint for n sites at bond cap chi (upper bound; any dims fit). */
TESSERA_QA_API size_t tessera_qa_checkpoint_bytes(size_t n, size_t chi);

/* Thin SVD of one rows x cols complex128 matrix (row-major, interleaved re/im) through the
 * engine's one-sided Jacobi kernel: s (min(rows,cols), descending), u (rows x k) and vh
 * (k x cols), both row-major interleaved; u / vh may be NULL.  The counterpart of the
 * reference's tessera::svd (cuda/src/linalg.cpp:107-172).  rows, cols <= 2048.  Singular
 * values under the noise floor 8 sqrt(rows) ulps of ||A||_F are not resolved (their columns
 * are frozen).  From about 1024 columns, a column whose norm dips under that floor during the
 * sweeps stays frozen: a few values within ~4x of the floor can come back at it, and the u / vh
 * columns of frozen values are then not orthogonal to the rest. */
TESSERA_QA_API int tessera_qa_svd(const double* a, size_t rows, size_t cols, double* s, double* u, double* vh);

/* Allocation-free SVD, for callers that cannot call cudaMalloc (their device memory belongs to
 * a host application's or framework's allocator, or allocation is forbidden after start-up).
 * No counterpart in the reference.  Same one-sided Jacobi kernel as tessera_qa_svd, but
 * d_a (rows x cols complex128, row-major interleaved re/im), d_s (min(rows,cols) singular
 * values, descending) and d_u (rows x k left singular vectors, row-major; may be NULL) are
 * DEVICE pointers on the current device, and all scratch is a fixed file-scope device array:
 * rows and cols must be 1..256 (larger sizes return TESSERA_QA_EINVAL), and no device memory
 * is allocated or freed.  Work is ordered on `stream` (a cudaStream_t; NULL = legacy default
 * stream) and the call waits for it before returning.  The first call on each device sets
 * the array up (device-address lookup, kernel load); make it before any stream capture.
 * All calls share the one array: calls that overlap on the GPU race and must be serialised. */
TESSERA_QA_API int tessera_qa_svd_noalloc(const double* d_a, size_t rows, size_t cols, double* d_s, double* d_u,
                                          void* stream);

/* Exact ground state by brute force over the 2^n patterns on the GPU (1 <= n <= 32): bit set
 * <-> spin +1, first minimum kept, as rust/src/ising.rs:46-61 (exact_ground_state).  Writes n
 * spins when out_spins is not NULL; returns the ground energy, or NaN on error. */
TESSERA_QA_API double tessera_qa_exact_ground(const double* h, size_t n, const size_t* ei, const size_t* ej,
                                              const double* ew, size_t m, int8_t* out_spins);

/* ---- exact state-vector anneal on the GPU (rust/src/quantum.rs:63-112), 1 <= n <= 30 ----
 * mode 0: the reference's splitting (quantum.rs:82-84): problem phase B dt/2, exp(+i A dt X) on
 *         every qubit, problem phase B dt/2.
 * mode 1: the MPS engine's splitting: single-site half steps exp(-i dt/2 (-A X - B h Z)) (with
 *         the problem's warm-start field when it has one), the exact ZZ block, half steps again.
 * |+>^n start, FP64 throughout, qubit-0 entropy per step (quantum.rs:138-175).  spins = the most
 * probable pattern (quantum.rs:94-103, first maximum); sign_spins = the sign<Z> pattern.
 * Memory: 32 bytes per basis state on the device. */
typedef struct tessera_qa_sv_result {
    int8_t* spins;          /* n, required */
    int8_t* sign_spins;     /* n, optional */
    double* entropy;        /* steps, optional */
    double* state;          /* 2 * 2^n doubles (interleaved complex), optional */
    double energy;          /* Ising energy of spins */
    double expected_energy; /* <psi|H_problem|psi> / <psi|psi> */
    double prob;            /* probability of spins */
    double sign_energy;     /* Ising energy of sign_spins */
    double sign_prob;       /* its probability (when state was requested, else -1) */
    double norm2;           /* <psi|psi> */
    double device_ms;
    double reserved[4];
} tessera_qa_sv_result;
TESSERA_QA_API int tessera_qa_sv_anneal(const tessera_qa_problem* problem, double dt, int mode,
                                        tessera_qa_sv_result* result);

/* ---- learned schedules: a message-passing GNN trained and run by the library's own kernels ----
 * No counterpart in the reference's engine; python/gnn_guide.py:81-135 (its warm-start spin
 * predictor) is the architectural starting point.  From an Ising graph it predicts `knots`
 * monotone schedule knots 0 = s_0 <= ... <= s_{K-1} = 1 at equally spaced anneal times and a
 * per-spin probability P(s_i = +1).  Weights are BF16 with FP32 accumulation (bf16_weights = 1)
 * or FP32. */
typedef struct tessera_qa_gnn tessera_qa_gnn;
TESSERA_QA_API tessera_qa_gnn* tessera_qa_gnn_create(int hidden, int layers, int knots, uint64_t seed,
                                                     int bf16_weights);
TESSERA_QA_API void tessera_qa_gnn_destroy(tessera_qa_gnn* g);
TESSERA_QA_API size_t tessera_qa_gnn_param_count(const tessera_qa_gnn* g);
TESSERA_QA_API int tessera_qa_gnn_get_params(tessera_qa_gnn* g, float* out, size_t count);
TESSERA_QA_API int tessera_qa_gnn_set_params(tessera_qa_gnn* g, const float* in, size_t count);
/* out_knots: count x knots; out_p: total nodes (problems concatenated). */
TESSERA_QA_API int tessera_qa_gnn_forward(tessera_qa_gnn* g, const tessera_qa_problem* problems, size_t count,
                                          float* out_knots, float* out_p);
/* One training step on a batch: loss = lambda_knots * mean (knot - target)^2 + lambda_spins *
 * mean BCE(p_i, target_spins_i) over nodes whose target is 0 or 1 (negative = no label);
 * forward and backward on the GPU, then Adam with step size lr (lr = 0: gradient only).
 * out_grads (optional, param_count floats) receives the gradient. */
TESSERA_QA_API int tessera_qa_gnn_train_step(tessera_qa_gnn* g, const tessera_qa_problem* problems, size_t count,
                                             const float* target_knots, const float* target_spins, float lr,
                                             float lambda_knots, float lambda_spins, float* out_loss,
                                             float* out_grads, size_t grads_count);
/* One Adam step with a gradient supplied by the caller (param_count floats), e.g. the average of
 * the train_step gradients of several data-parallel ranks; the same update train_step applies. */
TESSERA_QA_API int tessera_qa_gnn_apply_grads(tessera_qa_gnn* g, const float* grads, size_t count, float lr);
/* Schedule prediction (the learned layer's inference): out_knots count x knots; out_bias (total
 * nodes, may be NULL) = 2 P(s_i = +1) - 1 in [-1, 1]. */
TESSERA_QA_API int tessera_qa_schedule_predict(tessera_qa_gnn* g, const tessera_qa_problem* problems, size_t count,
                                               double* out_knots, double* out_bias);

/* Best-of-restarts simulated annealing on the GPU for `count` instances (n <= 128 each): the
 * best-known-energy scorer beyond brute force.  Restates rust/src/ising.rs:64-136 (sa_run,
 * sa_solve): random start, geometric temperatures t0 -> t_end over `sweeps` Metropolis sweeps in
 * spin order, lowest final energy over `restarts` runs (first on ties).  The uniforms come from a
 * counter-based splitmix64 stream keyed by (seed, instance, restart, sweep, spin) instead of the
 * reference's StdRng.  Writes each instance's best spins (concatenated, n per instance, +-1) and
 * energy.  The reference's own use is restarts 40, sweeps 400, t0 5.0, t_end 0.01
 * (rust/src/bin/bench.rs:46). */
TESSERA_QA_API int tessera_qa_sa_solve(const tessera_qa_problem* problems, size_t count, size_t restarts,
                                       size_t sweeps, double t0, double t_end, uint64_t seed,
                                       int8_t* out_spins, double* out_energy);

/* Copies the calling thread's last error message into buf; returns its full length. */
TESSERA_QA_API int tessera_qa_last_error(char* buf, size_t len);

/* Fault injection for tests (no counterpart in the reference, which has no error path): after
 * the next `after` device allocations made by the library (in any thread) succeed, the
 * `count` following ones fail as if cudaMalloc had returned cudaErrorMemoryAllocation;
 * count = 0 cancels what is left.  A call that meets the failure releases what it had
 * allocated and returns TESSERA_QA_ECUDA (tessera_qa_anneal: NaN) with its outputs
 * untouched.  Returns the number of injected failures that were still pending. */
TESSERA_QA_API int tessera_qa_debug_fail_allocations(int after, int count);

/* ---- sessions: device-resident anneal state (no host copies between calls) ---- */
typedef struct tessera_qa_session tessera_qa_session;

/* Uploads the problem and allocates the MPS at bond cap config->chi; state |+>^n. */
TESSERA_QA_API tessera_qa_session* tessera_qa_session_create(const tessera_qa_problem* problem,
                                              const tessera_qa_config* config);
/* A session over `count` independent instances run by the batched engine (see
 * tessera_qa_anneal_batch); randomize / run / run_gates / run_host / sync apply to all of
 * them (sync aggregates: summed updates, max discarded weight, ...). */
TESSERA_QA_API tessera_qa_session* tessera_qa_session_create_batch(const tessera_qa_problem* problems,
                                                                   const tessera_qa_config* configs, size_t count);
/* Replaces the state by a seeded random MPS with every bond at its cap (min(chi, 2^i,
 * 2^(n-i))), sites scaled so theta stays O(1). */
TESSERA_QA_API int tessera_qa_session_randomize(tessera_qa_session* s, uint64_t seed);
/* As tessera_qa_session_randomize, with column b of every site tensor scaled by exp(-b / decay),
 * so that each two-site theta has a graded singular spectrum (Schmidt values falling off as in a
 * TEBD state) instead of a flat one; decay 0 is tessera_qa_session_randomize.  A benchmark and
 * test input, like tessera_qa_session_randomize; the reference has neither. */
TESSERA_QA_API int tessera_qa_session_randomize_graded(tessera_qa_session* s, uint64_t seed, double decay);
/* Enqueues Trotter steps [step_begin, step_begin + nsteps) on the session's stream; returns
 * without waiting. */
TESSERA_QA_API int tessera_qa_session_run(tessera_qa_session* s, size_t step_begin, size_t nsteps);
/* Enqueues only gates [gate_begin, gate_end) of step `step`'s ZZ block (two-site updates in
 * the reference's order; no single-site half steps, no entropy); returns without waiting. */
TESSERA_QA_API int tessera_qa_session_run_gates(tessera_qa_session* s, size_t step, size_t gate_begin,
                                                size_t gate_end);
/* Host-buffer call: copies new h, J and schedule values from `problems` (host memory, one per
 * instance, same n / edges / step count as at creation), runs step `step` (or only its gates
 * [gate_begin, gate_end) when gate_end > 0), waits, and writes the run statistics to *result. */
TESSERA_QA_API int tessera_qa_session_run_host(tessera_qa_session* s, const tessera_qa_problem* problems,
                                               size_t count, size_t step, size_t gate_begin, size_t gate_end,
                                               tessera_qa_result* result);
/* The session's cudaStream_t. */
TESSERA_QA_API void* tessera_qa_session_stream(tessera_qa_session* s);
/* Waits for the stream and fills counters (updates, max_trunc, status, sweeps, bonds). */
TESSERA_QA_API int tessera_qa_session_sync(tessera_qa_session* s, tessera_qa_result* result);
/* Final observables of the current state into result (like tessera_qa_anneal_ex). */
TESSERA_QA_API int tessera_qa_session_observe(tessera_qa_session* s, tessera_qa_result* result);
/* Writes / reads a checkpoint of the current state. */
TESSERA_QA_API int tessera_qa_session_save(tessera_qa_session* s, void* buf, size_t bytes);
TESSERA_QA_API int tessera_qa_session_load(tessera_qa_session* s, const void* buf, size_t bytes);
/* Draws `count` basis patterns x from |<x|psi>|^2 / <psi|psi> of the session's MPS (perfect
 * sampling, site by site with the right environments): out_spins count x n (+1/-1), and the
 * Ising energy of each in out_energies (may be NULL).  The readout for instances whose <Z_i>
 * vanish (h = 0), where the sign readout of cuda/src/mps.cpp:370-371 carries no information.
 * Single-instance sessions; deterministic for a given seed. */
TESSERA_QA_API int tessera_qa_session_sample(tessera_qa_session* s, size_t count, uint64_t seed, int8_t* out_spins,
                                             double* out_energies);
/* Checkpoint of one instance of a batched session (index 0 for a single-instance session). */
TESSERA_QA_API int tessera_qa_session_save_instance(tessera_qa_session* s, size_t index, void* buf, size_t bytes);
TESSERA_QA_API void tessera_qa_session_destroy(tessera_qa_session* s);

#ifdef __cplusplus
}
#endif

#endif /* TESSERA_QA_H */
