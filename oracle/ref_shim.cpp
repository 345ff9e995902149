// ref_shim.cpp -- test infrastructure only.
//
// A thin extern "C" wrapper of ours over the reference engine's public C++ API, compiled
// together with the reference's own sources (cuda/src/linalg.cpp, mps.cpp, ffi.cpp) into
// oracle/_ref/libtessera_ref.so by oracle/Makefile. It exists because the reference's
// only C entry point, tessera_qa_anneal (cuda/src/ffi.cpp:10-37), hard-codes dt = 0.1 and
// returns only the readout energy; the parity tests need the other AnnealResult fields
// (cuda/include/mps.hpp:37-44) and a caller-chosen dt / zz_substeps
// (cuda/include/mps.hpp:76-82).
#include <chrono>
#include <complex>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>
// The reference's MPS keeps its site tensors private and offers no way to load a state; the
// saturated-bond timing below (ref_saturated_update) places random site tensors into it, so
// this one translation unit sees the class's members as public.  The class layout, the member
// functions compiled from the reference's mps.cpp and their behaviour are unchanged.
#define private public
#include "mps.hpp"
#undef private
#include "linalg.hpp"

using namespace tessera;

extern "C" {

// Runs tessera::mps_anneal (cuda/src/mps.cpp:295-381) on the given instance.
// stats[0..3] = energy, expected_energy, prob, max_trunc.  out_entropy may be null.
int ref_mps_anneal(const double* h, int n, const int* ei, const int* ej, const double* ew,
                   int m, const double* sa, const double* sb, int steps, double dt, int chi,
                   int zz_substeps, int8_t* out_spins, double* out_entropy, double* stats) {
    std::vector<double> hv(h, h + n), ewv(ew, ew + m), sav(sa, sa + steps), sbv(sb, sb + steps);
    std::vector<int> eiv(ei, ei + m), ejv(ej, ej + m);
    AnnealResult r = mps_anneal(hv, eiv, ejv, ewv, sav, sbv, dt, chi, zz_substeps);
    for (int i = 0; i < n; ++i) out_spins[i] = r.spins[i];
    if (out_entropy)
        for (int k = 0; k < steps; ++k) out_entropy[k] = r.entropy[k];
    stats[0] = r.energy;
    stats[1] = r.expected_energy;
    stats[2] = r.prob;
    stats[3] = r.max_trunc;
    return 0;
}

// tessera::svd (cuda/src/linalg.cpp:107-172) of a rows x cols complex matrix given
// row-major as interleaved (re, im).  S has min(rows, cols) entries; U is rows x k and
// Vh is k x cols, both row-major interleaved.
int ref_svd(int rows, int cols, const double* a, double* s, double* u, double* vh) {
    CMat A(rows, cols);
    for (int i = 0; i < rows * cols; ++i) A.a[i] = cd(a[2 * i], a[2 * i + 1]);
    CMat U, Vh;
    std::vector<double> S;
    svd(A, U, S, Vh);
    const int k = (int)S.size();
    for (int t = 0; t < k; ++t) s[t] = S[t];
    if (u) std::memcpy(u, U.a.data(), sizeof(cd) * (size_t)rows * k);
    if (vh) std::memcpy(vh, Vh.a.data(), sizeof(cd) * (size_t)k * cols);
    return k;
}

// tessera::hermitian_eig (cuda/src/linalg.cpp:56-105): n x n Hermitian, row-major
// interleaved.  Eigenvalues in returned order (descending); eigenvectors as columns.
int ref_hermitian_eig(int n, const double* a, double* w, double* v) {
    CMat H(n, n);
    for (int i = 0; i < n * n; ++i) H.a[i] = cd(a[2 * i], a[2 * i + 1]);
    std::vector<double> ev;
    CMat V;
    hermitian_eig(H, ev, V);
    for (int i = 0; i < n; ++i) w[i] = ev[i];
    std::memcpy(v, V.a.data(), sizeof(cd) * (size_t)n * n);
    return 0;
}

// tessera::hermitian_expm(H, coeff) (cuda/src/linalg.cpp:174-197).
int ref_hermitian_expm(int n, const double* a, double coeff_re, double coeff_im, double* out) {
    CMat H(n, n);
    for (int i = 0; i < n * n; ++i) H.a[i] = cd(a[2 * i], a[2 * i + 1]);
    CMat E = hermitian_expm(H, cd(coeff_re, coeff_im));
    std::memcpy(out, E.a.data(), sizeof(cd) * (size_t)n * n);
    return 0;
}

// One two-site update through the reference's own MPS class: builds |+>^n, applies
// `layers` brickwork layers of the given 4x4 gates (row-major interleaved, one per
// application, cycled) with bond cap chi, then returns the max bond reached.  Used to
// time MPS::apply_adjacent / apply_zz (cuda/src/mps.cpp:41-145) on grown bonds.
int ref_grow_and_apply(int n, int chi, int layers, const double* gates, int ngates,
                       int zz_i, int zz_j, double zz_theta, int zz_reps, double* trunc_out) {
    MPS psi(n);
    double trunc = 0.0;
    int g = 0;
    for (int l = 0; l < layers; ++l)
        for (int i = l % 2; i + 1 < n; i += 2) {
            cd G[4][4];
            const double* src = gates + (size_t)32 * (g % ngates);
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 4; ++c) G[r][c] = cd(src[2 * (4 * r + c)], src[2 * (4 * r + c) + 1]);
            psi.apply_adjacent(i, G, chi, trunc);
            ++g;
        }
    for (int r = 0; r < zz_reps; ++r) psi.apply_zz(zz_i, zz_j, zz_theta, chi, trunc);
    if (trunc_out) *trunc_out = trunc;
    return psi.max_bond();
}

// One saturated-bond update through the reference's own MPS::apply_adjacent
// (cuda/src/mps.cpp:41-100): a 4-site MPS with bond dimensions (1, chi, chi, chi, 1) filled
// with seeded Gaussian complex entries, then `reps` updates of the interior bond (1, 2) --
// theta is (2 chi) x (2 chi) -- with the ZZ gate exp(-i 0.3 Z Z) and cap chi, alternating
// with a SWAP so that the bond stays saturated.  Writes the wall time of each update to
// seconds[reps] and returns the bond dimension after the last one.
int ref_saturated_update(int chi, int reps, unsigned long long seed, double* seconds, double* trunc_out) {
    MPS psi(4);
    std::mt19937_64 g(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    const int dims[5] = {1, chi, chi, chi, 1};
    for (int i = 0; i < 4; ++i) {
        Site st(dims[i], dims[i + 1]);
        const double sc = 1.0 / std::sqrt(2.0 * dims[i]);
        for (auto& z : st.t) z = cd(nd(g) * sc, nd(g) * sc);
        psi.s_[i] = st;
    }
    cd Z[4][4] = {}, W[4][4] = {};
    const cd ph = std::exp(cd(0, -0.3)), phc = std::exp(cd(0, 0.3));
    Z[0][0] = ph; Z[1][1] = phc; Z[2][2] = phc; Z[3][3] = ph;
    W[0][0] = 1; W[1][2] = 1; W[2][1] = 1; W[3][3] = 1;
    double trunc = 0.0;
    for (int r = 0; r < reps; ++r) {
        const auto t0 = std::chrono::steady_clock::now();
        psi.apply_adjacent(1, (r % 2) ? W : Z, chi, trunc);
        seconds[r] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    if (trunc_out) *trunc_out = trunc;
    return psi.s_[1].Dr;
}

}  // extern "C"
