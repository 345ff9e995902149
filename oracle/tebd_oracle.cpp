// tebd_oracle.cpp -- CPU FP64 oracle.  TEST INFRASTRUCTURE ONLY: loaded by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker; never linked
// into or called by the product library.
//
// Three independent restatements, each citing the reference it follows:
//   1. mps_*  : the reference MPS-TEBD anneal (cuda/src/mps.cpp:9-381) on top of the
//               reference's dense kernels (cuda/src/linalg.cpp:7-197): cyclic Jacobi on a
//               real symmetric matrix, complex Hermitian eig through the real 2n
//               embedding, thin SVD through the smaller Gram matrix, Hermitian exp.
//               The steps (sweep order, thresholds, sort, de-dup, keep rule, gauge) are
//               kept alike on purpose so this restatement agrees with the reference to
//               rounding; it is pinned against the compiled reference and against the
//               golden fixtures in tests/golden/.
//   2. sv_*   : the exact 2^n state-vector anneal of rust/src/quantum.rs:46-207, in two
//               Trotter splittings: mode 0 = quantum.rs's own (Z-phase(dt/2) X(dt)
//               Z-phase(dt/2)), mode 1 = the MPS engine's (single-site(dt/2) ZZ(dt)
//               single-site(dt/2), cuda/src/mps.cpp:309-356) so that an exact-chi MPS
//               run can be compared state-for-state.
//   3. exact_ground: brute force over 2^n spin patterns (rust/src/ising.rs:46-61,
//               cuda/tests/test_mps.cpp:27-42).
// Spin convention of the MPS engine: physical index 0 <-> spin +1 (cuda/src/mps.cpp:203,
// 370).  Dense vectors exported here use that convention: basis index x has bit i equal
// to the physical index of site i.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

namespace {

using cplx = std::complex<double>;

// ---------------------------------------------------------------------------------
// Dense kernels (restating cuda/src/linalg.cpp)
// ---------------------------------------------------------------------------------

// Cyclic two-sided Jacobi eigensolver for a real symmetric n x n matrix (row-major).
// Stops when the squared off-diagonal upper triangle drops below 1e-30 or after 100
// sweeps; pairs with |a_pq| < 1e-300 are skipped (cuda/src/linalg.cpp:7-54).
// Eigenvectors are accumulated as the columns of V.
void sym_jacobi(std::vector<double> a, std::size_t n, std::vector<double>& evals,
                std::vector<double>& V) {
    V.assign(n * n, 0.0);
    for (std::size_t i = 0; i < n; ++i) V[i * n + i] = 1.0;
    if (n == 1) {
        evals.assign(1, a[0]);
        return;
    }
    auto at = [&](std::size_t r, std::size_t c) -> double& { return a[r * n + c]; };
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (std::size_t p = 0; p < n; ++p)
            for (std::size_t q = p + 1; q < n; ++q) off += at(p, q) * at(p, q);
        if (off < 1e-30) break;
        for (std::size_t p = 0; p < n; ++p) {
            for (std::size_t q = p + 1; q < n; ++q) {
                const double apq = at(p, q);
                if (std::fabs(apq) < 1e-300) continue;
                const double zeta = (at(q, q) - at(p, p)) / (2.0 * apq);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(zeta * zeta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0);
                const double s = t * c;
                for (std::size_t k = 0; k < n; ++k) {  // columns p, q
                    const double x = at(k, p), y = at(k, q);
                    at(k, p) = c * x - s * y;
                    at(k, q) = s * x + c * y;
                }
                for (std::size_t k = 0; k < n; ++k) {  // rows p, q
                    const double x = at(p, k), y = at(q, k);
                    at(p, k) = c * x - s * y;
                    at(q, k) = s * x + c * y;
                }
                for (std::size_t k = 0; k < n; ++k) {  // eigenvectors
                    const double x = V[k * n + p], y = V[k * n + q];
                    V[k * n + p] = c * x - s * y;
                    V[k * n + q] = s * x + c * y;
                }
            }
        }
    }
    evals.resize(n);
    for (std::size_t i = 0; i < n; ++i) evals[i] = at(i, i);
}

struct Dense {  // row-major complex matrix
    std::size_t r = 0, c = 0;
    std::vector<cplx> v;
    Dense() = default;
    Dense(std::size_t rows, std::size_t cols) : r(rows), c(cols), v(rows * cols) {}
    cplx& operator()(std::size_t i, std::size_t j) { return v[i * c + j]; }
    cplx operator()(std::size_t i, std::size_t j) const { return v[i * c + j]; }
};

// Hermitian eigendecomposition through the real embedding [[Re, -Im], [Im, Re]]; each
// eigenvalue appears twice there.  Embedding eigenpairs are sorted by value, descending,
// and complex candidates top + i*bottom are accepted greedily after Gram-Schmidt against
// those already accepted, skipping any whose residual norm is below 1e-7
// (cuda/src/linalg.cpp:56-105).
void herm_eig(const Dense& H, std::vector<double>& w, Dense& U) {
    const std::size_t n = H.r, m = 2 * n;
    std::vector<double> E(m * m, 0.0);
    for (std::size_t i = 0; i < n; ++i)
        for (std::size_t j = 0; j < n; ++j) {
            const double re = H(i, j).real(), im = H(i, j).imag();
            E[i * m + j] = re;
            E[(i + n) * m + (j + n)] = re;
            E[i * m + (j + n)] = -im;
            E[(i + n) * m + j] = im;
        }
    std::vector<double> w2, V2;
    sym_jacobi(E, m, w2, V2);
    std::vector<std::size_t> order(m);
    for (std::size_t i = 0; i < m; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](std::size_t x, std::size_t y) { return w2[x] > w2[y]; });
    w.assign(n, 0.0);
    U = Dense(n, n);
    std::size_t got = 0;
    std::vector<cplx> cand(n);
    for (std::size_t t = 0; t < m && got < n; ++t) {
        const std::size_t col = order[t];
        for (std::size_t i = 0; i < n; ++i) cand[i] = cplx(V2[i * m + col], V2[(i + n) * m + col]);
        for (std::size_t p = 0; p < got; ++p) {
            cplx d(0, 0);
            for (std::size_t i = 0; i < n; ++i) d += std::conj(U(i, p)) * cand[i];
            for (std::size_t i = 0; i < n; ++i) cand[i] -= d * U(i, p);
        }
        double nn = 0.0;
        for (std::size_t i = 0; i < n; ++i) nn += std::norm(cand[i]);
        nn = std::sqrt(nn);
        if (nn < 1e-7) continue;
        for (std::size_t i = 0; i < n; ++i) U(i, got) = cand[i] / nn;
        w[got] = w2[col];
        ++got;
    }
}

// Thin SVD from the eigendecomposition of the smaller Gram matrix; the other factor is
// recovered by one matrix product divided by sigma (cuda/src/linalg.cpp:107-172).
void gram_svd(const Dense& A, Dense& U, std::vector<double>& S, Dense& Vh) {
    const std::size_t r = A.r, c = A.c, k = std::min(r, c);
    S.assign(k, 0.0);
    U = Dense(r, k);
    Vh = Dense(k, c);
    std::vector<double> w;
    Dense Q;
    if (c <= r) {
        Dense G(c, c);
        for (std::size_t i = 0; i < c; ++i)
            for (std::size_t j = 0; j < c; ++j) {
                cplx acc(0, 0);
                for (std::size_t x = 0; x < r; ++x) acc += std::conj(A(x, i)) * A(x, j);
                G(i, j) = acc;
            }
        herm_eig(G, w, Q);  // Q = V
        for (std::size_t t = 0; t < k; ++t) {
            const double sv = std::sqrt(std::max(w[t], 0.0));
            S[t] = sv;
            for (std::size_t j = 0; j < c; ++j) Vh(t, j) = std::conj(Q(j, t));
            if (sv > 1e-300)
                for (std::size_t x = 0; x < r; ++x) {
                    cplx acc(0, 0);
                    for (std::size_t j = 0; j < c; ++j) acc += A(x, j) * Q(j, t);
                    U(x, t) = acc / sv;
                }
        }
    } else {
        Dense G(r, r);
        for (std::size_t i = 0; i < r; ++i)
            for (std::size_t j = 0; j < r; ++j) {
                cplx acc(0, 0);
                for (std::size_t x = 0; x < c; ++x) acc += A(i, x) * std::conj(A(j, x));
                G(i, j) = acc;
            }
        herm_eig(G, w, Q);  // Q = U
        for (std::size_t t = 0; t < k; ++t) {
            const double sv = std::sqrt(std::max(w[t], 0.0));
            S[t] = sv;
            for (std::size_t x = 0; x < r; ++x) U(x, t) = Q(x, t);
            if (sv > 1e-300)
                for (std::size_t j = 0; j < c; ++j) {
                    cplx acc(0, 0);
                    for (std::size_t x = 0; x < r; ++x) acc += std::conj(Q(x, t)) * A(x, j);
                    Vh(t, j) = acc / sv;
                }
        }
    }
}

// Accurate thin SVD by cyclic one-sided (Hestenes) Jacobi in FP64, used by the oracle's
// "accurate" mode: the same MPS algorithm as the reference but with an SVD that does not
// square the condition number.  Columns of X (r x c, c <= r) are rotated pairwise until
// every pair satisfies |x_p^H x_q| <= 1e-15 |x_p||x_q|; sigma = column norms, sorted
// descending; V accumulates the rotations.  For c > r the transpose-conjugate is used.
void jacobi_svd(const Dense& A, Dense& U, std::vector<double>& S, Dense& Vh) {
    const bool tr = A.c > A.r;
    const std::size_t r = tr ? A.c : A.r, c = tr ? A.r : A.c;
    std::vector<cplx> X(r * c), V(c * c, cplx(0, 0));  // column-major
    for (std::size_t i = 0; i < r; ++i)
        for (std::size_t j = 0; j < c; ++j) X[j * r + i] = tr ? std::conj(A(j, i)) : A(i, j);
    for (std::size_t j = 0; j < c; ++j) V[j * c + j] = 1.0;
    for (int sweep = 0; sweep < 80; ++sweep) {
        int rot = 0;
        for (std::size_t p = 0; p + 1 < c; ++p)
            for (std::size_t q = p + 1; q < c; ++q) {
                double al = 0, be = 0;
                cplx g(0, 0);
                for (std::size_t i = 0; i < r; ++i) {
                    al += std::norm(X[p * r + i]);
                    be += std::norm(X[q * r + i]);
                    g += std::conj(X[p * r + i]) * X[q * r + i];
                }
                const double ag = std::abs(g);
                if (!(al > 1e-300 && be > 1e-300 && ag > 1e-15 * std::sqrt(al * be))) continue;
                ++rot;
                const double zeta = (be - al) / (2.0 * ag);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                const double cs = 1.0 / std::sqrt(1.0 + t * t), sn = cs * t;
                const cplx e = g / ag;
                for (std::size_t i = 0; i < r; ++i) {
                    const cplx x = X[p * r + i], y = X[q * r + i];
                    X[p * r + i] = cs * x - sn * std::conj(e) * y;
                    X[q * r + i] = sn * e * x + cs * y;
                }
                for (std::size_t i = 0; i < c; ++i) {
                    const cplx x = V[p * c + i], y = V[q * c + i];
                    V[p * c + i] = cs * x - sn * std::conj(e) * y;
                    V[q * c + i] = sn * e * x + cs * y;
                }
            }
        if (!rot) break;
    }
    std::vector<double> nr(c);
    for (std::size_t j = 0; j < c; ++j) {
        double s2 = 0;
        for (std::size_t i = 0; i < r; ++i) s2 += std::norm(X[j * r + i]);
        nr[j] = std::sqrt(s2);
    }
    std::vector<std::size_t> ord(c);
    for (std::size_t j = 0; j < c; ++j) ord[j] = j;
    std::stable_sort(ord.begin(), ord.end(), [&](std::size_t x, std::size_t y) { return nr[x] > nr[y]; });
    const std::size_t k = c;
    S.assign(k, 0.0);
    // X = Uc diag(S) Vc^H with Uc (r x k), Vc (c x k)
    Dense Uc(r, k), Vc(c, k);
    for (std::size_t t = 0; t < k; ++t) {
        const std::size_t j = ord[t];
        S[t] = nr[j];
        for (std::size_t i = 0; i < r; ++i) Uc(i, t) = nr[j] > 0 ? X[j * r + i] / nr[j] : cplx(0, 0);
        for (std::size_t i = 0; i < c; ++i) Vc(i, t) = V[j * c + i];
    }
    if (!tr) {
        U = Uc;
        Vh = Dense(k, c);
        for (std::size_t t = 0; t < k; ++t)
            for (std::size_t i = 0; i < c; ++i) Vh(t, i) = std::conj(Vc(i, t));
    } else {  // A^H = Uc S Vc^H  =>  A = Vc S Uc^H
        U = Vc;
        Vh = Dense(k, r);
        for (std::size_t t = 0; t < k; ++t)
            for (std::size_t i = 0; i < r; ++i) Vh(t, i) = std::conj(Uc(i, t));
    }
}

// exp(coeff * H) = U diag(exp(coeff w)) U^dagger (cuda/src/linalg.cpp:174-197).
Dense herm_expm(const Dense& H, cplx coeff) {
    std::vector<double> w;
    Dense U;
    herm_eig(H, w, U);
    const std::size_t n = H.r;
    Dense out(n, n);
    for (std::size_t i = 0; i < n; ++i)
        for (std::size_t j = 0; j < n; ++j) {
            cplx acc(0, 0);
            for (std::size_t k = 0; k < n; ++k) acc += U(i, k) * std::exp(coeff * w[k]) * std::conj(U(j, k));
            out(i, j) = acc;
        }
    return out;
}

// ---------------------------------------------------------------------------------
// MPS-TEBD (restating cuda/src/mps.cpp)
// ---------------------------------------------------------------------------------

// Site tensor (Dl, 2, Dr); element (a, s, b) at (a*2 + s)*Dr + b (cuda/include/mps.hpp:27-35).
struct Tensor3 {
    int dl = 1, dr = 1;
    std::vector<cplx> t;
    Tensor3() : t(2) {}
    Tensor3(int l, int r) : dl(l), dr(r), t((std::size_t)l * 2 * r) {}
    cplx& at(int a, int s, int b) { return t[((std::size_t)a * 2 + s) * dr + b]; }
    cplx at(int a, int s, int b) const { return t[((std::size_t)a * 2 + s) * dr + b]; }
};

struct Chain {
    std::vector<Tensor3> site;
    double max_trunc = 0.0;
    long long updates = 0;
    // Diagnostics of the Gram-matrix SVD (not part of the reference's outputs): the largest
    // relative reconstruction error ||U S Vh - theta|| / ||theta|| of any update, and how many
    // updates exceeded 1e-8.  The Gram route squares the condition number and its eigenvector
    // de-duplication can mix degenerate eigenvalues, so a few updates can come back wrong.
    double max_recon = 0.0;
    long long bad_updates = 0;
    int svd_mode = 0;  // 0: the reference's Gram-matrix SVD; 1: accurate one-sided Jacobi SVD
    double min_gap = 1.0;  // min over truncating updates of (S[keep-1] - S[keep]) / S[0]

    explicit Chain(int n) : site(n) {  // |+>^n (cuda/src/mps.cpp:9-17)
        const double amp = 1.0 / std::sqrt(2.0);
        for (auto& s : site) {
            s = Tensor3(1, 1);
            s.at(0, 0, 0) = amp;
            s.at(0, 1, 0) = amp;
        }
    }
    int n() const { return (int)site.size(); }

    // B(a, s', b) = sum_s G[s'][s] A(a, s, b)   (cuda/src/mps.cpp:27-37)
    void single(int i, const cplx G[2][2]) {
        Tensor3& A = site[i];
        for (int a = 0; a < A.dl; ++a)
            for (int b = 0; b < A.dr; ++b) {
                const cplx x0 = A.at(a, 0, b), x1 = A.at(a, 1, b);
                A.at(a, 0, b) = G[0][0] * x0 + G[0][1] * x1;
                A.at(a, 1, b) = G[1][0] * x0 + G[1][1] * x1;
            }
    }

    // Two-site update on bond (i, i+1) (cuda/src/mps.cpp:41-100): theta, gate, SVD,
    // keep = min(chi, k) then drop trailing sigma < 1e-14, discarded weight, A <- U,
    // C <- diag(S) Vh.
    void two_site(int i, const cplx G[4][4], int chi) {
        Tensor3& A = site[i];
        Tensor3& C = site[i + 1];
        const int dl = A.dl, dr = C.dr, mid = A.dr;
        Dense M((std::size_t)2 * dl, (std::size_t)2 * dr);
        for (int a = 0; a < dl; ++a)
            for (int b = 0; b < dr; ++b) {
                cplx t[2][2];
                for (int s1 = 0; s1 < 2; ++s1)
                    for (int s2 = 0; s2 < 2; ++s2) {
                        cplx acc(0, 0);
                        for (int c = 0; c < mid; ++c) acc += A.at(a, s1, c) * C.at(c, s2, b);
                        t[s1][s2] = acc;
                    }
                for (int r1 = 0; r1 < 2; ++r1)
                    for (int r2 = 0; r2 < 2; ++r2) {
                        cplx acc(0, 0);
                        for (int s1 = 0; s1 < 2; ++s1)
                            for (int s2 = 0; s2 < 2; ++s2) acc += G[r1 * 2 + r2][s1 * 2 + s2] * t[s1][s2];
                        M((std::size_t)a * 2 + r1, (std::size_t)r2 * dr + b) = acc;
                    }
            }
        Dense U, Vh;
        std::vector<double> S;
        if (svd_mode == 1)
            jacobi_svd(M, U, S, Vh);
        else
            gram_svd(M, U, S, Vh);
        const int k = (int)S.size();
        {
            double err = 0.0, nrm = 0.0;
            for (std::size_t x = 0; x < M.r; ++x)
                for (std::size_t y = 0; y < M.c; ++y) {
                    cplx acc(0, 0);
                    for (int t = 0; t < k; ++t) acc += U(x, t) * S[t] * Vh(t, y);
                    err += std::norm(acc - M(x, y));
                    nrm += std::norm(M(x, y));
                }
            const double rel = nrm > 0 ? std::sqrt(err / nrm) : 0.0;
            max_recon = std::max(max_recon, rel);
            if (rel > 1e-8) ++bad_updates;
        }
        double total = 0.0;
        for (double x : S) total += x * x;
        int keep = std::min(chi, k);
        while (keep > 1 && S[keep - 1] < 1e-14) --keep;
        double disc = 0.0;
        for (int t = keep; t < k; ++t) disc += S[t] * S[t];
        if (keep < k && S[0] > 0) min_gap = std::min(min_gap, (S[keep - 1] - S[keep]) / S[0]);
        if (total > 0) max_trunc = std::max(max_trunc, disc / total);
        Tensor3 An(dl, keep), Cn(keep, dr);
        for (int a = 0; a < dl; ++a)
            for (int s1 = 0; s1 < 2; ++s1)
                for (int x = 0; x < keep; ++x) An.at(a, s1, x) = U((std::size_t)a * 2 + s1, x);
        for (int x = 0; x < keep; ++x)
            for (int s2 = 0; s2 < 2; ++s2)
                for (int b = 0; b < dr; ++b) Cn.at(x, s2, b) = S[x] * Vh(x, (std::size_t)s2 * dr + b);
        A = std::move(An);
        C = std::move(Cn);
        ++updates;
    }

    // exp(-i theta Z_i Z_j) for any i != j through a swap network
    // (cuda/src/mps.cpp:105-145): swaps (k-1,k) for k = j..i+2, the gate on (i, i+1),
    // swaps back (k, k+1) for k = i+1..j-1.  Every swap is a truncated two-site update.
    void zz(int i, int j, double theta, int chi) {
        if (i > j) std::swap(i, j);
        if (i == j) return;
        cplx Z[4][4] = {}, W[4][4] = {};
        const cplx ph = std::exp(cplx(0, -theta)), phc = std::exp(cplx(0, theta));
        Z[0][0] = ph; Z[1][1] = phc; Z[2][2] = phc; Z[3][3] = ph;
        W[0][0] = 1; W[1][2] = 1; W[2][1] = 1; W[3][3] = 1;
        for (int k = j; k > i + 1; --k) two_site(k - 1, W, chi);
        two_site(i, Z, chi);
        for (int k = i + 1; k < j; ++k) two_site(k, W, chi);
    }

    // <psi| prod_{k in zs} Z_k |psi> unnormalised, left-to-right transfer
    // (cuda/src/mps.cpp:150-178).
    cplx zstring(const std::vector<int>& zs) const {
        std::vector<cplx> E(1, cplx(1, 0));
        int d = 1;
        for (int st = 0; st < n(); ++st) {
            const Tensor3& A = site[st];
            const bool z = std::find(zs.begin(), zs.end(), st) != zs.end();
            const int nb = A.dr;
            std::vector<cplx> F((std::size_t)nb * nb, cplx(0, 0));
            for (int a = 0; a < d; ++a)
                for (int ap = 0; ap < d; ++ap) {
                    const cplx e = E[(std::size_t)a * d + ap];
                    if (e == cplx(0, 0)) continue;
                    for (int s = 0; s < 2; ++s) {
                        const double f = (z && s == 1) ? -1.0 : 1.0;
                        for (int b = 0; b < nb; ++b) {
                            const cplx ket = f * A.at(a, s, b) * e;
                            if (ket == cplx(0, 0)) continue;
                            for (int bp = 0; bp < nb; ++bp) F[(std::size_t)b * nb + bp] += ket * std::conj(A.at(ap, s, bp));
                        }
                    }
                }
            E.swap(F);
            d = nb;
        }
        return E[0];
    }
    double norm2() const { return zstring({}).real(); }
    double ez(int i) const {
        const double nr = norm2();
        return nr <= 0 ? 0.0 : zstring({i}).real() / nr;
    }
    double ezz(int i, int j) const {
        const double nr = norm2();
        if (nr <= 0) return 0.0;
        std::vector<int> z = {std::min(i, j), std::max(i, j)};
        return zstring(z).real() / nr;
    }
    // |<x|psi>|^2 / <psi|psi>, spin +1 <-> physical 0 (cuda/src/mps.cpp:197-216).
    double prob(const std::vector<int8_t>& spins) const {
        std::vector<cplx> v(1, cplx(1, 0));
        for (int st = 0; st < n(); ++st) {
            const Tensor3& A = site[st];
            const int s = spins[st] > 0 ? 0 : 1;
            std::vector<cplx> w((std::size_t)A.dr, cplx(0, 0));
            for (int b = 0; b < A.dr; ++b)
                for (int a = 0; a < A.dl && a < (int)v.size(); ++a) w[b] += v[a] * A.at(a, s, b);
            v.swap(w);
        }
        const double nr = norm2();
        return nr > 0 ? std::norm(v[0]) / nr : 0.0;
    }
    // Von Neumann entropy (bits) of site i's 2x2 reduced density matrix, eigenvalues in
    // closed form clamped to [0,1], terms with lambda <= 1e-12 dropped
    // (cuda/src/mps.cpp:218-291).
    double entropy(int i) const {
        std::vector<cplx> L(1, cplx(1, 0)), R(1, cplx(1, 0));
        int dL = 1, dR = 1;
        for (int st = 0; st < i; ++st) {
            const Tensor3& A = site[st];
            std::vector<cplx> F((std::size_t)A.dr * A.dr, cplx(0, 0));
            for (int a = 0; a < dL; ++a)
                for (int ap = 0; ap < dL; ++ap) {
                    const cplx e = L[(std::size_t)a * dL + ap];
                    for (int s = 0; s < 2; ++s)
                        for (int b = 0; b < A.dr; ++b)
                            for (int bp = 0; bp < A.dr; ++bp)
                                F[(std::size_t)b * A.dr + bp] += A.at(a, s, b) * e * std::conj(A.at(ap, s, bp));
                }
            L.swap(F);
            dL = A.dr;
        }
        for (int st = n() - 1; st > i; --st) {
            const Tensor3& A = site[st];
            std::vector<cplx> F((std::size_t)A.dl * A.dl, cplx(0, 0));
            for (int b = 0; b < dR; ++b)
                for (int bp = 0; bp < dR; ++bp) {
                    const cplx e = R[(std::size_t)b * dR + bp];
                    for (int s = 0; s < 2; ++s)
                        for (int a = 0; a < A.dl; ++a)
                            for (int ap = 0; ap < A.dl; ++ap)
                                F[(std::size_t)a * A.dl + ap] += A.at(a, s, b) * e * std::conj(A.at(ap, s, bp));
                }
            R.swap(F);
            dR = A.dl;
        }
        const Tensor3& A = site[i];
        cplx rho[2][2] = {};
        for (int s = 0; s < 2; ++s)
            for (int sp = 0; sp < 2; ++sp)
                for (int a = 0; a < A.dl; ++a)
                    for (int ap = 0; ap < A.dl; ++ap)
                        for (int b = 0; b < A.dr; ++b)
                            for (int bp = 0; bp < A.dr; ++bp)
                                rho[s][sp] += L[(std::size_t)a * A.dl + ap] * A.at(a, s, b) *
                                              std::conj(A.at(ap, sp, bp)) * R[(std::size_t)b * A.dr + bp];
        const double tr = (rho[0][0] + rho[1][1]).real();
        if (tr <= 0) return 0.0;
        const double p = rho[0][0].real() / tr, q = rho[1][1].real() / tr;
        const double off2 = std::norm(rho[0][1] / tr);
        const double mid = 0.5 * (p + q);
        const double rad = std::sqrt(std::max(0.0, 0.25 * (p - q) * (p - q) + off2));
        double h = 0.0;
        for (double lam : {std::min(1.0, std::max(0.0, mid + rad)), std::min(1.0, std::max(0.0, mid - rad))})
            if (lam > 1e-12) h -= lam * std::log2(lam);
        return h;
    }
    // Dense amplitudes psi[x], bit i of x = physical index of site i.
    void dense(cplx* out) const {
        const int nn = n();
        const std::size_t dim = (std::size_t)1 << nn;
        for (std::size_t x = 0; x < dim; ++x) {
            std::vector<cplx> v(1, cplx(1, 0));
            for (int st = 0; st < nn; ++st) {
                const Tensor3& A = site[st];
                const int s = (int)((x >> st) & 1);
                std::vector<cplx> w((std::size_t)A.dr, cplx(0, 0));
                for (int b = 0; b < A.dr; ++b)
                    for (int a = 0; a < A.dl; ++a) w[b] += v[a] * A.at(a, s, b);
                v.swap(w);
            }
            out[x] = v[0];
        }
    }
    int max_bond() const {
        int m = 1;
        for (const auto& s : site) m = std::max(m, s.dr);
        return m;
    }
};

// Single-site half-step gate exp(-i dt/2 g), g = [[-B h, -A], [-A, B h]]
// (cuda/src/mps.cpp:312-322), built with the Hermitian exponential as the reference does.
void half_gate(double A, double B, double hi, double dt, cplx G[2][2]) {
    Dense g(2, 2);
    g(0, 0) = cplx(-B * hi, 0);
    g(1, 1) = cplx(B * hi, 0);
    g(0, 1) = cplx(-A, 0);
    g(1, 0) = cplx(-A, 0);
    Dense U = herm_expm(g, cplx(0, -1) * (dt / 2.0));
    G[0][0] = U(0, 0); G[0][1] = U(0, 1); G[1][0] = U(1, 0); G[1][1] = U(1, 1);
}

double ising_energy(const std::vector<int8_t>& s, const double* h, int n, const int* ei,
                    const int* ej, const double* ew, int m) {
    double e = 0.0;
    for (int k = 0; k < m; ++k) e -= ew[k] * s[ei[k]] * s[ej[k]];
    for (int i = 0; i < n; ++i) e -= h[i] * s[i];
    return e;
}

}  // namespace

extern "C" {

// Full MPS anneal (cuda/src/mps.cpp:295-381).  svd_mode 0 = the reference's Gram SVD
// (bitwise the reference), 1 = accurate one-sided Jacobi SVD (same algorithm otherwise).  stats = {energy, expected_energy, prob,
// max_trunc, two_site_updates, max_bond, max SVD reconstruction error, updates with a
// reconstruction error above 1e-8, norm2, min relative gap at the truncation cut}.  out_state: optional 2^n interleaved dense
// final state (unnormalised, as the MPS holds it).
int orc_mps_anneal(const double* h, int n, const int* ei, const int* ej, const double* ew, int m,
                   const double* sa, const double* sb, int steps, double dt, int chi,
                   int zz_substeps, int8_t* out_spins, double* out_entropy, double* stats,
                   double* out_state, int svd_mode) {
    Chain psi(n);
    psi.svd_mode = svd_mode;
    for (int k = 0; k < steps; ++k) {
        const double A = sa[k], B = sb[k];
        for (int i = 0; i < n; ++i) {
            cplx G[2][2];
            half_gate(A, B, h[i], dt, G);
            psi.single(i, G);
        }
        const int ns = zz_substeps < 1 ? 1 : zz_substeps;
        const double sub = dt / ns;
        for (int s = 0; s < ns; ++s) {
            if (s % 2 == 0)
                for (int e = 0; e < m; ++e) psi.zz(ei[e], ej[e], -B * ew[e] * sub, chi);
            else
                for (int e = m - 1; e >= 0; --e) psi.zz(ei[e], ej[e], -B * ew[e] * sub, chi);
        }
        for (int i = 0; i < n; ++i) {
            cplx G[2][2];
            half_gate(A, B, h[i], dt, G);
            psi.single(i, G);
        }
        if (out_entropy) out_entropy[k] = psi.entropy(0);
    }
    double eexp = 0.0;
    for (int e = 0; e < m; ++e) eexp -= ew[e] * psi.ezz(ei[e], ej[e]);
    for (int i = 0; i < n; ++i) eexp -= h[i] * psi.ez(i);
    std::vector<int8_t> spins(n, 1);
    for (int i = 0; i < n; ++i) spins[i] = psi.ez(i) >= 0.0 ? 1 : -1;
    for (int i = 0; i < n; ++i) out_spins[i] = spins[i];
    stats[0] = ising_energy(spins, h, n, ei, ej, ew, m);
    stats[1] = eexp;
    stats[2] = psi.prob(spins);
    stats[3] = psi.max_trunc;
    stats[4] = (double)psi.updates;
    stats[5] = (double)psi.max_bond();
    stats[6] = psi.max_recon;
    stats[7] = (double)psi.bad_updates;
    stats[8] = psi.norm2();
    stats[9] = psi.min_gap;
    if (out_state) psi.dense(reinterpret_cast<cplx*>(out_state));
    return 0;
}

// Gate slots [q0, q1) of one step's ZZ block applied to a given MPS.  The slots are the
// two-site updates of the block in the reference's order: edges in list order (reverse order
// on odd substeps, cuda/src/mps.cpp:330-341), each through the swap network of
// cuda/src/mps.cpp:126-145 (swaps on bonds k-1 for k = j..i+2, the ZZ gate on bond i, swaps back
// on bonds k for k = i+1..j-1), the ZZ angle -B w dt/ns.  Every slot is apply_adjacent
// (cuda/src/mps.cpp:41-100): keep rule, discarded weight and gauge A <- U, C <- S Vh.
// dims: n+1 bond dimensions; sites: the n site tensors (Dl, 2, Dr) back to back, interleaved
// complex, element (a, s, b) at (a*2 + s)*Dr + b -- the payload of the engine's checkpoint.
// Writes the updated dims and sites (out_cap doubles available; returns -1 when too small,
// else the number of doubles written).  stats = {max_trunc, updates, min relative cut gap,
// max SVD reconstruction error}.
long long orc_mps_apply_slots(int n, const int* dims, const double* sites, const int* ei, const int* ej,
                              const double* ew, int m, double B, double dt, int zz_substeps, int chi,
                              int q0, int q1, int svd_mode, int* out_dims, double* out_sites,
                              long long out_cap, double* stats) {
    Chain psi(n);
    psi.svd_mode = svd_mode;
    size_t off = 0;
    for (int i = 0; i < n; ++i) {
        Tensor3 t(dims[i], dims[i + 1]);
        for (size_t e = 0; e < t.t.size(); ++e, ++off) t.t[e] = cplx(sites[2 * off], sites[2 * off + 1]);
        psi.site[i] = std::move(t);
    }
    struct Slot { int bond; bool zz; double theta; };
    std::vector<Slot> slots;
    const int ns = zz_substeps < 1 ? 1 : zz_substeps;
    const double sub = dt / ns;
    for (int sstep = 0; sstep < ns; ++sstep)
        for (int q = 0; q < m; ++q) {
            const int e = (sstep % 2 == 0) ? q : m - 1 - q;
            int i = ei[e], j = ej[e];
            if (i > j) std::swap(i, j);
            if (i == j) continue;
            const double th = -B * ew[e] * sub;
            for (int k = j; k > i + 1; --k) slots.push_back({k - 1, false, 0.0});
            slots.push_back({i, true, th});
            for (int k = i + 1; k < j; ++k) slots.push_back({k, false, 0.0});
        }
    if (q0 < 0 || q1 > (int)slots.size() || q0 > q1) return -2;
    cplx W[4][4] = {};
    W[0][0] = 1; W[1][2] = 1; W[2][1] = 1; W[3][3] = 1;
    for (int q = q0; q < q1; ++q) {
        const Slot& sl = slots[q];
        if (sl.zz) {
            cplx Z[4][4] = {};
            const cplx ph = std::exp(cplx(0, -sl.theta)), phc = std::exp(cplx(0, sl.theta));
            Z[0][0] = ph; Z[1][1] = phc; Z[2][2] = phc; Z[3][3] = ph;
            psi.two_site(sl.bond, Z, chi);
        } else {
            psi.two_site(sl.bond, W, chi);
        }
    }
    long long need = 0;
    for (int i = 0; i < n; ++i) need += 2LL * (long long)psi.site[i].t.size();
    if (need > out_cap) return -1;
    out_dims[0] = 1;
    size_t o = 0;
    for (int i = 0; i < n; ++i) {
        out_dims[i + 1] = psi.site[i].dr;
        for (const cplx& z : psi.site[i].t) { out_sites[o++] = z.real(); out_sites[o++] = z.imag(); }
    }
    stats[0] = psi.max_trunc;
    stats[1] = (double)psi.updates;
    stats[2] = psi.min_gap;
    stats[3] = psi.max_recon;
    return need;
}

// Gram-matrix thin SVD restatement (cuda/src/linalg.cpp:107-172); row-major interleaved.
int orc_svd(int rows, int cols, const double* a, double* s, double* u, double* vh) {
    Dense A(rows, cols);
    for (int i = 0; i < rows * cols; ++i) A.v[i] = cplx(a[2 * i], a[2 * i + 1]);
    Dense U, Vh;
    std::vector<double> S;
    gram_svd(A, U, S, Vh);
    const int k = (int)S.size();
    for (int t = 0; t < k; ++t) s[t] = S[t];
    if (u) std::memcpy(u, U.v.data(), sizeof(cplx) * (size_t)rows * k);
    if (vh) std::memcpy(vh, Vh.v.data(), sizeof(cplx) * (size_t)k * cols);
    return k;
}

int orc_hermitian_eig(int n, const double* a, double* w, double* v) {
    Dense H(n, n);
    for (int i = 0; i < n * n; ++i) H.v[i] = cplx(a[2 * i], a[2 * i + 1]);
    std::vector<double> ev;
    Dense U;
    herm_eig(H, ev, U);
    for (int i = 0; i < n; ++i) w[i] = ev[i];
    std::memcpy(v, U.v.data(), sizeof(cplx) * (size_t)n * n);
    return 0;
}

int orc_hermitian_expm(int n, const double* a, double cre, double cim, double* out) {
    Dense H(n, n);
    for (int i = 0; i < n * n; ++i) H.v[i] = cplx(a[2 * i], a[2 * i + 1]);
    Dense E = herm_expm(H, cplx(cre, cim));
    std::memcpy(out, E.v.data(), sizeof(cplx) * (size_t)n * n);
    return 0;
}

// Brute-force ground state (rust/src/ising.rs:46-61): bit b set <-> spin +1, first
// minimum kept.
double orc_exact_ground(const double* h, int n, const int* ei, const int* ej, const double* ew,
                        int m, int8_t* out_spins) {
    double best = INFINITY;
    std::vector<int8_t> s(n), bs(n, 1);
    const long long dim = 1LL << n;
    for (long long x = 0; x < dim; ++x) {
        for (int i = 0; i < n; ++i) s[i] = ((x >> i) & 1) ? 1 : -1;
        const double e = ising_energy(s, h, n, ei, ej, ew, m);
        if (e < best) { best = e; bs = s; }
    }
    if (out_spins) for (int i = 0; i < n; ++i) out_spins[i] = bs[i];
    return best;
}

// Best-of-restarts simulated annealing (rust/src/ising.rs:64-136: sa_run, simulated_annealing,
// sa_solve): random start; sweep k at t0 (t_end/t0)^(k/(max(sweeps,2)-1)); spins 0..n-1 in order,
// flip when dE = 2 s_i (h_i + sum_j J_ij s_j) < 0 or u < exp(-dE/t); energy of the final pattern
// (Ising::energy, rust/src/ising.rs:23-32); the lowest over restarts, the first on ties.  The
// uniforms follow the library's counter-based stream (splitmix64's finaliser over the counter
// (seed, instance, restart, sweep, spin); the start pattern uses sweep = sweeps), so the GPU
// solver can be checked against this one draw for draw; the reference's StdRng stream is not
// reproducible without its Rust crate.  Fields are summed over each spin's neighbours in the
// order the edge list lists them.
static double sa_u(uint64_t seed, uint64_t inst, uint64_t r, uint64_t k, uint64_t i, uint64_t sweeps, uint64_t n) {
    uint64_t x = seed + 0x9E3779B97F4A7C15ull * ((((inst * 0x100000001B3ull + r) * (sweeps + 1) + k) * n + i) + 1);
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x ^= x >> 31;
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

double orc_sa_solve(const double* h, int n, const int* ei, const int* ej, const double* ew, int m,
                    int restarts, int sweeps, double t0, double t_end, uint64_t seed, uint64_t inst,
                    int8_t* out_spins) {
    std::vector<std::vector<std::pair<int, double>>> adj(n);
    for (int e = 0; e < m; ++e) {
        if (ei[e] == ej[e]) continue;
        adj[ei[e]].push_back({ej[e], ew[e]});
        adj[ej[e]].push_back({ei[e], ew[e]});
    }
    const double den = (double)((sweeps < 2 ? 2 : sweeps) - 1);
    double best = INFINITY;
    std::vector<int8_t> s(n), bs(n, 1);
    for (int r = 0; r < restarts; ++r) {
        for (int i = 0; i < n; ++i) s[i] = sa_u(seed, inst, r, sweeps, i, sweeps, n) < 0.5 ? -1 : 1;
        for (int k = 0; k < sweeps; ++k) {
            const double t = t0 * std::pow(t_end / t0, (double)k / den);
            for (int i = 0; i < n; ++i) {
                double f = h[i];
                for (auto& pr : adj[i]) f += s[pr.first] < 0 ? -pr.second : pr.second;
                const double de = 2.0 * (s[i] < 0 ? -f : f);
                if (de < 0.0 || sa_u(seed, inst, r, k, i, sweeps, n) < std::exp(-de / t)) s[i] = -s[i];
            }
        }
        const double e = ising_energy(s, h, n, ei, ej, ew, m);
        if (e < best) { best = e; bs = s; }
    }
    if (out_spins) for (int i = 0; i < n; ++i) out_spins[i] = bs[i];
    return best;
}

// Exact state-vector anneal.  mode 0 restates rust/src/quantum.rs:63-112 exactly
// (diag phase b dt/2, Prod exp(+i a dt X), diag phase b dt/2; basis bit set <-> +1);
// mode 1 uses the MPS engine's splitting (exp(-i dt/2 g_i) per site, ZZ phases for dt,
// again the single-site half step; cuda/src/mps.cpp:309-356).
// stats = {argmax energy, expected energy, argmax prob, signZ energy, signZ prob}.
// out_spins_argmax: quantum.rs readout; out_spins_sign: engine's sign<Z> readout.
// out_state (optional): final amplitudes in the engine convention (bit i = physical
// index, 0 <-> +1), normalised to the evolved norm.
int orc_sv_anneal_bias(const double* h, int n, const int* ei, const int* ej, const double* ew, int m,
                       const double* sa, const double* sb, int steps, double dt, int mode,
                       int8_t* out_spins_argmax, int8_t* out_spins_sign, double* out_entropy,
                       double* stats, double* out_state, const double* bias, const double* sc);

int orc_sv_anneal(const double* h, int n, const int* ei, const int* ej, const double* ew, int m,
                  const double* sa, const double* sb, int steps, double dt, int mode,
                  int8_t* out_spins_argmax, int8_t* out_spins_sign, double* out_entropy,
                  double* stats, double* out_state) {
    return orc_sv_anneal_bias(h, n, ei, ej, ew, m, sa, sb, steps, dt, mode, out_spins_argmax, out_spins_sign,
                              out_entropy, stats, out_state, nullptr, nullptr);
}

// As orc_sv_anneal; in mode 1 an optional warm-start bias adds -C(s_k) sum_i b_i Z_i to the
// single-site term (the engine's tessera_qa_problem.bias / schedule_c extension, not part
// of the reference): g_i = -A X - (B h_i + C b_i) Z.
int orc_sv_anneal_bias(const double* h, int n, const int* ei, const int* ej, const double* ew, int m,
                       const double* sa, const double* sb, int steps, double dt, int mode,
                       int8_t* out_spins_argmax, int8_t* out_spins_sign, double* out_entropy,
                       double* stats, double* out_state, const double* bias, const double* sc) {
    const std::size_t dim = (std::size_t)1 << n;
    // Work in the engine basis: bit i = physical index s_i; spin = +1 when s_i = 0.
    std::vector<double> diag(dim);
    std::vector<int8_t> sp(n);
    for (std::size_t x = 0; x < dim; ++x) {
        for (int i = 0; i < n; ++i) sp[i] = ((x >> i) & 1) ? -1 : 1;
        diag[x] = ising_energy(sp, h, n, ei, ej, ew, m);
    }
    std::vector<cplx> psi(dim, cplx(1.0 / std::sqrt((double)dim), 0.0));
    auto phase = [&](double scale) {  // exp(-i scale diag)
        for (std::size_t x = 0; x < dim; ++x) psi[x] *= std::exp(cplx(0, -scale * diag[x]));
    };
    auto one_qubit = [&](int i, const cplx G[2][2]) {
        const std::size_t bit = (std::size_t)1 << i;
        for (std::size_t x = 0; x < dim; ++x)
            if (!(x & bit)) {
                const cplx u = psi[x], v = psi[x | bit];
                psi[x] = G[0][0] * u + G[0][1] * v;
                psi[x | bit] = G[1][0] * u + G[1][1] * v;
            }
    };
    auto ent0 = [&]() {  // rust/src/quantum.rs:138-175 (qubit 0 vs rest)
        if (n < 2) return 0.0;
        double r00 = 0, r11 = 0;
        cplx r01(0, 0);
        for (std::size_t x = 0; x < dim; x += 2) {
            r00 += std::norm(psi[x]);
            r11 += std::norm(psi[x + 1]);
            r01 += psi[x] * std::conj(psi[x + 1]);
        }
        const double tot = r00 + r11;
        if (tot <= 0) return 0.0;
        r00 /= tot; r11 /= tot;
        const double off2 = std::norm(r01) / (tot * tot);
        const double mid = 0.5 * (r00 + r11), rad = std::sqrt(0.25 * (r00 - r11) * (r00 - r11) + off2);
        double s = 0.0;
        for (double lam : {std::min(1.0, std::max(0.0, mid + rad)), std::min(1.0, std::max(0.0, mid - rad))})
            if (lam > 1e-12) s -= lam * std::log2(lam);
        return s;
    };
    for (int k = 0; k < steps; ++k) {
        const double A = sa[k], B = sb[k];
        if (mode == 0) {
            phase(B * dt * 0.5);
            const double th = A * dt;  // exp(+i th X)
            const cplx G[2][2] = {{std::cos(th), cplx(0, std::sin(th))}, {cplx(0, std::sin(th)), std::cos(th)}};
            for (int i = 0; i < n; ++i) one_qubit(i, G);
            phase(B * dt * 0.5);
        } else {
            auto gate = [&](int i, cplx G[2][2]) {  // longitudinal field B h_i (+ C b_i)
                if (bias) half_gate(A, 1.0, B * h[i] + sc[k] * bias[i], dt, G);
                else half_gate(A, B, h[i], dt, G);
            };
            for (int i = 0; i < n; ++i) { cplx G[2][2]; gate(i, G); one_qubit(i, G); }
            // ZZ block: exp(-i dt * (-B sum_e w_e z_i z_j)), exact (diagonal, commuting).
            for (std::size_t x = 0; x < dim; ++x) {
                double e = 0.0;
                for (int q = 0; q < m; ++q) {
                    const int zi = ((x >> ei[q]) & 1) ? -1 : 1, zj = ((x >> ej[q]) & 1) ? -1 : 1;
                    e -= ew[q] * zi * zj;
                }
                psi[x] *= std::exp(cplx(0, -dt * B * e));
            }
            for (int i = 0; i < n; ++i) { cplx G[2][2]; gate(i, G); one_qubit(i, G); }
        }
        if (out_entropy) out_entropy[k] = ent0();
    }
    double tot = 0, eexp = 0, bestp = -1;
    std::size_t best = 0;
    std::vector<double> ez(n, 0.0);
    for (std::size_t x = 0; x < dim; ++x) {
        const double p = std::norm(psi[x]);
        tot += p;
        eexp += p * diag[x];
        if (p > bestp) { bestp = p; best = x; }
        for (int i = 0; i < n; ++i) ez[i] += ((x >> i) & 1) ? -p : p;
    }
    for (int i = 0; i < n; ++i) out_spins_argmax[i] = ((best >> i) & 1) ? -1 : 1;
    std::size_t xs = 0;
    for (int i = 0; i < n; ++i) {
        const int8_t s = (ez[i] / tot >= 0.0) ? 1 : -1;
        out_spins_sign[i] = s;
        if (s < 0) xs |= (std::size_t)1 << i;
    }
    stats[0] = diag[best];
    stats[1] = eexp / tot;
    stats[2] = bestp / tot;
    stats[3] = diag[xs];
    stats[4] = std::norm(psi[xs]) / tot;
    if (out_state) std::memcpy(out_state, psi.data(), sizeof(cplx) * dim);
    return 0;
}

// Instances of cuda/tests/test_mps.cpp:99-111 / :159-167: std::mt19937_64(seed),
// U(-1,1); h_i = U; for i<j: if U > 0 add edge (i, j, U).  Several trials in sequence
// from one generator.  Returns the edge count of trial `want`.
int orc_mt_dense_instance(unsigned long long seed, int n, int trials, int want, double* h,
                          int* ei, int* ej, double* ew, int max_edges) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    int m = 0;
    for (int t = 0; t < trials; ++t) {
        std::vector<double> hh(n);
        for (auto& x : hh) x = U(rng);
        std::vector<int> a, b;
        std::vector<double> w;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j)
                if (U(rng) > 0.0) { a.push_back(i); b.push_back(j); w.push_back(U(rng)); }
        if (t == want) {
            for (int i = 0; i < n; ++i) h[i] = hh[i];
            m = (int)w.size();
            if (m > max_edges) return -1;
            for (int k = 0; k < m; ++k) { ei[k] = a[k]; ej[k] = b[k]; ew[k] = w[k]; }
        }
    }
    return m;
}

}  // extern "C"
