// Host sanitizer run of the oracle (test infrastructure only): builds with
// -fsanitize=address,undefined -fno-sanitize-recover=all (`make -C oracle sanitize`) and drives
// every extern "C" entry point of tebd_oracle.cpp on small inputs -- both SVD modes, a
// truncating chain with the swap network, the state vector in both splittings with and
// without the bias field, the Hermitian helpers, the brute-force ground state and the
// mt19937_64 instance generator.  Any out-of-bounds access, leak or undefined behaviour ends
// the process with a non-zero status; a clean run prints "sanitize ok" and exits 0.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>

extern "C" {
int orc_mps_anneal(const double* h, int n, const int* ei, const int* ej, const double* ew, int m, const double* sa,
                   const double* sb, int steps, double dt, int chi, int zz_substeps, int8_t* out_spins,
                   double* out_entropy, double* stats, double* out_state, int svd_mode);
int orc_svd(int rows, int cols, const double* a, double* s, double* u, double* vh);
int orc_hermitian_eig(int n, const double* a, double* w, double* v);
int orc_hermitian_expm(int n, const double* a, double cre, double cim, double* out);
double orc_exact_ground(const double* h, int n, const int* ei, const int* ej, const double* ew, int m,
                        int8_t* out_spins);
int orc_sv_anneal_bias(const double* h, int n, const int* ei, const int* ej, const double* ew, int m,
                       const double* sa, const double* sb, int steps, double dt, int mode, int8_t* out_spins_argmax,
                       int8_t* out_spins_sign, double* out_entropy, double* stats, double* out_state,
                       const double* bias, const double* sc);
int orc_mt_dense_instance(unsigned long long seed, int n, int trials, int want, double* h, int* ei, int* ej,
                          double* ew, int max_edges);
}

static int fail(const char* what) {
    std::fprintf(stderr, "sanitize: %s\n", what);
    return 1;
}

int main() {
    // the reference's n=6 dense test instance (mt19937_64(123), first trial)
    const int n = 6, cap = n * (n - 1) / 2;
    std::vector<double> h(n), ew(cap);
    std::vector<int> ei(cap), ej(cap);
    const int m = orc_mt_dense_instance(123, n, 1, 0, h.data(), ei.data(), ej.data(), ew.data(), cap);
    if (m <= 0) return fail("instance generator");
    const int steps = 12;
    std::vector<double> sa(steps), sb(steps);
    for (int k = 0; k < steps; ++k) {
        const double s = (double)k / (steps - 1);
        sa[k] = 1.0 - s;
        sb[k] = s;
    }
    std::vector<int8_t> spins(n), spins2(n);
    std::vector<double> ent(steps), stats(10), state(2 << n);
    for (int svd_mode = 0; svd_mode < 2; ++svd_mode)
        for (int chi : {2, 8})
            for (int zz : {1, 2}) {
                if (orc_mps_anneal(h.data(), n, ei.data(), ej.data(), ew.data(), m, sa.data(), sb.data(), steps, 0.1,
                                   chi, zz, spins.data(), ent.data(), stats.data(), state.data(), svd_mode) != 0)
                    return fail("mps_anneal");
                if (!std::isfinite(stats[0])) return fail("mps_anneal energy");
            }
    std::vector<double> bias(n, 0.3), sc(steps, 0.2);
    std::vector<double> st5(5);
    for (int mode = 0; mode < 2; ++mode) {
        if (orc_sv_anneal_bias(h.data(), n, ei.data(), ej.data(), ew.data(), m, sa.data(), sb.data(), steps, 0.1, mode,
                               spins.data(), spins2.data(), ent.data(), st5.data(), state.data(), nullptr,
                               nullptr) != 0)
            return fail("sv_anneal");
    }
    if (orc_sv_anneal_bias(h.data(), n, ei.data(), ej.data(), ew.data(), m, sa.data(), sb.data(), steps, 0.1, 1,
                           spins.data(), spins2.data(), ent.data(), st5.data(), nullptr, bias.data(), sc.data()) != 0)
        return fail("sv_anneal with bias");
    // n = 1: no bonds, no entropy pairs
    {
        const double h1 = 1.0;
        std::vector<int8_t> s1(1), s2(1);
        if (orc_sv_anneal_bias(&h1, 1, nullptr, nullptr, nullptr, 0, sa.data(), sb.data(), steps, 0.1, 0, s1.data(),
                               s2.data(), ent.data(), st5.data(), nullptr, nullptr, nullptr) != 0)
            return fail("sv_anneal n=1");
        if (orc_mps_anneal(&h1, 1, nullptr, nullptr, nullptr, 0, sa.data(), sb.data(), steps, 0.1, 4, 1, s1.data(),
                           ent.data(), stats.data(), nullptr, 1) != 0)
            return fail("mps_anneal n=1");
    }
    // SVDs: square, tall, wide, rank-deficient (a repeated column)
    static const int shapes[4][2] = {{5, 5}, {7, 3}, {3, 7}, {6, 4}};
    for (const auto& sh : shapes) {
        const int r = sh[0], c = sh[1], k = r < c ? r : c;
        std::vector<double> a(2 * r * c), s(k), u(2 * r * k), vh(2 * k * c);
        for (int i = 0; i < 2 * r * c; ++i) a[i] = std::sin(0.7 * i + 0.3);
        if (r == 6)
            for (int i = 0; i < r; ++i) {
                a[2 * (i * c + 1)] = a[2 * (i * c)];
                a[2 * (i * c + 1) + 1] = a[2 * (i * c) + 1];
            }
        if (orc_svd(r, c, a.data(), s.data(), u.data(), vh.data()) != k) return fail("svd");
    }
    {
        const double a[8] = {1.0, 0.0, 0.5, -0.25, 0.5, 0.25, -2.0, 0.0};  // 2x2 Hermitian
        double w[2], v[8], e[8];
        if (orc_hermitian_eig(2, a, w, v) != 0) return fail("hermitian_eig");
        if (orc_hermitian_expm(2, a, 0.0, -0.05, e) != 0) return fail("hermitian_expm");
    }
    if (!std::isfinite(orc_exact_ground(h.data(), n, ei.data(), ej.data(), ew.data(), m, spins.data())))
        return fail("exact_ground");
    std::printf("sanitize ok\n");
    return 0;
}
