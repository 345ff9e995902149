"""The freeze rules of the one-sided Jacobi, on the numpy model of the kernels (tests/jacobi_model.py).

Rule A (the kernels: a column under the noise floor is never rotated again) lets a column
whose norm dips under the floor mid-sweep stay frozen, so singular values a few times the
floor come back wrong.  Rule F (rotate every pair with one column above the floor while a
sweep still rotates >= 10% of its pairs, then rule A) resolves them at the same sweep count.
"""
import numpy as np
import pytest

from jacobi_model import graded, one_sided_jacobi, pivoted_lq, pivoted_lq_blocked, tournament_jacobi


@pytest.fixture(scope="module")
def runs():
    A, s = graded(96, 2.5, 7)
    return s, {rule: one_sided_jacobi(A, rule) for rule in ("A", "F")}


def _rel_err_above(s, sig, floor, k=4.0):
    keep = s > k * floor
    return float(np.max(np.abs(sig[keep] - s[keep]) / s[keep]))


def test_rule_a_loses_values_above_the_floor(runs):
    s, r = runs
    sig, _, _, floor = r["A"]
    assert _rel_err_above(s, sig, floor) > 1e-3


def test_rule_f_resolves_them_at_the_same_cost(runs):
    s, r = runs
    sig_f, W, sweeps_f, floor = r["F"]
    _, _, sweeps_a, _ = r["A"]
    assert _rel_err_above(s, sig_f, floor) < 1e-4
    assert np.max(np.abs(sig_f - s)) < floor  # everything else within the floor
    assert sweeps_f <= sweeps_a + 2
    kept = sig_f > floor
    U = W[:, kept] / sig_f[kept]
    assert np.linalg.norm(U.conj().T @ U - np.eye(U.shape[1])) < 1e-10


def test_model_rotation_matches_the_textbook_form():
    rng = np.random.default_rng(3)
    from jacobi_model import rotation
    for _ in range(200):
        v0, v1 = 10 ** rng.uniform(-3, 3, 2)
        g = np.sqrt(v0 * v1) * 10 ** rng.uniform(-6, 0)
        ph = rng.uniform(0, 2 * np.pi)
        c, s, e = rotation(v0, v1, g * np.cos(ph), g * np.sin(ph))
        zeta = 0.5 * (v1 - v0) / g
        t = np.sign(zeta if zeta != 0 else 1.0) / (abs(zeta) + np.sqrt(1 + zeta * zeta))
        assert c == pytest.approx(1 / np.sqrt(1 + t * t), rel=1e-14)
        assert s == pytest.approx(t / np.sqrt(1 + t * t), rel=1e-13, abs=1e-300)


def test_pivoted_lq_preconditioner_cuts_sweeps_on_a_graded_spectrum():
    """The batched Jacobi's preconditioner (lq.cu): P L equals A times a unitary (so the Jacobi on it
    gives A's singular values and, as W / sigma, A's left singular vectors in A's row order), L is
    lower trapezoidal in pivot order, and on a graded spectrum (values falling by 1e-10 over 96
    columns) the Jacobi on P L takes far fewer sweeps than on A."""
    A, s = graded(96, 4.0, 11)
    X = pivoted_lq(A)
    assert np.linalg.norm(X @ X.conj().T - A @ A.conj().T) < 1e-14 * np.linalg.norm(A) ** 2
    # row-pivot order: each row of P L has at most one more nonzero than the one pivoted before it
    nnz = sorted(int(np.max(np.flatnonzero(np.abs(r) > 0))) + 1 for r in X if np.any(np.abs(r) > 0))
    assert nnz == list(range(1, len(nnz) + 1))
    sig_a, _, sweeps_a, floor = one_sided_jacobi(A, "F")
    sig_x, W, sweeps_x, _ = one_sided_jacobi(X, "F")
    # absolute accuracy under the noise floor, as good as the Jacobi on A itself
    assert np.max(np.abs(sig_x - s)) < floor
    assert np.max(np.abs(sig_x - s)) <= 2 * np.max(np.abs(sig_a - s))
    assert sweeps_x * 2 <= sweeps_a, (sweeps_x, sweeps_a)  # observed 6 against 16
    # U = W / sigma spans A's leading left singular subspace
    U = W[:, :8] / sig_x[:8]
    Ua = np.linalg.svd(A)[0][:, :8]
    assert np.linalg.norm(Ua.conj().T @ U, 2) == pytest.approx(1.0, abs=1e-10)
    assert np.linalg.svd(Ua.conj().T @ U, compute_uv=False).min() > 1 - 1e-10


def test_pivoted_lq_of_wide_and_tall_matrices():
    rng = np.random.default_rng(5)
    for R, N in ((24, 40), (40, 24)):
        A = rng.normal(size=(R, N)) + 1j * rng.normal(size=(R, N))
        X = pivoted_lq(A)
        assert np.linalg.norm(X @ X.conj().T - A @ A.conj().T) < 1e-13 * np.linalg.norm(A) ** 2
        if N > R:
            assert np.all(X[:, R:] == 0)  # the Jacobi runs on min(R, N) columns


def test_blocked_lq_is_the_same_factorisation():
    """The panel-blocked form the kernel runs (updates delayed over 8 steps, products corrected
    for the pending updates) gives the same P L as the step-by-step LQ, to rounding, on square,
    wide, tall and rank-deficient matrices, with panels that end inside and at kmax."""
    rng = np.random.default_rng(8)
    for R, N, b in ((64, 64, 8), (40, 72, 8), (72, 40, 8), (33, 17, 4), (50, 50, 7)):
        A = rng.normal(size=(R, N)) + 1j * rng.normal(size=(R, N))
        if (R, N) == (50, 50):
            U, _, Vh = np.linalg.svd(A)
            A = (U[:, :20] * np.exp(-np.arange(20) / 3.0)) @ Vh[:20]  # rank 20
        Xb, Xr = pivoted_lq_blocked(A, b), pivoted_lq(A)
        scale = np.linalg.norm(A) ** 2
        assert np.linalg.norm(Xb @ Xb.conj().T - A @ A.conj().T) < 1e-13 * scale
        if (R, N) != (50, 50):  # full rank: the same pivots, so the same factor
            assert np.max(np.abs(Xb - Xr)) < 1e-12 * np.sqrt(scale)


def test_lq_preconditioner_in_the_cooperative_tournament_order():
    """The single-instance engine's Jacobi visits pairs in a block tournament without norm
    ordering; there the pivoted LQ cuts the sweeps by more than half, on a graded spectrum and on
    a product of two Gaussian matrices (the bench's random MPS form theta that way).  Observed at
    64 columns: 23 -> 8 and 22 -> 8; on the GPU at 512 rows the bench went 23.5 -> 11.3."""
    rng = np.random.default_rng(2)
    G = lambda r, c: rng.normal(size=(r, c)) + 1j * rng.normal(size=(r, c))
    for A in (graded(64, 4.0, 11)[0], G(64, 32) @ G(32, 64)):
        plain, pre = tournament_jacobi(A), tournament_jacobi(pivoted_lq(A))
        assert 2 * pre <= plain, (pre, plain)
