"""A numpy model of the engine's one-sided Jacobi SVD, for CPU experiments on its rules.

It restates what tessera_b200/csrc/kernels.cu does per column pair: FP64 sums alpha = |x|^2,
beta = |y|^2, gamma = x^H y; the convergence test |gamma|^2 > tol^2 alpha beta; the noise floor
tiny = (8 sqrt(R) eps)^2 ||A||_F^2 under which a column is frozen; the complex128 rotation of
jacobi_rotation (u = (|beta - alpha| + sqrt((beta - alpha)^2 + 4|gamma|^2)) / (2|gamma|),
c = u w, s = sgn(zeta) w, w = 1/sqrt(u^2 + 1)); and the update x' = c x - s conj(e) y,
y' = s e x + c y with e = gamma/|gamma|.  Columns are put in descending norm order at every
sweep and visited in row-cyclic order, as the batched kernel does (it groups them in blocks of
8, which changes the order of the pairs but not the rules).

freeze rules:
  "A": skip a pair when either column is under the floor;
  "C": skip only pairs with both columns under the floor;
  "F" (the kernels): while a sweep still rotates at least 10% of its pairs, and for at most
       8 + 3 log2(N) sweeps, rotate a pair when one column is above the floor and the other
       holds more than 1e-6 of it; then A.
"""
from __future__ import annotations

import numpy as np

EPS64 = 2.220446049250313e-16


def rotation(v0, v1, v2, v3):
    g2 = v2 * v2 + v3 * v3
    rg = 1.0 / np.sqrt(g2)
    zeta = 0.5 * (v1 - v0) * rg
    d = v1 - v0
    u = 0.5 * rg * (abs(d) + np.sqrt(d * d + 4.0 * g2))
    w = 1.0 / np.sqrt(u * u + 1.0)
    return u * w, (w if zeta >= 0 else -w), complex(v2 * rg, v3 * rg)


def one_sided_jacobi(A: np.ndarray, rule: str = "A", tol: float = 1e-13, max_sweeps: int = 60):
    """Returns (sigma descending, W with columns in the same order, sweeps, floor)."""
    W = np.array(A, dtype=np.complex128, copy=True)
    R, N = W.shape
    fro2 = float(np.sum(np.abs(W) ** 2))
    tiny = max(1e-200, (8.0 * np.sqrt(R) * EPS64) ** 2 * fro2)
    late = rule == "A"
    sweeps = max_sweeps
    for sweep in range(max_sweeps):
        W = W[:, np.argsort(-np.sum(np.abs(W) ** 2, axis=0), kind="stable")]
        rot = 0
        for i in range(N - 1):
            for j in range(i + 1, N):
                x, y = W[:, i], W[:, j]
                v0 = float(np.vdot(x, x).real)
                v1 = float(np.vdot(y, y).real)
                g = np.vdot(x, y)
                v2, v3 = float(g.real), float(g.imag)
                if late or rule == "A":
                    if not (v0 > tiny and v1 > tiny):
                        continue
                elif rule == "C":
                    if not (v0 > tiny or v1 > tiny):
                        continue
                elif not (max(v0, v1) > tiny and min(v0, v1) > 1e-6 * tiny):
                    continue
                if not (v2 * v2 + v3 * v3 > tol * tol * v0 * v1):
                    continue
                c, s, e = rotation(v0, v1, v2, v3)
                xn = c * x - s * np.conj(e) * y  # both from the old columns (x, y are views)
                yn = s * e * x + c * y
                W[:, i] = xn
                W[:, j] = yn
                rot += 1
        if rule == "F" and not late and (rot < 0.1 * N * (N - 1) / 2 or sweep + 1 >= 8 + 3 * int(np.ceil(np.log2(N)))):
            late = True
            if rot:
                continue
        if rot == 0:
            sweeps = sweep + 1
            break
    sig = np.sqrt(np.sum(np.abs(W) ** 2, axis=0))
    order = np.argsort(-sig, kind="stable")
    return sig[order], W[:, order], sweeps, float(np.sqrt(tiny))


def tournament_jacobi(A: np.ndarray, bw: int = 4, tol: float = 1e-13, max_sweeps: int = 60) -> int:
    """Sweeps to convergence in the cooperative kernel's order (k_svd): columns in blocks of bw,
    a round-robin tournament over the P blocks (P - 1 rounds of P/2 block pairs), a block pair's
    intra-block pairs in the first round of a sweep, then its bw x bw cross pairs in bw inner
    rounds; no norm ordering; the rotation and freeze rule F of one_sided_jacobi."""
    W = np.array(A, dtype=np.complex128, copy=True)
    R, N = W.shape
    tiny = max(1e-200, (8.0 * np.sqrt(R) * EPS64) ** 2 * float(np.sum(np.abs(W) ** 2)))
    P = (N + bw - 1) // bw
    P += P & 1
    late = False
    for sweep in range(max_sweeps):
        rot = 0

        def pair(p, q):
            nonlocal rot
            if p >= N or q >= N:
                return
            x, y = W[:, p], W[:, q]
            v0, v1 = float(np.vdot(x, x).real), float(np.vdot(y, y).real)
            g = np.vdot(x, y)
            if late and not (v0 > tiny and v1 > tiny):
                return
            if not late and not (max(v0, v1) > tiny and min(v0, v1) > 1e-6 * tiny):
                return
            if not (abs(g) ** 2 > tol * tol * v0 * v1):
                return
            c, s, e = rotation(v0, v1, float(g.real), float(g.imag))
            xn = c * x - s * np.conj(e) * y
            yn = s * e * x + c * y
            W[:, p], W[:, q] = xn, yn
            rot += 1

        for r in range(P - 1):
            for k in range(P // 2):
                I, J = (P - 1, r) if k == 0 else ((r + k) % (P - 1), (r - k + P - 1) % (P - 1))
                if r == 0:
                    for B in (I, J):
                        for a in range(bw):
                            for b in range(a + 1, bw):
                                pair(B * bw + a, B * bw + b)
                for t in range(bw):
                    for w in range(bw):
                        pair(I * bw + w, J * bw + (w + t) % bw)
        if not late and (rot < 0.1 * N * (N - 1) / 2 or sweep + 1 >= 8 + 3 * int(np.ceil(np.log2(N)))):
            late = True
            if rot:
                continue
        if rot == 0:
            return sweep + 1
    return max_sweeps


def pivoted_lq(A: np.ndarray) -> np.ndarray:
    """The preconditioner of tessera_b200/csrc/lq.cu, step for step: a row-pivoted Householder LQ
    P^T A = L Q^H returned as P L in A's own row order.  Step k takes the unpivoted row of largest
    remaining norm (downdated by its new column-k entry, recomputed exactly in each pass), forms
    the reflector u = x with u_0 = e (|x_0| + alpha), tau = 1/(alpha (alpha + |x_0|)) from that row
    x = X[p, k:], sets X[p, k] = -e alpha and zeroes the rest of the row, and updates every other
    unpivoted row z <- z - tau (z . conj(u)) u.  The kernel folds the update of the next pivot row
    into its reflector and fuses each update with the next step's products; the arithmetic is the
    same."""
    X = np.array(A, dtype=np.complex128, copy=True)
    R, N = X.shape
    nrm = np.sum(np.abs(X) ** 2, axis=1)
    free = np.ones(R, bool)
    for k in range(min(R, N)):
        key = np.where(free, nrm, -1.0)
        p = int(np.flatnonzero(key == key.max())[0])
        x = X[p, k:].copy()
        alpha, a0 = np.sqrt(np.sum(np.abs(x) ** 2)), abs(x[0])
        e = x[0] / a0 if a0 > 0 else 1.0
        free[p] = False
        X[p, k:] = 0
        if alpha == 0:
            continue
        X[p, k] = -e * alpha
        u = x.copy()
        u[0] = e * (a0 + alpha)
        tau = 1.0 / (alpha * (alpha + a0))
        rows = np.flatnonzero(free)
        w = X[rows, k:] @ np.conj(u)
        X[rows, k:] -= tau * np.outer(w, u)
        nrm[rows] = np.maximum(0.0, nrm[rows] - np.abs(X[rows, k]) ** 2)
    return X


def pivoted_lq_blocked(A: np.ndarray, panel: int = 8) -> np.ndarray:
    """pivoted_lq with the updates delayed over panels, as lq.cu's k_lq_batch runs it: within a
    panel the trailing block is not updated; row i's current values are X[i, c] - sum_j tw_j[i]
    u_j[c] over the panel's reflectors (tw_j = tau_j w_j), each step's products X[i, k:] . conj(u)
    are corrected by g_j = u_j . conj(u), only column k is written per step, and the panel's
    updates are applied at its end, where the row norms are recomputed exactly."""
    X = np.array(A, dtype=np.complex128, copy=True)
    R, N = X.shape
    kmax = min(R, N)
    free = np.ones(R, bool)
    nrm = np.sum(np.abs(X) ** 2, axis=1)
    k = 0
    while k < kmax:
        us, tws = [], []
        while k < kmax and len(us) < panel:
            key = np.where(free, nrm, -1.0)
            p = int(np.flatnonzero(key == key.max())[0])
            x = X[p, k:].copy()
            for u, tw in zip(us, tws):
                x -= tw[p] * u[k:]
            alpha, a0 = np.sqrt(np.sum(np.abs(x) ** 2)), abs(x[0])
            e = x[0] / a0 if a0 > 0 else 1.0
            u = np.zeros(N, complex)
            u[k:] = x
            tau = 0.0
            if alpha > 0:
                u[k] = e * (a0 + alpha)
                tau = 1.0 / (alpha * (alpha + a0))
            free[p] = False
            X[p, k] = -e * alpha if alpha > 0 else 0
            X[p, k + 1:] = 0
            rows = np.flatnonzero(free)
            w = np.zeros(R, complex)
            w[rows] = X[rows, k:] @ np.conj(u[k:])
            for uj, tj in zip(us, tws):
                w[rows] -= tj[rows] * np.sum(uj[k:] * np.conj(u[k:]))
            us.append(u)
            tws.append(tau * w)
            col = X[rows, k].copy()
            for uj, tj in zip(us, tws):
                col -= tj[rows] * uj[k]
            X[rows, k] = col
            nrm[rows] = np.maximum(0.0, nrm[rows] - np.abs(col) ** 2)
            k += 1
        rows = np.flatnonzero(free)
        for uj, tj in zip(us, tws):
            X[np.ix_(rows, np.arange(k, N))] -= np.outer(tj[rows], uj[k:])
        nrm[rows] = np.sum(np.abs(X[rows, k:]) ** 2, axis=1)
    return X


def graded(n: int, decay: float, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """n x n matrix U diag(exp(-k/decay)) V^H with Haar-like random unitary U, V."""
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    U, _, Vh = np.linalg.svd(X)
    s = np.exp(-np.arange(n) / decay)
    return (U * s) @ Vh, s
