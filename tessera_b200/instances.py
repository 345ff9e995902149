"""Seeded synthetic Ising instances and schedules for the anneal workloads.

Energies follow E(s) = -sum_e w_e s_i s_j - sum_i h_i s_i (rust/src/ising.rs:23-32).
Edge lists are upper-triangular (i < j) and sorted lexicographically by (i, j): the
engine applies ZZ gates in list order (cuda/src/mps.cpp:330-341), so the order is part of
the workload.  All generators use numpy's PCG64 with the seed given.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Problem:
    """An Ising instance plus its discretised schedule A(s_k), B(s_k)."""

    h: np.ndarray          # (n,) float64
    ei: np.ndarray         # (m,) int64, ei < ej
    ej: np.ndarray         # (m,) int64
    ew: np.ndarray         # (m,) float64
    sa: np.ndarray | None = None   # (steps,) transverse weight A(s)
    sb: np.ndarray | None = None   # (steps,) problem weight B(s)
    dt: float = 0.1
    chi: int = 32
    name: str = ""
    bias: np.ndarray | None = None  # optional warm-start bias b_i (field -C(s) sum b_i Z_i)
    sc: np.ndarray | None = None    # its schedule C(s_k)

    @property
    def n(self) -> int:
        return int(self.h.shape[0])

    @property
    def m(self) -> int:
        return int(self.ew.shape[0])

    @property
    def steps(self) -> int:
        return 0 if self.sa is None else int(self.sa.shape[0])

    def energy(self, spins) -> float:
        s = np.asarray(spins, dtype=np.float64)
        return float(-(self.ew * s[self.ei] * s[self.ej]).sum() - (self.h * s).sum())

    def updates_per_step(self) -> int:
        """Two-site updates one Trotter step costs: 2|i-j|-1 per edge (cuda/src/mps.cpp:126-145)."""
        d = np.abs(self.ej - self.ei)
        return int((2 * d[d > 0] - 1).sum())


def linear(steps: int):
    """A = 1 - s, B = s with s = k/(steps-1) (rust/src/schedule.rs:20-31)."""
    n = max(steps, 2)
    s = np.arange(n, dtype=np.float64) / (n - 1)
    return 1.0 - s, s


def smooth(steps: int):
    """A = cos^2(pi s/2), B = sin^2(pi s/2) (rust/src/schedule.rs:35-46)."""
    n = max(steps, 2)
    s = np.arange(n, dtype=np.float64) / (n - 1)
    th = 0.5 * np.pi * s
    return np.cos(th) ** 2, np.sin(th) ** 2


def from_knots(knots, steps: int):
    """Monotone piecewise-linear schedule through K knots s(u_j), u_j = j/(K-1).

    The learned-schedule layer predicts K knot values of the anneal fraction
    0 = s_0 <= s_1 <= ... <= s_{K-1} = 1 at equally spaced times; A = 1 - s, B = s.
    """
    kn = np.asarray(knots, dtype=np.float64)
    u = np.linspace(0.0, 1.0, kn.shape[0])
    t = np.arange(max(steps, 2), dtype=np.float64) / (max(steps, 2) - 1)
    s = np.interp(t, u, kn)
    return 1.0 - s, s


def _sorted_edges(ei, ej, ew):
    ei = np.asarray(ei, dtype=np.int64)
    ej = np.asarray(ej, dtype=np.int64)
    ew = np.asarray(ew, dtype=np.float64)
    lo, hi = np.minimum(ei, ej), np.maximum(ei, ej)
    order = np.lexsort((hi, lo))
    return lo[order], hi[order], ew[order]


def chain_nn(n: int = 16, seed: int = 1, T: float = 20.0, dt: float = 0.05, chi: int = 32) -> Problem:
    """Open chain, J_{i,i+1} ~ N(0,1), h ~ N(0, 0.5), linear schedule, T/dt steps."""
    rng = np.random.Generator(np.random.PCG64(seed))
    j = rng.normal(0.0, 1.0, n - 1)
    h = rng.normal(0.0, 0.5, n)
    ei = np.arange(n - 1)
    sa, sb = linear(int(round(T / dt)))
    return Problem(h, ei, ei + 1, j, sa, sb, dt, chi, f"chain_nn(n={n},seed={seed})")


def chain_range(n: int = 128, dmax: int = 4, seed: int = 2, T: float = 50.0, dt: float = 0.02,
                chi: int = 256, dist: str = "uniform", hzero: bool = True) -> Problem:
    """Chain with couplings to neighbours at distances 1..dmax.

    dist="uniform": J ~ U(-1, 1); dist="normal": J ~ N(0, 1).  h = 0 when hzero.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    ei, ej = [], []
    for i in range(n):
        for d in range(1, dmax + 1):
            if i + d < n:
                ei.append(i)
                ej.append(i + d)
    ei, ej = np.array(ei), np.array(ej)
    w = rng.uniform(-1.0, 1.0, len(ei)) if dist == "uniform" else rng.normal(0.0, 1.0, len(ei))
    ei, ej, w = _sorted_edges(ei, ej, w)
    h = np.zeros(n) if hzero else rng.normal(0.0, 0.5, n)
    sa, sb = linear(int(round(T / dt)))
    return Problem(h, ei, ej, w, sa, sb, dt, chi, f"chain_range(n={n},d<={dmax},seed={seed})")


def random_3_regular(n: int, rng: np.random.Generator, max_tries: int = 1000):
    """Random 3-regular graph by the configuration model, rejecting loops and multi-edges."""
    if n % 2:
        raise ValueError("3-regular graphs need even n")
    for _ in range(max_tries):
        stubs = np.repeat(np.arange(n), 3)
        rng.shuffle(stubs)
        a, b = stubs[0::2], stubs[1::2]
        if np.any(a == b):
            continue
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        key = lo * n + hi
        if len(np.unique(key)) != len(key):
            continue
        return lo, hi
    raise RuntimeError("no simple 3-regular graph found")


def batch_3_regular(count: int = 512, base_seed: int = 3, T: float = 30.0, dt: float = 0.05,
                    nmin: int = 32, nmax: int = 96):
    """Ragged batch: n ~ U{nmin..nmax} even, random 3-regular, J ~ N(0,1), h ~ N(0,0.1),
    chi_max ~ U{64, 128}; instance idx uses seed base_seed + idx."""
    out = []
    sa, sb = linear(int(round(T / dt)))
    for idx in range(count):
        rng = np.random.Generator(np.random.PCG64(base_seed + idx))
        n = int(rng.integers(nmin // 2, nmax // 2 + 1)) * 2
        lo, hi = random_3_regular(n, rng)
        w = rng.normal(0.0, 1.0, len(lo))
        h = rng.normal(0.0, 0.1, n)
        chi = int(rng.choice([64, 128]))
        ei, ej, w = _sorted_edges(lo, hi, w)
        out.append(Problem(h, ei, ej, w, sa, sb, dt, chi, f"3reg(n={n},seed={base_seed + idx})"))
    return out


def dense_er(n: int, seed: int, p: float = 0.5, T: float = 30.0, dt: float = 0.05, chi: int = 128) -> Problem:
    """Dense Erdos-Renyi: edge prob p, J ~ U(-1,1), h ~ U(-0.2, 0.2); linear schedule."""
    rng = np.random.Generator(np.random.PCG64(seed))
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(len(iu)) < p
    ei, ej = iu[keep], ju[keep]
    if len(ei) == 0:
        ei, ej = np.array([0]), np.array([1])
    w = rng.uniform(-1.0, 1.0, len(ei))
    h = rng.uniform(-0.2, 0.2, n)
    sa, sb = linear(int(round(T / dt)))
    ei, ej, w = _sorted_edges(ei, ej, w)
    return Problem(h, ei, ej, w, sa, sb, dt, chi, f"dense_er(n={n},seed={seed})")
