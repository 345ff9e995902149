"""Learned anneal schedules: the GNN of csrc/gnn.cu, its training data, and its evaluation.

Pipeline (every heavy step runs on the GPU through libtessera_qa.so):

1. candidates(): a fixed family of 16-knot monotone schedules s(u) (linear, power laws,
   slow-in-the-middle and sigmoid warps).
2. label(): anneal every training instance under every candidate with the batched engine
   (tessera_qa_anneal_batch), score each run by its readout energy against the exact ground
   energy (tessera_qa_exact_ground), and keep the best candidate's knots as the target;
   the exact ground-state spins are the per-spin target.
3. ScheduleGNN.train_step(): forward, backward and Adam in the library's own kernels.
4. solve(): predict knots and a warm-start bias, anneal under the predicted schedule and
   under the plain linear one in one batch, and keep whichever the engine's own final
   energy judges better (the fallback rule).
5. evaluate(): solves (readout within 1 % of the ground energy) per second of wall time,
   chosen (batched, complex64, learned + fallback) against plain (complex128, one instance
   at a time, linear schedule), on the same held-out instances.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _lib, ffi, instances

K_KNOTS = 16


def _setup(L):
    if getattr(L, "_gnn_ready", False):
        return L
    L.tessera_qa_exact_ground.argtypes = [_lib.c_double_p, C.c_size_t, _lib.c_size_p, _lib.c_size_p,
                                          _lib.c_double_p, C.c_size_t, _lib.c_int8_p]
    L.tessera_qa_exact_ground.restype = C.c_double
    L.tessera_qa_gnn_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int]
    L.tessera_qa_gnn_create.restype = C.c_void_p
    L.tessera_qa_gnn_destroy.argtypes = [C.c_void_p]
    L.tessera_qa_gnn_destroy.restype = None
    L.tessera_qa_gnn_param_count.argtypes = [C.c_void_p]
    L.tessera_qa_gnn_param_count.restype = C.c_size_t
    fp = C.POINTER(C.c_float)
    L.tessera_qa_gnn_get_params.argtypes = [C.c_void_p, fp, C.c_size_t]
    L.tessera_qa_gnn_get_params.restype = C.c_int
    L.tessera_qa_gnn_set_params.argtypes = [C.c_void_p, fp, C.c_size_t]
    L.tessera_qa_gnn_set_params.restype = C.c_int
    L.tessera_qa_gnn_forward.argtypes = [C.c_void_p, C.POINTER(_lib.Problem), C.c_size_t, fp, fp]
    L.tessera_qa_gnn_forward.restype = C.c_int
    L.tessera_qa_gnn_train_step.argtypes = [C.c_void_p, C.POINTER(_lib.Problem), C.c_size_t, fp, fp, C.c_float,
                                            C.c_float, C.c_float, fp, fp, C.c_size_t]
    L.tessera_qa_gnn_train_step.restype = C.c_int
    L.tessera_qa_gnn_apply_grads.argtypes = [C.c_void_p, fp, C.c_size_t, C.c_float]
    L.tessera_qa_gnn_apply_grads.restype = C.c_int
    L.tessera_qa_schedule_predict.argtypes = [C.c_void_p, C.POINTER(_lib.Problem), C.c_size_t, _lib.c_double_p,
                                              _lib.c_double_p]
    L.tessera_qa_schedule_predict.restype = C.c_int
    L._gnn_ready = True
    return L


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def exact_ground(p: instances.Problem):
    """Exact ground energy and spins on the GPU (tessera_qa_exact_ground, n <= 32)."""
    L = _setup(_lib.load())
    h = np.ascontiguousarray(p.h, np.float64)
    ei = np.ascontiguousarray(p.ei, np.uint64)
    ej = np.ascontiguousarray(p.ej, np.uint64)
    ew = np.ascontiguousarray(p.ew, np.float64)
    s = np.zeros(p.n, np.int8)
    e = L.tessera_qa_exact_ground(h.ctypes.data_as(_lib.c_double_p), p.n, ei.ctypes.data_as(_lib.c_size_p),
                                  ej.ctypes.data_as(_lib.c_size_p), ew.ctypes.data_as(_lib.c_double_p), p.m,
                                  s.ctypes.data_as(_lib.c_int8_p))
    if np.isnan(e):
        raise _lib.EngineError(_lib.EINVAL, _lib.last_error())
    return float(e), s


def reference_energies(problems, exact_max_n: int = 24, sa_restarts: int = 512, sa_sweeps: int = 4000,
                       seed: int = 0):
    """Energy each solve is scored against: the exact ground energy for n <= exact_max_n
    (tessera_qa_exact_ground, rust/src/ising.rs:46-61), else the best of a large simulated-annealing
    budget (tessera_qa_sa_solve, the reference's sa_solve, rust/src/ising.rs:118-136).  Returns
    (energies, kinds) with kind "exact" or "sa"."""
    e = np.zeros(len(problems))
    kinds = []
    big = [i for i, p in enumerate(problems) if p.n > exact_max_n]
    for i, p in enumerate(problems):
        if p.n <= exact_max_n:
            e[i] = exact_ground(p)[0]
            kinds.append("exact")
        else:
            kinds.append("sa")
    if big:
        en, _ = ffi.sa_solve([problems[i] for i in big], restarts=sa_restarts, sweeps=sa_sweeps, seed=seed)
        e[big] = en
    return e, kinds


def _problem_array(problems):
    arr = (_lib.Problem * len(problems))()
    keep = []
    for b, p in enumerate(problems):
        P, k = ffi.problem_struct(p.h, p.ei, p.ej, p.ew, np.zeros(0), np.zeros(0))
        arr[b] = P
        keep.append(k)
    return arr, keep


class ScheduleGNN:
    """The message-passing schedule predictor (tessera_qa_gnn_*)."""

    def __init__(self, hidden: int = 64, layers: int = 3, knots: int = K_KNOTS, seed: int = 0, bf16: bool = True):
        self.L = _setup(_lib.load())
        self.hidden, self.layers, self.knots = hidden, layers, knots
        self._h = self.L.tessera_qa_gnn_create(hidden, layers, knots, seed, 1 if bf16 else 0)
        if not self._h:
            raise _lib.EngineError(_lib.EINVAL, _lib.last_error())

    @property
    def param_count(self) -> int:
        return int(self.L.tessera_qa_gnn_param_count(self._h))

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.param_count, np.float32)
        self._ck(self.L.tessera_qa_gnn_get_params(self._h, _fptr(out), out.size))
        return out

    def set_params(self, params):
        a = np.ascontiguousarray(params, np.float32)
        self._ck(self.L.tessera_qa_gnn_set_params(self._h, _fptr(a), a.size))

    def _ck(self, rc):
        if rc != 0:
            raise _lib.EngineError(rc, _lib.last_error())

    def forward(self, problems):
        arr, keep = _problem_array(problems)
        kn = np.zeros((len(problems), self.knots), np.float32)
        p = np.zeros(sum(q.n for q in problems), np.float32)
        self._ck(self.L.tessera_qa_gnn_forward(self._h, arr, len(problems), _fptr(kn), _fptr(p)))
        return kn, p

    def train_step(self, problems, target_knots, target_spins, lr=1e-3, lambda_knots=1.0, lambda_spins=0.2,
                   want_grads=False):
        arr, keep = _problem_array(problems)
        tk = np.ascontiguousarray(target_knots, np.float32)
        ts = np.ascontiguousarray(target_spins, np.float32)
        loss = C.c_float(0)
        g = np.zeros(self.param_count, np.float32) if want_grads else None
        self._ck(self.L.tessera_qa_gnn_train_step(self._h, arr, len(problems), _fptr(tk), _fptr(ts), lr,
                                                  lambda_knots, lambda_spins, C.byref(loss),
                                                  _fptr(g) if g is not None else None, self.param_count))
        return float(loss.value), g

    def apply_grads(self, grads, lr=1e-3):
        """Adam step with a caller-supplied gradient (tessera_qa_gnn_apply_grads)."""
        a = np.ascontiguousarray(grads, np.float32)
        self._ck(self.L.tessera_qa_gnn_apply_grads(self._h, _fptr(a), a.size, lr))

    def predict(self, problems):
        """(knots (G, K), list of per-problem bias arrays in [-1, 1]) via tessera_qa_schedule_predict."""
        arr, keep = _problem_array(problems)
        kn = np.zeros((len(problems), self.knots))
        bias = np.zeros(sum(q.n for q in problems))
        self._ck(self.L.tessera_qa_schedule_predict(self._h, arr, len(problems), kn.ctypes.data_as(_lib.c_double_p),
                                                    bias.ctypes.data_as(_lib.c_double_p)))
        out, o = [], 0
        for q in problems:
            out.append(bias[o:o + q.n].copy())
            o += q.n
        return kn, out

    def close(self):
        if self._h:
            self.L.tessera_qa_gnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def candidates(k: int = K_KNOTS, count: int = 24) -> np.ndarray:
    """A fixed family of monotone schedules s(u), sampled at k equally spaced knots."""
    u = np.linspace(0.0, 1.0, k)
    out = [u.copy()]
    for p in (0.5, 0.65, 0.8, 1.25, 1.5, 2.0):
        out.append(u ** p)
    for a in (-0.9, -0.6, -0.3, 0.3, 0.6, 0.9):  # slow (a < 0) or fast through the middle
        out.append(u + a * np.sin(2 * np.pi * u) / (2 * np.pi))
    for kk, c in ((6, 0.5), (10, 0.5), (6, 0.35), (6, 0.65), (10, 0.3), (10, 0.7)):
        sg = 1 / (1 + np.exp(-kk * (u - c)))
        out.append((sg - sg[0]) / (sg[-1] - sg[0]))
    for q in (0.3, 0.5, 0.7):  # piecewise: slow before/after a kink
        out.append(np.where(u < q, 0.5 * u / q, 0.5 + 0.5 * (u - q) / (1 - q)))
    for q in (0.4, 0.6):
        out.append(np.minimum(1.0, np.maximum(0.0, u + 0.15 * np.sin(np.pi * u) * (1 if q > 0.5 else -1))))
    arr = np.array(out[:count])
    arr = np.maximum.accumulate(np.clip(arr, 0, 1), axis=1)
    arr[:, 0], arr[:, -1] = 0.0, 1.0
    return arr


@dataclass
class LearnConfig:
    T: float = 6.0          # anneal time
    dt: float = 0.1
    chi: int = 32
    bias_strength: float = 0.5
    precision: str = "c64"


def with_schedule(p: instances.Problem, knots, cfg: LearnConfig, bias=None) -> instances.Problem:
    steps = int(round(cfg.T / cfg.dt))
    sa, sb = instances.from_knots(knots, steps)
    q = instances.Problem(p.h, p.ei, p.ej, p.ew, sa, sb, cfg.dt, cfg.chi, p.name)
    if bias is not None:
        # warm-start field -C(s) sum b_i Z_i, C(s) = c0 4 s (1-s): zero at both ends
        q.bias = np.asarray(bias, np.float64)
        q.sc = cfg.bias_strength * 4.0 * sb * (1.0 - sb)
    return q


def plain_problem(p: instances.Problem, cfg: LearnConfig) -> instances.Problem:
    """The plain method: the linear schedule A = 1 - s, B = s (rust/src/schedule.rs:20-31), no bias."""
    sa, sb = instances.linear(int(round(cfg.T / cfg.dt)))
    return instances.Problem(p.h, p.ei, p.ej, p.ew, sa, sb, cfg.dt, cfg.chi, p.name)


def label(problems, cfg: LearnConfig, cands=None, chunk: int = 512):
    """Best candidate schedule (lowest readout energy, then lowest <H>) per problem, and the exact
    ground state.  Returns (target knots (G, K), ground energies, ground spins list, gaps per candidate)."""
    cands = candidates() if cands is None else cands
    jobs = [(g, c) for g in range(len(problems)) for c in range(len(cands))]
    E = np.full((len(problems), len(cands)), np.inf)
    H = np.full((len(problems), len(cands)), np.inf)
    for s in range(0, len(jobs), chunk):
        part = jobs[s:s + chunk]
        res = ffi.anneal_batch([with_schedule(problems[g], cands[c], cfg) for g, c in part], precision=cfg.precision,
                               raise_on_status=False)
        for (g, c), r in zip(part, res):
            E[g, c] = r.energy
            H[g, c] = r.expected_energy
    ground = [exact_ground(p) for p in problems]
    e0 = np.array([g[0] for g in ground])
    best = np.array([min(range(len(cands)), key=lambda c: (E[g, c], H[g, c])) for g in range(len(problems))])
    gaps = (E - e0[:, None]) / np.abs(e0)[:, None]
    return cands[best], e0, [g[1] for g in ground], gaps


def spin_targets(ground_spins):
    return np.concatenate([(np.asarray(s, np.float32) + 1.0) / 2.0 for s in ground_spins])


def train(gnn: ScheduleGNN, problems, target_knots, ground_spins, epochs=200, batch=32, lr=2e-3, seed=0,
          lambda_spins=0.2):
    """Mini-batch Adam on the GPU; returns the loss history (one value per step)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    losses = []
    idx = np.arange(len(problems))
    for ep in range(epochs):
        rng.shuffle(idx)
        for s in range(0, len(idx), batch):
            sel = idx[s:s + batch]
            ps = [problems[i] for i in sel]
            loss, _ = gnn.train_step(ps, target_knots[sel], spin_targets([ground_spins[i] for i in sel]), lr=lr,
                                     lambda_spins=lambda_spins)
            losses.append(loss)
    return losses


def train_data_parallel(gnn, problems, target_knots, ground_spins, epochs=100, batch=32, lr=2e-3, seed=0,
                        lambda_spins=0.2, group=None):
    """Data-parallel training over torch.distributed ranks (one GPU each): every rank draws the same
    mini-batch order, takes its contiguous share of each batch, computes loss and gradient with the
    library's kernels, and the gradients are averaged (weighted by the share sizes) with one
    all-reduce before the same Adam step on every rank, so the replicas stay identical.  Returns
    the averaged loss per step."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    rng = np.random.Generator(np.random.PCG64(seed))
    idx = np.arange(len(problems))
    losses = []
    for _ in range(epochs):
        rng.shuffle(idx)
        for s in range(0, len(idx), batch):
            sel = idx[s:s + batch]
            share = np.array_split(sel, world)[rank]
            buf = torch.zeros(gnn.param_count + 2, dtype=torch.float64, device=dev)
            if len(share):
                ps = [problems[i] for i in share]
                loss, g = gnn.train_step(ps, target_knots[share], spin_targets([ground_spins[i] for i in share]),
                                         lr=0.0, lambda_spins=lambda_spins, want_grads=True)
                w = float(len(share))
                buf[:-2] = torch.from_numpy(g.astype(np.float64) * w)
                buf[-2] = loss * w
                buf[-1] = w
            dist.all_reduce(buf, group=group)
            tot = float(buf[-1])
            gnn.apply_grads((buf[:-2] / tot).cpu().numpy(), lr=lr)
            losses.append(float(buf[-2]) / tot)
    return losses


def solve_chosen(gnn: ScheduleGNN, problems, cfg: LearnConfig, use_bias=True, detail=False):
    """Learned schedule (+ warm-start bias) and the plain linear schedule in one batch; per problem
    keep the run whose readout energy is lower (fallback to linear when the learned run is worse).
    Returns (chosen energy, learned run kept) per problem; with detail, also the learned run's and
    the linear run's energies (the method with and without the network, no fallback)."""
    kn, bias = gnn.predict(problems)
    runs = [with_schedule(p, kn[g], cfg, bias[g] if use_bias else None) for g, p in enumerate(problems)]
    runs += [plain_problem(p, cfg) for p in problems]
    res = ffi.anneal_batch(runs, precision=cfg.precision, raise_on_status=False)
    G = len(problems)
    out = []
    for g in range(G):
        a, b = res[g], res[G + g]
        chosen = a if (a.energy, a.expected_energy) <= (b.energy, b.expected_energy) else b
        out.append((chosen.energy, chosen is a, a.energy, b.energy) if detail else (chosen.energy, chosen is a))
    return out


def evaluate(gnn: ScheduleGNN, problems, cfg: LearnConfig, gap=0.01, plain_sample: int | None = None,
             plain_steps: int | None = None):
    """Solves per second, chosen (batched c64, learned + fallback) vs plain (c128, one instance at
    a time, linear schedule), on the same problems; reference energies from reference_energies()
    (exact for n <= 24, else the best of a large SA budget, stated per instance).  Also reported:
    the learned run and the linear run of the same batch each on their own (no fallback), which
    is what the network gains over the method without it.

    plain_sample = k: the plain arm is timed on the first k problems, one call each, and its
    per-instance time is taken as their mean; its energies for all problems come from one
    batched complex128 run of the same linear schedule, which executes the same per-instance
    code (the resident anneal kernel) and gives the same results -- checked on the timed
    sample.

    plain_steps = k: the timed single-instance plain calls run only the first k steps of the
    schedule (a full complex128 single-instance anneal at chi=128 takes hours); the plain time
    per instance is then that window's time scaled by steps / k, and is reported as
    extrapolated."""
    e0, kinds = reference_energies(problems)
    steps = int(round(cfg.T / cfg.dt))
    sa, sb = instances.linear(steps)
    timed = problems if plain_sample is None else problems[:plain_sample]
    win = steps if plain_steps is None else min(plain_steps, steps)
    t0 = time.perf_counter()
    single_e = []
    for p in timed:
        r = ffi.anneal(p.h, p.ei, p.ej, p.ew, sa[:win], sb[:win], dt=cfg.dt, chi=cfg.chi, precision="c128",
                       raise_on_status=False, skip_observables=win < steps)
        single_e.append(r.energy)
    t_timed = (time.perf_counter() - t0) * steps / win
    if win < steps:
        res = ffi.anneal_batch([plain_problem(p, cfg) for p in problems], precision="c128", raise_on_status=False)
        plain_e = np.array([r.energy for r in res])
        t_plain = t_timed / max(1, len(timed)) * len(problems)
    elif plain_sample is None:
        plain_e = np.array(single_e)
        t_plain = t_timed
    else:
        res = ffi.anneal_batch([plain_problem(p, cfg) for p in problems], precision="c128", raise_on_status=False)
        plain_e = np.array([r.energy for r in res])
        if not np.array_equal(plain_e[:len(timed)], np.array(single_e)):
            raise RuntimeError("batched complex128 plain runs differ from the single-instance runs")
        t_plain = t_timed / max(1, len(timed)) * len(problems)
    t0 = time.perf_counter()
    ch = solve_chosen(gnn, problems, cfg, detail=True)
    t_chosen = time.perf_counter() - t0
    chosen_e = np.array([c[0] for c in ch])
    learned_e = np.array([c[2] for c in ch])
    linear_e = np.array([c[3] for c in ch])
    rel = lambda e: (e - e0) / np.abs(e0)  # noqa: E731
    ok_plain = rel(plain_e) <= gap
    ok_chosen = rel(chosen_e) <= gap
    return {"instances": len(problems), "plain_solved": int(ok_plain.sum()), "chosen_solved": int(ok_chosen.sum()),
            "plain_seconds": t_plain, "chosen_seconds": t_chosen,
            "plain_timed_instances": len(timed), "plain_timed_steps": win, "steps": steps,
            "plain_extrapolated": bool(win < steps or len(timed) < len(problems)),
            "reference_energy": {"exact": kinds.count("exact"), "sa": kinds.count("sa")},
            "learned_solved_no_fallback": int((rel(learned_e) <= gap).sum()),
            "linear_c64_solved": int((rel(linear_e) <= gap).sum()),
            "learned_mean_gap_no_fallback": float(np.mean(rel(learned_e))),
            "linear_c64_mean_gap": float(np.mean(rel(linear_e))),
            "plain_solves_per_s": ok_plain.sum() / t_plain, "chosen_solves_per_s": ok_chosen.sum() / t_chosen,
            "learned_kept": int(sum(c[1] for c in ch)),
            "plain_mean_gap": float(np.mean((plain_e - e0) / np.abs(e0))),
            "chosen_mean_gap": float(np.mean((chosen_e - e0) / np.abs(e0)))}
