"""Host-side interface of the anneal path, mirroring the reference's Rust caller.

``quantum_anneal(model, sched, chi)`` is the counterpart of rust/src/ffi.rs:47-85: it
splits the model's couplings into ei/ej/ew arrays, rejects schedules shorter than two
steps with ``QaError.BadSchedule`` (rust/src/ffi.rs:49-51) and calls the legacy
``tessera_qa_anneal`` symbol of libtessera_qa.so exactly as the Rust wrapper does
(rust/src/ffi.rs:60-75).  ``anneal`` exposes the extended entry point (dt, precision,
Jacobi controls, checkpoints, every result field).
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _lib


class QaError(enum.Enum):
    """rust/src/ffi.rs:11-17 (EngineNotLinked cannot occur: the engine is always linked)."""

    EngineNotLinked = "EngineNotLinked"
    BadSchedule = "BadSchedule"


class QaException(Exception):
    def __init__(self, err: QaError):
        super().__init__(err.value)
        self.err = err


@dataclass
class Ising:
    """Problem model of rust/src/ising.rs:11-32: fields h and couplings (i, j, w)."""

    h: list
    j: list  # [(i, k, w), ...]

    @property
    def n(self) -> int:
        return len(self.h)

    def energy(self, s) -> float:
        e = 0.0
        for (i, k, w) in self.j:
            e -= w * s[i] * s[k]
        for hi, si in zip(self.h, s):
            e -= hi * si
        return e


@dataclass
class Schedule:
    """rust/src/schedule.rs:8-18."""

    a: list
    b: list

    def steps(self) -> int:
        return len(self.a)


@dataclass
class QaResult:
    """rust/src/ffi.rs:39-43."""

    spins: np.ndarray
    energy: float
    entropy: np.ndarray


def _arr(x, dtype):
    return np.ascontiguousarray(np.asarray(x, dtype=dtype))


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None and a.size else None


def quantum_anneal(model: Ising, sched: Schedule, chi: int) -> QaResult:
    steps = sched.steps()
    if steps < 2:
        raise QaException(QaError.BadSchedule)
    L = _lib.load()
    h = _arr(model.h, np.float64)
    ei = _arr([t[0] for t in model.j], np.uint64)
    ej = _arr([t[1] for t in model.j], np.uint64)
    ew = _arr([t[2] for t in model.j], np.float64)
    a = _arr(sched.a, np.float64)
    b = _arr(sched.b, np.float64)
    spins = np.zeros(model.n, np.int8)
    entropy = np.zeros(steps, np.float64)
    e = L.tessera_qa_anneal(_p(h, _lib.c_double_p), model.n, _p(ei, _lib.c_size_p), _p(ej, _lib.c_size_p),
                            _p(ew, _lib.c_double_p), len(model.j), _p(a, _lib.c_double_p), _p(b, _lib.c_double_p),
                            steps, chi, _p(spins, _lib.c_int8_p), _p(entropy, _lib.c_double_p))
    if np.isnan(e):
        raise _lib.EngineError(_lib.EINVAL, _lib.last_error())
    return QaResult(spins, float(e), entropy)


@dataclass
class AnnealResult:
    """All fields of tessera_qa_result (the reference's AnnealResult, cuda/include/mps.hpp:37-44, plus
    run statistics)."""

    spins: np.ndarray
    energy: float
    expected_energy: float
    prob: float
    max_trunc: float
    norm2: float
    entropy: np.ndarray
    two_site_updates: int
    status: int
    max_sweeps: int
    max_bond: int
    device_ms: float
    min_cut_gap: float = 1.0
    checkpoint: bytes | None = None
    z_expect: np.ndarray | None = None
    extra: dict = field(default_factory=dict)


def problem_struct(h, ei, ej, ew, sa, sb, bias=None, sc=None):
    """Build a tessera_qa_problem; returns (struct, keepalive arrays)."""
    h = _arr(h, np.float64)
    ei = _arr(ei, np.uint64)
    ej = _arr(ej, np.uint64)
    ew = _arr(ew, np.float64)
    sa = _arr(sa, np.float64)
    sb = _arr(sb, np.float64)
    bias = None if bias is None else _arr(bias, np.float64)
    sc = None if sc is None else _arr(sc, np.float64)
    P = _lib.Problem(len(h), _p(h, _lib.c_double_p), len(ew), _p(ei, _lib.c_size_p), _p(ej, _lib.c_size_p),
                     _p(ew, _lib.c_double_p), len(sa), _p(sa, _lib.c_double_p), _p(sb, _lib.c_double_p),
                     _p(bias, _lib.c_double_p) if bias is not None else None,
                     _p(sc, _lib.c_double_p) if sc is not None else None)
    return P, (h, ei, ej, ew, sa, sb, bias, sc)


def config_struct(dt=0.1, chi=32, precision="c128", zz_substeps=1, jacobi_tol=0.0, jacobi_max_sweeps=0,
                  jacobi_block=0, device=-1, step_begin=0, step_end=0, initial_mps=None, skip_observables=False,
                  theta_tensor_cores=False, jacobi_precondition=0):
    """jacobi_precondition: 0 default (on), 1 on, 2 off -- the pivoted LQ before the column-pair
    Jacobi of theta above 256 rows (batched: one CTA per theta; single instance: cooperative)."""
    L = _lib.load()
    c = _lib.Config()
    L.tessera_qa_config_init(C.byref(c))
    c.dt = dt
    c.chi = chi
    c.precision = _lib.TESSERA_QA_C64 if precision in ("c64", "complex64", 1) else _lib.TESSERA_QA_C128
    c.zz_substeps = zz_substeps
    c.jacobi_tol = jacobi_tol
    c.jacobi_max_sweeps = jacobi_max_sweeps
    c.jacobi_block = jacobi_block
    c.device = device
    c.step_begin = step_begin
    c.step_end = step_end
    keep = None
    if initial_mps is not None:
        if isinstance(initial_mps, np.ndarray) and initial_mps.flags["C_CONTIGUOUS"]:
            keep = initial_mps  # used in place (e.g. a pinned host buffer)
        else:
            keep = np.frombuffer(initial_mps, dtype=np.uint8).copy()
        c.initial_mps = keep.ctypes.data
    c.skip_observables = 1 if skip_observables else 0
    c.theta_tensor_cores = 1 if theta_tensor_cores else 0
    c.jacobi_precondition = int(jacobi_precondition)
    return c, keep


def anneal(h, ei, ej, ew, sa, sb, dt=0.1, chi=32, precision="c128", zz_substeps=1, want_checkpoint=False,
           raise_on_status=True, checkpoint_out: np.ndarray | None = None, bias=None, sc=None,
           **kw) -> AnnealResult:
    """tessera_qa_anneal_ex: the MPS-TEBD anneal with every result field.

    want_checkpoint returns the final MPS as checkpoint bytes; checkpoint_out (a contiguous uint8
    array of at least tessera_qa_checkpoint_bytes(n, chi) bytes, e.g. pinned memory) receives it
    in place instead."""
    L = _lib.load()
    P, keep = problem_struct(h, ei, ej, ew, sa, sb, bias, sc)
    c, keep2 = config_struct(dt=dt, chi=chi, precision=precision, zz_substeps=zz_substeps, **kw)
    n = int(P.n)
    k0 = int(c.step_begin)
    k1 = int(c.step_end) if c.step_end else int(P.steps)
    spins = np.zeros(n, np.int8)
    ent = np.zeros(max(k1 - k0, 1), np.float64)
    r = _lib.Result()
    r.spins = _p(spins, _lib.c_int8_p)
    zexp = np.zeros(n, np.float64)
    r.z_expect = _p(zexp, _lib.c_double_p)
    r.entropy = _p(ent, _lib.c_double_p) if k1 > k0 else None
    ck = None
    if checkpoint_out is not None:
        r.final_mps = checkpoint_out.ctypes.data
        r.final_mps_bytes = checkpoint_out.nbytes
    elif want_checkpoint:
        nb = L.tessera_qa_checkpoint_bytes(n, chi)
        ck = np.zeros(nb, np.uint8)
        r.final_mps = ck.ctypes.data
        r.final_mps_bytes = nb
    rc = L.tessera_qa_anneal_ex(C.byref(P), C.byref(c), C.byref(r))
    if rc != 0 and not (rc == _lib.ESTATUS and not raise_on_status):
        raise _lib.EngineError(rc, _lib.last_error())
    return AnnealResult(spins, r.energy, r.expected_energy, r.prob, r.max_trunc, r.norm2, ent[: k1 - k0],
                        int(r.two_site_updates), int(r.status), int(r.max_sweeps), int(r.max_bond),
                        float(r.device_ms), float(r.min_cut_gap), ck.tobytes() if ck is not None else None,
                        zexp)


def svd(a: np.ndarray):
    """Thin SVD through the engine's Jacobi kernel (tessera_qa_svd): returns u, s, vh."""
    L = _lib.load()
    a = np.ascontiguousarray(a, dtype=np.complex128)
    r, c = a.shape
    k = min(r, c)
    s = np.zeros(k)
    u = np.zeros((r, k), np.complex128)
    vh = np.zeros((k, c), np.complex128)
    rc = L.tessera_qa_svd(a.view(np.float64).ctypes.data_as(_lib.c_double_p), r, c, s.ctypes.data_as(_lib.c_double_p),
                          u.view(np.float64).ctypes.data_as(_lib.c_double_p),
                          vh.view(np.float64).ctypes.data_as(_lib.c_double_p))
    if rc != 0:
        raise _lib.EngineError(rc, _lib.last_error())
    return u, s, vh


def sa_solve(problems, restarts: int = 256, sweeps: int = 2000, t0: float = 5.0, t_end: float = 0.01,
             seed: int = 0):
    """Best-of-restarts simulated annealing on the GPU (tessera_qa_sa_solve) for a list of
    problems (objects with h, ei, ej, ew): returns (energies, [spins per problem])."""
    L = _lib.load()
    arr = (_lib.Problem * len(problems))()
    keep = []
    for b, p in enumerate(problems):
        P, k = problem_struct(p.h, p.ei, p.ej, p.ew, np.zeros(0), np.zeros(0))
        arr[b] = P
        keep.append(k)
    ns = [len(p.h) for p in problems]
    spins = np.zeros(sum(ns), np.int8)
    en = np.zeros(len(problems))
    rc = L.tessera_qa_sa_solve(arr, len(problems), restarts, sweeps, t0, t_end, seed,
                               spins.ctypes.data_as(_lib.c_int8_p), en.ctypes.data_as(_lib.c_double_p))
    if rc != 0:
        raise _lib.EngineError(rc, _lib.last_error())
    off = np.cumsum([0] + ns)
    return en, [spins[off[b]:off[b + 1]].copy() for b in range(len(problems))]


def checkpoint_to_sites(buf: bytes):
    """Decode a checkpoint into (dims, [site tensors (Dl, 2, Dr) complex128])."""
    raw = np.frombuffer(buf, dtype=np.uint8)
    if raw[:8].tobytes() != b"TQMPSv1\x00":
        raise ValueError("not a tessera_qa checkpoint")
    n = int(np.frombuffer(raw[8:12].tobytes(), np.uint32)[0])
    dims = np.frombuffer(raw[32:32 + 4 * (n + 1)].tobytes(), np.int32).copy()
    off = 32 + (4 * (n + 1) + 7) // 8 * 8
    sites = []
    for i in range(n):
        cnt = int(dims[i]) * 2 * int(dims[i + 1])
        t = np.frombuffer(raw[off:off + 16 * cnt].tobytes(), np.complex128).reshape(dims[i], 2, dims[i + 1])
        sites.append(t)
        off += 16 * cnt
    return dims, sites


def sites_to_dense(sites) -> np.ndarray:
    """Contract an MPS to its 2^n amplitudes; basis index bit i = physical index of site i."""
    v = np.ones((1, 1), np.complex128)  # (configurations so far, bond)
    for i, t in enumerate(sites):
        # v[x, a] * t[a, s, b] -> w[x + s 2^i, b]
        w = np.einsum("xa,asb->sxb", v, t)
        v = w.reshape(-1, t.shape[2])
    return v[:, 0]


class Session:
    """A device-resident anneal (tessera_qa_session_*): the MPS stays in HBM between calls.

    Session(h, ei, ej, ew, sa, sb, ...) holds one instance; Session.batch([problems], ...) holds
    many, run by the batched engine."""

    def __init__(self, h, ei, ej, ew, sa, sb, dt=0.1, chi=32, precision="c128", zz_substeps=1,
                 kernel_timing=False, **kw):
        L = _lib.load()
        self._L = L
        self._P, self._keep = problem_struct(h, ei, ej, ew, sa, sb)
        c, _ = config_struct(dt=dt, chi=chi, precision=precision, zz_substeps=zz_substeps, **kw)
        c.kernel_timing = 1 if kernel_timing else 0
        self.chi = chi
        self.n = int(self._P.n)
        self.count = 1
        self._h = L.tessera_qa_session_create(C.byref(self._P), C.byref(c))
        if not self._h:
            raise _lib.EngineError(_lib.ECUDA, _lib.last_error())

    @classmethod
    def batch(cls, problems, dt=None, chi=None, precision="c128", kernel_timing=False, **kw):
        self = cls.__new__(cls)
        L = _lib.load()
        self._L = L
        B = len(problems)
        self._Parr = (_lib.Problem * B)()
        Carr = (_lib.Config * B)()
        self._keep = []
        for b, p in enumerate(problems):
            Pb, kp = problem_struct(p.h, p.ei, p.ej, p.ew, p.sa, p.sb)
            self._keep.append(kp)
            self._Parr[b] = Pb
            cb, _ = config_struct(dt=dt if dt is not None else p.dt, chi=chi if chi is not None else p.chi,
                                  precision=precision, **kw)
            cb.kernel_timing = 1 if kernel_timing else 0
            Carr[b] = cb
        self._chis = [int(Carr[b].chi) for b in range(B)]
        self.chi = chi if chi is not None else max(self._chis)
        self.n = problems[0].n
        self.count = B
        self._h = L.tessera_qa_session_create_batch(self._Parr, Carr, B)
        if not self._h:
            raise _lib.EngineError(_lib.ECUDA, _lib.last_error())
        return self

    def run_gates(self, step: int, gate_begin: int, gate_end: int):
        self._ck(self._L.tessera_qa_session_run_gates(self._h, step, gate_begin, gate_end))

    def run_host(self, problems, step: int, gate_begin: int = 0, gate_end: int = 0) -> "_lib.Result":
        """Host-buffer call: new h/J/schedule values from `problems` (host numpy arrays), run, wait,
        return the run statistics."""
        B = len(problems)
        Parr = (_lib.Problem * B)()
        keep = []
        for b, p in enumerate(problems):
            Pb, kp = problem_struct(p.h, p.ei, p.ej, p.ew, p.sa, p.sb)
            keep.append(kp)
            Parr[b] = Pb
        r = _lib.Result()
        self._ck(self._L.tessera_qa_session_run_host(self._h, Parr, B, step, gate_begin, gate_end, C.byref(r)))
        return r

    def _ck(self, rc):
        if rc != 0:
            raise _lib.EngineError(rc, _lib.last_error())

    def randomize(self, seed: int, decay: float = 0.0):
        """Seeded random MPS with every bond at its cap; decay > 0 grades each theta's spectrum
        (site column b scaled by exp(-b / decay))."""
        if decay:
            self._ck(self._L.tessera_qa_session_randomize_graded(self._h, seed, float(decay)))
        else:
            self._ck(self._L.tessera_qa_session_randomize(self._h, seed))

    def run(self, step_begin: int, nsteps: int):
        self._ck(self._L.tessera_qa_session_run(self._h, step_begin, nsteps))

    @property
    def stream(self) -> int:
        return int(self._L.tessera_qa_session_stream(self._h))

    def sync(self) -> "_lib.Result":
        r = _lib.Result()
        self._ck(self._L.tessera_qa_session_sync(self._h, C.byref(r)))
        return r

    def observe(self, spins: np.ndarray | None = None) -> "_lib.Result":
        r = _lib.Result()
        if spins is not None:
            r.spins = spins.ctypes.data_as(_lib.c_int8_p)
        self._ck(self._L.tessera_qa_session_observe(self._h, C.byref(r)))
        return r

    def save(self) -> bytes:
        nb = self._L.tessera_qa_checkpoint_bytes(self.n, self.chi)
        buf = np.zeros(nb, np.uint8)
        self._ck(self._L.tessera_qa_session_save(self._h, buf.ctypes.data, nb))
        return buf.tobytes()

    def sample(self, count: int, seed: int = 0):
        """(spins (count, n) int8, energies (count,)): patterns drawn from |<x|psi>|^2
        (tessera_qa_session_sample)."""
        spins = np.zeros((count, self.n), np.int8)
        en = np.zeros(count)
        self._ck(self._L.tessera_qa_session_sample(self._h, count, seed, spins.ctypes.data_as(_lib.c_int8_p),
                                                   en.ctypes.data_as(_lib.c_double_p)))
        return spins, en

    def save_instance(self, index: int) -> bytes:
        """Checkpoint of instance `index` of a batched session (tessera_qa_session_save_instance)."""
        chi = self._chis[index] if hasattr(self, "_chis") else self.chi
        nb = self._L.tessera_qa_checkpoint_bytes(self.n_of(index), chi)
        buf = np.zeros(nb, np.uint8)
        self._ck(self._L.tessera_qa_session_save_instance(self._h, index, buf.ctypes.data, nb))
        return buf.tobytes()

    def n_of(self, index: int) -> int:
        return int(self._Parr[index].n) if hasattr(self, "_Parr") else self.n

    def load(self, buf: bytes):
        a = np.frombuffer(buf, np.uint8).copy()
        self._ck(self._L.tessera_qa_session_load(self._h, a.ctypes.data, a.size))

    def close(self):
        if self._h:
            self._L.tessera_qa_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class SvAnnealResult:
    spins: np.ndarray          # most probable pattern
    sign_spins: np.ndarray     # sign<Z> pattern
    energy: float
    expected_energy: float
    prob: float
    sign_energy: float
    entropy: np.ndarray
    norm2: float
    device_ms: float
    state: np.ndarray | None = None


def sv_anneal(h, ei, ej, ew, sa, sb, dt=0.1, mode=0, bias=None, sc=None, want_state=False) -> SvAnnealResult:
    """tessera_qa_sv_anneal: the exact 2^n state-vector anneal on the GPU (rust/src/quantum.rs:63-112).
    mode 0 = quantum.rs's splitting, mode 1 = the MPS engine's splitting."""
    L = _lib.load()
    P, keep = problem_struct(h, ei, ej, ew, sa, sb, bias, sc)
    n, steps = int(P.n), int(P.steps)
    spins = np.zeros(n, np.int8)
    sspins = np.zeros(n, np.int8)
    ent = np.zeros(steps)
    st = np.zeros(2 << n) if want_state else None
    r = _lib.SvResult()
    r.spins = _p(spins, _lib.c_int8_p)
    r.sign_spins = _p(sspins, _lib.c_int8_p)
    r.entropy = _p(ent, _lib.c_double_p)
    if st is not None:
        r.state = _p(st, _lib.c_double_p)
    rc = L.tessera_qa_sv_anneal(C.byref(P), dt, mode, C.byref(r))
    if rc != 0:
        raise _lib.EngineError(rc, _lib.last_error())
    return SvAnnealResult(spins, sspins, r.energy, r.expected_energy, r.prob, r.sign_energy, ent, r.norm2,
                          r.device_ms, st.view(np.complex128) if st is not None else None)


def anneal_batch(problems, dt=None, chi=None, precision="c128", zz_substeps=1, want_checkpoint=False,
                 raise_on_status=True, skip_observables=False, jacobi_block=0, device=-1, theta_tensor_cores=False):
    """tessera_qa_anneal_batch over a list of instances.Problem (each uses its own dt and chi unless
    overridden); returns a list of AnnealResult in the same order."""
    L = _lib.load()
    B = len(problems)
    P_arr = (_lib.Problem * B)()
    C_arr = (_lib.Config * B)()
    R_arr = (_lib.Result * B)()
    keep = []
    outs = []
    for b, p in enumerate(problems):
        Pb, kp = problem_struct(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, getattr(p, "bias", None), getattr(p, "sc", None))
        keep.append(kp)
        P_arr[b] = Pb
        cb, _ = config_struct(dt=dt if dt is not None else p.dt, chi=chi if chi is not None else p.chi,
                              precision=precision, zz_substeps=zz_substeps, jacobi_block=jacobi_block,
                              device=device, skip_observables=skip_observables, theta_tensor_cores=theta_tensor_cores)
        C_arr[b] = cb
        n, steps = p.n, p.steps
        spins = np.zeros(n, np.int8)
        zexp = np.zeros(n)
        ent = np.zeros(max(steps, 1))
        R_arr[b].spins = _p(spins, _lib.c_int8_p)
        R_arr[b].z_expect = _p(zexp, _lib.c_double_p)
        R_arr[b].entropy = _p(ent, _lib.c_double_p)
        ck = None
        if want_checkpoint:
            nb = L.tessera_qa_checkpoint_bytes(n, cb.chi)
            ck = np.zeros(nb, np.uint8)
            R_arr[b].final_mps = ck.ctypes.data
            R_arr[b].final_mps_bytes = nb
        outs.append((spins, zexp, ent, ck, steps))
    rc = L.tessera_qa_anneal_batch(P_arr, C_arr, R_arr, B)
    if rc != 0 and not (rc == _lib.ESTATUS and not raise_on_status):
        raise _lib.EngineError(rc, _lib.last_error())
    res = []
    for b in range(B):
        spins, zexp, ent, ck, steps = outs[b]
        r = R_arr[b]
        res.append(AnnealResult(spins, r.energy, r.expected_energy, r.prob, r.max_trunc, r.norm2, ent[:steps],
                                int(r.two_site_updates), int(r.status), int(r.max_sweeps), int(r.max_bond),
                                float(r.device_ms), float(r.min_cut_gap), ck.tobytes() if ck is not None else None,
                                zexp))
    return res
