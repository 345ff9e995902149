"""ctypes access to the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py as
the checker.  The product package (``tessera_b200``) never imports this module.

Two libraries are exposed:

* ``Oracle``    -- build/liboracle.so, our FP64 restatement (tebd_oracle.cpp) of the
  reference MPS-TEBD engine (cuda/src/mps.cpp, cuda/src/linalg.cpp), the exact
  state-vector anneal (rust/src/quantum.rs) and the brute-force ground state
  (rust/src/ising.rs:46-61).
* ``Reference`` -- _ref/libtessera_ref.so, the reference engine compiled from its own
  sources plus ref_shim.cpp.  Present only where it was built (it is built where the
  reference sources are mounted and then travels as a prebuilt file).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtessera_ref.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_i8p = C.POINTER(C.c_int8)


def build(ref_root: str | None = None) -> None:
    """Compile the oracle (and the reference when its sources are mounted)."""
    cmd = ["make", "-s", "-C", HERE]
    if ref_root:
        cmd.append(f"REF_ROOT={ref_root}")
    subprocess.run(cmd, check=True)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a, t):
    return a.ctypes.data_as(t)


@dataclass
class Instance:
    """An Ising instance: E(s) = -sum_e w_e s_i s_j - sum_i h_i s_i (rust/src/ising.rs:23-32)."""

    h: np.ndarray
    ei: np.ndarray
    ej: np.ndarray
    ew: np.ndarray

    @property
    def n(self) -> int:
        return int(len(self.h))

    @property
    def m(self) -> int:
        return int(len(self.ew))

    def energy(self, spins) -> float:
        s = np.asarray(spins, dtype=np.float64)
        return float(-(np.asarray(self.ew) * s[self.ei] * s[self.ej]).sum() - (np.asarray(self.h) * s).sum())


@dataclass
class AnnealOut:
    spins: np.ndarray
    energy: float
    expected_energy: float
    prob: float
    max_trunc: float
    entropy: np.ndarray
    updates: int = 0
    max_bond: int = 0
    state: np.ndarray | None = None
    extra: dict = field(default_factory=dict)


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        L = self.lib
        L.orc_mps_anneal.argtypes = [_dp, C.c_int, _ip, _ip, _dp, C.c_int, _dp, _dp, C.c_int,
                                     C.c_double, C.c_int, C.c_int, _i8p, _dp, _dp, _dp, C.c_int]
        L.orc_sv_anneal.argtypes = [_dp, C.c_int, _ip, _ip, _dp, C.c_int, _dp, _dp, C.c_int,
                                    C.c_double, C.c_int, _i8p, _i8p, _dp, _dp, _dp]
        L.orc_sv_anneal_bias.argtypes = [_dp, C.c_int, _ip, _ip, _dp, C.c_int, _dp, _dp, C.c_int,
                                         C.c_double, C.c_int, _i8p, _i8p, _dp, _dp, _dp, _dp, _dp]
        L.orc_exact_ground.argtypes = [_dp, C.c_int, _ip, _ip, _dp, C.c_int, _i8p]
        L.orc_exact_ground.restype = C.c_double
        L.orc_sa_solve.argtypes = [_dp, C.c_int, _ip, _ip, _dp, C.c_int, C.c_int, C.c_int, C.c_double,
                                   C.c_double, C.c_uint64, C.c_uint64, _i8p]
        L.orc_sa_solve.restype = C.c_double
        L.orc_svd.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp]
        L.orc_mps_apply_slots.argtypes = [C.c_int, _ip, _dp, _ip, _ip, _dp, C.c_int, C.c_double, C.c_double,
                                          C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _ip, _dp,
                                          C.c_longlong, _dp]
        L.orc_mps_apply_slots.restype = C.c_longlong
        L.orc_hermitian_eig.argtypes = [C.c_int, _dp, _dp, _dp]
        L.orc_hermitian_expm.argtypes = [C.c_int, _dp, C.c_double, C.c_double, _dp]
        L.orc_mt_dense_instance.argtypes = [C.c_ulonglong, C.c_int, C.c_int, C.c_int, _dp, _ip,
                                            _ip, _dp, C.c_int]

    def mps_anneal(self, inst: Instance, sa, sb, dt: float, chi: int, zz_substeps: int = 1,
                   want_state: bool = False, accurate_svd: bool = False) -> AnnealOut:
        """The reference MPS-TEBD anneal.  accurate_svd=False reproduces the reference bit for
        bit (its Gram-matrix SVD included); True swaps in an accurate one-sided Jacobi SVD and
        keeps everything else (gate order, keep rule, gauge A=U, C=S Vh)."""
        h, ei, ej, ew, sa, sb = _d(inst.h), _i(inst.ei), _i(inst.ej), _d(inst.ew), _d(sa), _d(sb)
        n, steps = len(h), len(sa)
        spins = np.zeros(n, np.int8)
        ent = np.zeros(steps)
        st = np.zeros(10)
        state = np.zeros(2 << n) if want_state else None
        self.lib.orc_mps_anneal(_ptr(h, _dp), n, _ptr(ei, _ip), _ptr(ej, _ip), _ptr(ew, _dp), len(ew),
                                _ptr(sa, _dp), _ptr(sb, _dp), steps, dt, chi, zz_substeps,
                                _ptr(spins, _i8p), _ptr(ent, _dp), _ptr(st, _dp),
                                _ptr(state, _dp) if state is not None else None, 1 if accurate_svd else 0)
        return AnnealOut(spins, st[0], st[1], st[2], st[3], ent, int(st[4]), int(st[5]),
                         state.view(np.complex128) if state is not None else None,
                         extra={"max_recon": st[6], "bad_updates": int(st[7]), "norm2": st[8],
                                "min_cut_gap": st[9]})

    def apply_slots(self, inst: Instance, sites, B: float, dt: float, chi: int, q0: int, q1: int,
                    zz_substeps: int = 1, accurate_svd: bool = True):
        """Gate slots [q0, q1) of one step's ZZ block (ZZ weight B) applied to the MPS given as a
        list of site tensors (Dl, 2, Dr); returns (sites, stats) with stats = {max_trunc,
        updates, min_cut_gap, max_recon}.  The slot order is the reference's gate order through
        the swap network, the update its apply_adjacent (cuda/src/mps.cpp:41-145, 330-341)."""
        ei, ej, ew = _i(inst.ei), _i(inst.ej), _d(inst.ew)
        n = len(sites)
        dims = np.array([1] + [int(t.shape[2]) for t in sites], np.int32)
        flat = np.ascontiguousarray(np.concatenate([np.asarray(t, np.complex128).reshape(-1) for t in sites]))
        cap = 2 * sum(int(dims[i]) * 2 * max(int(dims[i + 1]), chi) * 2 for i in range(n)) + 64
        out = np.zeros(cap)
        odims = np.zeros(n + 1, np.int32)
        st = np.zeros(4)
        rc = self.lib.orc_mps_apply_slots(n, _ptr(dims, _ip), _ptr(flat.view(np.float64), _dp), _ptr(ei, _ip),
                                          _ptr(ej, _ip), _ptr(ew, _dp), len(ew), B, dt, zz_substeps, chi, q0, q1,
                                          1 if accurate_svd else 0, _ptr(odims, _ip), _ptr(out, _dp), cap,
                                          _ptr(st, _dp))
        if rc < 0:
            raise ValueError(f"orc_mps_apply_slots failed ({rc})")
        z = out[:rc].view(np.complex128)
        res, off = [], 0
        for i in range(n):
            cnt = int(odims[i]) * 2 * int(odims[i + 1])
            res.append(z[off:off + cnt].reshape(odims[i], 2, odims[i + 1]).copy())
            off += cnt
        return res, {"max_trunc": st[0], "updates": int(st[1]), "min_cut_gap": st[2], "max_recon": st[3]}

    def sv_anneal(self, inst: Instance, sa, sb, dt: float, mode: int = 0,
                  want_state: bool = False, bias=None, sc=None) -> AnnealOut:
        h, ei, ej, ew, sa, sb = _d(inst.h), _i(inst.ei), _i(inst.ej), _d(inst.ew), _d(sa), _d(sb)
        bias = None if bias is None else _d(bias)
        sc = None if sc is None else _d(sc)
        n, steps = len(h), len(sa)
        s_arg = np.zeros(n, np.int8)
        s_sign = np.zeros(n, np.int8)
        ent = np.zeros(steps)
        st = np.zeros(5)
        state = np.zeros(2 << n) if want_state else None
        self.lib.orc_sv_anneal_bias(_ptr(h, _dp), n, _ptr(ei, _ip), _ptr(ej, _ip), _ptr(ew, _dp), len(ew),
                                    _ptr(sa, _dp), _ptr(sb, _dp), steps, dt, mode, _ptr(s_arg, _i8p),
                                    _ptr(s_sign, _i8p), _ptr(ent, _dp), _ptr(st, _dp),
                                    _ptr(state, _dp) if state is not None else None,
                                    _ptr(bias, _dp) if bias is not None else None,
                                    _ptr(sc, _dp) if sc is not None else None)
        return AnnealOut(s_arg, st[0], st[1], st[2], 0.0, ent,
                         state=state.view(np.complex128) if state is not None else None,
                         extra={"sign_spins": s_sign, "sign_energy": st[3], "sign_prob": st[4]})

    def exact_ground(self, inst: Instance):
        h, ei, ej, ew = _d(inst.h), _i(inst.ei), _i(inst.ej), _d(inst.ew)
        s = np.zeros(len(h), np.int8)
        e = self.lib.orc_exact_ground(_ptr(h, _dp), len(h), _ptr(ei, _ip), _ptr(ej, _ip),
                                      _ptr(ew, _dp), len(ew), _ptr(s, _i8p))
        return s, float(e)

    def sa_solve(self, inst: Instance, restarts: int, sweeps: int, t0: float = 5.0, t_end: float = 0.01,
                 seed: int = 0, index: int = 0):
        """Best-of-restarts simulated annealing (rust/src/ising.rs:64-136) with the library's
        counter-based uniforms; `index` is the instance's position in a tessera_qa_sa_solve batch."""
        h, ei, ej, ew = _d(inst.h), _i(inst.ei), _i(inst.ej), _d(inst.ew)
        s = np.zeros(len(h), np.int8)
        e = self.lib.orc_sa_solve(_ptr(h, _dp), len(h), _ptr(ei, _ip), _ptr(ej, _ip), _ptr(ew, _dp), len(ew),
                                  restarts, sweeps, t0, t_end, seed, index, _ptr(s, _i8p))
        return s, float(e)

    def svd(self, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        r, c = a.shape
        k = min(r, c)
        s = np.zeros(k)
        u = np.zeros((r, k), np.complex128)
        vh = np.zeros((k, c), np.complex128)
        self.lib.orc_svd(r, c, _ptr(a.view(np.float64), _dp), _ptr(s, _dp),
                         _ptr(u.view(np.float64), _dp), _ptr(vh.view(np.float64), _dp))
        return u, s, vh

    def hermitian_eig(self, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        n = a.shape[0]
        w = np.zeros(n)
        v = np.zeros((n, n), np.complex128)
        self.lib.orc_hermitian_eig(n, _ptr(a.view(np.float64), _dp), _ptr(w, _dp),
                                   _ptr(v.view(np.float64), _dp))
        return w, v

    def hermitian_expm(self, a: np.ndarray, coeff: complex):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        n = a.shape[0]
        out = np.zeros((n, n), np.complex128)
        self.lib.orc_hermitian_expm(n, _ptr(a.view(np.float64), _dp), coeff.real, coeff.imag,
                                    _ptr(out.view(np.float64), _dp))
        return out

    def mt_dense_instance(self, seed: int, n: int, trials: int, want: int) -> Instance:
        """Instance `want` of the std::mt19937_64 generator used by cuda/tests/test_mps.cpp."""
        h = np.zeros(n)
        cap = n * (n - 1) // 2
        ei = np.zeros(cap, np.int32)
        ej = np.zeros(cap, np.int32)
        ew = np.zeros(cap)
        m = self.lib.orc_mt_dense_instance(seed, n, trials, want, _ptr(h, _dp), _ptr(ei, _ip),
                                           _ptr(ej, _ip), _ptr(ew, _dp), cap)
        return Instance(h, ei[:m].copy(), ej[:m].copy(), ew[:m].copy())


class Reference:
    """The reference engine compiled from its own sources (oracle/_ref)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        L.ref_mps_anneal.argtypes = [_dp, C.c_int, _ip, _ip, _dp, C.c_int, _dp, _dp, C.c_int,
                                     C.c_double, C.c_int, C.c_int, _i8p, _dp, _dp]
        L.ref_svd.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp]
        L.ref_svd.restype = C.c_int
        L.ref_hermitian_eig.argtypes = [C.c_int, _dp, _dp, _dp]
        L.ref_hermitian_expm.argtypes = [C.c_int, _dp, C.c_double, C.c_double, _dp]
        L.ref_grow_and_apply.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.c_int, C.c_int, C.c_int,
                                         C.c_double, C.c_int, _dp]
        L.ref_grow_and_apply.restype = C.c_int
        if hasattr(L, "ref_saturated_update"):
            L.ref_saturated_update.argtypes = [C.c_int, C.c_int, C.c_ulonglong, _dp, _dp]
            L.ref_saturated_update.restype = C.c_int
        L.tessera_qa_anneal.argtypes = [_dp, C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                        _dp, C.c_size_t, _dp, _dp, C.c_size_t, C.c_size_t, _i8p, _dp]
        L.tessera_qa_anneal.restype = C.c_double

    @staticmethod
    def available(path: str = REF_SO) -> bool:
        return os.path.exists(path)

    def mps_anneal(self, inst: Instance, sa, sb, dt: float, chi: int, zz_substeps: int = 1) -> AnnealOut:
        h, ei, ej, ew, sa, sb = _d(inst.h), _i(inst.ei), _i(inst.ej), _d(inst.ew), _d(sa), _d(sb)
        n, steps = len(h), len(sa)
        spins = np.zeros(n, np.int8)
        ent = np.zeros(steps)
        st = np.zeros(4)
        self.lib.ref_mps_anneal(_ptr(h, _dp), n, _ptr(ei, _ip), _ptr(ej, _ip), _ptr(ew, _dp), len(ew),
                                _ptr(sa, _dp), _ptr(sb, _dp), steps, dt, chi, zz_substeps,
                                _ptr(spins, _i8p), _ptr(ent, _dp), _ptr(st, _dp))
        return AnnealOut(spins, st[0], st[1], st[2], st[3], ent)

    def legacy_anneal(self, inst: Instance, sa, sb, chi: int):
        """The reference's own C ABI, tessera_qa_anneal (cuda/src/ffi.cpp:10-37)."""
        h, ew, sa, sb = _d(inst.h), _d(inst.ew), _d(sa), _d(sb)
        ei = np.ascontiguousarray(inst.ei, dtype=np.uint64)
        ej = np.ascontiguousarray(inst.ej, dtype=np.uint64)
        n, steps = len(h), len(sa)
        spins = np.zeros(n, np.int8)
        ent = np.zeros(steps)
        szp = C.POINTER(C.c_size_t)
        e = self.lib.tessera_qa_anneal(_ptr(h, _dp), n, _ptr(ei, szp), _ptr(ej, szp), _ptr(ew, _dp),
                                       len(ew), _ptr(sa, _dp), _ptr(sb, _dp), steps, chi,
                                       _ptr(spins, _i8p), _ptr(ent, _dp))
        return float(e), spins, ent

    def svd(self, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        r, c = a.shape
        k = min(r, c)
        s = np.zeros(k)
        u = np.zeros((r, k), np.complex128)
        vh = np.zeros((k, c), np.complex128)
        self.lib.ref_svd(r, c, _ptr(a.view(np.float64), _dp), _ptr(s, _dp),
                         _ptr(u.view(np.float64), _dp), _ptr(vh.view(np.float64), _dp))
        return u, s, vh

    def hermitian_eig(self, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        n = a.shape[0]
        w = np.zeros(n)
        v = np.zeros((n, n), np.complex128)
        self.lib.ref_hermitian_eig(n, _ptr(a.view(np.float64), _dp), _ptr(w, _dp),
                                   _ptr(v.view(np.float64), _dp))
        return w, v

    def hermitian_expm(self, a: np.ndarray, coeff: complex):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        n = a.shape[0]
        out = np.zeros((n, n), np.complex128)
        self.lib.ref_hermitian_expm(n, _ptr(a.view(np.float64), _dp), coeff.real, coeff.imag,
                                    _ptr(out.view(np.float64), _dp))
        return out

    def saturated_update(self, chi: int, reps: int = 1, seed: int = 0):
        """Wall times of `reps` updates of a saturated bond (theta (2 chi) x (2 chi)) through the
        reference's own MPS::apply_adjacent (cuda/src/mps.cpp:41-100); returns (seconds, bond)."""
        sec = np.zeros(reps)
        tr = np.zeros(1)
        bond = self.lib.ref_saturated_update(chi, reps, seed, _ptr(sec, _dp), _ptr(tr, _dp))
        return sec, int(bond)

    def grow_and_apply(self, n, chi, layers, gates: np.ndarray, zz_i, zz_j, theta, reps):
        g = np.ascontiguousarray(gates, dtype=np.complex128)
        tr = np.zeros(1)
        mb = self.lib.ref_grow_and_apply(n, chi, layers, _ptr(g.view(np.float64), _dp), g.shape[0],
                                         zz_i, zz_j, theta, reps, _ptr(tr, _dp))
        return mb, float(tr[0])


def smooth_schedule(steps: int):
    """A = cos^2(pi s/2), B = sin^2(pi s/2), s = k/(steps-1) (cuda/tests/test_mps.cpp:44-52)."""
    k = np.arange(steps, dtype=np.float64)
    s = k / (steps - 1)
    th = np.pi / 2 * s
    return np.cos(th) ** 2, np.sin(th) ** 2
