"""The C ABI boundary, checked without a GPU: the library loads, exports every function that
include/tessera_qa.h declares, and rejects invalid input before touching a device (the
reference has no validation at all; cuda/src/ffi.cpp:10-37)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from tessera_b200 import _lib, ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "tessera_qa.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tessera_qa_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    names = header_functions()
    assert "tessera_qa_anneal" in names and len(names) >= 10
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (\w+)", out))
    for nme in names:
        assert nme in exported, nme
        getattr(L, nme)


def test_legacy_symbol_signature_matches_rust_binding():
    """rust/src/ffi.rs:21-34: (f64*, usize, usize*, usize*, f64*, usize, f64*, f64*, usize, usize, i8*, f64*) -> f64."""
    L = _lib.load()
    assert L.tessera_qa_anneal.restype is C.c_double
    assert len(L.tessera_qa_anneal.argtypes) == 12


def test_config_defaults_are_the_legacy_ones():
    c, _ = ffi.config_struct()
    assert c.dt == 0.1 and c.zz_substeps == 1 and c.chi == 32 and c.precision == 0


def test_bad_schedule_rejected_like_rust():
    m = ffi.Ising([1.0], [])
    with pytest.raises(ffi.QaException) as e:
        ffi.quantum_anneal(m, ffi.Schedule([1.0], [0.0]), 32)
    assert e.value.err is ffi.QaError.BadSchedule


@pytest.mark.parametrize("case", ["nan_h", "edge_oob", "chi0", "n0", "nan_sched", "bad_dt", "bad_block", "bad_precond"])
def test_invalid_input_returns_einval_without_a_gpu(case):
    h = np.array([0.1, -0.2, 0.3])
    ei, ej, ew = np.array([0, 1]), np.array([1, 2]), np.array([0.5, -0.5])
    sa, sb = np.linspace(1, 0, 5), np.linspace(0, 1, 5)
    kw = {}
    if case == "nan_h":
        h = np.array([np.nan, 0, 0])
    elif case == "edge_oob":
        ej = np.array([1, 3])
    elif case == "chi0":
        kw["chi"] = 0
    elif case == "n0":
        h = np.zeros(0)
        ei, ej, ew = np.zeros(0), np.zeros(0), np.zeros(0)
    elif case == "nan_sched":
        sb = np.array([0, np.inf, 0.5, 0.7, 1.0])
    elif case == "bad_dt":
        kw["dt"] = -1.0
    elif case == "bad_block":
        kw["jacobi_block"] = 3
    elif case == "bad_precond":
        kw["jacobi_precondition"] = 3
    with pytest.raises(_lib.EngineError) as e:
        ffi.anneal(h, ei, ej, ew, sa, sb, **kw)
    assert e.value.code == _lib.EINVAL
    assert len(_lib.last_error()) > 0


def test_legacy_symbol_returns_nan_on_invalid_input():
    L = _lib.load()
    h = np.array([np.nan])
    s = np.zeros(1, np.int8)
    e = L.tessera_qa_anneal(h.ctypes.data_as(_lib.c_double_p), 1, None, None, None, 0, None, None, 0, 8,
                            s.ctypes.data_as(_lib.c_int8_p), None)
    assert np.isnan(e)
    e = L.tessera_qa_anneal(h.ctypes.data_as(_lib.c_double_p), 1, None, None, None, 0, None, None, 0, 8, None, None)
    assert np.isnan(e)


def test_checkpoint_size_bound():
    L = _lib.load()
    assert L.tessera_qa_checkpoint_bytes(4, 2) >= 32 + 4 * 2 * 2 * 2 * 16


def test_checkpoint_decoder_roundtrip():
    # a hand-built 2-site checkpoint: dims [1, 2, 1]
    n = 2
    hdr = bytearray(32 + (4 * 3 + 7) // 8 * 8)
    hdr[0:8] = b"TQMPSv1\x00"
    hdr[8:12] = np.uint32(n).tobytes()
    hdr[32:44] = np.array([1, 2, 1], np.int32).tobytes()
    a = (np.arange(4) + 1j).astype(np.complex128).reshape(1, 2, 2)
    b = (np.arange(4) - 2j).astype(np.complex128).reshape(2, 2, 1)
    buf = bytes(hdr) + a.tobytes() + b.tobytes()
    dims, sites = ffi.checkpoint_to_sites(buf)
    assert list(dims) == [1, 2, 1]
    assert np.allclose(sites[0], a) and np.allclose(sites[1], b)
    psi = ffi.sites_to_dense(sites)
    ref = np.array([(a[0, s0] @ b[:, s1, 0]) for s1 in range(2) for s0 in range(2)])
    assert np.allclose(psi, ref)


@pytest.mark.parametrize("case", ["n31", "steps1", "bad_dt", "bad_mode", "bias_mode0", "edge_oob", "nan_h"])
def test_state_vector_rejects_invalid_input_without_a_gpu(case):
    """tessera_qa_sv_anneal validates before its first CUDA call: EINVAL and a message."""
    n = 31 if case == "n31" else 3
    h = np.full(n, 0.1)
    ei, ej, ew = np.array([0, 1]), np.array([1, 2]), np.array([0.5, -0.5])
    steps = 1 if case == "steps1" else 5
    sa, sb = np.linspace(1, 0, steps), np.linspace(0, 1, steps)
    kw = dict(dt=0.1, mode=0)
    if case == "bad_dt":
        kw["dt"] = 0.0
    elif case == "bad_mode":
        kw["mode"] = 2
    elif case == "bias_mode0":
        kw.update(bias=np.ones(n), sc=np.ones(steps))
    elif case == "edge_oob":
        ej = np.array([1, 3])
    elif case == "nan_h":
        h[1] = np.nan
    with pytest.raises(_lib.EngineError) as e:
        ffi.sv_anneal(h, ei, ej, ew, sa, sb, **kw)
    assert e.value.code == _lib.EINVAL
    assert len(_lib.last_error()) > 0


@pytest.mark.parametrize("shape", [(0, 4), (4, 0), (2049, 4), (4, 2049)])
def test_svd_rejects_out_of_range_shapes_without_a_gpu(shape):
    L = _lib.load()
    r, c = shape
    a = np.zeros(2 * max(r * c, 1))
    s = np.zeros(max(min(r, c), 1))
    rc = L.tessera_qa_svd(a.ctypes.data_as(_lib.c_double_p), r, c, s.ctypes.data_as(_lib.c_double_p), None, None)
    assert rc == _lib.EINVAL
    assert "shape" in _lib.last_error()


@pytest.mark.parametrize("shape", [(0, 4), (257, 4), (4, 257)])
def test_noalloc_svd_rejects_out_of_range_shapes_without_a_gpu(shape):
    import ctypes as C
    L = _lib.load()
    dummy = C.c_void_p(16)  # never dereferenced: the shape check comes first
    rc = L.tessera_qa_svd_noalloc(dummy, shape[0], shape[1], dummy, None, None)
    assert rc == _lib.EINVAL
    assert "rows and cols" in _lib.last_error()


def test_null_handles_and_structs_are_rejected_without_a_gpu():
    """Every handle-taking entry point returns EINVAL (or NULL / 0 / no-op for the void and
    size-returning ones) on a NULL handle or NULL struct, before any CUDA call."""
    import ctypes as C
    L = _lib.load()
    f0 = C.c_float(0.0)
    einval = {
        "session_randomize": lambda: L.tessera_qa_session_randomize(None, 1),
        "session_randomize_graded": lambda: L.tessera_qa_session_randomize_graded(None, 1, 24.0),
        "session_run": lambda: L.tessera_qa_session_run(None, 0, 1),
        "session_run_gates": lambda: L.tessera_qa_session_run_gates(None, 0, 0, 1),
        "session_run_host": lambda: L.tessera_qa_session_run_host(None, None, 0, 0, 0, 0, None),
        "session_sync": lambda: L.tessera_qa_session_sync(None, None),
        "session_observe": lambda: L.tessera_qa_session_observe(None, None),
        "session_save": lambda: L.tessera_qa_session_save(None, None, 0),
        "session_load": lambda: L.tessera_qa_session_load(None, None, 0),
        "session_sample": lambda: L.tessera_qa_session_sample(None, 1, 1, None, None),
        "session_save_instance": lambda: L.tessera_qa_session_save_instance(None, 0, None, 0),
        "gnn_get_params": lambda: L.tessera_qa_gnn_get_params(None, None, 0),
        "gnn_set_params": lambda: L.tessera_qa_gnn_set_params(None, None, 0),
        "gnn_forward": lambda: L.tessera_qa_gnn_forward(None, None, 0, None, None),
        "gnn_train_step": lambda: L.tessera_qa_gnn_train_step(None, None, 0, None, None, f0, f0, None, None),
        "gnn_apply_grads": lambda: L.tessera_qa_gnn_apply_grads(None, None, 0, f0),
        "schedule_predict": lambda: L.tessera_qa_schedule_predict(None, None, 0, None, None),
        "anneal_ex": lambda: L.tessera_qa_anneal_ex(None, None, None),
        "anneal_batch": lambda: L.tessera_qa_anneal_batch(None, None, None, 1),
        "sv_anneal": lambda: L.tessera_qa_sv_anneal(None, 0.1, 0, None),
    }
    for name, call in einval.items():
        assert call() == _lib.EINVAL, name
    assert not L.tessera_qa_session_stream(None)
    assert not L.tessera_qa_session_create(None, None)
    assert not L.tessera_qa_session_create_batch(None, None, 0)
    assert L.tessera_qa_gnn_param_count(None) == 0
    L.tessera_qa_session_destroy(None)
    L.tessera_qa_gnn_destroy(None)


def test_sa_solver_rejects_invalid_input_without_a_gpu():
    from tessera_b200 import instances
    p = instances.dense_er(8, 1, T=1.0, dt=0.1, chi=8)
    for kw in ({"restarts": 0}, {"sweeps": 0}, {"t0": 0.0}, {"t_end": float("nan")}):
        with pytest.raises(_lib.EngineError) as e:
            ffi.sa_solve([p], **kw)
        assert e.value.code == _lib.EINVAL, kw
    big = instances.chain_range(n=130, dmax=1, seed=1, T=1.0, dt=0.1, chi=8)
    with pytest.raises(_lib.EngineError) as e:
        ffi.sa_solve([big])
    assert e.value.code == _lib.EINVAL and "128" in str(e.value)
