"""Host-side fault injection on the GPU paths: device allocations that fail.

tessera_qa_debug_fail_allocations(after, count) makes the library's own cudaMalloc calls fail
(cudaErrorMemoryAllocation) after `after` successful ones, so every allocation of a call can be
made to fail in turn without exhausting a GPU.  A call that meets the failure must return
TESSERA_QA_ECUDA (the legacy symbol: NaN) with an "out of memory" message, leave its outputs
untouched, release what it had allocated before the failure (the device's free memory is the
same before and after), and leave the library usable: the next call succeeds.
"""
import numpy as np
import pytest

from tessera_b200 import _lib, ffi, instances

pytestmark = pytest.mark.gpu


def _problem():
    return instances.chain_range(n=8, dmax=2, seed=9, T=1.0, dt=0.1, chi=8, dist="normal", hzero=False)


def _legacy(L, p, spins, ent):
    ei = np.ascontiguousarray(p.ei, np.uint64)
    ej = np.ascontiguousarray(p.ej, np.uint64)
    return L.tessera_qa_anneal(p.h.ctypes.data_as(_lib.c_double_p), p.n, ei.ctypes.data_as(_lib.c_size_p),
                               ej.ctypes.data_as(_lib.c_size_p), p.ew.ctypes.data_as(_lib.c_double_p), p.m,
                               p.sa.ctypes.data_as(_lib.c_double_p), p.sb.ctypes.data_as(_lib.c_double_p),
                               p.steps, 8, spins.ctypes.data_as(_lib.c_int8_p), ent.ctypes.data_as(_lib.c_double_p))


@pytest.fixture
def lib():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    L = _lib.load()
    yield L, torch
    L.tessera_qa_debug_fail_allocations(0, 0)


def test_every_allocation_of_an_anneal_can_fail_cleanly(lib):
    L, torch = lib
    p = _problem()
    ok = ffi.anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=8)  # loads every kernel once
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    failed = 0
    for after in range(8):
        L.tessera_qa_debug_fail_allocations(after, 1)
        try:
            r = ffi.anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=8)
        except _lib.EngineError as e:
            assert e.code == _lib.ECUDA, after
            assert "out of memory" in str(e), after
            failed += 1
        else:  # fewer allocations than after + 1: the call ran clean and the failure is still pending
            assert L.tessera_qa_debug_fail_allocations(0, 0) == 1, after
            assert r.expected_energy == ok.expected_energy
            break
        assert L.tessera_qa_debug_fail_allocations(0, 0) == 0, after
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0, after  # nothing leaked
    assert failed >= 2  # the arena and at least one lazily made buffer
    again = ffi.anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=8)
    assert again.expected_energy == ok.expected_energy and list(again.spins) == list(ok.spins)


def test_legacy_symbol_returns_nan_and_leaves_outputs_untouched(lib):
    L, _ = lib
    p = _problem()
    spins = np.full(p.n, 7, np.int8)
    ent = np.full(p.steps, -5.0)
    L.tessera_qa_debug_fail_allocations(0, 1)
    e = _legacy(L, p, spins, ent)
    assert np.isnan(e)
    assert np.all(spins == 7) and np.all(ent == -5.0)
    assert "out of memory" in _lib.last_error()
    e = _legacy(L, p, spins, ent)
    assert np.isfinite(e) and set(spins.tolist()) <= {-1, 1}


def test_batch_session_state_vector_and_gnn_fail_cleanly(lib):
    L, torch = lib
    p = _problem()
    probs = [p, instances.chain_nn(n=10, seed=3, T=1.0, dt=0.1, chi=8)]
    ffi.anneal_batch(probs)
    ffi.sv_anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, mode=1)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for after in (0, 1, 2):  # the instances' arenas, then the batch's own
        L.tessera_qa_debug_fail_allocations(after, 1)
        with pytest.raises(_lib.EngineError) as err:
            ffi.anneal_batch(probs)
        assert err.value.code == _lib.ECUDA
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0, after
    # handle-returning calls give NULL; the message says why
    L.tessera_qa_debug_fail_allocations(0, 1)
    with pytest.raises(_lib.EngineError) as err:
        ffi.Session(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, chi=8)
    assert "out of memory" in str(err.value)
    L.tessera_qa_debug_fail_allocations(0, 1)
    with pytest.raises(_lib.EngineError) as err:
        ffi.sv_anneal(p.h, p.ei, p.ej, p.ew, p.sa, p.sb, dt=p.dt, mode=1)
    assert err.value.code == _lib.ECUDA
    from tessera_b200 import learned
    for after in (0, 1):  # the weights, then their BF16 copy
        L.tessera_qa_debug_fail_allocations(after, 1)
        with pytest.raises(_lib.EngineError) as err:
            learned.ScheduleGNN(hidden=16, layers=2, knots=8, seed=2)
        assert "out of memory" in str(err.value)
    L.tessera_qa_debug_fail_allocations(0, 0)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    r = ffi.anneal_batch(probs)
    assert all(x.status == 0 for x in r)
