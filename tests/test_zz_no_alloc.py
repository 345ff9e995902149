"""tessera_qa_svd_noalloc -- the SVD entry point for callers that cannot allocate device memory.

Such callers (code whose device heap is owned by a host application's or framework's
allocator, or services that forbid allocation after start-up) hand the library device
buffers they already own; the entry point keeps its scratch in a fixed file-scope device
array instead of calling cudaMalloc.  This file sorts last so that a run stopping at the
first failure has already run every other test; it also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

from tessera_b200 import _lib, ffi

pytestmark = pytest.mark.gpu


def _noalloc_svd(L, torch, a: np.ndarray):
    dev = torch.device("cuda", torch.cuda.current_device())
    d_a = torch.from_numpy(np.ascontiguousarray(a).view(np.float64).copy()).to(dev)
    r, c = a.shape
    k = min(r, c)
    d_s = torch.zeros(k, dtype=torch.float64, device=dev)
    d_u = torch.zeros(2 * r * k, dtype=torch.float64, device=dev)
    rc = L.tessera_qa_svd_noalloc(C.c_void_p(d_a.data_ptr()), r, c, C.c_void_p(d_s.data_ptr()),
                                  C.c_void_p(d_u.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, _lib.last_error()
    return d_s.cpu().numpy(), d_u.cpu().numpy().view(np.complex128).reshape(r, k)


@pytest.mark.parametrize("shape", [(64, 48), (256, 256)])
def test_noalloc_svd_matches_tessera_qa_svd_twice(shape):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    L = _lib.load()
    rng = np.random.Generator(np.random.PCG64(11 + shape[0]))
    for call in range(2):  # two calls in a row share (and must reset) the scratch array
        a = rng.normal(size=shape) + 1j * rng.normal(size=shape)
        U0, s0, _ = np.linalg.svd(a, full_matrices=False)
        a = (U0 * np.exp(-np.arange(len(s0)) / 10.0)) @ _  # decaying spectrum, distinct values
        u_ref, s_ref, _vh = ffi.svd(a)          # existing entry point (host buffers)
        s, u = _noalloc_svd(L, torch, a)
        assert np.allclose(s, s_ref, rtol=1e-10, atol=1e-13), call
        # singular vectors agree up to a phase per column
        ov = np.abs(np.sum(np.conj(u) * u_ref, axis=0))
        assert np.all(np.abs(ov - 1.0) < 1e-9), (call, ov.min())


def test_noalloc_svd_rejects_oversize():
    torch = pytest.importorskip("torch")
    L = _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    buf = torch.zeros(2 * 300 * 300, dtype=torch.float64, device=dev)
    s = torch.zeros(300, dtype=torch.float64, device=dev)
    rc = L.tessera_qa_svd_noalloc(C.c_void_p(buf.data_ptr()), 300, 300, C.c_void_p(s.data_ptr()), None, None)
    assert rc == _lib.EINVAL
    assert "256" in _lib.last_error()
