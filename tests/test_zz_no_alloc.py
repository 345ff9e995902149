"""tessera_qa_svd_noalloc -- the SVD entry point for callers that cannot allocate device memory.

Such callers (code whose device heap is owned by a host application's or framework's
allocator, or services that forbid allocation after start-up) hand the library device
buffers they already own; the entry point keeps its scratch in a fixed file-scope device
array instead of calling cudaMalloc.  This file sorts last so that a run stopping at the
first failure has already run every other test; it also passes when run alone.

Each case builds a matrix with a known spectrum, exp(-k/10), and checks the entry point
against that spectrum and its singular vectors, and against tessera_qa_svd (the existing
entry point, host buffers) within the same tolerances: singular values rel 1e-10 / abs
1e-13, singular vectors up to a phase to 1e-9.  Tall, square, wide and odd shapes are
covered, and the device's free memory is the same before and after a second call.
"""
import ctypes as C

import numpy as np
import pytest

from tessera_b200 import _lib, ffi

pytestmark = pytest.mark.gpu


def _known(shape, rng):
    """A matrix U diag(exp(-k/10)) Vh with random isometries U, Vh; returns (a, U, s)."""
    r, c = shape
    x = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    u0, _, vh0 = np.linalg.svd(x, full_matrices=False)
    s = np.exp(-np.arange(min(r, c)) / 10.0)
    return (u0 * s) @ vh0, u0, s


class _Buffers:
    """Device buffers owned by the caller (torch here), allocated once and reused."""

    def __init__(self, torch, shape):
        r, c = shape
        k = min(r, c)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.torch, self.shape, self.k = torch, shape, k
        self.a = torch.zeros(2 * r * c, dtype=torch.float64, device=dev)
        self.s = torch.zeros(k, dtype=torch.float64, device=dev)
        self.u = torch.zeros(2 * r * k, dtype=torch.float64, device=dev)

    def call(self, L, a: np.ndarray):
        torch = self.torch
        r, c = self.shape
        self.a.copy_(torch.from_numpy(np.ascontiguousarray(a).view(np.float64).reshape(-1)))
        rc = L.tessera_qa_svd_noalloc(C.c_void_p(self.a.data_ptr()), r, c, C.c_void_p(self.s.data_ptr()),
                                      C.c_void_p(self.u.data_ptr()),
                                      C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        return self.s.cpu().numpy(), self.u.cpu().numpy().view(np.complex128).reshape(r, self.k)


def _same_columns(u, v):
    """|<u_t, v_t>| for every column t (1 when equal up to a phase)."""
    return np.abs(np.sum(np.conj(u) * v, axis=0))


@pytest.mark.parametrize("shape", [(64, 48), (256, 256), (48, 64), (256, 17), (17, 33)])
def test_noalloc_svd_matches_known_spectrum_and_tessera_qa_svd_twice(shape):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    L = _lib.load()
    rng = np.random.Generator(np.random.PCG64(11 + shape[0] + 3 * shape[1]))
    buf = _Buffers(torch, shape)
    for call in range(2):  # two calls in a row share (and must reset) the scratch array
        a, u_true, s_true = _known(shape, rng)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        s, u = buf.call(L, a)
        if call == 1:  # the first call may set up the array; the second allocates nothing
            assert torch.cuda.mem_get_info()[0] == free_before
        assert np.allclose(s, s_true, rtol=1e-10, atol=1e-13), (call, np.max(np.abs(s - s_true)))
        assert np.all(np.abs(_same_columns(u, u_true) - 1.0) < 1e-9), call
        u_ref, s_ref, _vh = ffi.svd(a)  # existing entry point (host buffers)
        assert np.allclose(s, s_ref, rtol=1e-10, atol=1e-13), call
        assert np.all(np.abs(_same_columns(u, u_ref) - 1.0) < 1e-9), call


def test_noalloc_svd_rejects_oversize():
    torch = pytest.importorskip("torch")
    L = _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    buf = torch.zeros(2 * 300 * 300, dtype=torch.float64, device=dev)
    s = torch.zeros(300, dtype=torch.float64, device=dev)
    rc = L.tessera_qa_svd_noalloc(C.c_void_p(buf.data_ptr()), 300, 300, C.c_void_p(s.data_ptr()), None, None)
    assert rc == _lib.EINVAL
    assert "256" in _lib.last_error()
