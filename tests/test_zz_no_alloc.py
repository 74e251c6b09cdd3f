"""The allocation-free exchange entry point against the workspace entry point.

``ipie_b200_exchange_noalloc`` serves callers that cannot allocate device
memory where they need the exchange energy -- a code whose device memory is
owned by its own pool allocator, or a loop that must not take the implicit
synchronisation of cudaMalloc/cudaFree.  It keeps its partial sums in a fixed
16 MiB device array inside the library.  This file is collected last so a
failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = 1e-10  # relative, as in the other FP64 parity tests


def _lib():
    from ipie_b200._lib import lib

    return lib()


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _inputs(W, X, M, N, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    rchol = torch.randn(X, N * M, generator=g, dtype=torch.float64).cuda()
    ghalf = torch.complex(torch.randn(W, N, M, generator=g, dtype=torch.float64),
                          torch.randn(W, N, M, generator=g, dtype=torch.float64)).cuda()
    return rchol, ghalf


def _with_workspace(rchol, ghalf, W, X, M, N):
    lib = _lib()
    rows = lib.ipie_b200_exchange_rows(W, X, M, N)
    part = torch.empty(rows * W, dtype=torch.complex128, device="cuda")
    rc = lib.ipie_b200_exchange(_p(rchol), _p(ghalf), W, X, M, N, _p(part), _stream())
    assert rc == 0
    return part.view(rows, W).sum(dim=0)


@pytest.mark.parametrize("W,X,M,N", [(100, 300, 60, 12), (37, 120, 26, 5), (2048, 1600, 200, 32)])
def test_noalloc_matches_workspace_entry_point_twice(W, X, M, N):
    rchol, ghalf = _inputs(W, X, M, N, seed=W + X)
    ref = _with_workspace(rchol, ghalf, W, X, M, N)
    lib = _lib()
    for _ in range(2):  # two calls in a row share the library's scratch array
        exx = torch.full((W,), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda")
        rc = lib.ipie_b200_exchange_noalloc(_p(rchol), _p(ghalf), W, X, M, N, _p(exx), _stream())
        assert rc == 0
        torch.cuda.synchronize()
        err = (exx - ref).abs().max().item() / ref.abs().max().item()
        assert err < TOL, err


def test_noalloc_smaller_call_after_larger_one():
    """A large call leaves its partials in the shared array; a following call with fewer walkers
    (a different row stride) and other data must read only what it wrote itself."""
    lib = _lib()
    big = (2048, 1600, 200, 32)
    rchol, ghalf = _inputs(*big, seed=3)
    exx = torch.empty(big[0], dtype=torch.complex128, device="cuda")
    assert lib.ipie_b200_exchange_noalloc(_p(rchol), _p(ghalf), *big, _p(exx), _stream()) == 0
    del rchol, ghalf, exx
    small = (300, 500, 40, 8)
    rchol, ghalf = _inputs(*small, seed=11)
    ref = _with_workspace(rchol, ghalf, *small)
    exx = torch.full((small[0],), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda")
    assert lib.ipie_b200_exchange_noalloc(_p(rchol), _p(ghalf), *small, _p(exx), _stream()) == 0
    torch.cuda.synchronize()
    err = (exx - ref).abs().max().item() / ref.abs().max().item()
    assert err < TOL, err


def test_noalloc_rejects_sizes_beyond_its_scratch():
    """8192 walkers x 129 partial rows exceed the 1048576-entry array and are rejected before any
    launch.  The buffers are sized for the call (small M and N keep them cheap), so a broken size
    check would give a wrong answer here rather than touch memory outside them."""
    lib = _lib()
    W, X, M, N = 8192, 2064, 8, 8
    assert lib.ipie_b200_exchange_rows(W, X, M, N) * W > 1048576
    rchol, ghalf = _inputs(W, X, M, N, seed=1)
    exx = torch.zeros(W, dtype=torch.complex128, device="cuda")
    rc = lib.ipie_b200_exchange_noalloc(_p(rchol), _p(ghalf), W, X, M, N, _p(exx), _stream())
    assert rc == 1  # cudaErrorInvalidValue
    torch.cuda.synchronize()
    assert bool((exx == 0).all())
