"""The tcgen05 (5th-gen tensor core) TF32 GEMM core against FP64 products.

Plain TF32 carries ~2^-11 relative error per product; the 3-pass hi/lo split
~2^-22.  Errors are measured relative to sum_k |A||B| (the product's scale).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _split(x):
    from ipie_b200._lib import call, ptr, stream

    xd = x.contiguous()
    hi = torch.empty(xd.shape, dtype=torch.float32, device="cuda")
    lo = torch.empty_like(hi)
    call("ipie_b200_split_tf32", ptr(xd), ptr(hi), ptr(lo), xd.numel(), stream())
    return hi, lo


@pytest.mark.parametrize("M,N,K,na,nsplit", [(200, 300, 256, 1, 1), (200, 300, 256, 1, 3), (130, 64, 200, 2, 3),
                                             (1000, 512, 1600, 1, 3), (37, 70, 36, 1, 1)])
def test_umma_gemm_matches_fp64(M, N, K, na, nsplit):
    from ipie_b200._lib import call, ptr, stream

    g = torch.Generator(device="cpu").manual_seed(M + N + K)
    A = [torch.randn(M, K, generator=g, dtype=torch.float64).cuda() for _ in range(na)]
    B = torch.randn(N, K, generator=g, dtype=torch.float64).cuda()
    ah = [_split(a) for a in A]
    bh, bl = _split(B)
    a0h, a0l = ah[0]
    a1h, a1l = ah[1] if na == 2 else (None, None)
    c = torch.full((M, na, N), float("nan"), dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    call("ipie_b200_umma_gemm_test", ptr(a0h), ptr(a0l), ptr(a1h), ptr(a1l), ptr(bh), ptr(bl), ptr(c), M, N, K, na,
         nsplit, ptr(status), stream())
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    for a in range(na):
        ref = A[a] @ B.T
        scale = (A[a].abs() @ B.abs().T).max().item()
        err = (c[:, a, :].double() - ref).abs().max().item() / scale
        tol = 2e-3 if nsplit == 1 else 1e-5  # fp32 accumulation over K adds ~sqrt(K) 2^-24
        assert err < tol, (a, err)


def _split16(x, scale):
    from ipie_b200._lib import call, ptr, stream

    xd = x.contiguous()
    hi = torch.empty(xd.shape, dtype=torch.float16, device="cuda")
    lo = torch.empty_like(hi)
    call("ipie_b200_split_f16", ptr(xd), ptr(hi), ptr(lo), xd.numel(), scale, stream())
    return hi, lo


@pytest.mark.parametrize("M,N,K,nsplit", [(200, 300, 256, 1), (200, 300, 256, 3), (1000, 512, 1600, 3), (37, 70, 40, 3),
                                          (130, 260, 6400, 3)])
def test_umma_gemm_f16_matches_fp64(M, N, K, nsplit):
    """FP16 operands scaled by powers of two (max near 2^14): the 3-pass product carries ~2^-22
    of sum |A||B| like the TF32 one, a single pass ~2^-11; entries spread over six decades
    (most below the split's relative range) only add an absolute ~2^-25 per element."""
    from ipie_b200._lib import call, ptr, stream

    g = torch.Generator(device="cpu").manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g, dtype=torch.float64) * 10.0 ** (-6 * torch.rand(M, K, generator=g))
    B = torch.randn(N, K, generator=g, dtype=torch.float64) * 3.0
    A, B = A.cuda(), B.cuda()
    sa = 2.0 ** (14 - np.ceil(np.log2(A.abs().max().item())))
    sb = 2.0 ** (14 - np.ceil(np.log2(B.abs().max().item())))
    ah, al = _split16(A, sa)
    bh, bl = _split16(B, sb)
    c = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    call("ipie_b200_umma_gemm_f16_test", ptr(ah), ptr(al), ptr(bh), ptr(bl), ptr(c), M, N, K, nsplit, ptr(status),
         stream())
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    ref = A @ B.T
    scale = (A.abs() @ B.abs().T).max().item()
    err = (c.double() / (sa * sb) - ref).abs().max().item() / scale
    tol = 2e-3 if nsplit == 1 else 1e-5
    assert err < tol, err
