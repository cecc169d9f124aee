"""The tcgen05 BF16 GEMM against an FP32 matmul of the same BF16 inputs.

Bound: |C - C_ref| <= 1e-3 * max|C_ref| + 1e-3 -- both accumulate exact BF16
products in FP32, so only summation order differs."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from uph_b200 import _lib as L
    lib = L.lib()
    f = lib.uph_tc_gemm_bf16
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                  C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                  C.c_void_p]
    return lib


def tc_gemm(torch, A, B, bias=None, relu=False, splits=1, bf16_out=False):
    lib = _lib()
    M, K = A.shape
    N = B.shape[0]
    c32 = torch.zeros(M, N, dtype=torch.float32, device="cuda")
    c16 = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda") if bf16_out else None
    part = torch.empty(splits * M * N, dtype=torch.float32, device="cuda") if splits > 1 else None
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = lib.uph_tc_gemm_bf16(A.data_ptr(), K, B.data_ptr(), K, M, N, K,
                              bias.data_ptr() if bias is not None else None, int(relu), c32.data_ptr(),
                              c16.data_ptr() if c16 is not None else None, N, splits,
                              part.data_ptr() if part is not None else None, 0, err.data_ptr(),
                              torch.cuda.current_stream().cuda_stream)
    assert st == 0, lib.uph_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0, "device error word set"
    return c32, c16


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (300, 128, 128), (1000, 256, 384), (4096, 128, 256)])
def test_tc_gemm_matches_fp32_matmul(M, N, K):
    torch = pytest.importorskip("torch")
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    ref = A.float() @ B.float().T
    c, _ = tc_gemm(torch, A, B)
    tol = 1e-3 * ref.abs().max().item() + 1e-3
    assert (c - ref).abs().max().item() <= tol
    c, c16 = tc_gemm(torch, A, B, bias=bias, relu=True, bf16_out=True)
    ref2 = torch.relu(ref + bias)
    assert (c - ref2).abs().max().item() <= tol
    assert (c16.float() - ref2).abs().max().item() <= tol + 1e-2 * ref2.abs().max().item()


def test_tc_gemm_split_k_reduction():
    """dW-style product: a long K (nodes) split across CTAs, FP32 partials
    summed in a fixed order -- identical results on repeated calls."""
    torch = pytest.importorskip("torch")
    g = torch.Generator(device="cuda").manual_seed(7)
    M, N, K = 128, 256, 64 * 300
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    ref = A.float() @ B.float().T
    c1, _ = tc_gemm(torch, A, B, splits=24)
    c2, _ = tc_gemm(torch, A, B, splits=24)
    assert torch.equal(c1, c2)
    assert (c1 - ref).abs().max().item() <= 1e-3 * ref.abs().max().item() + 1e-3


def test_bounded_wait_gives_up_and_leaves_the_context_usable():
    """Failure detection on the GPU without a fault: the self test's CTA waits
    on an mbarrier that nothing arrives at.  The wait gives up after about a
    second, the kernel reports ERR_TIMEOUT (UPH_TIMEOUT), frees its TMEM and
    returns; a normal GEMM right after it is still correct."""
    import time
    torch = pytest.importorskip("torch")
    from uph_b200 import _lib as L
    lib = L.lib()
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(128, 64, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(128, 64, device="cuda", generator=g).to(torch.bfloat16)
    c = torch.zeros(128, 128, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    t0 = time.time()
    st = lib.uph_tc_wait_selftest(A.data_ptr(), B.data_ptr(), c.data_ptr(), err.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream)
    elapsed = time.time() - t0
    assert st == 5, (st, lib.uph_last_error())  # UPH_TIMEOUT
    assert int(err.item()) & 8  # ERR_TIMEOUT
    assert 0.5 <= elapsed <= 30.0, elapsed
    out, _ = tc_gemm(torch, A, B)
    ref = A.float() @ B.float().T
    assert (out - ref).abs().max().item() <= 1e-3 * ref.abs().max().item() + 1e-3
