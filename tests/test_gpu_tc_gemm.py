"""The BF16 tensor-core GEMM (tcgen05 + TMA, FP32 accumulation) that the
surrogate's training passes run on, against a float64 product of the same
BF16-rounded operands."""
import ctypes as C

import numpy as np
import pytest

from bhrt import lib

pytestmark = pytest.mark.gpu


def _run(M, N, K, splits=1, accumulate=False, bias=False, seed=0):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    C0 = torch.randn(M, N, generator=g).float().cuda() if accumulate else torch.zeros(M, N).cuda()
    b = torch.randn(N, generator=g).float().cuda() if bias else None
    Cg = C0.clone()
    L = lib.load()
    code = L.bhTcGemm(C.c_void_p(A.data_ptr()), K, C.c_void_p(B.data_ptr()), K, C.c_void_p(Cg.data_ptr()), N,
                      M, N, K, splits, 1 if accumulate else 0, C.c_void_p(b.data_ptr()) if bias else None,
                      C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert code == 0
    torch.cuda.synchronize()
    flags = C.c_uint(99)
    assert L.bhTcErrorFlags(C.byref(flags)) == 0 and flags.value == 0
    ref = A.double().cpu() @ B.double().cpu().T
    if bias:
        ref += b.double().cpu()
    if accumulate or splits > 1:
        ref += C0.double().cpu()
    got = Cg.double().cpu()
    err = (got - ref).abs().max().item()
    scale = ref.abs().max().item()
    return err, scale


@pytest.mark.parametrize("M,N,K,splits,acc,bias", [
    (128, 256, 64, 1, False, False),
    (256, 256, 256, 1, False, True),
    (300, 16, 256, 1, False, False),      # ragged M, the head's N
    (1000, 64, 128, 1, True, True),
    (256, 256, 4096, 8, False, False),    # split-K, the weight-gradient shape
    (384, 200, 192, 3, False, True),      # ragged N inside a 256 tile
])
def test_tc_gemm_matches_float64(cuda, M, N, K, splits, acc, bias):
    err, scale = _run(M, N, K, splits, acc, bias)
    print(f"M={M} N={N} K={K} splits={splits}: max abs err {err:.3g} (scale {scale:.3g})")
    # FP32 accumulation of K exact BF16 products: error ~ K * 2^-24 * |terms|
    assert err <= 1e-5 * K * 4.0 + 1e-4


def test_bounded_wait_times_out_reports_and_device_stays_usable(cuda):
    """A barrier wait that nothing completes gives up after its limit (1 ms here), sets the
    error flag that bhTcErrorFlags reads (and clears), and leaves the device usable: a GEMM
    right after it is exact and raises no flag."""
    import torch
    L = lib.load()
    flags = C.c_uint(99)
    assert L.bhTcErrorFlags(C.byref(flags)) == 0
    assert L.bhTcWaitProbe(0, None) != 0 and L.bhTcWaitProbe(2000000, None) != 0   # limits out of range
    assert L.bhTcWaitProbe(1000, C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    torch.cuda.synchronize()
    assert L.bhTcErrorFlags(C.byref(flags)) == 0 and flags.value & 1
    assert L.bhTcErrorFlags(C.byref(flags)) == 0 and flags.value == 0
    err, scale = _run(256, 256, 256)
    assert err <= 1e-5 * 256 * 4.0 + 1e-4
