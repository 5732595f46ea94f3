"""bhRenderPipelineNoAlloc: the pipeline for callers that cannot let a library
allocate device memory (a frame loop recorded inside CUDA stream capture, a
real-time loop that must not stall on the allocator, a plugin whose host owns
all device memory).  It keeps its scratch in a fixed array inside libbh.so, so
these checks call it through the C-ABI and compare it with launchRenderPipeline.

This file is named to be collected last, so that a run stopping at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu


def _call(L, out, acc, P, stream):
    return L.bhRenderPipelineNoAlloc(C.c_void_p(out.data_ptr()), C.c_void_p(acc.data_ptr()), C.byref(P),
                                     C.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("frame", [11, 3])
def test_no_alloc_pipeline_matches_pipeline_twice(cuda, frame):
    import torch
    from bhrt import lib, scenes
    from bhrt.device import Frame
    L = lib.load()
    P = scenes.kerr_pair_1080(lib.derive, 640, 360)[frame]   # disk, hot spots, bloom on
    ref = Frame(P.width, P.height)
    ref.pipeline(P)
    torch.cuda.synchronize()
    want, want_acc = ref.out.cpu().numpy(), ref.accum.cpu().numpy()

    out = torch.zeros_like(ref.out)
    acc = torch.zeros_like(ref.accum)
    stream = torch.cuda.current_stream()
    assert _call(L, out, acc, P, stream) == 0          # first call: scratch address looked up
    torch.cuda.synchronize()
    for call in range(2):
        out.zero_()
        free_before = torch.cuda.mem_get_info()[0]
        assert _call(L, out, acc, P, stream) == 0
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free_before, "the call must not allocate device memory"
        s = parity.compare_rgba(out.cpu().numpy(), want)
        assert s["alpha_ok"] and s["lsb1_frac"] >= 0.995, (call, s)
        np.testing.assert_allclose(acc.cpu().numpy(), want_acc, rtol=1e-6, atol=0)


def test_no_alloc_pipeline_rejects_frames_beyond_its_scratch(cuda):
    import torch
    from bhrt import lib, scenes
    L = lib.load()
    P = scenes.kerr_pair_1080(lib.derive, 2050, 1026)[0]    # (1025 * 513) half-res pixels > 524288
    out = torch.zeros((P.height, P.width, 4), dtype=torch.uint8, device="cuda")
    acc = torch.zeros((P.height, P.width, 4), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    assert _call(L, out, acc, P, stream) == 1            # cudaErrorInvalidValue, nothing launched
    torch.cuda.synchronize()
    assert int(out[..., 3].max()) == 0
    P.bloomEnabled = 0                                   # without bloom no half-res scratch is used
    P.width, P.height = 320, 180
    out = torch.zeros((180, 320, 4), dtype=torch.uint8, device="cuda")
    acc = torch.zeros((180, 320, 4), dtype=torch.float32, device="cuda")
    assert _call(L, out, acc, P, stream) == 0
    torch.cuda.synchronize()
    assert bool((out[..., 3] == 255).all())
