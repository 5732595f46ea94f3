"""bhRenderPipelineNoAlloc: the pipeline for callers that cannot let a library
allocate device memory (a plugin whose host application owns every byte of
device memory and hands out only its own buffers; a real-time frame loop that
must never stall on the allocator, since cudaMalloc can synchronise the
device).  It keeps its scratch in a fixed array inside libbh.so.  These checks
call it through the C-ABI and compare it with launchRenderPipeline.

The allocation check runs in a fresh process whose only libbh calls are
bhRenderPipelineNoAlloc and bhLibraryDeviceBytes (the library's count of the
device bytes it has allocated), then makes a launchRenderPipeline call to show
that the count does move when the library allocates.

This file is named to be collected last, so that a run stopping at the first
failure has already run every other test.
"""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _call(L, out, acc, P, stream):
    return L.bhRenderPipelineNoAlloc(C.c_void_p(out.data_ptr()), C.c_void_p(acc.data_ptr()), C.byref(P),
                                     C.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("frame", [11, 3])
def test_no_alloc_pipeline_matches_pipeline_twice(cuda, frame):
    """Two calls in a row, each compared with launchRenderPipeline's frame."""
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
    for call in range(2):
        out.zero_()
        assert _call(L, out, acc, P, stream) == 0
        torch.cuda.synchronize()
        s = parity.compare_rgba(out.cpu().numpy(), want)
        assert s["alpha_ok"] and s["lsb1_frac"] >= 0.995, (call, s)
        np.testing.assert_allclose(acc.cpu().numpy(), want_acc, rtol=1e-6, atol=0)


_CHILD = r"""
import ctypes as C, json, sys
sys.path.insert(0, sys.argv[1])
import torch
from bhrt import lib, scenes
L = lib.load()
torch.cuda.set_device(0)
P = scenes.kerr_pair_1080(lib.derive, 640, 360)[11]      # host-only derivation
out = torch.zeros((P.height, P.width, 4), dtype=torch.uint8, device="cuda")
acc = torch.zeros((P.height, P.width, 4), dtype=torch.float32, device="cuda")
s = torch.cuda.current_stream()
codes = []
for _ in range(3):
    codes.append(L.bhRenderPipelineNoAlloc(C.c_void_p(out.data_ptr()), C.c_void_p(acc.data_ptr()),
                                           C.byref(P), C.c_void_p(s.cuda_stream)))
torch.cuda.synchronize()
after_noalloc = L.bhLibraryDeviceBytes(0)
ok = bool((out[..., 3] == 255).all())
bA = torch.zeros(((P.height + 1) // 2, (P.width + 1) // 2, 4), dtype=torch.float32, device="cuda")
bB = torch.zeros_like(bA)
code = L.launchRenderPipeline(C.c_void_p(out.data_ptr()), C.c_void_p(acc.data_ptr()), C.c_void_p(bA.data_ptr()),
                              C.c_void_p(bB.data_ptr()), C.byref(P), C.c_void_p(s.cuda_stream))
torch.cuda.synchronize()
print(json.dumps({"codes": codes, "frame_ok": ok, "after_noalloc": after_noalloc,
                  "pipeline_code": code, "after_pipeline": L.bhLibraryDeviceBytes(0)}))
"""


def test_no_alloc_pipeline_allocates_nothing(cuda):
    r = subprocess.run([sys.executable, "-c", _CHILD, os.path.join(ROOT, "black-hole_b200")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    print(res)
    assert res["codes"] == [0, 0, 0] and res["frame_ok"], res
    assert res["after_noalloc"] == 0, "bhRenderPipelineNoAlloc allocated device memory"
    # the count is live: launchRenderPipeline allocates its work-counter ring on first use
    assert res["pipeline_code"] == 0 and res["after_pipeline"] > 0, res


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
