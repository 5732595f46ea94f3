"""launchRenderPipeline calls on different streams may overlap on the GPU (each
launch takes its own work counter): frames rendered concurrently on two streams
equal the same frames rendered one after another."""
import ctypes as C

import numpy as np
import pytest

from bhrt import lib, scenes
from bhrt.device import Frame

pytestmark = pytest.mark.gpu


def _launch(L, f, P, stream):
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    assert L.launchRenderPipeline(p(f.out), p(f.accum), p(f.bloomA), p(f.bloomB), C.byref(P),
                                  C.c_void_p(stream.cuda_stream)) == 0


def test_concurrent_streams_equal_sequential(cuda):
    import torch
    L = lib.load()
    frames = scenes.kerr_pair_1080(lib.derive, 640, 360)[::2]          # 8 frames, both metrics
    seq = [Frame(640, 360) for _ in frames]
    s0 = torch.cuda.current_stream()
    for f, P in zip(seq, frames):
        _launch(L, f, P, s0)
    torch.cuda.synchronize()
    want = [(f.out.cpu().numpy(), f.accum.cpu().numpy()) for f in seq]
    streams = [torch.cuda.Stream() for _ in range(4)]
    conc = [Frame(640, 360) for _ in frames]
    for rep in range(2):
        for i, (f, P) in enumerate(zip(conc, frames)):
            _launch(L, f, P, streams[i % 4])
        torch.cuda.synchronize()
        for (wo, wa), f in zip(want, conc):
            assert np.array_equal(f.out.cpu().numpy(), wo)
            assert np.array_equal(f.accum.cpu().numpy(), wa)
