"""Device-side front end: frame buffers and calls of the tracing entry points.

Buffers are torch CUDA tensors (allocation and streams only); every tracing
or post-processing call is a C-ABI call into libbh.so on the tensor memory.
"""
import ctypes as C

import numpy as np
import torch

from . import lib as _lib
from .abi import BH_PREC_FP32, PROBE_DTYPE

PROBE_BYTES = PROBE_DTYPE.itemsize


def _stream(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class Frame:
    """Caller-owned buffers of one W x H view, as the reference's interop allocates
    them (cuda_interop.cpp:45-59): RGBA8 output, float4 accumulation, two
    half-resolution float4 bloom buffers."""

    def __init__(self, width, height, device="cuda"):
        self.W, self.H = int(width), int(height)
        bw, bh = (self.W + 1) // 2, (self.H + 1) // 2
        self.out = torch.zeros((self.H, self.W, 4), dtype=torch.uint8, device=device)
        self.accum = torch.zeros((self.H, self.W, 4), dtype=torch.float32, device=device)
        self.bloomA = torch.zeros((bh, bw, 4), dtype=torch.float32, device=device)
        self.bloomB = torch.zeros((bh, bw, 4), dtype=torch.float32, device=device)

    def pipeline(self, P, precision=BH_PREC_FP32, stream=None):
        L = _lib.load()
        if precision == BH_PREC_FP32:
            code = L.launchRenderPipeline(_ptr(self.out), _ptr(self.accum), _ptr(self.bloomA),
                                          _ptr(self.bloomB), C.byref(P), _stream(stream))
        else:
            code = L.bhRenderPipelinePrec(_ptr(self.out), _ptr(self.accum), _ptr(self.bloomA),
                                          _ptr(self.bloomB), C.byref(P), int(precision), _stream(stream))
        _lib.check(code, "launchRenderPipeline")
        return self.out

    def accum_only(self, P, precision=BH_PREC_FP32, stream=None):
        _lib.check(_lib.load().bhRenderAccum(_ptr(self.accum), C.byref(P), int(precision), _stream(stream)),
                   "bhRenderAccum")
        return self.accum

    def render_kernel(self, P, stream=None):
        _lib.check(_lib.load().launchRenderKernel(_ptr(self.out), C.byref(P), _stream(stream)),
                   "launchRenderKernel")
        return self.out

    def post(self, P, stream=None):
        _lib.check(_lib.load().bhPostProcess(_ptr(self.out), _ptr(self.accum), _ptr(self.bloomA),
                                             _ptr(self.bloomB), C.byref(P), _stream(stream)),
                   "bhPostProcess")
        return self.out


def render_hdr(P, precision=BH_PREC_FP32, out=None, stream=None):
    Q, _ = _lib.sanitize(P)
    if out is None:
        out = torch.empty((Q.height, Q.width, 4), dtype=torch.float32, device="cuda")
    _lib.check(_lib.load().bhRenderHDR(_ptr(out), C.byref(P), int(precision), _stream(stream)),
               "bhRenderHDR")
    return out


def _probe_to_numpy(buf, shape):
    raw = buf.cpu().numpy().view(PROBE_DTYPE)
    return raw.reshape(shape)


def probe_grid(P, nx, ny, precision=BH_PREC_FP32, stream=None):
    buf = torch.zeros(nx * ny * PROBE_BYTES, dtype=torch.uint8, device="cuda")
    _lib.check(_lib.load().bhProbeGrid(_ptr(buf), C.byref(P), int(nx), int(ny), int(precision),
                                       _stream(stream)), "bhProbeGrid")
    torch.cuda.synchronize()
    return _probe_to_numpy(buf, (ny, nx))


def probe_rays(P, dirs, precision=BH_PREC_FP32, stream=None):
    d = torch.as_tensor(np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 3), device="cuda")
    n = d.shape[0]
    buf = torch.zeros(max(n, 1) * PROBE_BYTES, dtype=torch.uint8, device="cuda")
    _lib.check(_lib.load().bhProbeRays(_ptr(buf), _ptr(d), int(n), C.byref(P), int(precision),
                                       _stream(stream)), "bhProbeRays")
    torch.cuda.synchronize()
    return _probe_to_numpy(buf[: n * PROBE_BYTES], (n,))


def measure_fp32_peak():
    return _lib.load().bhMeasureFp32Peak()
