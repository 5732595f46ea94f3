"""TEST INFRASTRUCTURE ONLY -- ctypes front end of the CPU oracle.

`Oracle` wraps oracle/liboracle.so, the restated reference tracer
(oracle/bh_oracle.cpp; FP32 bit-exact with the reference built as host code,
FP64 as the small-step accuracy oracle).  `RefHost` wraps
oracle/_ref/libbhref_host.so, the reference's own headers compiled as host C++
(oracle/Makefile, target `ref`); `RefGpu` wraps oracle/_ref/libbhref_gpu.so,
the reference's kernels compiled for sm_100a.  Only tests/, the smoke check
and the benchmark's CPU-baseline leg use this module, as the checker.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "black-hole_b200"))
from bhrt.abi import PROBE_DTYPE, BHDerived, RenderParams  # noqa: E402

_P = C.POINTER(RenderParams)
_vp = C.c_void_p


def _ptr(a):
    return a.ctypes.data_as(_vp)


def ref_src():
    """The reference's src/ directory: $REF_SRC, else the Makefile's default."""
    if os.environ.get("REF_SRC"):
        return os.environ["REF_SRC"]
    import re
    with open(os.path.join(HERE, "Makefile")) as fh:
        m = re.search(r"^REF_SRC\s*\?=\s*(\S+)", fh.read(), flags=re.M)
    return m.group(1) if m else ""


def build(ref=None):
    """Build liboracle.so (and the reference builds when the reference tree exists)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    src = ref_src()
    if ref is None:
        ref = bool(src) and os.path.isdir(src)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_SRC={src}"], check=True)


class Oracle:
    """Restated reference tracer (CPU)."""

    def __init__(self, path=None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = self.lib = C.CDLL(path)
        L.orc_sanitize.argtypes = [_P]
        L.orc_sanitize.restype = C.c_int
        L.orc_derive.argtypes = [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                 C.POINTER(C.c_float), C.c_int, C.POINTER(BHDerived)]
        L.orc_camera_energy.argtypes = [_P]
        L.orc_camera_energy.restype = C.c_float
        L.orc_probe_grid.argtypes = [_P, C.c_int, C.c_int, C.c_int, C.c_int, _vp, C.c_int]
        L.orc_probe_dirs.argtypes = [_P, _vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int]
        L.orc_trace_pixels.argtypes = [_P, _vp, C.c_int, C.c_int, _vp, C.c_int]
        L.orc_render_hdr.argtypes = [_P, C.c_int, _vp, _vp, C.c_int]
        L.orc_post.argtypes = [_vp, _vp, _vp, _vp, _P, C.c_int]
        L.orc_pipeline.argtypes = [_vp, _vp, _vp, _vp, _P, C.c_int, C.c_int]
        L.orc_render_kernel.argtypes = [_vp, _P, C.c_int, C.c_int]

    def sanitize(self, P):
        Q = P.copy()
        fixed = self.lib.orc_sanitize(C.byref(Q))
        return Q, bool(fixed)

    def derive(self, model, M, a_star, q, allow_naked=False):
        m, a, qq = C.c_float(M), C.c_float(a_star), C.c_float(q)
        d = BHDerived()
        self.lib.orc_derive(model, C.byref(m), C.byref(a), C.byref(qq), int(allow_naked), C.byref(d))
        return d, m.value, a.value, qq.value

    def camera_energy(self, P):
        return self.lib.orc_camera_energy(C.byref(P))

    def probe_grid(self, P, nx, ny, precision=0, step_div=1, threads=0):
        out = np.zeros(nx * ny, dtype=PROBE_DTYPE)
        self.lib.orc_probe_grid(C.byref(P), nx, ny, precision, step_div, _ptr(out), threads)
        return out.reshape(ny, nx)

    def probe_dirs(self, P, dirs, precision=0, step_div=1, threads=0):
        d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 3)
        out = np.zeros(len(d), dtype=PROBE_DTYPE)
        self.lib.orc_probe_dirs(C.byref(P), _ptr(d), len(d), precision, step_div, _ptr(out), threads)
        return out

    def trace_pixels(self, P, pix, precision=0, threads=0):
        pix = np.ascontiguousarray(pix, dtype=np.int32)
        out = np.zeros(len(pix), dtype=PROBE_DTYPE)
        self.lib.orc_trace_pixels(C.byref(P), _ptr(pix), len(pix), precision, _ptr(out), threads)
        return out

    def render_hdr(self, P, precision=0, threads=0, rays=False):
        Q, _ = self.sanitize(P)
        hdr = np.zeros((Q.height, Q.width, 4), dtype=np.float32)
        rec = np.zeros(Q.height * Q.width, dtype=PROBE_DTYPE) if rays else None
        self.lib.orc_render_hdr(C.byref(P), precision, _ptr(hdr),
                                _ptr(rec) if rays else None, threads)
        return (hdr, rec.reshape(Q.height, Q.width)) if rays else hdr

    def _bufs(self, P, accum):
        Q, _ = self.sanitize(P)
        W, H = Q.width, Q.height
        bw, bh = (W + 1) // 2, (H + 1) // 2
        out = np.zeros((H, W, 4), dtype=np.uint8)
        acc = np.zeros((H, W, 4), dtype=np.float32) if accum is None else accum
        bA = np.zeros((bh, bw, 4), dtype=np.float32)
        bB = np.zeros((bh, bw, 4), dtype=np.float32)
        return out, acc, bA, bB

    def post(self, P, accum, threads=0):
        out, acc, bA, bB = self._bufs(P, np.ascontiguousarray(accum, dtype=np.float32))
        self.lib.orc_post(_ptr(out), _ptr(acc), _ptr(bA), _ptr(bB), C.byref(P), threads)
        return out, bA, bB

    def pipeline(self, P, accum=None, precision=0, threads=0):
        out, acc, bA, bB = self._bufs(P, accum)
        self.lib.orc_pipeline(_ptr(out), _ptr(acc), _ptr(bA), _ptr(bB), C.byref(P), precision, threads)
        return out, acc, bA, bB

    def render_kernel(self, P, precision=0, threads=0):
        Q, _ = self.sanitize(P)
        out = np.zeros((Q.height, Q.width, 4), dtype=np.uint8)
        self.lib.orc_render_kernel(_ptr(out), C.byref(P), precision, threads)
        return out


class RefHost:
    """The reference's own headers built as host C++ (oracle/_ref)."""

    PATH = os.path.join(HERE, "_ref", "libbhref_host.so")

    @classmethod
    def available(cls):
        return os.path.exists(cls.PATH)

    def __init__(self):
        L = self.lib = C.CDLL(self.PATH)
        L.ref_sanitize.argtypes = [_P]
        L.ref_sanitize.restype = C.c_int
        L.ref_derive.argtypes = [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                 C.POINTER(C.c_float), C.c_int, C.POINTER(BHDerived)]
        L.ref_probe_grid.argtypes = [_P, C.c_int, C.c_int, _vp, C.c_int]
        L.ref_probe_dirs.argtypes = [_P, _vp, C.c_int, _vp, C.c_int]
        L.ref_render_pixels.argtypes = [_P, _vp, C.c_int, _vp, C.c_int]
        L.ref_pipeline.argtypes = [_vp, _vp, _vp, _vp, _P, C.c_int]
        L.ref_render_kernel.argtypes = [_vp, _P, C.c_int]

    def sanitize(self, P):
        Q = P.copy()
        fixed = self.lib.ref_sanitize(C.byref(Q))
        return Q, bool(fixed)

    def derive(self, model, M, a_star, q, allow_naked=False):
        m, a, qq = C.c_float(M), C.c_float(a_star), C.c_float(q)
        d = BHDerived()
        self.lib.ref_derive(model, C.byref(m), C.byref(a), C.byref(qq), int(allow_naked), C.byref(d))
        return d, m.value, a.value, qq.value

    def probe_grid(self, P, nx, ny, threads=0):
        out = np.zeros(nx * ny, dtype=PROBE_DTYPE)
        self.lib.ref_probe_grid(C.byref(P), nx, ny, _ptr(out), threads)
        return out.reshape(ny, nx)

    def probe_dirs(self, P, dirs, threads=0):
        d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 3)
        out = np.zeros(len(d), dtype=PROBE_DTYPE)
        self.lib.ref_probe_dirs(C.byref(P), _ptr(d), len(d), _ptr(out), threads)
        return out

    def render_pixels(self, P, pix, threads=0):
        pix = np.ascontiguousarray(pix, dtype=np.int32)
        hdr = np.zeros((len(pix), 4), dtype=np.float32)
        self.lib.ref_render_pixels(C.byref(P), _ptr(pix), len(pix), _ptr(hdr), threads)
        return hdr

    def pipeline(self, P, accum=None, threads=0):
        Q, _ = self.sanitize(P)
        W, H = Q.width, Q.height
        bw, bh = (W + 1) // 2, (H + 1) // 2
        out = np.zeros((H, W, 4), dtype=np.uint8)
        acc = np.zeros((H, W, 4), dtype=np.float32) if accum is None else accum
        bA = np.zeros((bh, bw, 4), dtype=np.float32)
        bB = np.zeros((bh, bw, 4), dtype=np.float32)
        self.lib.ref_pipeline(_ptr(out), _ptr(acc), _ptr(bA), _ptr(bB), C.byref(P), threads)
        return out, acc, bA, bB

    def render_kernel(self, P, threads=0):
        Q, _ = self.sanitize(P)
        out = np.zeros((Q.height, Q.width, 4), dtype=np.uint8)
        self.lib.ref_render_kernel(_ptr(out), C.byref(P), threads)
        return out


class RefGpu:
    """The reference's kernels built for sm_100a (oracle/_ref); device pointers."""

    PATH = os.path.join(HERE, "_ref", "libbhref_gpu.so")

    @classmethod
    def available(cls):
        return os.path.exists(cls.PATH)

    def __init__(self):
        L = self.lib = C.CDLL(self.PATH)
        L.ref_gpu_probe_grid.argtypes = [_vp, _P, C.c_int, C.c_int, _vp]
        L.ref_gpu_probe_grid.restype = C.c_int
        L.ref_gpu_render_hdr.argtypes = [_vp, _P, _vp]
        L.ref_gpu_render_hdr.restype = C.c_int
        L.launchRenderPipeline.argtypes = [_vp, _vp, _vp, _vp, _P, _vp]
        L.launchRenderPipeline.restype = C.c_int
        L.launchRenderKernel.argtypes = [_vp, _P, _vp]
        L.launchRenderKernel.restype = C.c_int
