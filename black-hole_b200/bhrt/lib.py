"""ctypes binding of libbh.so -- every call goes through the C-ABI of include/bh_launch.h.

There is no fallback: if the library has not been built, or the GPU entry
points fail, the error is raised.  Device buffers may be any objects exposing
a device address (torch CUDA tensors are used by the tests and the benchmark;
PyTorch is only the allocator and stream provider here).
"""
import ctypes as C
import os

from .abi import BHDerived, RenderParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "libbh.so")

_P = C.POINTER(RenderParams)
_vp = C.c_void_p
_int = C.c_int

# name: (restype, argtypes)
_SIGNATURES = {
    "launchRenderPipeline": (_int, [_vp, _vp, _vp, _vp, _P, _vp]),
    "launchRenderKernel": (_int, [_vp, _P, _vp]),
    "bhSanitizeRenderParams": (_int, [_P]),
    "bhValidateAndDerive": (None, [_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                   C.POINTER(C.c_float), _int, C.POINTER(BHDerived)]),
    "bhDeriveBatch": (_int, [_vp, _vp, _int, _vp]),
    "bhProbeGrid": (_int, [_vp, _P, _int, _int, _int, _vp]),
    "bhProbeRays": (_int, [_vp, _vp, _int, _P, _int, _vp]),
    "bhRenderHDR": (_int, [_vp, _P, _int, _vp]),
    "bhRenderPipelinePrec": (_int, [_vp, _vp, _vp, _vp, _P, _int, _vp]),
    "bhRenderAccum": (_int, [_vp, _P, _int, _vp]),
    "bhPostProcess": (_int, [_vp, _vp, _vp, _vp, _P, _vp]),
    "bhSetTuning": (_int, [_int, _int, _int]),
    "bhGetTuning": (None, [_int, C.POINTER(_int), C.POINTER(_int)]),
    "bhSetTileOrder": (_int, [_int]),
    "bhGetTileOrder": (_int, []),
    "bhRenderBatch": (_int, [_vp, _int, _vp]),
    "bhBatchGraphCreate": (_int, [C.POINTER(_vp), _vp, _int]),
    "bhBatchGraphUpdate": (_int, [_vp, _vp, _int]),
    "bhBatchGraphLaunch": (_int, [_vp, _vp]),
    "bhBatchGraphDestroy": (None, [_vp]),
    "bhAutotune": (_int, [_P, C.POINTER(_int), C.POINTER(_int), C.POINTER(_int), C.POINTER(C.c_float)]),
    "bhAutotuneBatch": (_int, [_vp, _int, C.POINTER(_int), C.POINTER(_int), C.POINTER(C.c_float)]),
    "bhRenderPipelineNoAlloc": (_int, [_vp, _vp, _P, _vp]),
    "bhMeasureFp32Peak": (C.c_double, []),
    "bhLibraryDeviceBytes": (C.c_ulonglong, [_int]),
    "bhTcGemm": (_int, [_vp, _int, _vp, _int, _vp, _int, _int, _int, _int, _int, _int, _vp, _vp]),
    "bhTcErrorFlags": (_int, [C.POINTER(C.c_uint)]),
    "bhSurrogateParamCount": (_int, []),
    "bhSurrogateCreate": (_int, [C.POINTER(_vp), C.c_uint]),
    "bhSurrogateDestroy": (None, [_vp]),
    "bhSurrogateGetParams": (_int, [_vp, _vp]),
    "bhSurrogateSetParams": (_int, [_vp, _vp]),
    "bhSurrogateFeatures": (_int, [_vp, _vp, _int, _vp]),
    "bhSurrogateForward": (_int, [_vp, _vp, _vp, _int, _int, _vp]),
    "bhSurrogateGradients": (_int, [_vp, _vp, _vp, _int, _vp, _vp]),
    "bhSurrogateGenerate": (_int, [_vp, C.c_longlong, _int, C.c_uint]),
    "bhSurrogateDataset": (_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(C.c_longlong)]),
    "bhSurrogateDatasetCopy": (_int, [_vp, _vp, _vp, C.c_longlong, C.c_longlong]),
    "bhSurrogateTrain": (_int, [_vp, _int, _int, C.c_float, C.c_uint, _vp]),
    "bhSurrogateRender": (_int, [_vp, _vp, _vp, _vp, _vp, _P, _vp]),
    "bhSurrogateFrameStats": (_int, [_vp, _vp]),
    "bhSurrogateSetGate": (_int, [_vp, C.c_float, C.c_float, C.c_float, _int]),
    "bhSurrogateSetAnchors": (_int, [_vp, _int, _int, C.c_float, C.c_float]),
    "bhSurrogateSetAnchorSteps": (_int, [_vp, _int]),
    "bhSurrogateClone": (_int, [_vp, _vp]),
    "bhTcWaitProbe": (_int, [_int, _vp]),
    "bhVersion": (C.c_char_p, []),
}

EXPORTED = tuple(_SIGNATURES)

_lib = None


class CudaError(RuntimeError):
    pass


def load(path=None):
    """Load libbh.so once (raises if it is missing: build it with black-hole_b200/build.py)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(f"libbh.so not built ({path}); run python black-hole_b200/build.py")
    lib = C.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _lib = lib
    return lib


def check(code, what):
    if code != 0:
        raise CudaError(f"{what} failed with cudaError {code}")


def derive(model, M, a_star, q, allow_naked=False):
    """bhValidateAndDerive: returns (BHDerived, M, a*, q) with the clamped inputs."""
    L = load()
    m, a, qq = C.c_float(M), C.c_float(a_star), C.c_float(q)
    d = BHDerived()
    L.bhValidateAndDerive(int(model), C.byref(m), C.byref(a), C.byref(qq), int(bool(allow_naked)),
                          C.byref(d))
    return d, m.value, a.value, qq.value


def sanitize(P):
    """bhSanitizeRenderParams on a copy: returns (sanitised params, fixed flag)."""
    Q = P.copy()
    fixed = load().bhSanitizeRenderParams(C.byref(Q))
    return Q, bool(fixed)


def set_tuning(family, refill_min, blocks_per_sm=0):
    if not load().bhSetTuning(int(family), int(refill_min), int(blocks_per_sm)):
        raise ValueError("tuning out of range")


def get_tuning(family):
    r, b = C.c_int(), C.c_int()
    load().bhGetTuning(int(family), C.byref(r), C.byref(b))
    return r.value, b.value


def version():
    return load().bhVersion().decode()
