"""ctypes mirrors of the C-ABI in include/bh_render_params.h and include/bh_launch.h.

The RenderParams layout is the reference renderer's (src/render_params.h:21-87
of Sqhh99/Black-hole): 160 bytes, 4-byte aligned.  BHProbe is the per-ray
record of the probe entry points; PROBE_DTYPE is the same record as a numpy
structured dtype so device buffers can be viewed without copies.
"""
import ctypes as C

import numpy as np

BH_SCHWARZSCHILD, BH_REISSNER_NORDSTROM, BH_KERR, BH_KERR_NEWMAN = 0, 1, 2, 3
BH_PREC_FP32, BH_PREC_MIXED, BH_PREC_FP64 = 0, 1, 2
MODEL_NAMES = {0: "Schwarzschild", 1: "Reissner-Nordstrom", 2: "Kerr", 3: "Kerr-Newman"}


class Float3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]

    def tolist(self):
        return [self.x, self.y, self.z]


def f3(v):
    return Float3(float(v[0]), float(v[1]), float(v[2]))


class RenderParams(C.Structure):
    """Per-frame parameters; defaults are the reference's member initialisers."""

    _fields_ = [
        ("width", C.c_int), ("height", C.c_int), ("swapRB", C.c_int),
        ("camPos", Float3), ("camForward", Float3), ("camRight", Float3), ("camUp", Float3),
        ("tanHalfFov", C.c_float), ("aspect", C.c_float),
        ("model", C.c_int), ("M", C.c_float), ("aSpin", C.c_float), ("Qc", C.c_float),
        ("rPlus", C.c_float), ("rPhoton", C.c_float), ("rErgo", C.c_float),
        ("allowNaked", C.c_int),
        ("dPhi", C.c_float), ("maxSteps", C.c_int),
        ("diskEnabled", C.c_int), ("diskInner", C.c_float), ("diskOuter", C.c_float),
        ("diskTime", C.c_float), ("diskEmisScale", C.c_float), ("diskAbsScale", C.c_float),
        ("hotSpotsEnabled", C.c_int), ("hotSpotStrength", C.c_float),
        ("exposure", C.c_float), ("sampleIndex", C.c_int), ("accumMode", C.c_int),
        ("bloomEnabled", C.c_int), ("bloomStrength", C.c_float),
    ]

    def __init__(self, **kw):
        super().__init__()
        defaults = dict(
            width=1280, height=720, swapRB=0,
            camPos=(0.0, 0.0, 0.0), camForward=(0.0, 0.0, -1.0), camRight=(1.0, 0.0, 0.0),
            camUp=(0.0, 1.0, 0.0), tanHalfFov=0.5773503, aspect=1280.0 / 720.0,
            model=0, M=0.5, aSpin=0.0, Qc=0.0, rPlus=1.0, rPhoton=1.5, rErgo=1.0, allowNaked=0,
            dPhi=0.012, maxSteps=2000,
            diskEnabled=1, diskInner=3.0, diskOuter=8.0, diskTime=0.0,
            diskEmisScale=1.5, diskAbsScale=2.2, hotSpotsEnabled=1, hotSpotStrength=0.65,
            exposure=1.0, sampleIndex=0, accumMode=0, bloomEnabled=1, bloomStrength=0.35,
        )
        defaults.update(kw)
        for k, v in defaults.items():
            setattr(self, k, v)

    def __setattr__(self, k, v):
        if k in ("camPos", "camForward", "camRight", "camUp") and not isinstance(v, Float3):
            v = f3(v)
        super().__setattr__(k, v)

    def copy(self):
        c = RenderParams()
        C.memmove(C.byref(c), C.byref(self), C.sizeof(RenderParams))
        return c

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = v.tolist() if isinstance(v, Float3) else v
        return out


assert C.sizeof(RenderParams) == 160
assert C.alignment(RenderParams) == 4
assert RenderParams.camPos.offset == 12 and RenderParams.dPhi.offset == 100
assert RenderParams.bloomStrength.offset == 156


class BHView(C.Structure):
    """One view of a batch (include/bh_launch.h): parameters + device buffers."""
    _fields_ = [("params", RenderParams), ("out", C.c_void_p), ("accum", C.c_void_p),
                ("bloomA", C.c_void_p), ("bloomB", C.c_void_p)]


assert C.sizeof(BHView) == 160 + 4 * 8


class BHDerived(C.Structure):
    _fields_ = [("a", C.c_float), ("Q", C.c_float), ("rPlus", C.c_float), ("rMinus", C.c_float),
                ("rPhoton", C.c_float), ("rErgo", C.c_float), ("rIsco", C.c_float),
                ("clamped", C.c_int), ("naked", C.c_int)]


class BHDeriveRequest(C.Structure):
    _fields_ = [("model", C.c_int), ("M", C.c_float), ("aStar", C.c_float), ("q", C.c_float),
                ("allowNaked", C.c_int)]


DERIVE_REQ_DTYPE = np.dtype([("model", np.int32), ("M", np.float32), ("aStar", np.float32), ("q", np.float32),
                             ("allowNaked", np.int32)])
DERIVED_DTYPE = np.dtype([("a", np.float32), ("Q", np.float32), ("rPlus", np.float32), ("rMinus", np.float32),
                          ("rPhoton", np.float32), ("rErgo", np.float32), ("rIsco", np.float32),
                          ("clamped", np.int32), ("naked", np.int32)])
assert DERIVE_REQ_DTYPE.itemsize == 20 and DERIVED_DTYPE.itemsize == 36


PROBE_DTYPE = np.dtype([
    ("outcome", np.int32), ("cls", np.int32), ("steps", np.int32), ("diskSamples", np.int32),
    ("escDir", np.float32, (3,)), ("trans", np.float32), ("accum", np.float32, (3,)),
    ("maxHviol", np.float32), ("hdr", np.float32, (3,)),
    ("diskR", np.float32), ("diskG", np.float32), ("drift", np.float32),
])
assert PROBE_DTYPE.itemsize == 72
