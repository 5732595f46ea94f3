"""Loading helpers for tests/golden/golden.npz (made by tests/golden/make_golden.py)."""
import ctypes as C
import functools
import os

import numpy as np

from bhrt.abi import PROBE_DTYPE, RenderParams

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")
GRID_NAMES = ["S", "RN5", "K9", "Km7", "KN75", "S_disk", "RN6_disk", "K9_disk", "KNm74_disk", "K12_naked"]
PIPE_NAMES = ["S320_160x90", "K9_spots_96x54", "KNm74_cfg2_96x54", "KN995_sweep_96x54"]
GRID_NX, GRID_NY = 48, 27
# fields the reference itself produces (the rest are additions of the oracle)
REF_FIELDS = ("outcome", "cls", "steps", "escDir", "trans", "accum", "maxHviol", "hdr")


@functools.lru_cache(maxsize=1)
def load():
    return dict(np.load(PATH))


def params(raw):
    P = RenderParams()
    b = np.ascontiguousarray(raw, dtype=np.uint8).tobytes()
    assert len(b) == C.sizeof(RenderParams)
    C.memmove(C.addressof(P), b, len(b))
    return P


def grid(name):
    g = load()
    return params(g[f"grid_{name}_params"]), g[f"grid_{name}"].view(PROBE_DTYPE).reshape(GRID_NY, GRID_NX)


def same_bits(a, b):
    """Exact equality of float arrays, NaN matching NaN."""
    a, b = np.asarray(a), np.asarray(b)
    if a.dtype.kind == "f":
        return np.array_equal(a.view(np.uint32 if a.dtype == np.float32 else np.uint64),
                              b.view(np.uint32 if b.dtype == np.float32 else np.uint64)) or \
            bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
    return np.array_equal(a, b)
