"""Batched views: one persistent launch over many views (bhRenderBatch), its
CUDA-graph form, and the autotuner -- all through the C-ABI."""
import ctypes as C

import numpy as np
import pytest

import parity
from bhrt import lib, scenes
from bhrt.abi import BHView

pytestmark = pytest.mark.gpu


def _views(n=12, seed=5):
    """A mix of all four families, resolutions and bloom / hot-spot settings."""
    rng = np.random.default_rng(seed)
    sizes = [(64, 36), (96, 54), (160, 90), (200, 120), (320, 180)]
    out = []
    for i in range(n):
        w, h = sizes[i % len(sizes)]
        model = i % 4
        a = float(rng.uniform(-0.95, 0.95)) if model >= 2 else 0.0
        q = float(rng.uniform(0.0, 0.5)) if model in (1, 3) else 0.0
        P = scenes.scene(lib.derive, model, a, q, w, h, float(rng.uniform(8, 30)), float(rng.uniform(2, 80)),
                         float(rng.uniform(35, 80)), hot_spots=bool(i % 2), bloom=bool(i % 3), disk_time=0.3 * i)
        out.append(P)
    return out


def _buffers(P):
    import torch
    bw, bh = (P.width + 1) // 2, (P.height + 1) // 2
    return {"out": torch.zeros((P.height, P.width, 4), dtype=torch.uint8, device="cuda"),
            "accum": torch.zeros((P.height, P.width, 4), dtype=torch.float32, device="cuda"),
            "bloomA": torch.zeros((bh, bw, 4), dtype=torch.float32, device="cuda"),
            "bloomB": torch.zeros((bh, bw, 4), dtype=torch.float32, device="cuda")}


def _view_array(params, bufs):
    arr = (BHView * len(params))()
    for i, (P, b) in enumerate(zip(params, bufs)):
        arr[i].params = P
        arr[i].out, arr[i].accum = b["out"].data_ptr(), b["accum"].data_ptr()
        arr[i].bloomA, arr[i].bloomB = b["bloomA"].data_ptr(), b["bloomB"].data_ptr()
    return arr


def _singles(params):
    import torch
    from bhrt.device import Frame
    res = []
    for P in params:
        f = Frame(P.width, P.height)
        f.pipeline(P)
        torch.cuda.synchronize()
        res.append(f.out.cpu().numpy())
    return res


def _check(bufs, want):
    for b, w in zip(bufs, want):
        s = parity.compare_rgba(b["out"].cpu().numpy(), w)
        assert s["alpha_ok"] and s["max_diff"] <= 1 and s["exact_frac"] >= 0.999, s


def test_batch_equals_per_view_pipelines(cuda):
    import torch
    L = lib.load()
    params = _views()
    bufs = [_buffers(P) for P in params]
    arr = _view_array(params, bufs)
    assert L.bhRenderBatch(arr, len(params), C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    torch.cuda.synchronize()
    _check(bufs, _singles(params))


def test_batch_graph_launch_and_update(cuda):
    import torch
    L = lib.load()
    params = _views(8, seed=11)
    bufs = [_buffers(P) for P in params]
    arr = _view_array(params, bufs)
    g = C.c_void_p()
    assert L.bhBatchGraphCreate(C.byref(g), arr, len(params)) == 0
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    try:
        assert L.bhBatchGraphLaunch(g, stream) == 0
        torch.cuda.synchronize()
        _check(bufs, _singles(params))
        # new cameras and animation time, same buffers: update, relaunch
        moved = []
        for i, P in enumerate(params):
            Q = P.copy()
            scenes.orbit_camera(Q, 0.3 + 0.1 * i, np.radians(20.0 + 5 * i), 14.0 + i, 50.0)
            Q.diskTime = P.diskTime + 0.5
            moved.append(Q)
        arr2 = _view_array(moved, bufs)
        assert L.bhBatchGraphUpdate(g, arr2, len(moved)) == 0
        assert L.bhBatchGraphLaunch(g, stream) == 0
        torch.cuda.synchronize()
        _check(bufs, _singles(moved))
        # a changed resolution, or a view moved to the other metric family, is refused
        bad = _view_array([params[0].copy()] + moved[1:], bufs)
        bad[0].params.width += 2
        assert L.bhBatchGraphUpdate(g, bad, len(moved)) != 0
        other = params[0].copy()
        scenes.apply_black_hole(other, 2 if other.model < 2 else 0, 0.5 if other.model < 2 else 0.0, 0.0,
                                lib.derive)
        bad = _view_array([other] + moved[1:], bufs)
        assert L.bhBatchGraphUpdate(g, bad, len(moved)) != 0
    finally:
        L.bhBatchGraphDestroy(g)


def test_autotune_applies_a_valid_setting(cuda):
    L = lib.load()
    P = scenes.kerr_pair_1080(lib.derive, 480, 270)[3]
    r, b, o, ms = C.c_int(), C.c_int(), C.c_int(), C.c_float()
    before = lib.get_tuning(1), L.bhGetTileOrder()
    try:
        assert L.bhAutotune(C.byref(P), C.byref(r), C.byref(b), C.byref(o), C.byref(ms)) == 0
        assert r.value in (8, 16, 32) and b.value >= 1 and o.value in (0, 1) and 0.0 < ms.value < 1e4
        assert lib.get_tuning(1) == (r.value, b.value) and L.bhGetTileOrder() == o.value
        print("autotune:", r.value, b.value, o.value, ms.value)
    finally:
        lib.set_tuning(1, *before[0])
        L.bhSetTileOrder(before[1])


def test_batch_autotune_then_batch_still_matches(cuda):
    L = lib.load()
    params = _views(8, seed=3)
    bufs = [_buffers(P) for P in params]
    arr = _view_array(params, bufs)
    bk, bs, ms = C.c_int(-1), C.c_int(-1), C.c_float()
    before = lib.get_tuning(0), lib.get_tuning(1)
    try:
        assert L.bhAutotuneBatch(arr, len(params), C.byref(bk), C.byref(bs), C.byref(ms)) == 0
        assert bk.value >= 1 and bs.value >= 1 and 0.0 < ms.value < 1e4
        assert lib.get_tuning(1)[1] == bk.value and lib.get_tuning(0)[1] == bs.value
        import torch
        for b in bufs:
            b["out"].zero_()
        assert L.bhRenderBatch(arr, len(params), C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
        torch.cuda.synchronize()
        _check(bufs, _singles(params))
    finally:
        lib.set_tuning(0, *before[0])
        lib.set_tuning(1, *before[1])


def test_refill_kernel_agrees_with_tile_kernel(cuda):
    """Under the default work distribution frames run the tile-synchronous
    kernel; with refillMin < 32 they run the refill-queue kernel.  Both trace
    every ray with the same step loop, so the frames agree to rounding (the two
    kernels are compiled separately and may contract a multiply-add
    differently): every pixel within +-1 LSB but a handful."""
    params = _views(12, seed=7)
    tile = _singles(params)
    before = lib.get_tuning(0), lib.get_tuning(1)
    try:
        lib.set_tuning(0, 16, before[0][1])
        lib.set_tuning(1, 16, before[1][1])
        refill = _singles(params)
    finally:
        lib.set_tuning(0, *before[0])
        lib.set_tuning(1, *before[1])
    for a, b in zip(refill, tile):
        s = parity.compare_rgba(a, b)
        assert s["alpha_ok"] and s["lsb1_frac"] >= 0.9995 and s["exact_frac"] >= 0.99, s
