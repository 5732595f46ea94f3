"""Headless driver: render named or custom scenes through the C-ABI.

    python black-hole_b200/bhrt/cli.py render --scene kerr1080 --frame 3 --out kerr.png
    python black-hole_b200/bhrt/cli.py render --model 3 --astar 0.8 --q 0.3 --r 25 --el 15 \\
        --fov 50 --width 1280 --height 720 --preset high --ori 0 30 0 --out kn.ppm
    python black-hole_b200/bhrt/cli.py sweep --scene kn4k --frames 120 --step 12 --width 960 \\
        --height 540 --outdir frames/
    python black-hole_b200/bhrt/cli.py render --scene kn1080 --repeat 5      (timing)
    python black-hole_b200/bhrt/cli.py batch --scene pair1080 --frames 16 --repeat 3   (one queue)
    python black-hole_b200/bhrt/cli.py mlp --rays 2097152 --repeat 3      (surrogate MLP timing)
    python black-hole_b200/bhrt/cli.py surrogate --scene orbit4k --stride 8 --repeat 3 --out s.png
                                                      (anchored surrogate frame vs the plain frame)

Replaces the reference application's interactive loop (src/main.cpp): the
orbit camera, body orientation and quality presets become arguments; frames
go to a device buffer and, on request, to PPM/PNG files.  Named scenes are the
workloads of the benchmark and the tests (bhrt.scenes).
"""
import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from bhrt import lib, scenes  # noqa: E402
from bhrt.abi import BH_PREC_FP32, BH_PREC_FP64, BH_PREC_MIXED, MODEL_NAMES  # noqa: E402


def named(name, frame, width, height):
    d = lib.derive
    if name == "schw320":
        return scenes.schwarzschild_320(d, width or 320, height or 180)
    if name in ("kerr1080", "kn1080"):
        fr = scenes.kerr_pair_1080(d, width or 1920, height or 1080)
        return fr[(0 if name == "kerr1080" else 8) + (frame % 8)]
    if name == "pair1080":
        return scenes.kerr_pair_1080(d, width or 1920, height or 1080)[frame % 16]
    if name == "kn4k":
        return scenes.kn_sweep_4k(d, width or 3840, height or 2160, frame_ids=[frame % 120])[0]
    if name == "orbit4k":
        return scenes.kn_orbit_4k(d, width or 3840, height or 2160, 300, [frame % 300])[0]
    if name == "batch":
        v = scenes.batch_views(d)[frame % 256]
        return v
    raise SystemExit(f"unknown scene {name}")


def custom(a):
    return scenes.scene(lib.derive, a.model, a.astar, a.q, a.width or 1280, a.height or 720, a.r, a.el, a.fov,
                        az_deg=a.az, preset=a.preset, disk=not a.no_disk, hot_spots=not a.no_spots,
                        bloom=not a.no_bloom, disk_time=a.time, exposure=a.exposure, ori_deg=tuple(a.ori),
                        allow_naked=a.naked)


def render(P, precision, repeat, out_path):
    import torch
    from bhrt.device import Frame
    from bhrt.imageio import write_image
    f = Frame(P.width, P.height)
    times = []
    for _ in range(max(1, repeat)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        f.pipeline(P, precision)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    if out_path:
        write_image(out_path, f.out.cpu().numpy())
    return times


def render_batch(views, repeat):
    """All views in one bhRenderBatch call (one work queue), timed."""
    import ctypes as C
    import torch
    from bhrt.abi import BHView
    from bhrt.device import Frame
    fs = [Frame(P.width, P.height) for P in views]
    arr = (BHView * len(views))()
    for i, (P, f) in enumerate(zip(views, fs)):
        arr[i].params = P
        arr[i].out, arr[i].accum = f.out.data_ptr(), f.accum.data_ptr()
        arr[i].bloomA, arr[i].bloomB = f.bloomA.data_ptr(), f.bloomB.data_ptr()
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    times = []
    for _ in range(max(1, repeat)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        lib.check(lib.load().bhRenderBatch(arr, len(views), sp), "bhRenderBatch")
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return times


def time_mlp(rays, repeat):
    """The fused tensor-core surrogate inference on `rays` synthetic input rows (untrained network)."""
    import ctypes as C
    import torch
    L = lib.load()
    h = C.c_void_p()
    lib.check(L.bhSurrogateCreate(C.byref(h), 7), "bhSurrogateCreate")
    x = torch.zeros((rays, 8), device="cuda")
    x[:, 2] = 1.0
    y = torch.empty((rays, 16), device="cuda")
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    times = []
    for _ in range(max(1, repeat)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        lib.check(L.bhSurrogateForward(h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), rays, 1, sp),
                  "bhSurrogateForward")
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    L.bhSurrogateDestroy(h)
    return times


def render_surrogate(P, stride, use_net, repeat, out_path):
    """The anchored (stride >= 2) or network (stride 0) surrogate frame of an untrained
    network (the anchored form without its cell gate needs none), timed, against the
    plain frame: returns (times, plain ms, fraction within 1 LSB, frame statistics)."""
    import ctypes as C
    import numpy as np
    import torch
    from bhrt.device import Frame
    from bhrt.imageio import write_image
    L = lib.load()
    h = C.c_void_p()
    lib.check(L.bhSurrogateCreate(C.byref(h), 7), "bhSurrogateCreate")
    try:
        lib.check(L.bhSurrogateSetAnchors(h, stride, use_net, C.c_float(1e-4), C.c_float(0.5)), "anchors")
        plain, f = Frame(P.width, P.height), Frame(P.width, P.height)
        sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        plain.pipeline(P)
        e0.record()
        plain.pipeline(P)
        e1.record()
        torch.cuda.synchronize()
        plain_ms = e0.elapsed_time(e1)
        times = []
        for _ in range(max(1, repeat)):
            e0.record()
            lib.check(L.bhSurrogateRender(h, C.c_void_p(f.out.data_ptr()), C.c_void_p(f.accum.data_ptr()),
                                          C.c_void_p(f.bloomA.data_ptr()), C.c_void_p(f.bloomB.data_ptr()),
                                          C.byref(P), sp), "bhSurrogateRender")
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        st = np.zeros(16, dtype=np.uint32)
        lib.check(L.bhSurrogateFrameStats(h, st.ctypes.data_as(C.c_void_p)), "bhSurrogateFrameStats")
        d = (plain.out[..., :3].int() - f.out[..., :3].int()).abs().amax(dim=-1)
        within = float((d <= 1).float().mean())
        if out_path:
            write_image(out_path, f.out.cpu().numpy())
        return times, plain_ms, within, st
    finally:
        L.bhSurrogateDestroy(h)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("cmd", choices=["render", "sweep", "batch", "mlp", "surrogate", "info"])
    ap.add_argument("--stride", type=int, default=8, help="surrogate: anchor stride (0: the network form)")
    ap.add_argument("--net", type=int, default=0, help="surrogate: 1 applies the network's gate (untrained)")
    ap.add_argument("--rays", type=int, default=3840 * 2160)
    ap.add_argument("--scene", default=None, help="schw320 | kerr1080 | kn1080 | pair1080 | kn4k | orbit4k | batch")
    ap.add_argument("--frame", type=int, default=0)
    ap.add_argument("--frames", type=int, default=120)
    ap.add_argument("--step", type=int, default=1)
    ap.add_argument("--width", type=int, default=0)
    ap.add_argument("--height", type=int, default=0)
    ap.add_argument("--model", type=int, default=3)
    ap.add_argument("--astar", type=float, default=0.8)
    ap.add_argument("--q", type=float, default=0.3)
    ap.add_argument("--r", type=float, default=25.0)
    ap.add_argument("--el", type=float, default=15.0)
    ap.add_argument("--az", type=float, default=0.0)
    ap.add_argument("--fov", type=float, default=60.0)
    ap.add_argument("--ori", type=float, nargs=3, default=[0.0, 0.0, 0.0], metavar=("X", "Y", "Z"))
    ap.add_argument("--preset", default="balanced", choices=list(scenes.PRESETS))
    ap.add_argument("--time", type=float, default=0.0)
    ap.add_argument("--exposure", type=float, default=1.0)
    ap.add_argument("--no-disk", action="store_true")
    ap.add_argument("--no-spots", action="store_true")
    ap.add_argument("--no-bloom", action="store_true")
    ap.add_argument("--naked", action="store_true")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "mixed", "fp64"])
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--out", default=None)
    ap.add_argument("--outdir", default=None)
    a = ap.parse_args(argv)
    prec = {"fp32": BH_PREC_FP32, "mixed": BH_PREC_MIXED, "fp64": BH_PREC_FP64}[a.precision]

    if a.cmd == "info":
        P = named(a.scene, a.frame, a.width, a.height) if a.scene else custom(a)
        Q, _ = lib.sanitize(P)
        print(f"{MODEL_NAMES[Q.model]}  M={Q.M} a={Q.aSpin:.4f} Q={Q.Qc:.4f} r+={Q.rPlus:.4f} "
              f"r_ph={Q.rPhoton:.4f} disk=[{Q.diskInner:.4f}, {Q.diskOuter}] {Q.width}x{Q.height} "
              f"dPhi={Q.dPhi} maxSteps={Q.maxSteps}")
        return 0
    if a.cmd == "render":
        P = named(a.scene, a.frame, a.width, a.height) if a.scene else custom(a)
        t = render(P, prec, a.repeat, a.out)
        print(f"{P.width}x{P.height} {MODEL_NAMES[P.model]} {a.precision}: {min(t):.3f} ms (best of {len(t)})"
              + (f" -> {a.out}" if a.out else ""))
        return 0
    if a.cmd == "mlp":
        t = time_mlp(a.rays, a.repeat)
        flop = 2.0 * (4 * 256 * 256 + 256 * 16) * a.rays
        print(f"fused surrogate MLP, {a.rays} rays: {min(t):.3f} ms (best of {len(t)}), "
              f"{flop / min(t) / 1e9:.1f} TFLOP/s")
        return 0
    if a.cmd == "surrogate":
        P = named(a.scene, a.frame, a.width, a.height) if a.scene else custom(a)
        t, pm, within, st = render_surrogate(P, a.stride, a.net, a.repeat, a.out)
        print(f"{P.width}x{P.height} surrogate stride {a.stride}: {min(t):.3f} ms (best of {len(t)}), "
              f"plain {pm:.3f} ms, {100 * within:.3f} % within 1 LSB, {st[7]} interpolated, "
              f"{st[1]} traced by RK4" + (f" -> {a.out}" if a.out else ""))
        return 0
    if a.cmd == "batch":
        views = [named(a.scene, k, a.width, a.height) if a.scene else custom(a)
                 for k in range(a.frame, a.frames, max(1, a.step))]
        t = render_batch(views, a.repeat)
        npx = sum(P.width * P.height for P in views)
        print(f"{len(views)} views, {npx / 1e6:.2f} Mpx in one batch: {min(t):.3f} ms (best of {len(t)}), "
              f"{npx / min(t) / 1e3:.1f} Mrays/s")
        return 0
    # sweep
    if a.outdir:
        os.makedirs(a.outdir, exist_ok=True)
    for k in range(a.frame, a.frames, max(1, a.step)):
        P = named(a.scene, k, a.width, a.height) if a.scene else custom(a)
        out = os.path.join(a.outdir, f"frame_{k:04d}.png") if a.outdir else None
        t = render(P, prec, a.repeat, out)
        print(f"frame {k}: {min(t):.3f} ms")
    return 0


if __name__ == "__main__":
    sys.exit(main())
