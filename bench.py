"""Benchmark of the B200 null-geodesic tracer (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (the configuration the headline metric is quoted on): 3840x2160
Kerr-Newman a*=0.8 q=0.3, camera r = 25, inclination 75 deg, FOV 45 deg, disk
+ hot spots, bloom + tonemap, balanced preset, plain FP32 RK4.  A step is 30
frames of the 300-frame camera orbit (azimuth 360 k / 300 deg, every 10th
frame; rank r of a multi-GPU run takes the frames offset by r).  Metric:
Mrays/s (one primary ray per pixel) over the whole job, and 4K frame ms.

  value      device-resident throughput of the reference-facing pipeline: per
             step an L2 flush (256 MiB memset, outside the timed events), then
             per frame bhRenderAccum + bhPostProcess (together exactly
             launchRenderPipeline) with CUDA events around each, on the launch
             stream; max over ranks.  frame_ms = median frame time.
  e2e        launchRenderPipeline per frame with RenderParams from the host,
             each RGBA8 frame copied back to pinned host memory, inside the
             timed region; frames alternate between two streams, so a frame's
             tail and read-back overlap the next frame.
  roofline   the tracing kernel (dominant): algorithmic FLOPs / its event time
             (the bhRenderAccum intervals of the timed steps) against the FP32
             FMA peak measured in the same run.  Algorithmic FLOPs follow the
             reference's work on the same inputs: RK4 steps x 420 (Kerr
             family) or x 115 (spherical), + 500 per contributing disk
             sub-sample + 250 per escaped ray, counted by the CPU oracle on a
             1/24^2 pixel sample of every frame.
  cpu_baseline  the reference's own tracer (src/trace.cuh built as host code,
             oracle/_ref) on all host cores, on a bounded pixel sample.
  reference_gpu_kernel  the reference's own black_hole_kernel.cu built
             unchanged for sm_100a (oracle/_ref/libbhref_gpu.so, its
             launchRenderPipeline) on the same 30 frames and buffers, CUDA
             events, L2 flushed: frame ms and this build's speed-up over it.
  surrogate  (1 GPU; --no-surrogate skips it) the learned lensing surrogate
             on the same scene: training from RK4-traced rays, then
             bhSurrogateRender vs the plain frame in its anchored and network
             forms under the strict acceptance gate (and a permissive one),
             pixels within +-1 LSB; and the default anchored form with two
             frames in flight (the handle and its clone on two streams).
  mixed_precision_4k, batch_256_views, post_process, accuracy, kerr_pair_1080
             (1 GPU; --no-configs skips them) the other workloads: the
             near-extremal 4K elevation sweep (FP32 vs mixed precision, frame
             ms and accuracy against the FP64 integration), the 256 random
             views of seed 1234 (one batch / CUDA graph vs 256 calls), bloom +
             tonemap HBM throughput at 4K, FP32 against the FP64 small-step
             integration with conserved-quantity drift, and the 1920x1080
             Kerr / Kerr-Newman pair through bhRenderBatch.

Multi-GPU: one process per GPU (torchrun); every rank renders its own 30
frames (no collective on the data path, "scaling": "weak"); timing is the max
over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "black-hole_b200"))

C_STEP_KERR, C_STEP_SPH, C_DISK, C_BG = 420.0, 115.0, 500.0, 250.0
W, H = 3840, 2160
ORBIT_FRAMES, FRAMES_PER_STEP = 300, 30
PAIR_FRAMES = 8     # frames per scene of the 1920x1080 Kerr / Kerr-Newman pair
L2_FLUSH_BYTES = 256 << 20
PARAM_BYTES = 160   # RenderParams per frame, passed by value to the launch
METRIC = "Mrays/s and 4K frame ms, plain FP32 RK4 (3840x2160 Kerr-Newman a*=0.8 q=0.3 orbit)"
CONFIG = {"workload": "kn_a0.8_q0.3_r25_incl75_fov45_3840x2160_orbit",
          "frames_per_step": FRAMES_PER_STEP, "orbit_frames": ORBIT_FRAMES,
          "step": "30 frames: every 10th frame of the 300-frame orbit (azimuth 360 k / 300 deg), offset by the rank",
          "width": W, "height": H, "preset": "balanced dPhi=0.012 maxSteps=2000",
          "scene": "disk + hot spots on (diskTime 0), bloom + tonemap on, exposure 1",
          "precision": "fp32", "l2": "flushed (256 MiB memset) before every timed step; frame buffers > L2"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--baseline-seconds", type=float, default=12.0)
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--no-configs", action="store_true")
    return ap.parse_args()


def workload(derive, rank=0):
    """The 30 orbit frames of a rank (distinct frames per rank, weak scaling)."""
    from bhrt import ranks, scenes
    ids = ranks.orbit_frames_for_rank(ORBIT_FRAMES, FRAMES_PER_STEP, rank)
    return scenes.kn_orbit_4k(derive, W, H, ORBIT_FRAMES, ids)


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock / throttle samples every 50 ms.  Started before the warm-up (nvidia-smi takes a
    few hundred ms to start); only the samples whose own timestamps fall inside the timed window
    (mark_start .. mark_stop, host wall clock) are reported."""
    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def mark_start(self):
        self.t0 = time.time()

    def mark_stop(self):
        self.t1 = time.time()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 8:
                self.rows.append(parts)

    @staticmethod
    def _when(stamp):
        from datetime import datetime
        try:
            return datetime.strptime(stamp, "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)    # let the samples of the window's last 50 ms arrive
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = self.rows
        if self.t0 is not None and self.t1 is not None:
            inside = [r for r in rows if (w := self._when(r[0])) is not None and self.t0 <= w <= self.t1]
            rows = inside or rows[-1:]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# baseline legs: the reference's tracer on the host cores (+ the work census)
# and the reference's own GPU kernel
# ---------------------------------------------------------------------------
def sample_pixels(frame_idx, stride, W_, H_):
    ys = np.arange((frame_idx * 7) % stride, H_, stride)
    xs = np.arange((frame_idx * 13) % stride, W_, stride)
    yy, xx = np.meshgrid(ys, xs, indexing="ij")
    return (yy * W_ + xx).ravel().astype(np.int32)


def work_census(frames):
    """The reference's algorithmic work on the frames: the restated oracle
    (bit-exact with the reference) on a 1/24^2 pixel sample of every frame."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    port = orc.Oracle()
    census = []
    for k, P in enumerate(frames):
        rec = port.trace_pixels(P, sample_pixels(k, 24, P.width, P.height))
        kerr = P.model in (2, 3)
        flops = (rec["steps"].astype(np.float64) * (C_STEP_KERR if kerr else C_STEP_SPH)
                 + rec["diskSamples"] * C_DISK + (rec["outcome"] == 1) * C_BG)
        census.append({"flops_per_ray": float(flops.mean()), "steps_per_ray": float(rec["steps"].mean()),
                       "disk_per_ray": float(rec["diskSamples"].mean())})
    return census


def cpu_baseline_leg(frames, seconds):
    """The reference tracer on a pixel sample of the workload, all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    cores = os.cpu_count() or 1
    kind = "reference" if orc.RefHost.available() else "port"
    ref = orc.RefHost() if kind == "reference" else orc.Oracle()
    done, t0, chunks = 0, time.perf_counter(), 0
    while True:
        k = chunks % len(frames)
        pix = sample_pixels(k + 31 * (chunks // len(frames)), 64, frames[k].width, frames[k].height)
        if kind == "reference":
            ref.render_pixels(frames[k], pix, threads=cores)
        else:
            ref.trace_pixels(frames[k], pix, threads=cores)
        done += len(pix)
        chunks += 1
        if time.perf_counter() - t0 >= seconds and chunks >= len(frames):
            break
    el = time.perf_counter() - t0
    return {"value": done / el / 1e6, "unit": "Mrays/s", "cores": cores, "kind": kind,
            "sample": f"{done} rays: 1/64^2 strided pixel samples of the {len(frames)} workload frames, "
                      f"{el:.1f} s on {cores} threads"}


def reference_gpu_leg(frames, fs, flush, our_frame_ms):
    """The reference's black_hole_kernel.cu, unchanged, built for sm_100a with its own flags
    (oracle/_ref/libbhref_gpu.so): launchRenderPipeline on the same frames and buffers."""
    import ctypes as C
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    if not orc.RefGpu.available():
        return {"unavailable": "oracle/_ref/libbhref_gpu.so not built (reference tree absent at build time)"}
    R = orc.RefGpu().lib
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731

    def run(evs=None):
        for i, (P, f) in enumerate(zip(frames, fs)):
            if evs is not None:
                evs[i][0].record(stream)
            code = R.launchRenderPipeline(ptr(f.out), ptr(f.accum), ptr(f.bloomA), ptr(f.bloomB), C.byref(P), sp)
            if code != 0:
                raise RuntimeError(f"reference launchRenderPipeline failed: {code}")
            if evs is not None:
                evs[i][1].record(stream)

    run()
    torch.cuda.synchronize()
    flush.zero_()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in frames]
    run(evs)
    torch.cuda.synchronize()
    ms = np.array([a.elapsed_time(b) for a, b in evs])
    med = float(np.median(ms))
    return {"kernel": "reference src/black_hole_kernel.cu built unchanged for sm_100a (--use_fast_math, "
                      "CMakeLists.txt:63)", "frame_ms": med, "mrays_s": W * H / (med * 1e-3) / 1e6,
            "frames": len(frames), "speedup_of_this_build": med / our_frame_ms}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_b200(args, rank, world, local_rank):
    import ctypes as C
    import torch
    import torch.distributed as dist
    from bhrt import lib, ranks
    from bhrt.device import Frame, measure_fp32_peak

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    frames = workload(lib.derive, rank)
    nF = len(frames)
    fs = [Frame(W, H, device=dev) for _ in frames]
    L = lib.load()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    peak = measure_fp32_peak()

    def step(evs=None):
        for i, (P, fr) in enumerate(zip(frames, fs)):
            if evs is not None:
                evs[i][0].record(stream)
            lib.check(L.bhRenderAccum(ptr(fr.accum), C.byref(P), 0, sp), "bhRenderAccum")
            if evs is not None:
                evs[i][1].record(stream)
            lib.check(L.bhPostProcess(ptr(fr.out), ptr(fr.accum), ptr(fr.bloomA), ptr(fr.bloomB), C.byref(P), sp),
                      "bhPostProcess")
            if evs is not None:
                evs[i][2].record(stream)

    clocks = ClockSampler(local_rank)
    clocks.start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    evs = [[[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(nF)] for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.mark_start()
    for s in range(args.steps):
        flush.zero_()
        step(evs[s])
    torch.cuda.synchronize()
    clocks.mark_stop()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    step_ms = np.array([evs[s][0][0].elapsed_time(evs[s][-1][2]) for s in range(args.steps)])
    trace_ms = np.array([[evs[s][i][0].elapsed_time(evs[s][i][1]) for i in range(nF)] for s in range(args.steps)])
    post_ms = np.array([[evs[s][i][1].elapsed_time(evs[s][i][2]) for i in range(nF)] for s in range(args.steps)])
    total_ms = float(step_ms.sum())
    trace_total = float(trace_ms.sum())
    frame_ms = float(np.median(trace_ms + post_ms))

    # e2e: the reference-facing call per frame, params from the host, each RGBA8 frame read back to
    # pinned host memory on a copy stream (overlapping the next frame's tracing); the step ends when
    # the last read-back has landed
    hosts = [torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    side = torch.cuda.Stream(device=dev)
    sps = (sp, C.c_void_p(side.cuda_stream))
    e2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for s in range(-1, args.steps):
        flush.zero_()
        if s >= 0:
            e2[s][0].record(stream)
        side.wait_stream(stream)
        for i, (P, fr) in enumerate(zip(frames, fs)):
            st = stream if i % 2 == 0 else side
            lib.check(L.launchRenderPipeline(ptr(fr.out), ptr(fr.accum), ptr(fr.bloomA), ptr(fr.bloomB),
                                             C.byref(P), sps[i % 2]), "launchRenderPipeline")
            with torch.cuda.stream(st):
                hosts[i % 2].copy_(fr.out, non_blocking=True)
        stream.wait_stream(side)
        if s >= 0:
            e2[s][1].record(stream)
    torch.cuda.synchronize()
    e2e_ms = float(sum(a.elapsed_time(b) for a, b in e2))

    total_ms, e2e_ms, trace_total = ranks.max_over_ranks([total_ms, e2e_ms, trace_total], world, dev)
    rays_step = nF * W * H
    out = {
        "metric": METRIC,
        "value": world * rays_step * args.steps / (total_ms * 1e-3) / 1e6,
        "unit": "Mrays/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "frame_ms": frame_ms,
        "trace_ms_per_frame": float(np.median(trace_ms)),
        "post_ms_per_frame": float(np.median(post_ms)),
        "api": "bhRenderAccum + bhPostProcess per frame (= launchRenderPipeline), device-resident",
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (procedural scene of the named configuration)",
        "config": dict(CONFIG, parallelism=f"replicas x{world} (frames per rank, no collective)"),
        "e2e": {"value": world * rays_step * args.steps / (e2e_ms * 1e-3) / 1e6, "unit": "Mrays/s",
                "api": "launchRenderPipeline per frame + RGBA8 read-back to pinned host memory",
                "h2d_bytes_per_step": nF * PARAM_BYTES, "d2h_bytes_per_step": nF * W * H * 4},
        "gpu_launches": args.steps * nF * 3,
        "clocks": clk,
        "fp32_peak_tflops_measured": peak,
    }
    return out, trace_total, frames, fs, flush


def kerr_pair_leg(steps=3):
    """The 1920x1080 Kerr a*=+0.9 / Kerr-Newman a*=-0.7 q=0.4 pair (r = 20, inclination 80, FOV 45,
    8 frames each, disk + hot spots + bloom): the 16 frames through one bhRenderBatch, L2 flushed."""
    import ctypes as C
    import torch
    from bhrt import lib, scenes
    from bhrt.abi import BHView
    from bhrt.device import Frame
    L = lib.load()
    frames = scenes.kerr_pair_1080(lib.derive, 1920, 1080, PAIR_FRAMES)
    fs = [Frame(1920, 1080) for _ in frames]
    views = (BHView * len(frames))()
    for i, (P, fr) in enumerate(zip(frames, fs)):
        views[i].params = P
        views[i].out, views[i].accum = fr.out.data_ptr(), fr.accum.data_ptr()
        views[i].bloomA, views[i].bloomB = fr.bloomA.data_ptr(), fr.bloomB.data_ptr()
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lib.check(L.bhRenderBatch(views, len(frames), sp), "bhRenderBatch")
    ts = []
    for _ in range(steps):
        flush.zero_()
        e0.record()
        lib.check(L.bhRenderBatch(views, len(frames), sp), "bhRenderBatch")
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    ms = float(np.median(ts))
    return {"workload": "kerr_a0.9+kn_a-0.7_q0.4_1920x1080_8frames_each_bloom (16 frames per call)",
            "api": "bhRenderBatch", "ms_per_16_frames": ms, "frame_ms": ms / len(frames),
            "mrays_s": len(frames) * 1920 * 1080 / (ms * 1e-3) / 1e6}


# ---------------------------------------------------------------------------
# learned surrogate leg (single GPU): train, then 3840x2160 frames, plain vs surrogate
# ---------------------------------------------------------------------------
SG_W, SG_H = 3840, 2160
SG_FRAMES = (0, 50, 100, 150, 200, 250)        # of the 300-frame orbit (azimuth 360 k / 300 deg)


def two_stream_frames(L, h, scene, fa):
    """The default anchored form with two frames in flight: a clone of the handle (same weights and
    settings, its own scratch) renders every other orbit frame on its own stream (the frames of a pair overlap, so one
    frame's anchor pass and resolve passes fill the other's tails).  frame_ms = a pair's time / 2."""
    import ctypes as C
    import torch
    from bhrt import lib
    from bhrt.device import Frame
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    lib.check(L.bhSurrogateSetAnchors(h, 8, 1, C.c_float(1e-4), C.c_float(0.5)), "anchors")
    lib.check(L.bhSurrogateSetGate(h, C.c_float(0.95), C.c_float(0.95), C.c_float(0.02), 256), "gate")
    h2 = C.c_void_p()
    lib.check(L.bhSurrogateClone(h, C.byref(h2)), "bhSurrogateClone")   # same weights and settings
    try:
        hs = (h, h2)
        fs = (Frame(SG_W, SG_H), Frame(SG_W, SG_H))
        ss = (torch.cuda.Stream(), torch.cuda.Stream())
        cur = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def pair(Ps):
            for s in ss:
                s.wait_stream(cur)
            for i in range(2):
                lib.check(L.bhSurrogateRender(hs[i], ptr(fs[i].out), ptr(fs[i].accum), ptr(fs[i].bloomA),
                                              ptr(fs[i].bloomB), C.byref(Ps[i]), C.c_void_p(ss[i].cuda_stream)),
                          "bhSurrogateRender")
            for s in ss:
                cur.wait_stream(s)

        ms, within = [], []
        for k in range(0, len(SG_FRAMES), 2):
            Ps = (scene(SG_FRAMES[k]), scene(SG_FRAMES[k + 1]))
            pair(Ps)                                     # warm-up
            torch.cuda.synchronize()
            e0.record()
            pair(Ps)
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1) / 2)
            for i in range(2):
                fa.pipeline(Ps[i])
                d = (fa.out[..., :3].int() - fs[i].out[..., :3].int()).abs().amax(dim=-1)
                within.append(float((d <= 1).float().mean()))
            torch.cuda.synchronize()
        return {"gate": {"anchor_stride": 8, "network_cell_gate": True, "min_prob": 0.95, "min_conf": 0.95,
                         "crit_band": 0.02, "held_stride": 256, "frames_in_flight": 2},
                "frame_ms": float(np.median(ms)), "px_within_1lsb": float(np.min(within))}
    finally:
        L.bhSurrogateDestroy(h2)


def surrogate_leg():
    import ctypes as C
    import torch
    from bhrt import lib, scenes
    from bhrt.device import Frame
    L = lib.load()
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    h = C.c_void_p()
    lib.check(L.bhSurrogateCreate(C.byref(h), 7), "bhSurrogateCreate")
    try:
        views, rays, steps, batch = 16384, 16384 * 4096, 24000, 16384   # 67 M rays (the 64 Mi of the spec)
        t0 = time.perf_counter()
        lib.check(L.bhSurrogateGenerate(h, rays, views, 7), "bhSurrogateGenerate")
        t_gen = time.perf_counter() - t0
        hist = np.zeros((steps, 5), dtype=np.float32)
        t0 = time.perf_counter()
        lib.check(L.bhSurrogateTrain(h, steps, batch, C.c_float(2e-3), 11, hist.ctypes.data_as(C.c_void_p)),
                  "bhSurrogateTrain")
        t_train = time.perf_counter() - t0
        # fused tensor-core inference alone on one 4K frame of rays
        n = SG_W * SG_H
        x = torch.zeros((n, 8), device="cuda")
        x[:, 2] = 1.0
        y = torch.empty((n, 16), device="cuda")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(2):
            lib.check(L.bhSurrogateForward(h, ptr(x), ptr(y), n, 1, sp), "bhSurrogateForward")
        torch.cuda.synchronize()
        e0.record()
        for _ in range(5):
            L.bhSurrogateForward(h, ptr(x), ptr(y), n, 1, sp)
        e1.record()
        torch.cuda.synchronize()
        mlp_ms = e0.elapsed_time(e1) / 5
        del x, y
        flops = 2.0 * (4 * 256 * 256 + 256 * 16) * n
        peaks = _peaks()
        bf16_peak = peaks.get("bf16_tflops", 1590.0)
        fa, fb = Frame(SG_W, SG_H), Frame(SG_W, SG_H)

        def scene(k):
            return scenes.scene(lib.derive, 3, 0.8, 0.3, SG_W, SG_H, 25.0, 15.0, 45.0, az_deg=360.0 * k / 300.0)

        def timed(fn):
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1)

        def sur(P):
            lib.check(L.bhSurrogateRender(h, ptr(fb.out), ptr(fb.accum), ptr(fb.bloomA), ptr(fb.bloomB),
                                          C.byref(P), sp), "bhSurrogateRender")

        t0 = time.perf_counter()
        sur(scene(0))                                   # first frame: critical curve by RK4 bisection
        torch.cuda.synchronize()
        t_first = time.perf_counter() - t0
        # (anchor stride, network cell gate, minProb, minConf, critBand, held-out stride)
        gates = {"anchored_strict": (8, 1, 0.95, 0.95, 0.02, 256),
                 "anchored_no_network": (8, 0, 0.95, 0.95, 0.02, 256),
                 "anchored_stride4": (4, 1, 0.95, 0.95, 0.02, 256),
                 "network_strict": (0, 1, 0.95, 0.95, 0.02, 256),
                 "network_permissive": (0, 1, 0.5, 0.0, 0.02, 256)}
        res = {}
        plain_ms = []
        for gname, gg in gates.items():
            lib.check(L.bhSurrogateSetAnchors(h, gg[0], gg[1], C.c_float(1e-4), C.c_float(0.5)), "anchors")
            g = gg[2:]
            lib.check(L.bhSurrogateSetGate(h, C.c_float(g[0]), C.c_float(g[1]), C.c_float(g[2]), g[3]), "gate")
            sur_ms, within, rk4, held, held_bad = [], [], [], 0, 0
            for k in SG_FRAMES:
                P = scene(k)
                fa.pipeline(P)
                sur(P)
                torch.cuda.synchronize()
                if gname == "anchored_strict":
                    plain_ms.append(timed(lambda: fa.pipeline(P)))
                sur_ms.append(timed(lambda: sur(P)))
                d = (fa.out[..., :3].int() - fb.out[..., :3].int()).abs().amax(dim=-1)
                within.append(float((d <= 1).float().mean()))
                st = np.zeros(16, dtype=np.uint32)
                lib.check(L.bhSurrogateFrameStats(h, st.ctypes.data_as(C.c_void_p)), "stats")
                rk4.append(float(st[1]) / (SG_W * SG_H))
                held += int(st[2])
                held_bad += int(st[3])
            res[gname] = {"gate": {"anchor_stride": gg[0], "network_cell_gate": bool(gg[1]), "min_prob": g[0],
                                   "min_conf": g[1], "crit_band": g[2], "held_stride": g[3]},
                          "interpolated_frac": float(st[7]) / (SG_W * SG_H),
                          "sky_sampled_frac": float(st[11]) / (SG_W * SG_H),
                          "frame_ms": float(np.median(sur_ms)),
                          "px_within_1lsb": float(np.min(within)),
                          "rk4_pixel_frac": float(np.mean(rk4)),
                          "held_out": held, "held_out_over_1lsb": held_bad}
        res["anchored_strict_two_streams"] = two_stream_frames(L, h, scene, fa)
        pm = float(np.median(plain_ms))
        for r in res.values():
            r["speedup_vs_plain"] = pm / r["frame_ms"]
            r["mrays_s"] = SG_W * SG_H / (r["frame_ms"] * 1e-3) / 1e6
        mlp_tflops = flops / (mlp_ms * 1e-3) / 1e12
        return {
            "workload": "kn_a0.8_q0.3_r25_incl75_fov45_3840x2160_orbit (6 of 300 frames)",
            "plain_frame_ms": pm, "plain_mrays_s": SG_W * SG_H / (pm * 1e-3) / 1e6,
            "train": {"rays": rays, "views": views, "steps": steps, "batch": batch, "seed": 7,
                      "generate_s": t_gen, "train_s": t_train, "final_loss": hist[-50:].mean(axis=0).tolist()},
            "first_frame_s": t_first,
            "gates": res,
            "mlp": {"ms_per_4k_frame": mlp_ms,
                    "roofline": {"bound": "tensor", "achieved": mlp_tflops, "peak": bf16_peak, "unit": "TFLOP/s",
                                 "frac": mlp_tflops / bf16_peak,
                                 "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)" if peaks else "fallback"}},
        }
    finally:
        L.bhSurrogateDestroy(h)


# ---------------------------------------------------------------------------
# configuration legs (single GPU)
# ---------------------------------------------------------------------------
def mixed_leg():
    """3840x2160 Kerr-Newman a*=0.998 (0.995 after the clamp) q=0.05, r=12, FOV 50, elevation sweep:
    frame ms of plain FP32 and of the mixed-precision mode on 5 of the 120 sweep frames."""
    import torch
    from bhrt import lib, scenes
    from bhrt.abi import BH_PREC_FP32, BH_PREC_MIXED
    from bhrt.device import Frame
    ids = (0, 30, 60, 90, 119)
    frames = scenes.kn_sweep_4k(lib.derive, 3840, 2160, frames=120, frame_ids=ids)
    f = Frame(3840, 2160)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    res = {}
    for name, prec in (("fp32", BH_PREC_FP32), ("mixed", BH_PREC_MIXED)):
        ms = []
        for P in frames:
            f.pipeline(P, prec)
            e0.record()
            f.pipeline(P, prec)
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        res[name] = {"frame_ms": float(np.median(ms)), "mrays_s": 3840 * 2160 / (np.median(ms) * 1e-3) / 1e6,
                     "frame_ms_by_elevation_deg": {str(round(89.0 * k / 119, 1)): m for k, m in zip(ids, ms)}}
    res["workload"] = "kn_a0.998_q0.05_r12_fov50_3840x2160_sweep (frames 0, 30, 60, 90, 119 of 120)"
    res["mixed_over_fp32_time"] = res["mixed"]["frame_ms"] / res["fp32"]["frame_ms"]
    # accuracy: FP32 and mixed against the all-FP64 integration (same step control) of the same
    # frames, per-ray records on a 480x270 grid of each camera
    from bhrt.abi import BH_PREC_FP64
    from bhrt.device import probe_grid
    acc = {}
    for k, P in zip(ids, frames):
        ref = probe_grid(P, 480, 270, BH_PREC_FP64)
        acc[str(round(89.0 * k / 119, 1))] = {
            "fp32": _ray_errors(probe_grid(P, 480, 270, BH_PREC_FP32), ref),
            "mixed": _ray_errors(probe_grid(P, 480, 270, BH_PREC_MIXED), ref)}
    res["accuracy_vs_fp64_by_elevation_deg"] = acc
    res["accuracy_grid"] = "480x270 per frame, reference: the all-FP64 GPU integration"
    return res


def _class_edge(cls):
    """True where the 3x3 pixel neighbourhood (clamped) holds more than one class."""
    c = np.asarray(cls)
    p = np.pad(c, 1, mode="edge")
    edge = np.zeros(c.shape, dtype=bool)
    for dy in (0, 1, 2):
        for dx in (0, 1, 2):
            edge |= p[dy:dy + c.shape[0], dx:dx + c.shape[1]] != c
    return edge


def _ray_errors(x, ref):
    """Statistics of probe records x against ref (same grid): class mismatches off class boundaries,
    escape-direction angle (from the difference vector in float64, resolving ~1e-7 rad) and HDR
    relative error on rays off the boundary."""
    inner = ~_class_edge(ref["cls"])
    esc = inner & (x["cls"] == 2) & (ref["cls"] == 2)
    d = x["escDir"][esc].astype(np.float64) - ref["escDir"][esc].astype(np.float64)
    ang = 2.0 * np.arcsin(np.minimum(1.0, np.sqrt((d * d).sum(-1)) / 2.0))
    hx, hr = x["hdr"][inner].astype(np.float64), ref["hdr"][inner].astype(np.float64)
    hrel = (np.abs(hx - hr) / np.maximum(np.abs(hr), 1e-3)).max(-1)
    return {"class_mismatch_off_boundary": int(((x["cls"] != ref["cls"]) & inner).sum()),
            "rays_off_boundary": int(inner.sum()),
            "escape_dir_err_rad": {"median": float(np.median(ang)), "p99": float(np.quantile(ang, 0.99)),
                                   "frac_within_1e-4": float((ang <= 1e-4).mean())},
            "hdr_rel_err": {"median": float(np.median(hrel)), "frac_within_1e-3": float((hrel <= 1e-3).mean())}}


def accuracy_leg():
    """The plain FP32 integration against the FP64 small-step integration (dPhi / 16, 16x the step
    budget; the library's own FP64 kernel) at 480x270: frame 0 of the headline orbit and frame 0 of
    each scene of the 1920x1080 pair, per-ray records from bhProbeGrid.  FP64 at the FP32 step size against the same small-step run
    separates the method's truncation error from FP32 rounding.  Conserved quantities along the FP32
    rays: E and L_z are constants of both integrators' equations, so only the Carter constant (Binet
    first integral) and the null Hamiltonian can drift."""
    from bhrt import lib, scenes
    from bhrt.abi import BH_PREC_FP32, BH_PREC_FP64
    from bhrt.device import probe_grid
    nx, ny = 480, 270
    frames = scenes.kerr_pair_1080(lib.derive, nx, ny, PAIR_FRAMES)
    orbit = scenes.kn_orbit_4k(lib.derive, nx, ny, ORBIT_FRAMES, [0])[0]
    res = {"workload": "kn_a0.8_q0.3 orbit frame 0, kerr_a0.9 and kn_a-0.7_q0.4 frame 0, at 480x270 (disk, hot "
                       "spots on); reference: FP64 with dPhi/16 and 16x maxSteps; all on the GPU",
           "off_boundary": "rays whose reference 3x3 pixel neighbourhood holds one class"}
    for name, P in (("kn_a0.8_q0.3_orbit", orbit), ("kerr_a0.9", frames[0]), ("kn_a-0.7_q0.4", frames[PAIR_FRAMES])):
        a = probe_grid(P, nx, ny, BH_PREC_FP32)
        c = probe_grid(P, nx, ny, BH_PREC_FP64)
        Q = P.copy()
        Q.dPhi, Q.maxSteps = P.dPhi / 16.0, P.maxSteps * 16
        b = probe_grid(Q, nx, ny, BH_PREC_FP64)
        live = a["cls"] != 0
        res[name] = {
            "fp32_vs_small_step": _ray_errors(a, b),
            "fp64_same_step_vs_small_step": _ray_errors(c, b),
            "fp32_drift": {"carter_q_rel_median": float(np.median(a["drift"][live])),
                           "carter_q_rel_max": float(a["drift"][live].max()),
                           "null_hamiltonian_median": float(np.median(a["maxHviol"][live])),
                           "null_hamiltonian_max": float(a["maxHviol"][live].max()),
                           "energy_and_lz": "exact (constants of the integrated equations)"},
            "fp64_same_step_drift": {"carter_q_rel_median": float(np.median(c["drift"][c["cls"] != 0])),
                                     "null_hamiltonian_median": float(np.median(c["maxHviol"][c["cls"] != 0]))},
            "steps_per_ray": {"fp32": float(a["steps"].mean()), "fp64_small_step": float(b["steps"].mean())},
        }
    return res


def post_leg():
    """Bloom + tonemap (bloom_h_kernel + composite_kernel through bhPostProcess) on a rendered
    3840x2160 accumulation buffer (frame 60 of the Kerr-Newman a*=0.998 sweep): 133 MB of float4,
    larger than L2, and L2 flushed before every launch.  Achieved HBM GB/s uses the fused-minimum
    algorithmic traffic of 32 B per full-resolution pixel with bloom (16 B accumulation read, 4 B RGBA8
    write, ~8 B half-resolution horizontal blur written and read, 4 B finished bloom written to
    bloomA) and 20 B without."""
    import torch
    from bhrt import lib, scenes
    from bhrt.device import Frame
    P = scenes.kn_sweep_4k(lib.derive, 3840, 2160, frames=120, frame_ids=(60,))[0]
    f = Frame(3840, 2160)
    f.pipeline(P)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    peaks = _peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    res = {"workload": "bhPostProcess on kn_a0.998_q0.05_r12_fov50_3840x2160 frame 60 (accum 133 MB > L2, "
                       "L2 flushed per launch)",
           "kernels": ["bloom_h_kernel", "composite_kernel"], "algorithmic_bytes_per_px": {"bloom_on": 32.0,
                                                                                          "bloom_off": 20.0},
           "peak_gbs": hbm, "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback"}
    npx = 3840 * 2160
    for bloom in (1, 0):
        P.bloomEnabled = bloom
        for _ in range(3):
            f.post(P)
        ts = []
        for _ in range(20):
            flush.zero_()
            e0.record()
            f.post(P)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        us = float(np.median(ts)) * 1e3
        byts = (32.0 if bloom else 20.0) * npx
        key = "bloom_on" if bloom else "bloom_off"
        res[key] = {"us_per_frame": us, "achieved_gbs": byts / (us * 1e-6) / 1e9,
                    "frac": byts / (us * 1e-6) / 1e9 / hbm}
    return res


def batch256_leg():
    """The 256 random views of seed 1234 (all four families, 128x72 .. 1920x1080): one bhRenderBatch
    call vs 256 launchRenderPipeline calls, and the CUDA-graph replay."""
    import ctypes as C
    import torch
    from bhrt import lib, scenes
    from bhrt.abi import BHView
    from bhrt.device import Frame
    L = lib.load()
    views = scenes.batch_views(lib.derive, 256, 1234)
    fs = [Frame(P.width, P.height) for P in views]
    arr = (BHView * len(views))()
    for i, (P, f) in enumerate(zip(views, fs)):
        arr[i].params = P
        arr[i].out, arr[i].accum = f.out.data_ptr(), f.accum.data_ptr()
        arr[i].bloomA, arr[i].bloomB = f.bloomA.data_ptr(), f.bloomB.data_ptr()
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    npx = sum(P.width * P.height for P in views)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    def seq():
        for P, f in zip(views, fs):
            f.pipeline(P)

    g = C.c_void_p()
    lib.check(L.bhBatchGraphCreate(C.byref(g), arr, len(views)), "bhBatchGraphCreate")
    try:
        t_seq = timed(seq)
        t_batch = timed(lambda: lib.check(L.bhRenderBatch(arr, len(views), sp), "bhRenderBatch"))
        t_graph = timed(lambda: lib.check(L.bhBatchGraphLaunch(g, sp), "bhBatchGraphLaunch"))
    finally:
        L.bhBatchGraphDestroy(g)
    mr = lambda t: npx / (t * 1e-3) / 1e6  # noqa: E731
    return {"workload": "batch_views seed 1234: 256 views, %.1f Mpx" % (npx / 1e6),
            "sequential_ms": t_seq, "batch_ms": t_batch, "graph_ms": t_graph,
            "sequential_mrays_s": mr(t_seq), "batch_mrays_s": mr(t_batch), "graph_mrays_s": mr(t_graph)}


def highlights(out):
    """The figures of every leg in one short object, last on the line."""
    h = {"frame_ms": out.get("frame_ms"), "value_mrays_s": out.get("value"),
         "e2e_mrays_s": out.get("e2e", {}).get("value"), "roofline_frac": out.get("roofline", {}).get("frac")}
    rg = out.get("reference_gpu_kernel", {})
    if "frame_ms" in rg:
        h["reference_gpu_frame_ms"] = rg["frame_ms"]
        h["speedup_over_reference_gpu"] = rg["speedup_of_this_build"]
    sg = out.get("surrogate")
    if sg:
        for g, r in sg["gates"].items():
            h[f"surrogate_{g}"] = {"frame_ms": r["frame_ms"], "speedup": r["speedup_vs_plain"],
                                   "px_within_1lsb": r["px_within_1lsb"], "rk4_frac": r.get("rk4_pixel_frac")}
        h["surrogate_mlp_frac"] = sg["mlp"]["roofline"]["frac"]
    mx = out.get("mixed_precision_4k")
    if mx:
        acc89 = mx["accuracy_vs_fp64_by_elevation_deg"].get("89.0", {})
        h["mixed_vs_fp32_time"] = mx["mixed_over_fp32_time"]
        h["esc_1e4_at_89deg"] = {k: v["escape_dir_err_rad"]["frac_within_1e-4"] for k, v in acc89.items()}
    if out.get("batch_256_views"):
        b = out["batch_256_views"]
        h["batch256_ms"] = {"sequential": b["sequential_ms"], "batch": b["batch_ms"], "graph": b["graph_ms"]}
    if out.get("post_process"):
        h["post_frac_bloom_on"] = out["post_process"]["bloom_on"]["frac"]
    if out.get("kerr_pair_1080"):
        h["kerr_pair_1080_mrays_s"] = out["kerr_pair_1080"]["mrays_s"]
    return h


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        return run_reference(args)

    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    out, trace_total_ms, frames, fs, flush = run_b200(args, rank, world, local_rank)
    if rank == 0:
        if not args.no_cpu_baseline:
            census = work_census(frames)
            flops_step = float(sum(c["flops_per_ray"] * W * H for c in census))
            achieved = flops_step * args.steps / (trace_total_ms * 1e-3) / 1e12
            peak = out["fp32_peak_tflops_measured"]
            out["roofline"] = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                               "frac": achieved / peak if peak else None, "traffic": None,
                               "peak_source": "measured FP32 FMA microbenchmark, max of scalar and packed "
                                              "fma.rn.f32x2 (bhMeasureFp32Peak), same run",
                               "kernel": "tile_kernel<KerrRay<float>> (bhRenderAccum)",
                               "flops_per_frame": flops_step / len(frames),
                               "steps_per_ray": float(np.mean([c["steps_per_ray"] for c in census]))}
            out["cpu_baseline"] = cpu_baseline_leg(frames, args.baseline_seconds)
            if world == 1:
                out["reference_gpu_kernel"] = reference_gpu_leg(frames, fs, flush, out["frame_ms"])
        del fs, flush
        if world == 1 and not args.no_configs:
            import torch
            torch.cuda.empty_cache()
            out["kerr_pair_1080"] = kerr_pair_leg()
            out["mixed_precision_4k"] = mixed_leg()
            out["batch_256_views"] = batch256_leg()
            out["post_process"] = post_leg()
            out["accuracy"] = accuracy_leg()
        if world == 1 and not args.no_surrogate:
            import torch
            torch.cuda.empty_cache()
            out["surrogate"] = surrogate_leg()
        out["highlights"] = highlights(out)
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    """The reference's own tracer (src/trace.cuh and post_process.cuh built as host
    code, oracle/_ref) on the host cores, on the same frames as this build's arm.
    Scenes are derived with the reference's own bhValidateAndDerive, so nothing of
    this build is loaded; each step traces a 1/6^2 strided pixel sample of one
    workload frame through the reference's renderSampleHDR."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    cores = os.cpu_count() or 1
    if orc.RefHost.available():
        kind, impl = "reference", orc.RefHost()
    else:
        kind, impl = "port", orc.Oracle()
    frames = workload(impl.derive, 0)

    def one(k):
        P = frames[k % len(frames)]
        pix = sample_pixels(k, 6, P.width, P.height)
        if kind == "reference":
            impl.render_pixels(P, pix, threads=cores)
        else:
            impl.trace_pixels(P, pix, threads=cores)
        return len(pix)

    for k in range(args.warmup):
        one(k)
    t0 = time.perf_counter()
    n = sum(one(args.warmup + k) for k in range(args.steps))
    el = time.perf_counter() - t0
    v = n / el / 1e6
    out = {"impl": "reference", "metric": METRIC,
           "value": v, "unit": "Mrays/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": el * 1e3 / args.steps, "frame_ms": W * H / (v * 1e6) * 1e3,
           "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (procedural scene of the named configuration)",
           "config": dict(CONFIG, parallelism="replicas x1 (frames per rank, no collective)"),
           "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": cores, "kind": kind,
                            "sample": f"{n} rays over {args.steps} steps (1/6^2 strided pixel samples of the "
                                      f"workload frames) on {cores} threads"},
           "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
