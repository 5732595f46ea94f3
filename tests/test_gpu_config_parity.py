"""Parity at the benchmark workloads' own configurations and sizes.

Each workload is rendered by the CUDA tracer through the C-ABI at its stated
size and compared with the oracle on every pixel (the comparison pattern of
the reference's compareGrids, tests/test_main.cu:195-221, extended to
radiance and 8-bit output):

  1  Schwarzschild 320x180, disk on, bloom off: the reference's own output
     (golden fixture made by the reference's sources built as host code);
  2  the 1920x1080 Kerr a*=+0.9 and Kerr-Newman a*=-0.7 q=0.4 frames 0 of
     both scenes (disk, hot spots, bloom, tonemap): the CPU oracle, live;
  3  the near-extremal Kerr-Newman elevation sweep (a*=0.995 after the clamp,
     q=0.05, r=12, FOV 50) at 480x270, elevations 0, 45 and 89 deg: FP32
     against the FP32 oracle, and the mixed-precision mode against the CPU
     FP64 oracle at the same step control;
  4  32 of the 256 random views of seed 1234 (every 8th), rendered in one
     bhRenderBatch call with the other 224: the CPU oracle, live.

Bars (asserted per configuration at the levels measured on B200): outcome
class identical off the class boundaries; escape directions within 1e-4 rad
on >= 99.9 % of off-boundary escaped rays (config 1: 100 %); RGBA8 within
+-1 LSB on >= 99.95 % of pixels; HDR within 1e-3 relative (floor 1e-3) on the
off-boundary fraction stated in HDR_1E3 below (measured: config 1 99.83 %,
config 2 99.67 / 99.65 %, config 3 99.31-99.65 %, config 4 99.02 % in the
worst of the 32 views, 99.6 % on average).  The HDR misses are rays that graze a sub-pixel star core or a
disk-noise cell edge, where a ~1e-7 rad difference in direction, from
different (correctly rounded vs hardware) sin/cos and reciprocal roundings,
moves the sample across a steep texture edge.
"""
import ctypes as C

import numpy as np
import pytest

import golden_data as G
import parity
from bhrt import lib, scenes
from bhrt.abi import BH_PREC_FP32, BH_PREC_FP64, BH_PREC_MIXED, PROBE_DTYPE

pytestmark = pytest.mark.gpu

# off-boundary fraction of pixels whose HDR is within 1e-3 relative of the oracle's
HDR_1E3 = {"config1": 0.998, "config2": 0.996, "config3": 0.99, "config4_worst": 0.985, "config4_mean": 0.995}


def _hdr_frac(got, ref, mask):
    g = np.asarray(got, np.float64)[..., :3]
    r = np.asarray(ref, np.float64)[..., :3]
    rel = (np.abs(g - r) / np.maximum(np.abs(r), 1e-3)).max(axis=-1)
    return float((rel[mask] <= 1e-3).mean())


def _frame(P):
    import torch
    from bhrt.device import Frame
    f = Frame(P.width, P.height)
    f.pipeline(P)
    torch.cuda.synchronize()
    return f.out.cpu().numpy(), f.accum.cpu().numpy()


def test_config1_schwarzschild_320x180_full_frame(cuda):
    from bhrt.device import probe_grid
    z = np.load(G.PATH.replace("golden.npz", "config1_schwarzschild_320x180.npz"))
    P = G.params(z["params"])
    ref = np.zeros((P.height, P.width), dtype=PROBE_DTYPE)
    for k in ("outcome", "cls", "steps", "escDir", "trans", "hdr"):
        ref[k] = z[k]
    out, acc = _frame(P)
    s = parity.compare_rgba(out, z["rgba"])
    rays = probe_grid(P, P.width, P.height)
    st = parity.compare_rays(rays, ref)
    inner = ~parity.boundary_mask(ref["cls"])
    hf = _hdr_frac(acc, ref["hdr"], inner)
    print("config1", s, st, "frame hdr within 1e-3:", hf)
    assert s["alpha_ok"] and s["lsb1_frac"] >= 0.9995, s
    assert st["cls_mismatch_inner"] == 0, st
    assert st["esc_frac_1e4"] == 1.0, st
    assert st["hdr_frac_1e3"] >= HDR_1E3["config1"] and hf >= HDR_1E3["config1"], (st, hf)


@pytest.mark.parametrize("k", [0, 8])
def test_config2_full_hd_frame(cuda, oracle, k):
    from bhrt.device import probe_grid
    P = scenes.kerr_pair_1080(lib.derive)[k]
    ref_hdr, ref_rays = oracle.render_hdr(P, rays=True)
    ref_out, _, _ = oracle.post(P, ref_hdr)
    out, acc = _frame(P)
    s = parity.compare_rgba(out, ref_out)
    rays = probe_grid(P, P.width, P.height)
    st = parity.compare_rays(rays, ref_rays)
    inner = ~parity.boundary_mask(ref_rays["cls"])
    hf = _hdr_frac(acc, ref_hdr, inner)
    print(f"config2 frame {k}", s, st, "frame hdr within 1e-3:", hf)
    assert s["alpha_ok"] and s["lsb1_frac"] >= 0.9995, s
    assert st["cls_mismatch_inner"] == 0, st
    assert st["esc_frac_1e4"] >= 0.999, st
    assert hf >= HDR_1E3["config2"], hf


@pytest.mark.parametrize("fid", [0, 60, 119])
def test_config3_sweep_frame_480x270(cuda, oracle, fid):
    """FP32 against the FP32 oracle (the reference's method); MIXED and the GPU
    FP64 integration against the CPU FP64 oracle at the same step control."""
    from bhrt.device import probe_grid
    P = scenes.kn_sweep_4k(lib.derive, 480, 270, frames=120, frame_ids=[fid])[0]
    nx, ny = 480, 270
    ref32 = oracle.probe_grid(P, nx, ny, precision=0)
    ref64 = oracle.probe_grid(P, nx, ny, precision=2)
    g32 = probe_grid(P, nx, ny, BH_PREC_FP32)
    gmx = probe_grid(P, nx, ny, BH_PREC_MIXED)
    g64 = probe_grid(P, nx, ny, BH_PREC_FP64)
    s32 = parity.compare_rays(g32, ref32)
    smx = parity.compare_rays(gmx, ref64)
    s64 = parity.compare_rays(g64, ref64)
    f32_vs_64 = parity.compare_rays(g32, ref64)
    el = 89.0 * fid / 119
    print(f"config3 el={el:.1f} fp32-vs-oracle32 {s32}\n  mixed-vs-oracle64 {smx}\n  "
          f"fp64-vs-oracle64 {s64}\n  fp32-vs-oracle64 {f32_vs_64}")
    for st in (s32, smx, s64):
        assert st["cls_mismatch_inner"] <= max(2, int(1e-4 * nx * ny)), st
    assert s64["esc_frac_1e4"] >= 0.999, s64
    # mixed: within 1e-4 rad of the FP64 integration on >= 99.9 % of rays up to 45 deg
    # and >= 99.5 % at 89 deg (measured 99.79 % with the 0.9 deg polar cap), and
    # closer to it than plain FP32 (measured 98.5 % at 89 deg: the polar passages)
    assert smx["esc_frac_1e4"] >= (0.999 if el < 80 else 0.995), smx
    assert smx["esc_frac_1e4"] >= f32_vs_64["esc_frac_1e4"], (smx, f32_vs_64)
    # FP32 against the reference's own FP32 method (both start from the same rounded
    # initial state, so they agree even where both drift from FP64)
    assert s32["esc_frac_1e4"] >= 0.999, s32
    assert s32["hdr_frac_1e3"] >= HDR_1E3["config3"], s32


def test_config4_batch_views_against_oracle(cuda, oracle):
    import torch
    from bhrt.abi import BHView
    L = lib.load()
    views = scenes.batch_views(lib.derive, 256, 1234)
    bufs = []
    arr = (BHView * len(views))()
    for i, P in enumerate(views):
        W, H = P.width, P.height
        bw, bh = (W + 1) // 2, (H + 1) // 2
        b = {"out": torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda"),
             "accum": torch.zeros((H, W, 4), dtype=torch.float32, device="cuda"),
             "bloomA": torch.zeros((bh, bw, 4), dtype=torch.float32, device="cuda"),
             "bloomB": torch.zeros((bh, bw, 4), dtype=torch.float32, device="cuda")}
        bufs.append(b)
        arr[i].params = P
        arr[i].out, arr[i].accum = b["out"].data_ptr(), b["accum"].data_ptr()
        arr[i].bloomA, arr[i].bloomB = b["bloomA"].data_ptr(), b["bloomB"].data_ptr()
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib.check(L.bhRenderBatch(arr, len(views), sp), "bhRenderBatch")
    torch.cuda.synchronize()
    worst_lsb, worst_hdr, hdrs = 1.0, 1.0, []
    for i in range(0, len(views), 8):
        P = views[i]
        ref_hdr, ref_rays = oracle.render_hdr(P, rays=True)
        ref_out, ref_bA, _ = oracle.post(P, ref_hdr)
        out = bufs[i]["out"].cpu().numpy()
        acc = bufs[i]["accum"].cpu().numpy()
        s = parity.compare_rgba(out, ref_out)
        inner = ~parity.boundary_mask(ref_rays["cls"])
        hf = _hdr_frac(acc, ref_hdr, inner)
        print(f"config4 view {i} {P.width}x{P.height} model {P.model}", s, "hdr within 1e-3:", hf)
        assert s["alpha_ok"] and s["lsb1_frac"] >= 0.9995, (i, s)
        worst_lsb, worst_hdr = min(worst_lsb, s["lsb1_frac"]), min(worst_hdr, hf)
        hdrs.append(hf)
    print("config4 worst view: rgba within 1 LSB", worst_lsb, "hdr within 1e-3", worst_hdr, "mean", np.mean(hdrs))
    assert worst_hdr >= HDR_1E3["config4_worst"], worst_hdr
    assert np.mean(hdrs) >= HDR_1E3["config4_mean"], np.mean(hdrs)
