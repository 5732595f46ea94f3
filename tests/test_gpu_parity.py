"""Parity of the CUDA tracer (through the C-ABI of libbh.so) with the oracle.

The oracle here is the reference itself: golden fixtures produced by the
reference's own sources (tests/golden), plus the restated CPU oracle, which
those fixtures pin bit for bit, for cases computed live.

Tolerances (the bar set for this tracer):
  * outcome class (captured / disk / escaped) identical except within one
    pixel of a class boundary of the oracle image;
  * escape directions within 1e-4 rad (chord) for >= 99% of escaped rays off
    the class boundary;
  * HDR radiance within 1e-3 relative (floor 1e-3 absolute) for >= 97% of
    off-boundary rays and within 1e-2 for >= 99%; the rest are rays that
    graze a sub-pixel star core or the photon ring, where an FP32 rounding
    difference moves the sample across a steep texture edge;
  * RGBA8 within +-1 LSB for >= 99.5% of pixels.
"""
import numpy as np
import pytest

import golden_data as G
import parity

pytestmark = pytest.mark.gpu


def _device():
    from bhrt import device
    return device


@pytest.mark.parametrize("name", G.GRID_NAMES)
def test_probe_grid_matches_reference(cuda, name):
    P, want = G.grid(name)
    got = _device().probe_grid(P, G.GRID_NX, G.GRID_NY)
    s = parity.compare_rays(got, want)
    print(name, s)
    assert s["cls_mismatch_inner"] == 0, s
    assert s["esc_frac_1e4"] >= 0.99, s
    assert s["hdr_frac_1e3"] >= 0.97 and s["hdr_frac_1e2"] >= 0.99, s


@pytest.mark.parametrize("name", ["K9_disk", "KNm74_disk", "S_disk"])
def test_probe_grid_fp64_matches_fp64_oracle(cuda, oracle, name):
    P, _ = G.grid(name)
    got = _device().probe_grid(P, G.GRID_NX, G.GRID_NY, precision=2)
    want = oracle.probe_grid(P, G.GRID_NX, G.GRID_NY, precision=2)
    s = parity.compare_rays(got, want)
    print(name, s)
    assert s["cls_mismatch_inner"] == 0, s
    assert s["esc_frac_1e4"] >= 0.995, s
    assert s["hdr_frac_1e2"] >= 0.99, s


@pytest.mark.parametrize("name", G.PIPE_NAMES)
def test_pipeline_matches_reference(cuda, name):
    from bhrt.device import Frame
    import torch
    g = G.load()
    P = G.params(g[f"pipe_{name}_params"])
    f = Frame(P.width, P.height)
    f.pipeline(P)
    torch.cuda.synchronize()
    out = f.out.cpu().numpy()
    s = parity.compare_rgba(out, g[f"pipe_{name}_rgba"])
    print(name, s)
    assert s["alpha_ok"]
    assert s["lsb1_frac"] >= 0.995, s


@pytest.mark.parametrize("name", G.PIPE_NAMES)
def test_post_process_is_exact_given_the_same_hdr(cuda, name):
    """Bloom + tonemap alone: feed the reference's accumulation buffer."""
    from bhrt.device import Frame
    import torch
    g = G.load()
    P = G.params(g[f"pipe_{name}_params"])
    f = Frame(P.width, P.height)
    f.accum.copy_(torch.from_numpy(g[f"pipe_{name}_accum"]))
    f.post(P)
    torch.cuda.synchronize()
    s = parity.compare_rgba(f.out.cpu().numpy(), g[f"pipe_{name}_rgba"])
    print(name, s)
    assert s["max_diff"] <= 1 and s["exact_frac"] >= 0.999, s
    if P.bloomEnabled:   # bloomB: the horizontally blurred half-res image; bloomA: the finished bloom
        bB = f.bloomB.cpu().numpy()
        assert np.array_equal(bB[..., :3], g[f"pipe_{name}_bloomB"][..., :3])
        bA = f.bloomA.cpu().numpy()
        assert np.array_equal(bA, g[f"pipe_{name}_bloomA"])


@pytest.mark.parametrize("name", ["badKN", "K9"])
def test_render_kernel_matches_reference(cuda, name):
    from bhrt.device import Frame
    import torch
    g = G.load()
    P = G.params(g[f"kern_{name}_params"])
    Q, _ = _lib_sanitize(P)
    f = Frame(Q.width, Q.height)
    f.render_kernel(P)
    torch.cuda.synchronize()
    s = parity.compare_rgba(f.out.cpu().numpy(), g[f"kern_{name}_rgba"])
    print(name, s)
    assert s["alpha_ok"] and s["lsb1_frac"] >= 0.995, s


def _lib_sanitize(P):
    from bhrt import lib
    return lib.sanitize(P)


def test_progressive_accumulation_from_poisoned_buffer(cuda):
    from bhrt.device import Frame
    import torch
    g = G.load()
    f = Frame(64, 36)
    f.accum.fill_(float("nan"))
    for raw in g["accum_seq_params"]:
        f.pipeline(G.params(raw))
    torch.cuda.synchronize()
    s = parity.compare_rgba(f.out.cpu().numpy(), g["accum_seq_rgba"])
    print(s)
    assert s["alpha_ok"] and s["lsb1_frac"] >= 0.995, s
    assert np.all(np.isfinite(f.accum.cpu().numpy()))


@pytest.mark.parametrize("w,h,model,swap,bloom", [
    (1, 1, 3, 0, 1),        # one pixel (bloom's half-res image is 1 x 1)
    (3, 5, 2, 1, 1),        # smaller than one 8x4 tile, BGRA
    (97, 61, 3, 0, 1),      # ragged in both directions
    (8, 4, 0, 0, 0),        # exactly one tile
    (33, 200, 1, 1, 0),     # tall and narrow, BGRA, no bloom
])
def test_edge_frame_sizes_match_oracle(cuda, oracle, derive, w, h, model, swap, bloom):
    """Frame shapes the 8x4 tiling and the half-resolution bloom must handle,
    against the oracle (bit-exact with the reference's host build)."""
    import torch
    from bhrt import scenes
    from bhrt.device import Frame
    a = {0: 0.0, 1: 0.0, 2: 0.9, 3: -0.7}[model]
    q = {0: 0.0, 1: 0.5, 2: 0.0, 3: 0.4}[model]
    P = scenes.scene(derive, model, a, q, w, h, 20.0, 10.0, 45.0, bloom=bool(bloom), disk_time=0.4)
    P.swapRB = swap
    f = Frame(w, h)
    f.pipeline(P)
    torch.cuda.synchronize()
    want, _, _, _ = oracle.pipeline(P)
    s = parity.compare_rgba(f.out.cpu().numpy(), want)
    print(w, h, s)
    assert s["alpha_ok"]
    # tiny frames: every pixel must be within 1 LSB; larger ones: the usual 99.5 %
    assert s["lsb1_frac"] >= (1.0 if w * h < 64 else 0.995), s
