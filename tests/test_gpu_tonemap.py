"""Bloom + tonemap kernels against a plain PyTorch fp32 restatement.

The post-process is exact arithmetic: every operation of the reference's
display chain (src/post_process.cuh:34-148, src/black_hole_kernel.cu:41-103)
is one correctly rounded fp32 operation, in the reference's order.  Here the
same chain is written as separate torch fp32 ops on the GPU (one rounding per
op, no contraction), with torch.pow for the gamma, and the kernels' RGBA8 must
equal it byte for byte -- which also shows that the tonemap's MUFU gamma with
its boundary fallback decides every byte as the full-accuracy power does.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

f32 = np.float32
G9 = [f32(v) for v in (0.02907, 0.06794, 0.12458, 0.17925, 0.20236, 0.17925, 0.12458, 0.06794, 0.02907)]


def _fract(x):
    import torch
    return x - torch.floor(x)


def _hash12(px, py):
    """post_process.cuh dither hash (vec_math.cuh hash12): p.x enters twice."""
    ax = _fract(px * f32(0.1031))
    ay = _fract(py * f32(0.1031))
    az = ax
    d = (ax * (ay + f32(33.33)) + ay * (az + f32(33.33))) + az * (ax + f32(33.33))
    ax, ay, az = ax + d, ay + d, az + d
    return _fract((ax + ay) * az)


def _clamp01(x):
    import torch
    return torch.clamp(x, 0.0, 1.0)


def _half_bloom(acc, exposure):
    """Half-resolution bright pass, then the 9-tap horizontal and vertical
    blurs with clamp-to-edge addressing; returns (hblur, vblur) [bh, bw, 3]."""
    import torch
    H, W = acc.shape[:2]
    bw, bh = (W + 1) // 2, (H + 1) // 2
    dev = acc.device
    x0 = torch.arange(bw, device=dev) * 2
    y0 = torch.arange(bh, device=dev) * 2
    x1 = torch.where(x0 + 1 < W, x0 + 1, x0)
    y1 = torch.where(y0 + 1 < H, y0 + 1, y0)
    a = acc[y0][:, x0, :3]
    b = acc[y0][:, x1, :3]
    c = acc[y1][:, x0, :3]
    d = acc[y1][:, x1, :3]
    avg = (((a + b) + c) + d) * f32(0.25)
    e = avg * f32(exposure)
    lum = (f32(0.2126) * e[..., 0] + f32(0.7152) * e[..., 1]) + f32(0.0722) * e[..., 2]
    # (a tensor divisor: torch turns division by a scalar into a reciprocal multiply)
    t = _clamp01((lum - f32(0.95)) / torch.full_like(lum, f32(2.2) - f32(0.95)))
    w = (t * t) * (f32(3.0) - f32(2.0) * t)
    s = e * w[..., None]
    cols = torch.arange(bw, device=dev)
    hb = torch.zeros_like(s)
    for k in range(9):
        hb = hb + s[:, torch.clamp(cols - 4 + k, 0, bw - 1)] * G9[k]
    rows = torch.arange(bh, device=dev)
    vb = torch.zeros_like(hb)
    for k in range(9):
        vb = vb + hb[torch.clamp(rows - 4 + k, 0, bh - 1)] * G9[k]
    return hb, vb


def _finalize(acc, P, bloom_on):
    """RGBA8 of the whole frame from the float4 accumulation buffer."""
    import torch
    H, W = acc.shape[:2]
    dev = acc.device
    c = acc[..., :3] * f32(P.exposure)
    hb = vb = None
    if bloom_on:
        hb, vb = _half_bloom(acc, P.exposure)
        bh, bw = vb.shape[:2]
        px = torch.arange(W, device=dev, dtype=torch.float32)
        py = torch.arange(H, device=dev, dtype=torch.float32)
        x = (px + f32(0.5)) * f32(0.5) - f32(0.5)
        y = (py + f32(0.5)) * f32(0.5) - f32(0.5)
        ix, iy = torch.floor(x), torch.floor(y)
        fx, fy = (x - ix)[None, :, None], (y - iy)[:, None, None]
        ix, iy = ix.long(), iy.long()
        cx0, cx1 = torch.clamp(ix, 0, bw - 1), torch.clamp(ix + 1, 0, bw - 1)
        cy0, cy1 = torch.clamp(iy, 0, bh - 1), torch.clamp(iy + 1, 0, bh - 1)
        c00, c10 = vb[cy0][:, cx0], vb[cy0][:, cx1]
        c01, c11 = vb[cy1][:, cx0], vb[cy1][:, cx1]
        top = c00 + (c10 - c00) * fx
        bot = c01 + (c11 - c01) * fx
        bloom = top + (bot - top) * fy
        c = c + bloom * f32(P.bloomStrength)
    num = c * (c * f32(2.51) + f32(0.03))
    den = c * (c * f32(2.43) + f32(0.59)) + f32(0.14)
    c = _clamp01(num / den)
    lum = (f32(0.2126) * c[..., 0] + f32(0.7152) * c[..., 1]) + f32(0.0722) * c[..., 2]
    lum = lum[..., None]
    c = _clamp01(lum + (c - lum) * f32(1.12))
    v = torch.pow(c, float(f32(1.0) / f32(2.2)))
    fxp = torch.arange(W, device=dev, dtype=torch.float32)[None, :].expand(H, W)
    fyp = torch.arange(H, device=dev, dtype=torch.float32)[:, None].expand(H, W)
    dth = (_hash12(fxp, fyp) + _hash12(fxp + f32(41.3), fyp + f32(17.7))) - f32(1.0)
    dd = (dth * (f32(1.0) / f32(255.0)))[..., None]
    q = torch.trunc(_clamp01(v + dd) * f32(255.0) + f32(0.5)).to(torch.uint8)
    if P.swapRB:
        q = q[..., [2, 1, 0]]
    out = torch.full((H, W, 4), 255, dtype=torch.uint8, device=dev)
    out[..., :3] = q
    return out, hb, vb


def _hdr(H, W, seed):
    """Synthetic HDR radiance over the tonemap's whole range: black, deep
    shadows (where the gamma is steep), mid tones, bright-pass values and
    over-exposed highlights."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    mag = torch.pow(10.0, torch.rand((H, W, 1), generator=g, device="cuda") * 8.0 - 6.0)
    tint = torch.rand((H, W, 3), generator=g, device="cuda")
    acc = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    acc[..., :3] = (mag * tint).float()
    acc[..., 3] = 1.0
    acc[torch.rand((H, W), generator=g, device="cuda") < 0.1] = 0.0     # captured pixels
    return acc


@pytest.mark.parametrize("W,H,bloom,swap,seed", [
    (1920, 1080, 0, 0, 1),
    (1920, 1080, 1, 0, 2),
    (3840, 2160, 1, 0, 3),
    (333, 197, 1, 1, 4),       # odd sizes: clamped half-res edge, BGRA
    (1, 1, 1, 0, 5),
])
def test_post_matches_torch_fp32_chain(cuda, W, H, bloom, swap, seed):
    import torch
    from bhrt import lib, scenes
    from bhrt.device import Frame
    P = scenes.make_params(lib.derive, 0, 0.0, 0.0)
    P.width, P.height = W, H
    P.bloomEnabled, P.swapRB = bloom, swap
    P.exposure, P.bloomStrength = 1.0, 0.35
    f = Frame(W, H)
    f.accum.copy_(_hdr(H, W, seed))
    f.bloomA.fill_(-7.0)
    f.post(P)
    torch.cuda.synchronize()
    ref, hb, vb = _finalize(f.accum, P, bool(bloom))
    diff = (f.out.int() - ref.int()).abs()
    n_bad = int((diff > 0).any(dim=-1).sum())
    assert n_bad == 0, f"{n_bad} of {W * H} pixels differ, max {int(diff.max())}"
    if bloom:   # bloomB: the horizontally blurred half-res image; bloomA: the finished bloom
        assert torch.equal(f.bloomB[..., :3], hb)
        assert torch.equal(f.bloomA[..., :3], vb)
        assert bool((f.bloomA[..., 3] == 1.0).all())
    else:       # bloom off: the reference's passes leave both buffers alone
        assert bool((f.bloomA == -7.0).all())
