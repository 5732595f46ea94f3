"""The reference's own verification battery (tests/test_main.cu of
Sqhh99/Black-hole, T3-T6) run on the CUDA tracer through the C-ABI, with the
reference's tolerances, plus full-size property checks."""
import math

import numpy as np
import pytest

import parity
from bhrt import lib, scenes
from bhrt.abi import BH_KERR, BH_KERR_NEWMAN, BH_REISSNER_NORDSTROM, BH_SCHWARZSCHILD

pytestmark = pytest.mark.gpu
NX, NY = 96, 54


def grid(model, a, q, dPhi=0.012, max_steps=4000, naked=False, nx=NX, ny=NY, precision=0):
    from bhrt import device
    P = scenes.make_params(lib.derive, model, a, q, dPhi, max_steps, naked)
    return device.probe_grid(P, nx, ny, precision)


def grid_diff(A, B):
    """compareGrids (tests/test_main.cu:195-221)."""
    same = A["outcome"] == B["outcome"]
    esc = same & (A["outcome"] == 1)
    ang = np.sort(parity.chord(A["escDir"], B["escDir"])[esc])
    return {"mismatch": int((~same).sum()), "n": int(A.size),
            "median": float(ang[ang.size // 2]) if ang.size else 0.0,
            "max": float(ang[-1]) if ang.size else 0.0}


def test_T3_model_limits(cuda):
    S = grid(BH_SCHWARZSCHILD, 0, 0)
    RN0 = grid(BH_REISSNER_NORDSTROM, 0, 0)
    RN5 = grid(BH_REISSNER_NORDSTROM, 0, 0.5)
    K0 = grid(BH_KERR, 0, 0)
    K6 = grid(BH_KERR, 0.6, 0)
    KN60 = grid(BH_KERR_NEWMAN, 0.6, 0)
    KN05 = grid(BH_KERR_NEWMAN, 0, 0.5)
    KN00 = grid(BH_KERR_NEWMAN, 0, 0)
    d = grid_diff(S, RN0)
    assert d["mismatch"] == 0 and d["max"] < 1e-4, d
    d = grid_diff(K6, KN60)
    assert d["mismatch"] == 0 and d["max"] < 1e-4, d
    for A, B in ((S, K0), (RN5, KN05), (S, KN00)):
        d = grid_diff(A, B)
        assert d["mismatch"] <= int(0.025 * d["n"]) and d["median"] < 0.02, d
    assert (RN5["outcome"] == 0).sum() < (S["outcome"] == 0).sum()
    Kp, Km = grid(BH_KERR, 0.7, 0), grid(BH_KERR, -0.7, 0)
    d = grid_diff(Kp, Km)
    assert d["mismatch"] > 0 or d["median"] > 1e-3

    def bias(v):
        cap = v["outcome"] == 0
        return int(cap[:, : NX // 2].sum()) - int(cap[:, NX // 2:].sum())
    bp, bm = bias(Kp), bias(Km)
    if bp != 0 or bm != 0:
        assert bp * bm <= 0, (bp, bm)
    naked = grid(BH_KERR, 1.2, 0, naked=True, nx=48, ny=27)
    assert np.all((naked["outcome"] == 0) | (naked["outcome"] == 1))


@pytest.mark.parametrize("model,a,q", [(BH_KERR, 0.9, 0.0), (BH_KERR_NEWMAN, 0.7, 0.5)])
def test_T4_null_constraint(cuda, model, a, q):
    v = np.sort(grid(model, a, q)["maxHviol"].ravel())
    med, mx = v[v.size // 2], v[-1]
    assert med < 5e-3 and mx < 5e-2, (med, mx)


def test_T5_convergence(cuda):
    A = grid(BH_KERR, 0.9, 0, 0.012, 4000)
    B = grid(BH_KERR, 0.9, 0, 0.006, 8000)
    Cc = grid(BH_KERR, 0.9, 0, 0.003, 16000)
    dAB, dBC = grid_diff(A, B), grid_diff(B, Cc)
    assert dBC["median"] <= dAB["median"] * 1.2 + 1e-5 and dBC["median"] < 1e-2, (dAB, dBC)


def test_T5_schwarzschild_shadow_edge(cuda):
    from bhrt import device
    P = scenes.make_params(lib.derive, BH_SCHWARZSCHILD, 0, 0, 0.006, 8000)
    r0 = 30.0
    P.camPos, P.camForward, P.camRight, P.camUp = (r0, 0, 0), (-1, 0, 0), (0, 0, -1), (0, 1, 0)
    M = 0.5
    bc = 3.0 * math.sqrt(3.0) * M
    alpha_th = math.asin(bc * math.sqrt(1.0 - 2.0 * M / r0) / r0)
    lo, hi = 0.0, 0.2
    for _ in range(30):
        mid = 0.5 * (lo + hi)
        d = np.array([[-math.cos(mid), math.sin(mid), 0.0]], dtype=np.float32)
        d /= np.linalg.norm(d)
        rec = device.probe_rays(P, d)[0]
        if rec["outcome"] == 0:
            lo = mid
        else:
            hi = mid
    rel = abs(0.5 * (lo + hi) - alpha_th) / alpha_th
    assert rel < 0.01, rel


def test_T6_stability_and_determinism(cuda):
    import torch
    from bhrt.device import Frame
    W, H = 160, 90
    bad = []
    for k in range(4):
        P = scenes.make_params(lib.derive, BH_KERR_NEWMAN, 0.7, 0.5)
        P.width, P.height, P.diskEnabled = W, H, 1
        bad.append(P)
    bad[0].dPhi = 0.0
    bad[1].maxSteps = 0
    bad[2].camPos = (float("nan"), float("nan"), 0.0)
    bad[3].aSpin, bad[3].Qc, bad[3].rPlus = 7.0, 9.0, -1.0
    f = Frame(W, H)
    for P in bad:
        f.out.zero_()
        f.render_kernel(P)
        torch.cuda.synchronize()
        assert bool((f.out[..., 3] == 255).all())

    P = scenes.make_params(lib.derive, BH_KERR, 0.9, 0)
    P.width, P.height, P.diskEnabled, P.bloomEnabled = W, H, 1, 1
    a = f.pipeline(P).clone()
    b = f.pipeline(P).clone()
    torch.cuda.synchronize()
    assert torch.equal(a, b), "two fresh frames must be bit-identical"

    f.accum.fill_(float("nan"))
    for s in range(8):
        P.sampleIndex, P.accumMode = s, (0 if s == 0 else 1)
        f.pipeline(P)
    torch.cuda.synchronize()
    assert bool((f.out[..., 3] == 255).all()) and bool(torch.isfinite(f.accum).all())

    P.sampleIndex, P.accumMode, P.bloomStrength = -7, 99, float("nan")
    f.pipeline(P)
    torch.cuda.synchronize()

    P = scenes.make_params(lib.derive, BH_KERR, 0.9, 0)
    P.width, P.height, P.diskEnabled, P.bloomEnabled = W, H, 1, 1
    P.hotSpotsEnabled, P.hotSpotStrength, P.diskTime = 1, 1.0, 1.25
    a = f.pipeline(P).clone()
    b = f.pipeline(P).clone()
    torch.cuda.synchronize()
    assert torch.equal(a, b)


@pytest.mark.parametrize("which", [0, 8])
def test_full_hd_frame_matches_oracle_on_pixel_sample(cuda, oracle, which):
    """1920x1080 frames of the Kerr / Kerr-Newman pair: every pixel of a strided
    sample compared with the oracle, and frame-level properties."""
    import torch
    from bhrt.device import Frame, render_hdr
    P = scenes.kerr_pair_1080(lib.derive)[which + 3]
    f = Frame(P.width, P.height)
    out1 = f.pipeline(P).clone()
    out2 = f.pipeline(P).clone()
    hdr = render_hdr(P)
    torch.cuda.synchronize()
    assert torch.equal(out1, out2)
    assert bool((out1[..., 3] == 255).all())
    ys, xs = np.meshgrid(np.arange(3, P.height, 17), np.arange(5, P.width, 17), indexing="ij")
    pix = (ys * P.width + xs).ravel().astype(np.int32)
    ref = oracle.trace_pixels(P, pix)
    got = hdr.cpu().numpy().reshape(-1, 4)[pix, :3].astype(np.float64)
    rel = np.abs(got - ref["hdr"]) / np.maximum(np.abs(ref["hdr"].astype(np.float64)), 1e-3)
    frac = float((rel.max(axis=-1) <= 1e-2).mean())
    print("hdr within 1e-2:", frac, "within 1e-3:", float((rel.max(axis=-1) <= 1e-3).mean()))
    assert frac >= 0.98
