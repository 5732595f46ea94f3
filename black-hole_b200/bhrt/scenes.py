"""Scene construction: orbit camera, quality presets and the named workloads.

The orbit camera restates the reference application's fillCamera
(src/main.cpp:186-228): spin axis +Y, camera at (d cos(el) cos(az), d sin(el),
d cos(el) sin(az)) looking at the origin, then the body orientation R = Rz Ry Rx
(main.cpp:147-166; identity by default).  Inclination i maps to elevation 90 deg - i.  Distances are code units
with M = 0.5, so "r = 20 rs" is 20.0.

make_params restates the reference test helper makeParams
(tests/test_main.cu:132-154): derive the metric quantities on the host with
bhValidateAndDerive, disk inner edge at the numeric ISCO, outer edge 8.
"""
import math

import numpy as np

from .abi import (BH_KERR, BH_KERR_NEWMAN, BH_REISSNER_NORDSTROM, BH_SCHWARZSCHILD, BHDerived,
                  RenderParams)

# Quality presets (reference src/main.cpp:307-309): (dPhi, maxSteps)
PRESETS = {"fast": (0.020, 1200), "balanced": (0.012, 2000), "high": (0.007, 3500)}


def _rotate_body(v, ori):
    """R = Rz(ori_z) Ry(ori_y) Rx(ori_x) applied to a vector (main.cpp:147-166)."""
    f32 = np.float32
    cx, sx = f32(math.cos(ori[0])), f32(math.sin(ori[0]))
    cy, sy = f32(math.cos(ori[1])), f32(math.sin(ori[1]))
    cz, sz = f32(math.cos(ori[2])), f32(math.sin(ori[2]))
    x0, y0, z0 = (f32(t) for t in v)
    x1, y1, z1 = x0, cx * y0 - sx * z0, sx * y0 + cx * z0
    x2, y2, z2 = cy * x1 + sy * z1, y1, -sy * x1 + cy * z1
    return np.array([cz * x2 - sz * y2, sz * x2 + cz * y2, z2], dtype=f32)


def _unit(v):
    f32 = np.float32
    n = f32(np.sqrt(np.sum(v * v, dtype=f32)))
    if n < 1e-8:
        return np.array([0.0, 1.0, 0.0], dtype=f32)
    return (v / n).astype(f32)


def orbit_camera(P, az, el, dist, fov_deg=60.0, ori=(0.0, 0.0, 0.0)):
    """fillCamera (main.cpp:186-228) in float32: orbit camera looking at the hole,
    mapped through the body orientation `ori` (Euler X, Y, Z; identity by default)."""
    f32 = np.float32
    ca, sa = f32(math.cos(az)), f32(math.sin(az))
    ce, se = f32(math.cos(el)), f32(math.sin(el))
    d = f32(dist)
    p = np.array([d * ce * ca, d * se, d * ce * sa], dtype=f32)
    fl = f32(np.sqrt(np.sum(p * p, dtype=f32)))
    f = (-p / fl).astype(f32)
    r = np.array([-f[2], 0.0, f[0]], dtype=f32)
    rl = f32(np.sqrt(r[0] * r[0] + r[2] * r[2]))
    if rl < 1e-6:
        r, rl = np.array([1.0, 0.0, 0.0], dtype=f32), f32(1.0)
    r = (r / rl).astype(f32)
    p, f, r = (_rotate_body(v, ori) for v in (p, f, r))   # identity for ori = 0
    f, r = _unit(f), _unit(r)
    u = _unit(np.cross(r, f).astype(f32))                  # re-orthogonalised up
    P.camPos, P.camForward, P.camRight, P.camUp = p, f, r, u
    P.tanHalfFov = float(f32(math.tan(math.radians(fov_deg) * 0.5)))
    P.aspect = float(f32(P.width) / f32(P.height)) if P.height > 0 else 16.0 / 9.0
    return P


def test_camera(P, az, el, dist):
    """The reference test suite's setCamera (tests/test_main.cu:111-130): 60 deg FOV, 16:9."""
    f32 = np.float32
    ca, sa = f32(math.cos(az)), f32(math.sin(az))
    ce, se = f32(math.cos(el)), f32(math.sin(el))
    d = f32(dist)
    p = np.array([d * ce * ca, d * se, d * ce * sa], dtype=f32)
    fl = f32(np.sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]))
    f = np.array([-p[0] / fl, -p[1] / fl, -p[2] / fl], dtype=f32)
    r = np.array([-f[2], 0.0, f[0]], dtype=f32)
    rl = f32(np.sqrt(r[0] * r[0] + r[2] * r[2]))
    if rl < 1e-6:
        r, rl = np.array([1.0, 0.0, 0.0], dtype=f32), f32(1.0)
    r = np.array([r[0] / rl, 0.0, r[2] / rl], dtype=f32)
    u = np.array([r[1] * f[2] - r[2] * f[1], r[2] * f[0] - r[0] * f[2], r[0] * f[1] - r[1] * f[0]],
                 dtype=f32)
    P.camPos, P.camForward, P.camRight, P.camUp = p, f, r, u
    P.tanHalfFov = float(f32(math.tan(60.0 * 3.14159265 / 180.0 * 0.5)))
    P.aspect = float(f32(16.0) / f32(9.0))
    return P


def apply_black_hole(P, model, a_star, q, derive, allow_naked=False, disk_outer=8.0):
    """applyBlackHole (main.cpp:97-134): validate, derive, disk inner edge at the ISCO.

    `derive(model, M, aStar, q, allowNaked) -> (BHDerived, M, aStar, q)` is the
    host derivation to use (the product library's bhValidateAndDerive)."""
    d, M, a_eff, q_eff = derive(model, 0.5, a_star, q, allow_naked)
    P.model = model
    P.M = M
    P.aSpin, P.Qc = d.a, d.Q
    P.rPlus, P.rPhoton, P.rErgo = d.rPlus, d.rPhoton, d.rErgo
    P.allowNaked = 1 if allow_naked else 0
    P.diskInner = d.rIsco
    P.diskOuter = disk_outer
    return P, a_eff, q_eff


def make_params(derive, model, a_star, q, dPhi=0.012, max_steps=4000, allow_naked=False):
    """tests/test_main.cu:132-154: geometry-only test scene (disk off)."""
    P = RenderParams()
    apply_black_hole(P, model, a_star, q, derive, allow_naked)
    P.diskEnabled = 0
    P.dPhi, P.maxSteps = dPhi, max_steps
    test_camera(P, 0.6, 0.25, 16.0)
    return P


def scene(derive, model, a_star, q, width, height, dist, el_deg, fov_deg, az_deg=0.0,
          preset="balanced", disk=True, hot_spots=True, bloom=True, disk_time=0.0,
          exposure=1.0, ori_deg=(0.0, 0.0, 0.0), allow_naked=False):
    """A rendered frame as the application sets it up (main.cpp:376-478), accumMode 0."""
    P = RenderParams(width=width, height=height)
    apply_black_hole(P, model, a_star, q, derive, allow_naked)
    orbit_camera(P, math.radians(az_deg), math.radians(el_deg), dist, fov_deg,
                 tuple(math.radians(o) for o in ori_deg))
    P.dPhi, P.maxSteps = PRESETS[preset]
    P.diskEnabled = 1 if disk else 0
    P.hotSpotsEnabled = 1 if (hot_spots and disk) else 0
    P.hotSpotStrength = 0.65
    P.bloomEnabled = 1 if bloom else 0
    P.bloomStrength = 0.35
    P.diskTime = disk_time
    P.exposure = exposure
    P.sampleIndex, P.accumMode = 0, 0
    return P


# ---- the named workloads --------------------------------------------------

def schwarzschild_320(derive, width=320, height=180):
    """Schwarzschild, r = 15, elevation 15 deg, azimuth 0, FOV 60, balanced,
    disk on at t = 0, hot spots off, bloom off, exposure 1."""
    return scene(derive, BH_SCHWARZSCHILD, 0.0, 0.0, width, height, 15.0, 15.0, 60.0,
                 hot_spots=False, bloom=False)


def kerr_pair_1080(derive, width=1920, height=1080, frames=8):
    """Kerr a* = +0.9 and Kerr-Newman a* = -0.7 q = 0.4 at r = 20, inclination
    80 deg, FOV 45, disk + hot spots, bloom + tonemap, diskTime = k/(frames-1)."""
    out = []
    for model, a, q in ((BH_KERR, 0.9, 0.0), (BH_KERR_NEWMAN, -0.7, 0.4)):
        for k in range(frames):
            t = k / (frames - 1) if frames > 1 else 0.0
            out.append(scene(derive, model, a, q, width, height, 20.0, 10.0, 45.0, disk_time=t))
    return out


def kn_sweep_4k(derive, width=3840, height=2160, frames=120, frame_ids=None):
    """Kerr-Newman a* = 0.998 (the host clamp makes it 0.995) q = 0.05, r = 12,
    FOV 50, disk and bloom on, elevation swept 0 -> 89 deg over `frames`."""
    ids = range(frames) if frame_ids is None else frame_ids
    out = []
    for k in ids:
        el = 89.0 * k / (frames - 1) if frames > 1 else 0.0
        out.append(scene(derive, BH_KERR_NEWMAN, 0.998, 0.05, width, height, 12.0, el, 50.0,
                         disk_time=0.0))
    return out


def kn_orbit_4k(derive, width=3840, height=2160, frames=300, frame_ids=None):
    """Kerr-Newman a* = 0.8 q = 0.3 at r = 25, inclination 75 deg (elevation 15),
    FOV 45, disk + hot spots, bloom + tonemap, static disk (diskTime 0): frame k
    of the `frames`-frame orbit has camera azimuth 360 k / frames deg."""
    ids = range(frames) if frame_ids is None else frame_ids
    return [scene(derive, BH_KERR_NEWMAN, 0.8, 0.3, width, height, 25.0, 15.0, 45.0,
                  az_deg=360.0 * k / frames) for k in ids]


BATCH_RESOLUTIONS = ((128, 72), (320, 180), (640, 360), (1280, 720), (1920, 1080))


def batch_views(derive, n=256, seed=1234):
    """Random views for the batched launch: resolution uniform over
    BATCH_RESOLUTIONS, model uniform over the four families, a* U(-0.998, 0.998),
    q U(0, 0.6) rejected unless a*^2 + q^2 <= 0.98, camera r U(6, 60),
    inclination U(2, 88) deg, FOV U(30, 90) deg, disk on, hot spots on/off."""
    rng = np.random.default_rng(seed)
    views = []
    for _ in range(n):
        w, h = BATCH_RESOLUTIONS[rng.integers(len(BATCH_RESOLUTIONS))]
        model = int(rng.integers(4))
        while True:
            a = float(rng.uniform(-0.998, 0.998))
            q = float(rng.uniform(0.0, 0.6))
            if a * a + q * q <= 0.98:
                break
        if model in (BH_SCHWARZSCHILD, BH_REISSNER_NORDSTROM):
            a = 0.0
        if model in (BH_SCHWARZSCHILD, BH_KERR):
            q = 0.0
        r = float(rng.uniform(6.0, 60.0))
        inc = float(rng.uniform(2.0, 88.0))
        fov = float(rng.uniform(30.0, 90.0))
        hs = bool(rng.integers(2))
        views.append(scene(derive, model, a, q, int(w), int(h), r, 90.0 - inc, fov,
                           hot_spots=hs, bloom=True))
    return views
