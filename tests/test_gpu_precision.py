"""Precision modes of the CUDA tracer against FP64 oracles.

* FP32 and MIXED (FP32 steps; FP64 initial data, FP64 steps at radial turning
  points and on horizon approach, FP64 bisection of the equatorial crossing)
  are compared with the all-FP64 GPU integration on the Kerr-Newman
  a* = 0.998 (0.995 after the host clamp), q = 0.05 scene at r = 12 rs,
  FOV 50 deg, over the elevation sweep 0 -> 89 deg;
* the GPU integrations are compared with the CPU FP64 small-step oracle
  (dPhi / 16, 16x the step budget), and the conserved-quantity drift (Carter
  constant, null Hamiltonian, Binet first integral) is checked to shrink with
  precision;
* the disk-hit radius (first equatorial crossing inside the disk) matches the
  oracle's.
"""
import numpy as np
import pytest

import golden_data as G
import parity
from bhrt import lib, scenes
from bhrt.abi import BH_PREC_FP32, BH_PREC_FP64, BH_PREC_MIXED

pytestmark = pytest.mark.gpu
NX, NY = 160, 90


def _probe(P, prec, nx=NX, ny=NY):
    from bhrt import device
    return device.probe_grid(P, nx, ny, prec)


def _sweep_scene(el):
    P = scenes.kn_sweep_4k(lib.derive, NX, NY, frames=90, frame_ids=[0])[0]
    return scenes.orbit_camera(P, 0.0, np.radians(el), 12.0, 50.0)


def _errors(got, ref):
    edge = parity.boundary_mask(ref["cls"])
    esc = (got["outcome"] == 1) & (ref["outcome"] == 1) & ~edge
    ang = parity.chord(got["escDir"], ref["escDir"])[esc]
    return {"cls_all": int((got["cls"] != ref["cls"]).sum()),
            "cls_inner": int(((got["cls"] != ref["cls"]) & ~edge).sum()),
            "esc_med": float(np.median(ang)) if ang.size else 0.0,
            "esc_p99": float(np.quantile(ang, 0.99)) if ang.size else 0.0,
            "esc_1e4": float((ang <= 1e-4).mean()) if ang.size else 1.0}


@pytest.mark.parametrize("el", [0.0, 30.0, 60.0, 85.0, 89.0])
def test_mixed_and_fp32_against_fp64_on_the_4k_sweep_scene(cuda, el):
    P = _sweep_scene(el)
    ref = _probe(P, BH_PREC_FP64)
    e32 = _errors(_probe(P, BH_PREC_FP32), ref)
    emx = _errors(_probe(P, BH_PREC_MIXED), ref)
    print(f"el={el}: fp32 {e32}  mixed {emx}")
    for e in (e32, emx):
        assert e["cls_inner"] <= max(2, int(0.001 * NX * NY)), e
    # Within a few degrees of the spin axis the reference's FP32 set-up itself is
    # ill-conditioned (theta0 = acos(y / r) loses ~1e-5 rad), so plain FP32
    # may leave up to 2 % of escape directions beyond 1e-4 rad there; the mixed
    # mode, with its FP64 set-up, must meet the 1e-4 rad bar everywhere.
    assert e32["esc_1e4"] >= (0.99 if el < 80 else 0.98), e32
    assert emx["esc_1e4"] >= 0.99, emx
    # mixed precision is at least as close to the FP64 integration as plain FP32
    assert emx["esc_med"] <= e32["esc_med"] * 1.05 + 1e-9
    assert emx["cls_all"] <= e32["cls_all"] + 2


@pytest.mark.parametrize("name", ["K9_disk", "KNm74_disk", "S_disk"])
def test_fp32_and_fp64_against_small_step_fp64_oracle(cuda, oracle, name):
    """Errors against the FP64 small-step oracle (dPhi/16, 16x budget) and drift."""
    P, _ = G.grid(name)
    small = oracle.probe_grid(P, G.GRID_NX, G.GRID_NY, precision=2, step_div=16)
    g32 = _probe(P, BH_PREC_FP32, G.GRID_NX, G.GRID_NY)
    g64 = _probe(P, BH_PREC_FP64, G.GRID_NX, G.GRID_NY)
    e32, e64 = _errors(g32, small), _errors(g64, small)
    esc32 = g32["outcome"] == 1
    d32, d64 = float(np.median(g32["drift"][esc32])), float(np.median(g64["drift"][esc32]))
    print(f"{name}: fp32 vs small-step {e32}, fp64 vs small-step {e64}, drift fp32 {d32:.3g} fp64 {d64:.3g}")
    # the step-size (truncation) error dominates both: same method, similar error
    assert e32["esc_med"] < 2e-3 and e64["esc_med"] < 2e-3
    assert abs(e32["esc_med"] - e64["esc_med"]) <= 0.1 * e64["esc_med"] + 1e-6
    # conserved quantities: FP64 integration drifts no more than FP32
    assert d64 <= d32 * 1.05 + 1e-12
    if P.model in (2, 3):
        assert float(np.median(g32["maxHviol"])) < 5e-3


@pytest.mark.parametrize("name", ["K9_disk", "KNm74_disk", "S_disk", "RN6_disk"])
def test_disk_hit_radius_matches_oracle(cuda, oracle, name):
    P, _ = G.grid(name)
    want = oracle.probe_grid(P, G.GRID_NX, G.GRID_NY)
    edge = parity.boundary_mask(want["cls"])
    for prec in (BH_PREC_FP32, BH_PREC_MIXED):
        got = _probe(P, prec, G.GRID_NX, G.GRID_NY)
        both = (got["diskR"] > 0) & (want["diskR"] > 0) & ~edge
        only = ((got["diskR"] > 0) != (want["diskR"] > 0)) & ~edge
        rel = np.abs(got["diskR"][both] - want["diskR"][both]) / want["diskR"][both]
        print(name, prec, "hits", int(both.sum()), "presence mismatch", int(only.sum()),
              "max rel", float(rel.max()) if rel.size else 0.0)
        assert both.sum() > 20
        assert only.sum() <= max(1, int(0.01 * both.sum()))
        assert float(np.quantile(rel, 0.99)) < 1e-3
        grel = np.abs(got["diskG"][both] - want["diskG"][both]) / want["diskG"][both]
        assert float(np.quantile(grel, 0.99)) < 1e-3
