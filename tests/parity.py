"""Parity metrics between two per-ray records or frames (GPU vs oracle).

Outcome class per ray: 0 captured, 1 disk hit (transmittance < 0.5), 2 escaped.
A ray is "on a class boundary" when the oracle's 3x3 pixel neighbourhood holds
more than one class; the class must match bit for bit everywhere else.
"""
import numpy as np


def boundary_mask(cls):
    """True where any pixel of the 3x3 neighbourhood (clamped) has another class."""
    c = np.asarray(cls)
    H, W = c.shape
    pad = np.pad(c, 1, mode="edge")
    m = np.zeros((H, W), dtype=bool)
    for dy in (0, 1, 2):
        for dx in (0, 1, 2):
            m |= pad[dy:dy + H, dx:dx + W] != c
    return m


def chord(a, b):
    """|a - b| of unit vectors = 2 sin(angle/2), the reference test's angle measure."""
    return np.sqrt(np.sum((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2, axis=-1))


def compare_rays(got, ref):
    """Statistics of a GPU record grid against the oracle's (2-D structured arrays)."""
    edge = boundary_mask(ref["cls"])
    inner = ~edge
    cls_bad = got["cls"] != ref["cls"]
    esc = (got["outcome"] == 1) & (ref["outcome"] == 1) & inner
    ang = chord(got["escDir"], ref["escDir"])[esc]
    h_got, h_ref = got["hdr"].astype(np.float64), ref["hdr"].astype(np.float64)
    rel = np.abs(h_got - h_ref) / np.maximum(np.abs(h_ref), 1e-3)
    rel_px = rel.max(axis=-1)
    return {
        "n": int(ref["cls"].size),
        "boundary_frac": float(edge.mean()),
        "cls_mismatch": int(cls_bad.sum()),
        "cls_mismatch_inner": int((cls_bad & inner).sum()),
        "outcome_mismatch_inner": int(((got["outcome"] != ref["outcome"]) & inner).sum()),
        "esc_n": int(esc.sum()),
        "esc_frac_1e4": float((ang <= 1e-4).mean()) if ang.size else 1.0,
        "esc_median": float(np.median(ang)) if ang.size else 0.0,
        "esc_max": float(ang.max()) if ang.size else 0.0,
        "hdr_frac_1e3": float((rel_px[inner] <= 1e-3).mean()),
        "hdr_frac_1e2": float((rel_px[inner] <= 1e-2).mean()),
        "steps_equal_frac": float((got["steps"] == ref["steps"]).mean()),
    }


def compare_rgba(got, ref):
    d = np.abs(got[..., :3].astype(np.int32) - ref[..., :3].astype(np.int32)).max(axis=-1)
    return {
        "n": int(d.size),
        "exact_frac": float((d == 0).mean()),
        "lsb1_frac": float((d <= 1).mean()),
        "max_diff": int(d.max()),
        "alpha_ok": bool(np.all(got[..., 3] == 255)),
    }
