"""The CPU oracle is pinned to the reference: bit-exact against fixtures made by
running the reference's own sources (tests/golden/make_golden.py)."""
import numpy as np
import pytest

import golden_data as G


def test_derive_matches_reference(oracle):
    g = G.load()
    for (model, M, a, q, naked), want in zip(g["derive_in"], g["derive_out"]):
        d, m, a2, q2 = oracle.derive(int(model), float(M), float(a), float(q), bool(naked))
        got = np.array([d.a, d.Q, d.rPlus, d.rMinus, d.rPhoton, d.rErgo, d.rIsco, d.clamped, d.naked,
                        m, a2, q2], dtype=np.float64)
        assert G.same_bits(got.astype(np.float32), want.astype(np.float32)), (model, M, a, q, naked)


def test_sanitize_matches_reference(oracle):
    g = G.load()
    for raw, want, fixed in zip(g["sanitize_in"], g["sanitize_out"], g["sanitize_fixed"]):
        Q, f = oracle.sanitize(G.params(raw))
        got = np.frombuffer(bytes(Q), dtype=np.uint8)
        assert np.array_equal(got, want)
        assert int(f) == int(fixed)


@pytest.mark.parametrize("name", G.GRID_NAMES)
def test_probe_grid_bit_exact(oracle, name):
    P, want = G.grid(name)
    got = oracle.probe_grid(P, G.GRID_NX, G.GRID_NY)
    for f in G.REF_FIELDS:
        assert G.same_bits(got[f], want[f]), f"{name}: field {f} differs"


@pytest.mark.parametrize("name", G.PIPE_NAMES)
def test_pipeline_bit_exact(oracle, name):
    g = G.load()
    P = G.params(g[f"pipe_{name}_params"])
    out, acc, bA, bB = oracle.pipeline(P)
    assert np.array_equal(out, g[f"pipe_{name}_rgba"])
    assert G.same_bits(acc, g[f"pipe_{name}_accum"])
    if P.bloomEnabled:
        assert G.same_bits(bB, g[f"pipe_{name}_bloomB"])
        assert G.same_bits(bA, g[f"pipe_{name}_bloomA"])


def test_config1_full_frame_bit_exact(oracle):
    """The full 320x180 Schwarzschild frame: RGBA8 and every pixel's ray record."""
    z = np.load(G.PATH.replace("golden.npz", "config1_schwarzschild_320x180.npz"))
    P = G.params(z["params"])
    out, acc, _, _ = oracle.pipeline(P)
    assert np.array_equal(out, z["rgba"])
    rec = oracle.probe_grid(P, P.width, P.height)
    for f in ("outcome", "cls", "steps", "escDir", "trans", "hdr"):
        assert G.same_bits(rec[f].astype(z[f].dtype), z[f]), f
    assert G.same_bits(acc[..., :3], z["hdr"])


def test_progressive_accumulation_bit_exact(oracle):
    g = G.load()
    acc = np.full((36, 64, 4), np.nan, dtype=np.float32)
    for raw in g["accum_seq_params"]:
        out, acc, _, _ = oracle.pipeline(G.params(raw), accum=acc)
    assert np.array_equal(out, g["accum_seq_rgba"])
    assert G.same_bits(acc, g["accum_seq_accum"])
    assert np.all(out[..., 3] == 255)


@pytest.mark.parametrize("name", ["badKN", "K9"])
def test_render_kernel_bit_exact(oracle, name):
    g = G.load()
    out = oracle.render_kernel(G.params(g[f"kern_{name}_params"]))
    assert np.array_equal(out, g[f"kern_{name}_rgba"])
