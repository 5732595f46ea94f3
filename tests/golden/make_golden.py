"""Generate the golden fixtures of tests/golden from the reference's own sources.

    python tests/golden/make_golden.py        (needs the reference tree; see oracle/Makefile)

The reference repository ships no golden images or vectors, so they are made
here by running its own code: src/metric.cuh, src/trace.cuh and
src/post_process.cuh compiled unmodified as host C++ (oracle/_ref/libbhref_host.so,
built by `make -C oracle ref`), driven through the pixel loops of
oracle/ref_host.cpp.  Every fixture stores its inputs (RenderParams bytes,
derivation arguments) next to the outputs, so the tests need neither the
reference tree nor this script.

Fixtures (golden.npz):
  derive_*      bhValidateAndDerive over a grid of (model, M, a*, q, allowNaked)
  sanitize_*    sanitizeRenderParams over poisoned and random parameter blocks
  grid_<name>   the reference test probe (tests/test_main.cu:71-89) on 48x27
                rays of the test camera, plus the HDR shading of each ray
  pipe_<name>   launchRenderPipeline: RGBA8, accumulation and bloom buffers
  kern_<name>   launchRenderKernel: RGBA8

and (config1_schwarzschild_320x180.npz) the full 320x180 Schwarzschild frame
of the single-frame CPU workload (r = 15, elevation 15 deg, FOV 60, balanced,
disk on at t = 0, hot spots and bloom off): launchRenderPipeline's RGBA8 and,
per pixel, the reference probe record of the pixel's ray (outcome, class,
steps, escape direction, transmittance, HDR).
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "black-hole_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from bhrt import scenes  # noqa: E402
from bhrt.abi import BHDerived, RenderParams  # noqa: E402
import oracle as orc  # noqa: E402

GRID_NX, GRID_NY = 48, 27

GRID_CASES = [  # name, model, a*, q, disk, hot spots
    ("S", 0, 0.0, 0.0, False, False),
    ("RN5", 1, 0.0, 0.5, False, False),
    ("K9", 2, 0.9, 0.0, False, False),
    ("Km7", 2, -0.7, 0.0, False, False),
    ("KN75", 3, 0.7, 0.5, False, False),
    ("S_disk", 0, 0.0, 0.0, True, True),
    ("RN6_disk", 1, 0.0, 0.6, True, True),
    ("K9_disk", 2, 0.9, 0.0, True, True),
    ("KNm74_disk", 3, -0.7, 0.4, True, True),
    ("K12_naked", 2, 1.2, 0.0, False, False),
]


def params_bytes(P):
    return np.frombuffer(C.string_at(C.addressof(P), C.sizeof(P)), dtype=np.uint8).copy()


def derive_table(ref):
    rows_in, rows_out = [], []
    a_vals = [-5.0, -0.998, -0.9, -0.7, 0.0, 0.3, 0.6, 0.9, 0.998, 1.2, 5.0, float("nan")]
    q_vals = [-3.0, 0.0, 0.05, 0.3, 0.5, 0.6, 0.9, 2.0, float("nan")]
    for model in range(4):
        for a in a_vals:
            for q in q_vals:
                for naked in (0, 1):
                    for M in (0.5, 0.5, 1.0) if (a == 0.0 and q == 0.0) else (0.5,):
                        d, m, a2, q2 = ref.derive(model, M, a, q, naked)
                        rows_in.append((model, M, a, q, naked))
                        rows_out.append((d.a, d.Q, d.rPlus, d.rMinus, d.rPhoton, d.rErgo, d.rIsco,
                                         d.clamped, d.naked, m, a2, q2))
    for M in (float("nan"), -1.0, 0.0):
        d, m, a2, q2 = ref.derive(3, M, float("nan"), -3.0, 0)
        rows_in.append((3, M, float("nan"), -3.0, 0))
        rows_out.append((d.a, d.Q, d.rPlus, d.rMinus, d.rPhoton, d.rErgo, d.rIsco, d.clamped, d.naked,
                         m, a2, q2))
    return np.array(rows_in, dtype=np.float64), np.array(rows_out, dtype=np.float64)


def sanitize_cases(ref, derive):
    rng = np.random.default_rng(20241203)
    cases = []
    base = scenes.make_params(derive, 3, 0.7, 0.5)
    base.width, base.height = 160, 90
    nan = float("nan")
    bad = [("dPhi", 0.0), ("maxSteps", 0), ("camPos", (nan, nan, 0.0)), ("exposure", -5.0),
           ("model", 99), ("aSpin", 7.0), ("Qc", 9.0), ("rPlus", -1.0), ("sampleIndex", -7),
           ("accumMode", 99), ("bloomStrength", nan), ("width", 0), ("height", -3), ("M", nan),
           ("tanHalfFov", 100.0), ("aspect", nan), ("diskInner", 0.0), ("diskOuter", 0.0),
           ("hotSpotsEnabled", 7), ("maxSteps", 10 ** 7), ("dPhi", 1.0), ("camPos", (0.1, 0.0, 0.0))]
    for k, v in bad:
        P = base.copy()
        setattr(P, k, v)
        cases.append(P)
    P = base.copy()
    P.aSpin, P.Qc, P.rPlus = 7.0, 9.0, -1.0
    cases.append(P)
    fields = [f for f, _ in RenderParams._fields_]
    for _ in range(60):
        P = base.copy()
        for _k in range(int(rng.integers(1, 5))):
            f = fields[int(rng.integers(len(fields)))]
            cur = getattr(P, f)
            if isinstance(cur, int):
                setattr(P, f, int(rng.choice([-100, -1, 0, 1, 2, 3, 4, 5, 100000, 10 ** 7])))
            elif hasattr(cur, "x"):
                setattr(P, f, tuple(float(rng.choice([nan, -1e3, 0.0, 0.3, 5.0])) for _ in range(3)))
            else:
                setattr(P, f, float(rng.choice([nan, float("inf"), -1e6, -1.0, 0.0, 1e-5, 0.7, 3.0, 1e6])))
        cases.append(P)
    ins = np.stack([params_bytes(P) for P in cases])
    outs, fixed = [], []
    for P in cases:
        Q, f = ref.sanitize(P)
        outs.append(params_bytes(Q))
        fixed.append(int(f))
    return ins, np.stack(outs), np.array(fixed, dtype=np.int32)


def pipeline_scenes(derive):
    out = {}
    P = scenes.schwarzschild_320(derive, 160, 90)
    out["S320_160x90"] = P
    P = scenes.make_params(derive, 2, 0.9, 0.0)
    P.width, P.height = 96, 54
    P.diskEnabled, P.bloomEnabled, P.hotSpotsEnabled = 1, 1, 1
    P.hotSpotStrength, P.diskTime = 1.0, 1.25
    out["K9_spots_96x54"] = P
    P = scenes.kerr_pair_1080(derive, 96, 54, frames=8)[8 + 3]
    out["KNm74_cfg2_96x54"] = P
    P = scenes.kn_sweep_4k(derive, 96, 54, frames=120, frame_ids=[60])[0]
    out["KN995_sweep_96x54"] = P
    return out


def main():
    if not orc.RefHost.available():
        raise SystemExit("oracle/_ref/libbhref_host.so missing: run make -C oracle ref")
    ref = orc.RefHost()
    derive = ref.derive
    data = {}
    data["derive_in"], data["derive_out"] = derive_table(ref)
    data["sanitize_in"], data["sanitize_out"], data["sanitize_fixed"] = sanitize_cases(ref, derive)

    for name, model, a, q, disk, spots in GRID_CASES:
        P = scenes.make_params(derive, model, a, q, allow_naked=(name == "K12_naked"))
        P.diskEnabled = 1 if disk else 0
        P.hotSpotsEnabled = 1 if spots else 0
        data[f"grid_{name}_params"] = params_bytes(P)
        data[f"grid_{name}"] = ref.probe_grid(P, GRID_NX, GRID_NY).view(np.uint8)

    for name, P in pipeline_scenes(derive).items():
        out, acc, bA, bB = ref.pipeline(P)
        data[f"pipe_{name}_params"] = params_bytes(P)
        data[f"pipe_{name}_rgba"] = out
        data[f"pipe_{name}_accum"] = acc
        data[f"pipe_{name}_bloomA"] = bA
        data[f"pipe_{name}_bloomB"] = bB

    # progressive accumulation from a poisoned buffer (tests/test_main.cu:596-610)
    P = scenes.make_params(derive, 2, 0.9, 0.0)
    P.width, P.height, P.diskEnabled, P.bloomEnabled = 64, 36, 1, 1
    acc = np.full((36, 64, 4), np.nan, dtype=np.float32)
    seq = []
    for s in range(6):
        Ps = P.copy()
        Ps.sampleIndex, Ps.accumMode = s, (0 if s == 0 else (1 if s < 4 else 2))
        out, acc, _, _ = ref.pipeline(Ps, accum=acc)
        seq.append(params_bytes(Ps))
    data["accum_seq_params"] = np.stack(seq)
    data["accum_seq_rgba"] = out
    data["accum_seq_accum"] = acc

    P = scenes.make_params(derive, 3, 0.7, 0.5)
    P.width, P.height, P.diskEnabled = 64, 36, 1
    P.aSpin, P.Qc, P.rPlus = 7.0, 9.0, -1.0     # invalid a*/q (tests/test_main.cu:547)
    data["kern_badKN_params"] = params_bytes(P)
    data["kern_badKN_rgba"] = ref.render_kernel(P)
    P = scenes.kerr_pair_1080(derive, 64, 36, frames=2)[1]
    data["kern_K9_params"] = params_bytes(P)
    data["kern_K9_rgba"] = ref.render_kernel(P)

    path = os.path.join(HERE, "golden.npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB, {len(data)} arrays)")
    config1(ref, derive)


CONFIG1_FIELDS = ("outcome", "cls", "steps", "escDir", "trans", "hdr")


def config1(ref, derive):
    """The full 320x180 Schwarzschild frame: pipeline RGBA8 + per-pixel ray records.  For
    accumMode 0 the pixel's ray is the probe ray through the pixel centre, so the
    reference probe grid at W x H gives the frame's own rays."""
    P = scenes.schwarzschild_320(derive)
    out, acc, _, _ = ref.pipeline(P)
    rec = ref.probe_grid(P, P.width, P.height)
    # the probe's HDR is the frame's accumulation value (mode 0, one sample)
    assert np.array_equal(rec["hdr"], acc[..., :3])
    data = {"params": params_bytes(P), "rgba": out}
    for k in CONFIG1_FIELDS:
        v = rec[k]
        data[k] = v.astype(np.int8) if k in ("outcome", "cls") else v
    path = os.path.join(HERE, "config1_schwarzschild_320x180.npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB)")


if __name__ == "__main__":
    main()
