"""Host-side scene construction and headless image output (no GPU)."""
import math
import os
import struct
import tempfile
import zlib

import numpy as np

from bhrt import lib, scenes
from bhrt.abi import BH_KERR, BH_KERR_NEWMAN, BH_REISSNER_NORDSTROM, BH_SCHWARZSCHILD
from bhrt.imageio import read_ppm, write_png, write_ppm


def _vec(v):
    return np.array(v.tolist(), dtype=np.float64)


def test_orbit_camera_is_orthonormal_and_looks_at_the_hole():
    for ori in ((0, 0, 0), (10, 20, 30), (-45, 5, 90)):
        P = scenes.scene(lib.derive, BH_KERR, 0.9, 0.0, 640, 360, 20.0, 10.0, 45.0, ori_deg=ori)
        f, r, u, p = _vec(P.camForward), _vec(P.camRight), _vec(P.camUp), _vec(P.camPos)
        for v in (f, r, u):
            assert abs(np.linalg.norm(v) - 1.0) < 1e-6
        assert abs(f @ r) < 1e-6 and abs(f @ u) < 1e-6 and abs(r @ u) < 1e-5
        assert np.allclose(-p / np.linalg.norm(p), f, atol=1e-6)       # looks at the origin
        assert abs(np.linalg.norm(p) - 20.0) < 1e-4
    P = scenes.scene(lib.derive, BH_KERR, 0.9, 0.0, 640, 360, 20.0, 10.0, 45.0)
    assert abs(P.camPos.y - 20.0 * math.sin(math.radians(10.0))) < 1e-5       # elevation = 90 - inclination
    assert abs(P.tanHalfFov - math.tan(math.radians(22.5))) < 1e-6 and abs(P.aspect - 640 / 360) < 1e-6


def test_named_workloads():
    fr = scenes.kerr_pair_1080(lib.derive)
    assert len(fr) == 16 and fr[0].model == BH_KERR and fr[8].model == BH_KERR_NEWMAN
    assert [round(P.diskTime, 6) for P in fr[:8]] == [round(k / 7, 6) for k in range(8)]
    assert all(P.bloomEnabled and P.hotSpotsEnabled and P.diskEnabled for P in fr)
    kn = scenes.kn_sweep_4k(lib.derive, frame_ids=[0, 119])
    assert abs(kn[0].aSpin / kn[0].M - 0.995) < 1e-6          # a* = 0.998 clamped by the host derivation
    assert abs(kn[1].camPos.y / 12.0 - math.sin(math.radians(89.0))) < 1e-5
    s = scenes.schwarzschild_320(lib.derive)
    assert (s.width, s.height, s.model, s.bloomEnabled, s.hotSpotsEnabled) == (320, 180, BH_SCHWARZSCHILD, 0, 0)


def test_batch_views_distribution():
    v = scenes.batch_views(lib.derive, 256, seed=1234)
    assert len(v) == 256
    assert {(P.width, P.height) for P in v} <= set(scenes.BATCH_RESOLUTIONS)
    assert {P.model for P in v} == {0, 1, 2, 3}
    for P in v:
        r = math.sqrt(P.camPos.x ** 2 + P.camPos.y ** 2 + P.camPos.z ** 2)
        assert 6.0 - 1e-4 <= r <= 60.0 + 1e-4
        a, q = P.aSpin / P.M, P.Qc / P.M
        assert a * a + q * q <= 0.98 + 1e-4
        if P.model in (BH_SCHWARZSCHILD, BH_REISSNER_NORDSTROM):
            assert P.aSpin == 0.0
    again = scenes.batch_views(lib.derive, 256, seed=1234)
    assert all(bytes(a) == bytes(b) for a, b in zip(v, again))


def test_ppm_and_png_round_trip():
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, size=(37, 53, 4), dtype=np.uint8)
    img[..., 3] = 255
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "a.ppm")
        write_ppm(p, img)
        assert np.array_equal(read_ppm(p), img[..., :3])
        q = os.path.join(d, "a.png")
        write_png(q, img)
        data = open(q, "rb").read()
        assert data[:8] == b"\x89PNG\r\n\x1a\n"
        w, h = struct.unpack(">II", data[16:24])
        assert (w, h) == (53, 37)
        i = data.index(b"IDAT")
        n = struct.unpack(">I", data[i - 4:i])[0]
        raw = zlib.decompress(data[i + 4:i + 4 + n])
        rows = np.frombuffer(raw, dtype=np.uint8).reshape(37, 1 + 53 * 4)
        assert np.all(rows[:, 0] == 0) and np.array_equal(rows[:, 1:].reshape(37, 53, 4), img)
