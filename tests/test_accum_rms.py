"""Progressive accumulation: an 8-sample running mean (accumMode 1, R2 sub-pixel
jitter) has a lower full-image RMS error against a 64-sample accumulation than
the single centred sample.  The reference's README reports 1.78x for this
comparison (README.md:266-268); the sample sequence is the application's
(src/main.cpp:473-478: sample 0 overwrites with accumMode 0, samples k >= 1
blend with accumMode 1 and sampleIndex k).

Error measure: RMS over all pixels and the three colour channels of the
tonemapped RGBA8 image (bloom off, so each pixel depends on its own samples).
The gain depends on how much of the image is silhouette edge: measured on the
oracle 1.38-1.56 for Schwarzschild and 1.58-1.74 for Kerr a* = 0.9 (r = 20,
inclination 80 deg, FOV 45 deg) at 96x54 and 192x108; the bar is 1.3.
"""
import numpy as np
import pytest

from bhrt import scenes


def _scene(derive, model, w, h):
    a = 0.9 if model >= 2 else 0.0
    P = scenes.scene(derive, model, a, 0.0, w, h, 20.0, 10.0, 45.0, hot_spots=True, bloom=False)
    return P


def _progressive(render, P, counts=(1, 8, 64)):
    """render(P) -> RGBA8 after blending sample P.sampleIndex; images after `counts` samples."""
    out = {}
    for k in range(max(counts)):
        Q = P.copy()
        Q.sampleIndex, Q.accumMode = k, (0 if k == 0 else 1)
        img = render(Q)
        if k + 1 in counts:
            out[k + 1] = img[..., :3].astype(np.float64)
    return out


def _ratio(imgs):
    rms = lambda a: float(np.sqrt(np.mean((a - imgs[64]) ** 2)))
    return rms(imgs[1]) / rms(imgs[8]), rms(imgs[1]), rms(imgs[8])


def _oracle_progressive(oracle, P):
    state = {"acc": None}

    def render(Q):
        out, acc, _, _ = oracle.pipeline(Q, state["acc"])
        state["acc"] = acc
        return out
    return _progressive(render, P)


@pytest.mark.parametrize("model", [0, 2])
def test_oracle_eight_samples_beat_one(oracle, derive, model):
    P = _scene(derive, model, 96, 54)
    ratio, r1, r8 = _ratio(_oracle_progressive(oracle, P))
    print(f"model {model}: RMS 1 spp {r1:.3f}, 8 spp {r8:.3f}, ratio {ratio:.2f}")
    assert ratio >= 1.3


@pytest.mark.gpu
@pytest.mark.parametrize("model", [0, 2])
def test_gpu_accumulation_rms_matches_oracle_and_gains(cuda, oracle, derive, model):
    import torch
    from bhrt.device import Frame

    def gpu_run(P):
        f = Frame(P.width, P.height)

        def render(Q):
            f.pipeline(Q)
            torch.cuda.synchronize()
            return f.out.cpu().numpy()
        return _progressive(render, P)

    small = _scene(derive, model, 96, 54)
    g_ratio = _ratio(gpu_run(small))[0]
    o_ratio = _ratio(_oracle_progressive(oracle, small))[0]
    big = _scene(derive, model, 640, 360)
    b_ratio, r1, r8 = _ratio(gpu_run(big))
    print(f"model {model}: 96x54 gpu {g_ratio:.3f} oracle {o_ratio:.3f}; 640x360 RMS 1 spp {r1:.3f} "
          f"8 spp {r8:.3f} ratio {b_ratio:.2f}")
    assert abs(g_ratio - o_ratio) <= 0.03 * o_ratio
    assert b_ratio >= 1.3
