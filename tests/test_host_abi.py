"""libbh.so on CPU: it loads without a GPU, exports every entry point that
include/*.h declares, keeps the reference's RenderParams layout, and its host
derivation / sanitising equals the reference's bit for bit."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import golden_data as G
from bhrt import lib
from bhrt.abi import RenderParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = []
    for h in sorted(os.listdir(INCLUDE)):
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof", "static_assert", "offsetof",
                            "alignof", "BH_DEFAULT"):
                names.append(name)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = lib.load()
    names = declared_functions()
    assert "launchRenderPipeline" in names and "launchRenderKernel" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert set(names) == set(lib.EXPORTED), "ctypes signatures must cover the header"


def test_exports_are_unmangled_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", lib.LIB_PATH], capture_output=True, text=True).stdout
    for n in declared_functions():
        assert re.search(rf"\bT {n}$", out, flags=re.M), n


def test_render_params_layout_in_c_and_cpp():
    prog = r"""
#include <stdio.h>
#include <stddef.h>
#include "bh_render_params.h"
int main(void){
  printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(RenderParams), offsetof(RenderParams, camPos),
         offsetof(RenderParams, model), offsetof(RenderParams, dPhi), offsetof(RenderParams, diskEnabled),
         offsetof(RenderParams, hotSpotsEnabled), offsetof(RenderParams, sampleIndex),
         offsetof(RenderParams, bloomStrength));
  return 0; }
"""
    want = [C.sizeof(RenderParams), RenderParams.camPos.offset, RenderParams.model.offset,
            RenderParams.dPhi.offset, RenderParams.diskEnabled.offset, RenderParams.hotSpotsEnabled.offset,
            RenderParams.sampleIndex.offset, RenderParams.bloomStrength.offset]
    assert want == [160, 12, 68, 100, 108, 132, 144, 156]   # the reference layout
    with tempfile.TemporaryDirectory() as d:
        for lang, comp in (("c", "gcc"), ("c++", "g++")):
            src = os.path.join(d, "t." + ("c" if lang == "c" else "cpp"))
            open(src, "w").write(prog)
            exe = os.path.join(d, "t_" + lang)
            subprocess.run(["/usr/bin/" + comp, "-I" + INCLUDE, "-I/usr/local/cuda/include", src, "-o", exe],
                           check=True)
            got = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
            assert got == want, lang


def test_defaults_match_reference_initialisers():
    P = RenderParams()
    assert (P.width, P.height, P.model, P.maxSteps, P.diskEnabled, P.bloomEnabled) == (1280, 720, 0, 2000, 1, 1)
    assert abs(P.dPhi - 0.012) < 1e-9 and abs(P.bloomStrength - 0.35) < 1e-7
    assert abs(P.diskEmisScale - 1.5) < 1e-7 and abs(P.diskAbsScale - 2.2) < 1e-6


def test_derive_matches_reference():
    g = G.load()
    for (model, M, a, q, naked), want in zip(g["derive_in"], g["derive_out"]):
        d, m, a2, q2 = lib.derive(int(model), float(M), float(a), float(q), bool(naked))
        got = np.array([d.a, d.Q, d.rPlus, d.rMinus, d.rPhoton, d.rErgo, d.rIsco, d.clamped, d.naked,
                        m, a2, q2], dtype=np.float64)
        assert G.same_bits(got.astype(np.float32), want.astype(np.float32)), (model, M, a, q, naked)


def test_sanitize_matches_reference():
    g = G.load()
    for raw, want, fixed in zip(g["sanitize_in"], g["sanitize_out"], g["sanitize_fixed"]):
        Q, f = lib.sanitize(G.params(raw))
        assert np.array_equal(np.frombuffer(bytes(Q), dtype=np.uint8), want)
        assert int(f) == int(fixed)


def test_sanitize_never_modifies_the_callers_struct():
    P = RenderParams(dPhi=0.0, maxSteps=0, model=42)
    before = bytes(P)
    Q, fixed = lib.sanitize(P)
    assert fixed and bytes(P) == before and Q.maxSteps >= 16 and 0 <= Q.model <= 3


@pytest.mark.parametrize("family,refill,blocks,ok", [(0, 4, 0, True), (1, 32, 3, True), (1, 0, 0, False),
                                                     (2, 8, 0, False), (0, 33, 0, False)])
def test_tuning_validation(family, refill, blocks, ok):
    before = [lib.get_tuning(0), lib.get_tuning(1)]
    if ok:
        lib.set_tuning(family, refill, blocks)
        assert lib.get_tuning(family) == (refill, blocks)
    else:
        with pytest.raises(ValueError):
            lib.set_tuning(family, refill, blocks)
    for fam, (r, b) in enumerate(before):
        lib.set_tuning(fam, r, b)
