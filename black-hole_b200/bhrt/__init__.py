"""bhrt -- host front end of the B200 null-geodesic tracer (libbh.so).

    from bhrt import lib, scenes, abi
    P = scenes.kerr_pair_1080(lib.derive)[0]
    from bhrt.device import Frame
    f = Frame(P.width, P.height); f.pipeline(P)

The tracer itself is CUDA (black-hole_b200/csrc) behind the C-ABI declared in
include/bh_launch.h; this package builds RenderParams, calls that ABI and
owns device buffers through torch.
"""
from . import abi, lib, scenes  # noqa: F401
from .abi import (BH_KERR, BH_KERR_NEWMAN, BH_PREC_FP32, BH_PREC_FP64, BH_PREC_MIXED,  # noqa: F401
                  BH_REISSNER_NORDSTROM, BH_SCHWARZSCHILD, PROBE_DTYPE, BHDerived, RenderParams)
