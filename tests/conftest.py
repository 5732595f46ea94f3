"""Shared test set-up.

`-m "not gpu"`: the oracle against the reference's golden fixtures, the host
logic of libbh.so (parameter derivation and sanitising, ABI layout and
exports) and the multi-process plumbing, all on CPU.
`-m gpu`: parity of the CUDA tracer, called through the C-ABI, with the oracle.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "black-hole_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA tracer")


def _ensure_built():
    lib = os.path.join(ROOT, "black-hole_b200", "libbh.so")
    orc = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(orc):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all"], check=True)
    if not os.path.exists(lib):
        subprocess.run([sys.executable, os.path.join(ROOT, "black-hole_b200", "build.py")], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def derive():
    from bhrt import lib
    return lib.derive


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch
    torch.cuda.init()
    return torch.device("cuda:0")
