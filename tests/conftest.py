import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "paulioperators.jl_b200"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libpauliprop.so")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def _ensure_built():
    """Build the oracle and the product library in-tree if a fresh checkout lacks them."""
    import subprocess
    lib = os.path.join(ROOT, "paulioperators.jl_b200", "lib", "libpauliprop.so")
    orc = os.path.join(ROOT, "oracle", "_build", "liborc.so")
    if not os.path.exists(orc):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "paulioperators.jl_b200")], check=True)


_ensure_built()
