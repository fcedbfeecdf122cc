import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA kernels through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    """liboracle.so (the checker) is built on demand; the reference harness
    (oracle/_ref) only where the reference tree exists."""
    so = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True,
                       capture_output=True)
    yield


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(os.path.join(GOLDEN, "trace_golden.npz")))


@pytest.fixture(scope="session")
def cornell_tris():
    from cudaraytracer_b200 import scenes

    return scenes.cornell_box().triangles()


@pytest.fixture(scope="session")
def ico_tris():
    from cudaraytracer_b200 import scenes

    return scenes.icosphere_field(with_env=False).triangles()


@pytest.fixture(scope="session")
def crt_ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cudaraytracer_b200 import Context

    ctx = Context(0)
    yield ctx
    ctx.close()
