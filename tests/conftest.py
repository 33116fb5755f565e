import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


def _built(*paths):
    return all(os.path.exists(os.path.join(ROOT, p)) for p in paths)


@pytest.fixture(scope="session", autouse=True)
def native_built():
    """Build the in-tree native artefacts once if they are missing."""
    if not _built("gfsm_b200/libgfsm.so", "gfsm_b200/GFSM", "gfsm_b200/libgfsm_synth.so"):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "gfsm_b200")], check=True)
    if not _built("oracle/liboracle.so"):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True)
    yield


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_ctx():
    """One device context for the GPU tests (limits from the environment)."""
    import gfsm_b200
    ctx = gfsm_b200.GFSM(device=0)
    yield ctx
    ctx.close()


@pytest.fixture(scope="session")
def gpu_ctx_vl():
    """Device context matching vertex labels."""
    import gfsm_b200
    ctx = gfsm_b200.GFSM(device=0, vertex_labels=1)
    yield ctx
    ctx.close()


@pytest.fixture(scope="session")
def host_ctx():
    """Host-only context: parsing and planning without a device."""
    import gfsm_b200
    ctx = gfsm_b200.GFSM(device=-1)
    yield ctx
    ctx.close()
