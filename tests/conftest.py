import importlib
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (CUDA library calls)")
    config.addinivalue_line("markers", "slow: long-running CPU oracle work")


@pytest.fixture(scope="session")
def rtb():
    return importlib.import_module("2023_render_engine_b200")


@pytest.fixture(scope="session")
def core(rtb):
    return importlib.import_module("2023_render_engine_b200.core")


@pytest.fixture(scope="session")
def restated():
    from oracle import bindings

    if not bindings.RESTATE_SO.exists():
        bindings.build(ref=False)
    return bindings.Restated()


@pytest.fixture(scope="session")
def refo():
    """The reference's own code (prebuilt oracle/_ref library); skipped when absent."""
    from oracle import bindings

    if not bindings.REF_SO.exists():
        if bindings.reference_dir() is not None:
            bindings.build(ref=True)
        else:
            pytest.skip("reference harness library not built and REF_DIR does not name the reference tree")
    return bindings.RefOracle()


@pytest.fixture(scope="session")
def gpu_ctx(core):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return core.Context(0)
