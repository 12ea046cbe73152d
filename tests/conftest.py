"""Test configuration: the `gpu` marker, the package loader, and the built
native libraries."""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "vlasov.jl_b200"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def load_package():
    """Import the package directory `vlasov.jl_b200` as module `vlasov_b200`."""
    if "vlasov_b200" in sys.modules:
        return sys.modules["vlasov_b200"]
    spec = importlib.util.spec_from_file_location("vlasov_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["vlasov_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def built():
    """Builds (if stale) the CUDA library and the oracle, once per session."""
    spec = importlib.util.spec_from_file_location("vlb_build", PKG_DIR / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    b.build_all()
    return b


@pytest.fixture(scope="session")
def vb(built):
    return load_package()


@pytest.fixture(scope="session")
def orc(built):
    from oracle import oracle
    return oracle


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    return 0
