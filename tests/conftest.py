import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "l-norms_bruteforce_b200"
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT))


def load_package():
    """Import the package directory (its name has hyphens) as `lnorms_b200`."""
    if "lnorms_b200" in sys.modules:
        return sys.modules["lnorms_b200"]
    spec = importlib.util.spec_from_file_location("lnorms_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["lnorms_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def ld():
    return load_package()


@pytest.fixture(scope="session")
def workloads():
    load_package()
    import lnorms_b200.workloads as w
    return w
