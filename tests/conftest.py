"""Shared test set-up.

* registers the ``gpu`` marker (tests that need a B200; run with ``-m gpu``);
* imports the package directory ``volcano-ash3d_b200`` as ``volcano_ash3d_b200``
  and the oracle (test infrastructure) from ``oracle/``.
"""
import importlib.util
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _load_pkg():
    if "volcano_ash3d_b200" in sys.modules:
        return sys.modules["volcano_ash3d_b200"]
    d = ROOT / "volcano-ash3d_b200"
    spec = importlib.util.spec_from_file_location("volcano_ash3d_b200", d / "__init__.py",
                                                  submodule_search_locations=[str(d)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["volcano_ash3d_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_pkg()
if str(ROOT / "oracle") not in sys.path:
    sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def pkg():
    return _load_pkg()


@pytest.fixture(scope="session")
def oracle_mod():
    import ash3d_oracle as orc
    orc.build()
    return orc
