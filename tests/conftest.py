"""Shared pytest fixtures: the package loader, the FP64 oracle and the GPU marker."""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def load_package():
    """Import ``irsounderlbl.jl_b200/`` (a folder name with a dot) as ``irs_b200``."""
    if "irs_b200" in sys.modules:
        return sys.modules["irs_b200"]
    d = ROOT / "irsounderlbl.jl_b200"
    spec = importlib.util.spec_from_file_location("irs_b200", d / "__init__.py",
                                                  submodule_search_locations=[str(d)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["irs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def oracle():
    import oracle as orc_mod
    return orc_mod.Oracle()


@pytest.fixture(scope="session")
def orc_mod():
    import oracle as orc_mod
    return orc_mod


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return {"wofz": np.load(ROOT / "tests" / "golden" / "wofz_grid.npz"),
            "xsec": np.load(ROOT / "tests" / "golden" / "xsec_fixtures.npz")}
