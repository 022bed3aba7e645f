import importlib.util
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _load_package():
    if "pssfss_b200" in sys.modules:
        return sys.modules["pssfss_b200"]
    pkgdir = os.path.join(ROOT, "pssfss.jl_b200")
    spec = importlib.util.spec_from_file_location(
        "pssfss_b200", os.path.join(pkgdir, "__init__.py"), submodule_search_locations=[pkgdir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pssfss_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def pkg():
    return _load_package()


_GOLDEN = None


def golden(key):
    """Golden values from the reference's own tests (tests/golden/reference_golden.json,
    made by tests/golden/extract_reference_golden.py): complex values and their record."""
    global _GOLDEN
    if _GOLDEN is None:
        with open(os.path.join(ROOT, "tests", "golden", "reference_golden.json")) as f:
            _GOLDEN = json.load(f)
    g = _GOLDEN[key]
    return [complex(re_, im) for re_, im in g.get("values", [])], g
