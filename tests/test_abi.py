"""The C-ABI library loads and exports every symbol the public header declares (no GPU
calls), and the Python binding declares a signature for each of them."""
import os
import re

import pytest

from pssfss_b200 import _build, engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "pssfss_b200.h")).read()
    return sorted(set(re.findall(r"\b(pss_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header_symbols():
    _build.build()
    L = engine.lib()
    syms = header_symbols()
    assert len(syms) >= 12
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(engine.SIGNATURES)
    assert L.pss_version() >= 100


def test_no_device_error_is_reported_not_raised_in_c():
    # Without a GPU the context creation must fail cleanly with a message.
    import ctypes
    if os.environ.get("CUDA_VISIBLE_DEVICES") is None:
        try:
            import torch
            if torch.cuda.is_available():
                pytest.skip("a GPU is present")
        except Exception:
            pass
    h = ctypes.c_void_p()
    rc = engine.lib().pss_ctx_create(0, 1, ctypes.byref(h))
    assert rc != 0
    assert b"device" in engine.lib().pss_last_error().lower() or b"cuda" in engine.lib().pss_last_error().lower()
