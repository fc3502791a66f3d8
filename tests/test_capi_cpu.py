"""CPU-only checks of the C-ABI library: it builds for sm_100a, loads, and
exports every entry point declared in include/elastica_b200.h; the host-side
argument checks answer without a GPU."""
import ctypes
import os
import re

import pytest

import elasticapp_b200 as eb
from elasticapp_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "elastica_b200.h"), encoding="utf-8") as f:
        text = f.read()
    return sorted(set(re.findall(r"EB_API\s+[^;(]*?\b(eb_\w+)\s*\(", text)))


def test_library_builds_and_loads():
    from elasticapp_b200 import build

    path = build.build()
    assert os.path.exists(path)
    lib = L.load()
    assert lib.eb_version().startswith(b"elastica_b200")


def test_every_declared_symbol_is_exported_and_bound():
    lib = L.load()
    syms = declared_symbols()
    assert len(syms) >= 20
    for name in syms:
        assert hasattr(lib, name), name
        assert name in L.SIGNATURES, f"{name} has no ctypes signature"


def test_null_arguments_are_rejected():
    lib = L.load()
    n = ctypes.c_int64()
    assert lib.eb_rod_count(None, ctypes.byref(n)) == 1  # EB_ERR_INVALID_ARGUMENT
    assert b"null" in lib.eb_last_error()
    assert lib.eb_sim_create(None, None) == 1
    assert lib.eb_sim_destroy(None) == 0


def test_unknown_precision_rejected_before_touching_cuda():
    lib = L.load()
    cfg = L.EbConfig()
    cfg.precision = 7
    h = ctypes.c_void_p()
    assert lib.eb_sim_create(ctypes.byref(cfg), ctypes.byref(h)) == 1


def test_no_device_reports_cuda_error_not_fallback():
    """Without a GPU the library must fail loudly (no CPU fallback)."""
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    with pytest.raises(L.EbError) as exc:
        eb.Simulator()
    assert exc.value.status == 5  # EB_ERR_CUDA
