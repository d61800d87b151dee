"""The C-ABI library loads without a GPU and exports every entry point that
include/kynema_b200.h declares (no compute call is made)."""
import ctypes
import os
import re

from openturbine_b200 import build as kbuild

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "kynema_b200.h")


def declared_symbols() -> list[str]:
    text = open(HEADER).read()
    return sorted(set(re.findall(r"KYN_API\s+[\w\s\*]+?\b(kyn_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "kyn_step" in names and "kyn_model_create" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(kbuild.build())
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_no_device_is_an_error_not_a_fallback():
    """Without a GPU the context cannot be created: there is no CPU path."""
    import torch
    if torch.cuda.is_available():
        return
    lib = ctypes.CDLL(kbuild.build())
    lib.kyn_ctx_create.restype = ctypes.c_void_p
    lib.kyn_ctx_create.argtypes = [ctypes.c_int, ctypes.c_size_t]
    assert not lib.kyn_ctx_create(0, 0)
