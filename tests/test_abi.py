"""The C-ABI library loads and exports every symbol include/hplb.h declares
(no compute call: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "hplb.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hplb_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    from rochpl_b200.lib import EXPORTS

    assert sorted(EXPORTS) == declared_symbols()


def test_library_exports_every_declared_symbol():
    from rochpl_b200 import build as B

    if not os.path.exists(B.LIB):
        B.build()
    lib = ctypes.CDLL(B.LIB)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_host_only_entry_points():
    from rochpl_b200.lib import load

    L = load()
    assert L.hplb_default_ld(4096) == 4128
    assert L.hplb_default_ld(131072) == 131104
    assert L.hplb_default_ld(0) == 32 and L.hplb_default_ld(33) == 160
    assert L.hplb_status_string(4) == b"device wait timed out"


def test_create_fails_cleanly_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from rochpl_b200.lib import HplError, Library

    with pytest.raises(HplError):
        Library(0)
