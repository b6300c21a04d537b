"""The C ABI boundary: the library loads, exports every symbol include/fwi3d.h
declares, and fails loudly (no CPU fallback) when no GPU is present."""
import ctypes as C
import re
from pathlib import Path

import pytest

from conftest import HAS_GPU, ROOT
from fwi3d_b200 import lib

HEADER = ROOT / "include" / "fwi3d.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fwi_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    so = lib.load()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, f"missing exports: {missing}"


def test_binding_covers_the_header():
    assert set(declared_functions()) == set(lib.SIGNATURES)


def test_binding_constants_match_the_header():
    """FWI_FLAG_*, FWI_BOUNDARY_* and the status codes have the header's values
    in the Python binding."""
    text = HEADER.read_text()
    macros = {k: int(v, 0) for k, v in re.findall(r"#define\s+(FWI_[A-Z0-9_]+)\s+(0x[0-9a-fA-F]+|\d+)", text)}
    for name, value in macros.items():
        if name.startswith(("FWI_FLAG_", "FWI_BOUNDARY_")):
            assert getattr(lib, name[len("FWI_"):]) == value, name
        if name.startswith("FWI_ERR_") or name == "FWI_OK":
            assert value == 0 or value in lib.STATUS_NAMES, name
    flags = [v for k, v in macros.items() if k.startswith("FWI_FLAG_")]
    assert len(flags) == 3 and len(set(flags)) == 3 and all(f & (f - 1) == 0 for f in flags)


def test_status_strings():
    so = lib.load()
    assert so.fwi_status_string(0) == b"ok"
    assert so.fwi_status_string(8) == b"no CUDA device"


def test_tile_table_is_valid():
    for tz, tx in lib.tile_table():
        assert tz % 4 == 0 and (tz + 8) * 4 % 16 == 0 and tz + 8 <= 256 and tx + 8 <= 256


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device path")
def test_create_without_gpu_fails_loudly():
    with pytest.raises(lib.FwiError) as e:
        lib.Context(20, 20, 20, 4, 10.0, 10, 1e-3, 30.0)
    assert e.value.code == 8


def test_null_arguments_are_rejected():
    so = lib.load()
    assert so.fwi_create(None, None, None) == 1
    assert so.fwi_destroy(None) == 1
