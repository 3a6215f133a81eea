"""The C ABI library loads without a GPU and exports every entry point that
include/magtense_b200.h declares (no compute calls here)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "magtense_b200.h"


def declared_functions():
    src = HEADER.read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\s*\*)\s+(\w+)\s*\(", src, flags=re.M)))


@pytest.fixture(scope="module")
def built_lib():
    from magtense_b200 import _lib
    if not _lib.LIB_PATH.exists():
        _lib.build()
    return _lib


def test_header_declares_the_reference_shims():
    names = declared_functions()
    for ref in ("icl_initDemagMatrices", "icl_MVMult_GetH", "icl_destroy", "icl_initDemagMatrices_sparse",
                "icl_MVMult_GetH_sparse"):
        assert ref in names
    assert "mt_integrate" in names and "mt_rhs" in names and "mt_assemble_demag" in names


def test_library_exports_every_declared_symbol(built_lib):
    lib = ctypes.CDLL(str(built_lib.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header(built_lib):
    assert set(declared_functions()) <= set(built_lib.SIGNATURES)


def test_build_targets_sm100a_only():
    mk = (ROOT / "magtense_b200" / "csrc" / "Makefile").read_text()
    assert "arch=compute_100a,code=sm_100a" in mk
    assert "sm_90" not in mk and "compute_90" not in mk


def test_version_string_without_device(built_lib):
    assert b"sm_100a" in built_lib.lib().mt_version()
