"""CPU-side checks of the C-ABI boundary: the library loads and exports every
entry point ``include/fvx.h`` declares (no compute calls: no GPU here)."""

import ctypes
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "fvx.h"
LIB = ROOT / "finitevolx_b200" / "libfvx.so"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(?:int|long long)\s+(fvx_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not LIB.exists():
        from finitevolx_b200.build import build
        build()
    return ctypes.CDLL(str(LIB))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert len(syms) >= 20
    assert "fvx_advect2d_f32" in syms and "fvx_mask2d_build" in syms


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"declared but not exported: {missing}"


def test_library_is_sm100a(lib):
    # the fatbin must carry sm_100a code (cuobjdump is not used: read the ELF
    # note of the embedded arch name that nvcc writes into the host object)
    data = LIB.read_bytes()
    assert b"sm_100a" in data


def test_python_package_imports_without_gpu():
    import finitevolx_b200 as fvx  # noqa: F401
    assert hasattr(fvx, "Advection2D") and hasattr(fvx, "Mask2D")
