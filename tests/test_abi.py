"""The drop-in boundary, checked without a GPU: libmublis.so loads and
exports every function and object that include/*.h declares, and the
library refuses to work (nonzero status, no fallback) when no B200 is
present."""
import ctypes
import re
from pathlib import Path

import pytest

import mublis_b200 as mb

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"#define[^\n]*(\\\n[^\n]*)*", "", text)
        for m in re.finditer(r"\b((?:cblas|mublis)_\w+)\s*\(", text):
            names.add(m.group(1))
        for m in re.finditer(r"REGISTER_TARGET_CONTEXT\((\w+)\)", h.read_text()):
            if m.group(1) != "name":
                names.add(m.group(1))
    return sorted(names)


def test_header_surface_is_complete():
    names = declared_symbols()
    for p in "sd":
        for r in ("gemm", "symm", "syrk", "syr2k", "trmm", "trsm"):
            assert f"cblas_{p}{r}" in names
            assert f"mublis_{p}{r}" in names
        assert f"mublis_l3_{p}driver" in names
    assert "cblas_xerbla" in names and "mublis_get_context" in names
    assert "b200_context" in names


@pytest.mark.parametrize("name", declared_symbols())
def test_library_exports(name):
    lib = ctypes.CDLL(str(mb.LIB_PATH))
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_declared_signatures_bind():
    lib = mb.load()
    assert lib.cblas_sgemm.restype is None
    assert lib.mublis_dtrsm.restype is ctypes.c_int


def test_no_silent_fallback_without_gpu():
    """With no CUDA device the library reports failure instead of computing
    on the CPU."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    lib = mb.load()
    assert lib.mublis_b200_init() != 0
    a = (ctypes.c_float * 4)(1, 2, 3, 4)
    c = (ctypes.c_float * 4)(0, 0, 0, 0)
    st = lib.mublis_sgemm(0, 0, 2, 2, 2, 1.0, a, 1, 2, a, 1, 2, 0.0, c, 1, 2)
    assert st != 0
    assert list(c) == [0, 0, 0, 0]
    assert "device" in mb.last_error(lib).lower() or "cuda" in mb.last_error(lib).lower()
    ctx = ctypes.create_string_buffer(256)
    assert lib.mublis_get_context(ctx) != 0
