"""CPU checks of the C ABI library: it loads, and exports every symbol the header declares.

No compute call is made here (there may be no GPU)."""
import ctypes
import re
from pathlib import Path

import pytest

from adamixture_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "adamixture_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(adx_\w+)\s*\(", text, re.M)))


def test_library_loads_and_exports_header_symbols():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), f"{n} declared in {HEADER.name} but not exported"
    assert set(names) == set(_lib.SIGNATURES), "ctypes signatures out of sync with the header"


def test_version_string():
    assert "sm_100a" in _lib.version()


def test_library_is_built_for_sm100a():
    # the fatbin only has sm_100a code: check with cuobjdump-free means, the ELF notes
    # are not inspected; the build flags are the contract (see csrc/build.py)
    from adamixture_b200.csrc import build

    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "nope.so")
    with pytest.raises(_lib.AdxError, match="missing"):
        _lib.load()


def test_argument_errors_are_reported_without_a_gpu():
    # invalid K is rejected before any CUDA call
    with pytest.raises(_lib.AdxError, match="invalid argument"):
        _lib.query_size("adx_em_workspace_bytes", 10, 10, 0, _lib.ADX_F32)
    with pytest.raises(_lib.AdxError, match="invalid argument"):
        _lib.query_size("adx_em_workspace_bytes", 10, 10, 65, _lib.ADX_F32)
    assert _lib.query_size("adx_em_workspace_bytes", 1000, 100, 7, _lib.ADX_F64) > 0
    assert isinstance(ctypes.c_int(0).value, int)
