"""The C ABI library loads and exports every function include/*.h declares (no GPU needed)."""

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from tractography_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(tg_[a-z_0-9]+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_the_abi():
    names = declared_functions()
    assert "tg_tractogram" in names and "tg_tracker_run" in names
    assert names == set(_lib.EXPORTS)


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.tg_abi_version() == 1
    assert lib.tg_status_string(0) == b"ok"
    assert lib.tg_status_string(5) == b"point pool exhausted"


def test_exports_are_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert declared_functions() <= exported


def test_invalid_arguments_fail_without_a_device():
    lib = _lib.load()
    out = ctypes.c_void_p()
    # null values are rejected before any CUDA call
    status = lib.tg_field_create(0, None, 1, 1, 1, 1, None, None, ctypes.byref(out))
    assert status == _lib.TG_ERR_INVALID_ARGUMENT
    assert b"null" in lib.tg_last_error()
    with pytest.raises(ValueError):
        _lib.check(status)


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    """No CPU fallback: without libtg_b200.so the package raises instead of tracking on the host."""
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "absent.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="not built"):
        _lib.load()
