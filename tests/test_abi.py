"""The C-ABI library: it builds, loads without a GPU, exports every function that
include/*.h declares, and the ctypes signature table covers exactly those functions.
Also the host-side argument checks that need no device."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

from mertens_bound_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([a-z_][A-Za-z0-9_]*)\s*\(", src, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof"):
                names.add(name)
    return names


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_function(k2lib):
    decl = declared_functions()
    assert len(decl) >= 20
    exported = exported_symbols(_lib.LIB_PATH)
    missing = decl - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"


def test_ctypes_table_matches_header(k2lib):
    assert set(_lib.SIGNATURES) == declared_functions()
    for name in _lib.SIGNATURES:
        assert getattr(k2lib, name) is not None


def test_abi_version_and_error_channel(k2lib):
    assert k2lib.mb_abi_version() >= 1
    # argument errors are reported without touching a device
    out = C.c_void_p()
    assert k2lib.mb_table_create(None, None, None, None, 10, 0, C.byref(out)) == -1
    assert b"null array" in k2lib.mb_last_error()
    assert k2lib.mb_table_count_below(None, 1.0, None) == -1


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError):
        _lib.lib()
