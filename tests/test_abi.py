"""The C-ABI library loads and exports every entry point include/spt_b200.h
declares, and the ctypes structures match the C layout (CPU only: no
compute calls)."""

import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from conftest import REPO
from bem_b200 import _lib

HEADER = os.path.join(REPO, "include", "spt_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*int\s+(spt_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_expected_entry_points():
    names = declared_functions()
    assert set(names) == set(_lib.SIGNATURES), names


def test_library_loads_and_exports_every_symbol():
    lib = _lib.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.spt_abi_version() == _lib.ABI_VERSION == 4


STRUCTS = {
    "SptGeometry": _lib.SptGeometry,
    "SptBem": _lib.SptBem,
    "SptState": _lib.SptState,
    "SptTraceParams": _lib.SptTraceParams,
    "SptAccelArgs": _lib.SptAccelArgs,
    "SptGemmArgs": _lib.SptGemmArgs,
    "SptImage": _lib.SptImage,
}


def test_struct_layout_matches_c():
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "spt_b200.h"', "int main(void) {"]
    for name, cls in STRUCTS.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        r = subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), src, "-o", exe], capture_output=True, text=True)
        if r.returncode != 0:
            pytest.fail(r.stderr)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(l.split() for l in out if l.strip())
    for name, cls in STRUCTS.items():
        assert int(got[name]) == ctypes.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert int(got[f"{name}.{fname}"]) == getattr(cls, fname).offset, f"{name}.{fname}"


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_LIB", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(_lib.SptError):
        _lib.lib()
