"""The C-ABI libraries load without a GPU and export every function that
include/*.h declares (no compute calls) -- CPU only."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header: str):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(ms[h]?_[A-Za-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.mark.parametrize("header", ["morphoshell_gpu.h", "morphoshell_host.h"])
def test_library_exports_every_declared_symbol(header):
    from morphoshell_b200 import LIB_PATH
    L = C.CDLL(LIB_PATH)
    names = declared_functions(header)
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_lists_match_headers():
    import morphoshell_b200 as m
    assert sorted(m.GPU_SYMBOLS) == declared_functions("morphoshell_gpu.h")
    assert sorted(m.HOST_SYMBOLS) == declared_functions("morphoshell_host.h")


def test_status_strings_and_no_device_error():
    from morphoshell_b200 import lib
    L = lib()
    assert L.ms_status_string(3) == b"implausibly_high_force"
    assert L.ms_status_string(0) == b"ok"


def test_cli_rejects_bad_arguments(tmp_path):
    import subprocess
    exe = os.path.join(ROOT, "morphoshell_b200", "lib", "morphoshell_gpu")
    r = subprocess.run([exe, "only_one_arg"], capture_output=True, text=True)
    assert r.returncode != 0
    assert "settings file path" in r.stderr
    r = subprocess.run([exe, str(tmp_path / "missing.txt"), str(tmp_path / "missing.vtk")], capture_output=True,
                       text=True)
    assert r.returncode != 0
    assert "settings file" in r.stderr
