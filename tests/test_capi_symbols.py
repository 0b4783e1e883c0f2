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


def test_headers_compile_as_c_and_cpp_and_ms_check_throws(tmp_path):
    """Both headers compile as C11; in C++ the header's ms_check turns a guard
    trip into the reference's "implausibly_high_force" and other codes into
    their status names (no handle)."""
    import shutil
    import subprocess
    if not shutil.which("g++") or not shutil.which("gcc"):
        pytest.skip("no host compiler")
    from morphoshell_b200 import LIB_PATH
    inc = os.path.join(ROOT, "include")
    c = tmp_path / "h.c"
    c.write_text('#include "morphoshell_gpu.h"\n#include "morphoshell_host.h"\nint main(void) { return 0; }\n')
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-fsyntax-only", "-I", inc, str(c)], check=True)
    cpp = tmp_path / "h.cpp"
    cpp.write_text(
        '#include "morphoshell_gpu.h"\n#include <cstdio>\n'
        "int main() {\n"
        "  const int codes[2] = {MS_ERR_IMPLAUSIBLE_FORCE, MS_ERR_INVALID_ARGUMENT};\n"
        "  for (int rc : codes) {\n"
        '    try { ms_check(rc, nullptr); std::puts("no throw"); }\n'
        '    catch (const std::runtime_error& e) { std::puts(e.what()); }\n'
        "  }\n"
        "  ms_check(MS_OK, nullptr);\n"
        "  return 0;\n}\n")
    exe = tmp_path / "h"
    lib_dir = os.path.dirname(LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", inc, str(cpp), "-L", lib_dir, "-lmorphoshell",
                    "-Wl,-rpath," + lib_dir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    assert out[0] == "implausibly_high_force"
    assert out[1] and out[1] != "no throw"
