"""The C ABI from C: tests/c/abi_check.c compiles against include/mbd_b200.h
as C (and the header as C++), links libmbd_b200.so and calls the entry points
that need no GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "mbd_b200")


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_program_links_and_runs(tmp_path):
    exe = tmp_path / "abi_check"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "abi_check.c"), "-L", LIB_DIR, "-lmbd_b200",
                    "-Wl,-rpath," + LIB_DIR, "-lm", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "abi_check ok" in out.stdout


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_header_compiles_as_cpp(tmp_path):
    src = tmp_path / "h.cpp"
    src.write_text('#include "mbd_b200.h"\nint main() { return mbd_rsscs_element_z("C") == 6 ? 0 : 1; }\n')
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                    str(src)], check=True)
