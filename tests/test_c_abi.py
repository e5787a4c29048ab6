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


def _c_struct_fields(header, name):
    import re
    body = dict((n, b) for b, n in re.findall(r"typedef struct \{([^{}]*)\} (\w+);", header))[name]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        for part in decl.split(","):
            m = re.search(r"(\w+)\s*(\[\w+\])?\s*$", part.strip())
            fields.append(m.group(1).lower())
    return fields


def _f_type_fields(src, name):
    import re
    body = re.search(r"TYPE, BIND\(C\) :: " + name + r"\n(.*?)END TYPE", src, re.S).group(1)
    fields = []
    for line in body.splitlines():
        line = line.split("!")[0]
        if "::" not in line:
            continue
        for part in line.split("::")[1].split(","):
            fields.append(re.match(r"\s*(\w+)", part).group(1).lower())
    return fields


def test_fortran_module_matches_the_header_and_the_library():
    """include/mbd_b200.f90 (not compiled here: no Fortran compiler): every
    name it binds is declared in the header and exported by the library, and
    its BIND(C) types list the C structs' members in the same order."""
    import ctypes
    import re
    with open(os.path.join(ROOT, "include", "mbd_b200.h")) as fh:
        header = fh.read()
    with open(os.path.join(ROOT, "include", "mbd_b200.f90")) as fh:
        src = fh.read()
    names = [n for n in re.findall(r"NAME='(\w+)'", src) if n != "strlen"]
    assert len(names) >= 20
    lib = ctypes.CDLL(os.path.join(LIB_DIR, "libmbd_b200.so"))
    for n in names:
        assert re.search(r"\b" + n + r"\(", header), n
        assert hasattr(lib, n), n
    for st in ("mbd_geom", "mbd_result"):
        assert _f_type_fields(src, st) == _c_struct_fields(header, st), st
