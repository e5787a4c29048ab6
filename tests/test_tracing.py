"""Tracing on CPU: the engine's NVTX ranges, seen through the NVTX v3
injection interface that profilers use.  tests/c/nvtx_record.c, built as an
injection library and named by NVTX_INJECTION64_PATH, records every range
push and pop; each public call opens its range on entry (before its argument
checks, so calls with a null context show it without a GPU) and closes it
on every return."""
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _cuda_include():
    from mbd_b200 import build
    try:
        inc = os.path.join(os.path.dirname(os.path.dirname(build.nvcc())), "include")
    except RuntimeError:
        return None
    return inc if os.path.isdir(os.path.join(inc, "nvtx3")) else None


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_public_calls_open_and_close_their_nvtx_ranges(tmp_path):
    from mbd_b200 import build
    inc = _cuda_include()
    if inc is None or not os.path.exists(build.LIB):
        pytest.skip("CUDA headers or libmbd_b200.so missing")
    inj = tmp_path / "libnvtx_record.so"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-shared", "-fPIC", "-I", inc,
                    os.path.join(ROOT, "tests", "c", "nvtx_record.c"), "-o", str(inj), "-ldl"], check=True)
    rec = tmp_path / "ranges.txt"
    script = (
        "import ctypes, sys\n"
        "lib = ctypes.CDLL(sys.argv[1])\n"
        "codes = [lib.mbd_rsscs_upload(None, 0, None)]\n"
        "codes += [lib.mbd_rsscs_compute(None, m) for m in (0, 1, 2, 7)]\n"
        "codes += [lib.mbd_rsscs_download(None, None), lib.mbd_rsscs_eigvalsh(None, None, 0, 0, None),\n"
        "          lib.mbd_rsscs_eigh(None, None, 0, 0, None, None, 0), lib.mbd_rsscs_autotune(None, 0)]\n"
        "print(codes)\n")
    env = dict(os.environ, NVTX_INJECTION64_PATH=str(inj), MBD_NVTX_RECORD=str(rec))
    out = subprocess.run([sys.executable, "-c", script, build.LIB], capture_output=True, text=True, env=env,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == str([1] * 9)          # MBD_ERR_ARG everywhere
    names = ["upload", "compute plain", "compute mixed", "compute mixed_learned", "compute", "download",
             "eigvalsh", "eigh", "autotune"]
    expect = []
    for nm in names:
        expect += [f"push mbd_b200 {nm}", "pop"]
    assert rec.read_text().splitlines() == expect
