"""The command line on the GPU: `python -m mbd_b200 run` prints the MBD
section of pmbd.x's report for the reference's examples/C6H6.in byte for byte
as examples/C6H6.out prints it; `train` writes a network checkpoint that
`run --mode mixed_learned --network` loads, with the energy within the mixed
forms' 1e-6 Ha of the printed one."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _c6h6(tmp_path):
    with open(os.path.join(GOLDEN, "C6H6.json")) as fh:
        fix = json.load(fh)
    g = tmp_path / "C6H6.in"
    g.write_text(fix["geometry_in"])
    s = tmp_path / "settings.in"
    s.write_text(fix["settings_in"])
    return fix, str(g), str(s)


def _energy(report):
    line = [ln for ln in report.splitlines() if "MBD@rsSCS energy   :" in ln][0]
    return float(line.split(":")[1].split()[0])


def test_cli_run_prints_reference_report(tmp_path):
    fix, g, s = _c6h6(tmp_path)
    out = subprocess.run([sys.executable, "-m", "mbd_b200", "run", g, s], capture_output=True, text=True, cwd=ROOT,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    assert out.stdout.splitlines() == fix["printed"]["report_lines"]


def test_cli_train_then_run_learned(tmp_path):
    fix, g, s = _c6h6(tmp_path)
    net = tmp_path / "net.bin"
    tr = subprocess.run([sys.executable, "-m", "mbd_b200", "train", "--out", str(net), "--geoms", "12",
                         "--epochs", "2"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert tr.returncode == 0, tr.stderr
    out = subprocess.run([sys.executable, "-m", "mbd_b200", "run", g, s, "--mode", "mixed_learned", "--network",
                          str(net)], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert out.returncode == 0, out.stderr
    assert abs(_energy(out.stdout) - fix["printed"]["energy"]) <= 1e-6


def test_cli_run_reports_unknown_element(tmp_path):
    g = tmp_path / "bad.in"
    g.write_text("1\n\nXx 0 0 0 1.0\n")
    out = subprocess.run([sys.executable, "-m", "mbd_b200", "run", str(g)], capture_output=True, text=True,
                         cwd=ROOT, timeout=600)
    assert out.returncode == 1
    assert "VdW parameters not defined" in out.stderr
