"""The command lines on the GPU: `python -m mbd_b200 run` and the C++
executable mbd_b200/pmbd_b200 print the MBD section of pmbd.x's report for
the reference's examples/C6H6.in byte for byte as examples/C6H6.out prints
it; `train` writes a network checkpoint that both load with `--mode
mixed_learned --network`, with the energy within the mixed forms' 1e-6 Ha of
the printed one."""
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


@pytest.fixture(scope="module")
def network(tmp_path_factory):
    net = tmp_path_factory.mktemp("net") / "net.bin"
    tr = subprocess.run([sys.executable, "-m", "mbd_b200", "train", "--out", str(net), "--geoms", "12",
                         "--epochs", "2"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert tr.returncode == 0, tr.stderr
    return str(net)


@pytest.fixture(scope="module")
def pmbd():
    from mbd_b200 import build
    return build.build_host()


def test_cli_train_then_run_learned(tmp_path, network):
    fix, g, s = _c6h6(tmp_path)
    out = subprocess.run([sys.executable, "-m", "mbd_b200", "run", g, s, "--mode", "mixed_learned", "--network",
                          network], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert out.returncode == 0, out.stderr
    assert abs(_energy(out.stdout) - fix["printed"]["energy"]) <= 1e-6


def test_pmbd_b200_prints_reference_report(tmp_path, pmbd):
    fix, g, s = _c6h6(tmp_path)
    out = subprocess.run([pmbd, g, s], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    assert out.stdout.splitlines() == fix["printed"]["report_lines"]


def test_pmbd_b200_modes(tmp_path, pmbd, network):
    """mixed, and mixed_learned from zero and from the trained network: the
    report's energy within 1e-6 Ha of the printed one."""
    fix, g, s = _c6h6(tmp_path)
    for extra in (["--mode", "mixed"], ["--mode", "mixed_learned"], ["--mode", "mixed_learned", "--network", network]):
        out = subprocess.run([pmbd, g, s] + extra, capture_output=True, text=True, timeout=600)
        assert out.returncode == 0, (extra, out.stderr)
        assert abs(_energy(out.stdout) - fix["printed"]["energy"]) <= 1e-6, extra


def test_cli_run_reports_unknown_element(tmp_path):
    g = tmp_path / "bad.in"
    g.write_text("1\n\nXx 0 0 0 1.0\n")
    out = subprocess.run([sys.executable, "-m", "mbd_b200", "run", str(g)], capture_output=True, text=True,
                         cwd=ROOT, timeout=600)
    assert out.returncode == 1
    assert "VdW parameters not defined" in out.stderr


def test_pmbd_b200_reports_unknown_element(tmp_path, pmbd):
    g = tmp_path / "bad.in"
    g.write_text("1\n\nXx 0 0 0 1.0\n")
    out = subprocess.run([pmbd, str(g)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 1
    assert "VdW parameters not defined" in out.stderr and "(status 2)" in out.stderr


def test_pmbd_b200_batch_reports(tmp_path, pmbd):
    """--batch: C6H6 and PBBA in one energy_batch call, one report file each
    with the reference's lines (numbers to the last printed digit, which a
    batch's different summation order may move by one)."""
    lst = tmp_path / "list.txt"
    fixes = {}
    for name in ("C6H6", "PBBA"):
        with open(os.path.join(GOLDEN, name + ".json")) as fh:
            fixes[name] = json.load(fh)
        (tmp_path / f"{name}.in").write_text(fixes[name]["geometry_in"])
        (tmp_path / f"{name}.set").write_text(fixes[name]["settings_in"])
    lst.write_text("C6H6.in C6H6.set\nPBBA.in PBBA.set\n")
    out_dir = tmp_path / "reports"
    out_dir.mkdir()
    out = subprocess.run([pmbd, "--batch", str(lst), "--out-dir", str(out_dir)], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    for name, fix in fixes.items():
        got = (out_dir / f"{name}.out").read_text().splitlines()
        want = fix["printed"]["report_lines"]
        assert len(got) == len(want)
        for a, b in zip(got, want):
            ta, tb = a.split(), b.split()
            assert len(ta) == len(tb), (a, b)
            for x, y in zip(ta, tb):
                if x != y:
                    fx, fy = float(x), float(y)
                    assert abs(fx - fy) <= 1.01 * 10.0 ** -(len(y.split(".")[1].split("E")[0])) * \
                        (10.0 ** int(y.split("E")[1]) if "E" in y else 1.0), (a, b)
        assert abs(_energy("\n".join(got)) - fix["printed"]["energy"]) <= 2e-9
