"""The C++ host above the C ABI (mbd_b200/host/pmbd_io.h and the pmbd_b200
executable), checked on CPU.

* tests/c/host_io_check.cpp drives the header: its report, fed the FP64
  oracle's values, reproduces the lines of the reference's examples/C6H6.out
  and examples/PBBA.out byte for byte (the committed golden fixtures); its
  parsers and Fortran edit descriptors agree with the Python host's
  (mbd_b200/io.py) on the same inputs, malformed ones included; its SHA-256
  agrees with hashlib and its network-checkpoint reader reads what
  write_network_file writes and rejects a corrupted, truncated or
  wrong-version file;
* the linked pmbd_b200 answers a bad command line with status 2 and an
  unreadable input or a machine without an sm_100 GPU with status 1 and the
  engine's message;
* pmbd_b200 linked against a stub engine (tests/c/fake_mbd.c) hands the C
  ABI exactly the atomic numbers, bohr coordinates, lattice, settings and
  mode the Python host would, loads a network checkpoint, prints the
  reference's report from the engine's results and reports engine errors.
"""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")


@pytest.fixture(scope="module")
def check(tmp_path_factory):
    d = tmp_path_factory.mktemp("hostio")
    exe = d / "host_io_check"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I",
                    os.path.join(ROOT, "mbd_b200", "host"), os.path.join(ROOT, "tests", "c", "host_io_check.cpp"),
                    "-o", str(exe)], check=True)

    def run(*args, files=None, ok=True):
        paths = []
        for k, text in enumerate(files or []):
            p = d / f"in{k}"
            if isinstance(text, bytes):
                p.write_bytes(text)
            else:
                p.write_text(text, newline="")
            paths.append(str(p))
        out = subprocess.run([str(exe)] + list(args) + paths, capture_output=True, text=True, timeout=60)
        if ok:
            assert out.returncode == 0, out.stderr
        return out
    return run


def _values(o, omega):
    eig = np.asarray(o["mol_pol_eig"], dtype=np.float64)          # (21, 3)
    vals = [o["energy"], o["c6_mol"], o["nimag"], *o["supercell"], *o["c6_eff"], *o["alpha_eff"],
            *eig.T.ravel(), *omega]
    return "\n".join(float(v).hex() for v in vals) + "\n"


@pytest.mark.parametrize("name", ["C6H6", "PBBA"])
def test_report_matches_reference_bytes(check, name):
    from oracle import mbd_oracle as mo
    with open(os.path.join(GOLDEN, name + ".json")) as fh:
        fix = json.load(fh)
    out = check("report", files=[fix["geometry_in"], _values(fix["oracle"], mo.CASIMIR_OMEGA)])
    assert out.stdout.splitlines() == fix["printed"]["report_lines"]


def test_report_warning_and_supercell_lines_match_python(check):
    import types

    from mbd_b200 import format_report, parse_geometry
    text = "2\n\nC 0 0 0 0.8\nH 0 0 1.1 0.6\n"
    o = {"energy": -0.5, "c6_mol": 10.0, "nimag": 3, "supercell": [2, 2, 1], "c6_eff": [1.0, 2.0],
         "alpha_eff": [3.0, 4.0], "mol_pol_eig": np.ones((21, 3)).tolist()}
    omega = np.linspace(0.0, 2.0, 21)
    res = types.SimpleNamespace(energy=o["energy"], c6_mol=o["c6_mol"], nimag=3, supercell=(2, 2, 1),
                                c6_eff=np.array(o["c6_eff"]), alpha_eff=np.array(o["alpha_eff"]),
                                mol_pol_eig=np.ones((21, 3)))
    expect = format_report(parse_geometry(text), res, omega_grid=omega).splitlines()
    got = check("report", files=[text, _values(o, omega)]).stdout.splitlines()
    assert got == expect
    assert " ***WARNING: found    3 negative eigenvalues in MBD energy calculation." in got


GEOMETRIES = [
    "3\ncomment\nO 0.0 0.0 0.1173 0.85\nH 0.0 0.7572 -0.4692 0.62\nH,0.0,-0.7572,-0.4692,0.62\n",
    "2\r\n\r\nC 1.0d0 -2.5D-1 3.25E+00 0.8\r\nHe 0 0 1.1 0.6\r\n",
    "2\nx\nCl 0 0 0 0.9 extra tokens\nTi 1 2 3 1.0\nlattice_vector 10.0 0 0\nlattice_vector 0 11.5 0\n"
    "lattice_vector 0.5 0 12d0\n",
    "1\n\nC 0 0 0 1\n\nlattice_vector 1 0 0\n",          # a blank line: no lattice
]


def _py_geometry_lines(text):
    from mbd_b200 import parse_geometry
    g = parse_geometry(text)
    lines = [f"{len(g.names)} {g.n_periodic}"]
    for name, xyz, h in zip(g.names, g.coords, g.hirshfeld):
        lines.append(" ".join([name] + [float(v).hex() for v in (*xyz, h)]))
    lines += [float(v).hex() for v in g.lattice.ravel()]
    return lines


def _norm_hex(lines):
    # %a prints 0x0p+0 and 0x1.8p+1 where float.hex prints 0x0.0p+0 and 0x1.8000000000000p+1
    out = []
    for ln in lines:
        toks = []
        for t in ln.split():
            toks.append(float.fromhex(t).hex() if t.startswith(("0x", "-0x")) else t)
        out.append(" ".join(toks))
    return out


@pytest.mark.parametrize("k", range(len(GEOMETRIES)))
def test_geometry_parser_matches_python(check, k):
    text = GEOMETRIES[k]
    got = check("geometry", files=[text]).stdout.splitlines()
    assert _norm_hex(got) == _norm_hex(_py_geometry_lines(text))


def test_golden_geometries_parse_alike(check):
    for name in ("C6H6", "H2O", "PBBA", "TiOCHF", "graphene_111"):
        with open(os.path.join(GOLDEN, name + ".json")) as fh:
            text = json.load(fh)["geometry_in"]
        got = check("geometry", files=[text]).stdout.splitlines()
        assert _norm_hex(got) == _norm_hex(_py_geometry_lines(text)), name


SETTINGS = [
    "",
    "xc 2\nmbd_supercell_cutoff 30.0\nmbd_cfdm_dip_cutoff 80d0\nmbd_scs_dip_cutoff 90\n"
    "mbd_scs_vacuum_axis .false. .false. .true.\nnprow 2\nnpcol 4\n",
    "mbd_scs_vacuum_axis T,F,f\nsomething else\nxc 3 # comment\n",
]


@pytest.mark.parametrize("k", range(len(SETTINGS)))
def test_settings_parser_matches_python(check, k):
    from mbd_b200 import parse_settings
    text = SETTINGS[k]
    s = parse_settings(text)
    expect = " ".join([str(s.xc)] + [float(v).hex() for v in (s.mbd_supercell_cutoff, s.mbd_cfdm_dip_cutoff,
                                                                s.mbd_scs_dip_cutoff)] +
                      [str(int(v)) for v in s.mbd_scs_vacuum_axis] + [str(s.nprow), str(s.npcol)])
    got = check("settings", files=[text]).stdout.strip()
    assert _norm_hex([got]) == _norm_hex([expect])


@pytest.mark.parametrize("text,which", [
    ("x\n\nC 0 0 0 1\n", "geometry"),
    ("0\n\n", "geometry"),
    ("2\n\nC 0 0 0 1\n", "geometry"),
    ("1\n\nC 0 0 0\n", "geometry"),
    ("1\n\nC 0 0 zero 1\n", "geometry"),
    ("1\n\nC 0 0 0 1\nlattice_vector 1 0 0\nlattice_vector 0 1 0\n", "geometry"),
    ("1\n\nC 0 0 0 1\nlattice_vector 1 0 0\nlattice_vector 0 1\nlattice_vector 0 0 1\n", "geometry"),
    ("1\n\nC 0 0 0 1\nlattice_vector 1 0 0\nlattice_vector 0 1 0\nlattice_vector 0 0 x\n", "geometry"),
    ("mbd_scs_vacuum_axis .maybe. .false. .true.\n", "settings"),
    ("xc\n", "settings"),
    ("mbd_scs_dip_cutoff far\n", "settings"),
])
def test_malformed_inputs_are_errors_in_both_hosts(check, text, which):
    from mbd_b200 import parse_geometry, parse_settings
    from mbd_b200.io import InputError
    with pytest.raises(InputError):
        (parse_geometry if which == "geometry" else parse_settings)(text)
    out = check(which, files=[text], ok=False)
    assert out.returncode == 1 and out.stderr.strip().startswith(which), out.stderr


def test_edit_descriptors_match_python(check):
    from mbd_b200 import io
    rng = np.random.default_rng(5)
    cases = [(65.6629, 15, 6), (0.0212703, 15, 6), (-1234.5, 15, 6), (0.0, 15, 6), (0.9999999, 15, 6),
             (1622.14013676, 20, 8), (123456.0, 5, 1), (1e-120, 15, 6), (-9.9999996e99, 15, 6), (5e-324, 15, 6),
             (-0.0, 10, 6), (0.5, 3, 1), (-0.05, 4, 1)]
    for w, d in ((15, 6), (10, 6), (20, 8), (20, 9), (12, 6)):
        for v in rng.standard_normal(60) * 10.0 ** rng.integers(-12, 14, 60):
            cases.append((float(v), w, d))
    text = "".join(f"{float(v).hex()} {w} {d}\n" for v, w, d in cases)
    got = check("edit", files=[text]).stdout.splitlines()
    expect = [f"{io._fortran_e(v, w, d)}|{io._fortran_f(v, w, d)}" for v, w, d in cases]
    assert got == expect


def test_sha256_matches_hashlib(check):
    import hashlib
    rng = np.random.default_rng(1)
    for n in (0, 1, 3, 55, 56, 57, 63, 64, 65, 119, 120, 128, 1000, 4103):
        data = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        got = check("sha256", files=[data]).stdout.strip()
        assert got == hashlib.sha256(data).hexdigest(), n


def test_network_checkpoint_reader(check, tmp_path):
    from mbd_b200.engine import write_network_file
    rng = np.random.default_rng(2)
    p = rng.standard_normal(1234).astype(np.float32)
    path = tmp_path / "net.bin"
    write_network_file(str(path), p)
    data = path.read_bytes()
    got = check("network", files=[data]).stdout.split()
    assert int(got[0]) == p.size
    np.testing.assert_array_equal(np.array([float.fromhex(t) for t in got[1:]], dtype=np.float32), p)
    bad = bytearray(data)
    bad[100] ^= 1
    out = check("network", files=[bytes(bad)], ok=False)
    assert out.returncode == 1 and "SHA-256 mismatch" in out.stderr
    out = check("network", files=[data[:-5]], ok=False)
    assert out.returncode == 1 and "SHA-256 mismatch" in out.stderr
    bad = bytearray(data)
    bad[8] = 2
    out = check("network", files=[bytes(bad)], ok=False)
    assert out.returncode == 1 and "version 2, expected 1" in out.stderr
    out = check("network", files=[b"not a checkpoint at all"], ok=False)
    assert out.returncode == 1 and "not a network checkpoint" in out.stderr


@pytest.fixture(scope="module")
def pmbd():
    from mbd_b200 import build
    if not os.path.exists(build.LIB):
        pytest.skip("libmbd_b200.so not built")
    return build.build_host()


def test_pmbd_b200_command_line(pmbd, tmp_path):
    def run(*args):
        return subprocess.run([pmbd] + list(args), capture_output=True, text=True, timeout=120)
    assert run("--help").returncode == 0
    for args in ((), ("a", "b", "c"), ("g.in", "--mode", "fast"), ("g.in", "--device"), ("g.in", "--bogus")):
        out = run(*args)
        assert out.returncode == 2 and out.stderr.startswith("usage: pmbd_b200"), args
    out = run(str(tmp_path / "missing.in"))
    assert out.returncode == 1 and "cannot open" in out.stderr
    g = tmp_path / "g.in"
    g.write_text("1\n\nC 0 0 0\n")
    out = run(str(g))
    assert out.returncode == 1 and "needs name x y z hirshfeld" in out.stderr


def test_pmbd_b200_without_a_gpu(pmbd, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    g = tmp_path / "g.in"
    g.write_text("2\n\nC 0 0 0 0.8\nH 0 0 1.1 0.6\n")
    out = subprocess.run([pmbd, str(g)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 1 and out.stderr.strip().endswith("(status 6)"), out.stderr


@pytest.fixture(scope="module")
def fake_pmbd(tmp_path_factory):
    """pmbd_b200 linked against tests/c/fake_mbd.c built as libmbd_b200.so:
    the executable's own code runs unchanged, the engine is a stub that
    records what it is given and returns fixed values."""
    d = tmp_path_factory.mktemp("fakembd")
    inc = os.path.join(ROOT, "include")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-shared", "-fPIC", "-I", inc,
                    os.path.join(ROOT, "tests", "c", "fake_mbd.c"), "-o", str(d / "libmbd_b200.so")], check=True)
    exe = d / "pmbd_b200"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", inc, "-I",
                    os.path.join(ROOT, "mbd_b200", "host"), os.path.join(ROOT, "mbd_b200", "host", "pmbd_b200.cpp"),
                    "-L", str(d), "-lmbd_b200", "-Wl,-rpath," + str(d), "-o", str(exe)], check=True)
    return str(exe)


def _run_fake(exe, args, tmp_path, values, status=None):
    vals = tmp_path / "values.txt"
    vals.write_text(values)
    rec = tmp_path / "record.txt"
    if rec.exists():
        rec.unlink()
    env = dict(os.environ, FAKE_MBD_VALUES=str(vals), FAKE_MBD_RECORD=str(rec))
    if status is not None:
        env["FAKE_MBD_STATUS"] = str(status)
    out = subprocess.run([exe] + list(args), capture_output=True, text=True, timeout=60, env=env)
    lines = rec.read_text().splitlines() if rec.exists() else []
    return out, lines


def _record_fields(lines):
    atoms = [ln.split()[1:] for ln in lines if ln.startswith("atom ")]
    rec = {"atoms": [(int(a[0]), *[float.fromhex(t) for t in a[1:]]) for a in atoms],
           "lattice": [float.fromhex(ln.split()[1]) for ln in lines if ln.startswith("lattice ")]}
    for ln in lines:
        key, *rest = ln.split()
        if key in ("mode", "n_atoms", "n_periodic", "xc", "device", "use_network"):
            rec[key] = int(rest[0])
        elif key == "cuts":
            rec[key] = [float.fromhex(t) for t in rest]
        elif key == "vacuum":
            rec[key] = [int(t) for t in rest]
        elif key == "set_params":
            rec[key] = (int(rest[0]), float.fromhex(rest[1]))
    return rec


@pytest.mark.parametrize("name", ["C6H6", "PBBA", "graphene_111", "H2O"])
def test_pmbd_b200_host_with_a_stub_engine(fake_pmbd, tmp_path, name):
    """What the executable hands the C ABI for the reference's inputs: atomic
    numbers, coordinates and lattice vectors converted to bohr exactly as the
    Python host converts them (MBD_rsSCS.f90:211-212), Hirshfeld ratios, the
    settings' cut-offs, vacuum axes and xc, the mode; and the report it
    prints from the engine's results (byte for byte the reference's report
    where the fixture holds it, else the Python host's)."""
    import types

    from mbd_b200 import format_report, parse_geometry, parse_settings
    from mbd_b200.engine import BOHR, element_z
    from oracle import mbd_oracle as mo
    with open(os.path.join(GOLDEN, name + ".json")) as fh:
        fix = json.load(fh)
    g = tmp_path / "geometry.in"
    g.write_text(fix["geometry_in"])
    s = tmp_path / "setting.in"
    s.write_text(fix["settings_in"])
    o = fix["oracle"]
    out, lines = _run_fake(fake_pmbd, [str(g), str(s), "--device", "3"], tmp_path, _values(o, mo.CASIMIR_OMEGA))
    assert out.returncode == 0, out.stderr
    rec = _record_fields(lines)
    geo = parse_geometry(fix["geometry_in"])
    st = parse_settings(fix["settings_in"])
    assert rec["device"] == 3 and rec["mode"] == 0 and "use_network" not in rec
    assert rec["n_atoms"] == len(geo.names) and rec["n_periodic"] == geo.n_periodic
    assert [a[0] for a in rec["atoms"]] == [element_z(nm) for nm in geo.names]
    np.testing.assert_array_equal(np.array([a[1:4] for a in rec["atoms"]]), geo.coords / BOHR)
    np.testing.assert_array_equal(np.array([a[4] for a in rec["atoms"]]), geo.hirshfeld)
    np.testing.assert_array_equal(np.array(rec["lattice"]).reshape(3, 3), geo.lattice / BOHR)
    assert rec["cuts"] == [st.mbd_scs_dip_cutoff, st.mbd_cfdm_dip_cutoff, st.mbd_supercell_cutoff]
    assert rec["vacuum"] == [int(v) for v in st.mbd_scs_vacuum_axis] and rec["xc"] == st.xc
    if "report_lines" in fix.get("printed", {}):
        expect = fix["printed"]["report_lines"]
    else:
        res = types.SimpleNamespace(energy=o["energy"], c6_mol=o["c6_mol"], nimag=o["nimag"],
                                    supercell=tuple(o["supercell"]), c6_eff=np.array(o["c6_eff"]),
                                    alpha_eff=np.array(o["alpha_eff"]), mol_pol_eig=np.array(o["mol_pol_eig"]))
        expect = format_report(geo, res, omega_grid=mo.CASIMIR_OMEGA).splitlines()
    assert out.stdout.splitlines() == expect


def test_pmbd_b200_modes_network_and_errors_with_a_stub_engine(fake_pmbd, tmp_path):
    from mbd_b200.engine import write_network_file
    from oracle import mbd_oracle as mo
    with open(os.path.join(GOLDEN, "C6H6.json")) as fh:
        fix = json.load(fh)
    g = tmp_path / "geometry.in"
    g.write_text(fix["geometry_in"])
    vals = _values(fix["oracle"], mo.CASIMIR_OMEGA)
    out, lines = _run_fake(fake_pmbd, [str(g), "--mode", "mixed"], tmp_path, vals)
    rec = _record_fields(lines)
    assert out.returncode == 0 and rec["mode"] == 1 and "use_network" not in rec
    assert rec["cuts"] == [120.0, 100.0, 25.0] and rec["vacuum"] == [0, 0, 0] and rec["xc"] == 1
    out, lines = _run_fake(fake_pmbd, [str(g), "--mode", "mixed_learned"], tmp_path, vals)
    rec = _record_fields(lines)
    assert out.returncode == 0 and rec["mode"] == 2 and rec["use_network"] == 0 and "set_params" not in rec
    p = np.random.default_rng(4).standard_normal(16274).astype(np.float32)
    net = tmp_path / "net.bin"
    write_network_file(str(net), p)
    out, lines = _run_fake(fake_pmbd, [str(g), "--mode", "mixed_learned", "--network", str(net)], tmp_path, vals)
    rec = _record_fields(lines)
    checksum = 0.0
    for i, x in enumerate(p):
        checksum += float(x) * (i % 7 + 1)
    assert out.returncode == 0 and rec["mode"] == 2 and "use_network" not in rec
    assert rec["set_params"] == (p.size, checksum)
    # the network is read before the engine is touched
    bad = bytearray(net.read_bytes())
    bad[40] ^= 4
    net.write_bytes(bytes(bad))
    out, lines = _run_fake(fake_pmbd, [str(g), "--mode", "mixed_learned", "--network", str(net)], tmp_path, vals)
    assert out.returncode == 1 and "SHA-256 mismatch" in out.stderr and lines == []
    write_network_file(str(net), p[:100])
    out, lines = _run_fake(fake_pmbd, [str(g), "--mode", "mixed_learned", "--network", str(net)], tmp_path, vals)
    assert out.returncode == 1 and "100 parameters, the engine's network has 16274" in out.stderr and lines == []
    # an engine status: message and exit status 1, nothing on stdout
    out, _ = _run_fake(fake_pmbd, [str(g)], tmp_path, vals, status=3)
    assert out.returncode == 1 and out.stdout == ""
    assert out.stderr.strip() == "pmbd_b200: fake error (status 3)"
    x = tmp_path / "bad.in"
    x.write_text("1\n\nXx 0 0 0 1.0\n")
    out, _ = _run_fake(fake_pmbd, [str(x)], tmp_path, vals)
    assert out.returncode == 1 and out.stderr.strip() == "pmbd_b200: fake: unknown element (status 2)"


def test_pmbd_b200_batch_with_a_stub_engine(fake_pmbd, tmp_path):
    """--batch: every listed geometry in one energy_batch call, a report file
    per geometry (byte for byte the reference's for C6H6), a failing geometry
    reported on stderr while the others are still written; relative paths in
    the list are taken from the list's directory."""
    from oracle import mbd_oracle as mo
    with open(os.path.join(GOLDEN, "C6H6.json")) as fh:
        fix = json.load(fh)
    d = tmp_path / "inputs"
    (d / "sub").mkdir(parents=True)
    (d / "benzene.in").write_text(fix["geometry_in"])
    (d / "sub" / "second.in").write_text(fix["geometry_in"])
    (d / "setting.in").write_text(fix["settings_in"])
    (d / "bad.in").write_text("1\n\nXx 0 0 0 1.0\n")
    lst = d / "list.txt"
    lst.write_text("# three geometries\nbenzene.in setting.in\n\nsub/second.in\n" + str(d / "bad.in") + "\n")
    out_dir = tmp_path / "reports"
    out_dir.mkdir()
    vals = _values(fix["oracle"], mo.CASIMIR_OMEGA)
    out, lines = _run_fake(fake_pmbd, ["--batch", str(lst), "--out-dir", str(out_dir), "--mode", "mixed"], tmp_path,
                           vals)
    assert out.returncode == 1 and out.stdout == ""
    assert out.stderr.strip() == f"pmbd_b200: {d / 'bad.in'}: fake: unknown element (status 2)"
    assert sorted(p.name for p in out_dir.iterdir()) == ["benzene.out", "second.out"]
    for name in ("benzene.out", "second.out"):
        assert (out_dir / name).read_text().splitlines() == fix["printed"]["report_lines"]
    rec = _record_fields(lines)
    assert rec["mode"] == 1 and len(rec["atoms"]) == 12 + 12 + 1
    assert sum(1 for ln in lines if ln.startswith("mode ")) == 3
    # two geometries that would write the same report, and a bad list line
    lst.write_text("benzene.in\nsub/benzene.in\n")
    (d / "sub" / "benzene.in").write_text(fix["geometry_in"])
    out, _ = _run_fake(fake_pmbd, ["--batch", str(lst), "--out-dir", str(out_dir)], tmp_path, vals)
    assert out.returncode == 1 and "would both write" in out.stderr
    lst.write_text("benzene.in\nmissing.in\n")
    out, lines = _run_fake(fake_pmbd, ["--batch", str(lst), "--out-dir", str(out_dir)], tmp_path, vals)
    assert out.returncode == 1 and "missing.in: cannot open" in out.stderr and lines == []
    lst.write_text("benzene.in setting.in extra\n")
    out, _ = _run_fake(fake_pmbd, ["--batch", str(lst), "--out-dir", str(out_dir)], tmp_path, vals)
    assert out.returncode == 1 and "expected geometry.in [setting.in]" in out.stderr
    for args in (["--batch", str(lst)], ["--out-dir", str(out_dir), str(d / "benzene.in")],
                 ["--batch", str(lst), "--out-dir", str(out_dir), str(d / "benzene.in")]):
        out, _ = _run_fake(fake_pmbd, args, tmp_path, vals)
        assert out.returncode == 2 and out.stderr.startswith("usage: pmbd_b200"), args
