"""Input tooling and the network checkpoint, on the CPU.

* write_geometry / parse_geometry round-trip a geometry exactly (full double
  precision), periodic or not;
* tile replicates a periodic cell as the reference's examples/process.py
  tiles the graphene cell (same coordinates, lattice vectors scaled), along
  all three vectors;
* the network checkpoint (magic, version, count, FP32 parameters, SHA-256)
  round-trips and refuses a corrupted or foreign file;
* the command line's tile subcommand writes a readable geometry.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from mbd_b200 import InputError, parse_geometry, tile, write_geometry
from mbd_b200.engine import read_network_file, write_network_file

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _graphene():
    with open(os.path.join(GOLDEN, "graphene_111.json")) as fh:
        return parse_geometry(json.load(fh)["geometry_in"])


def test_geometry_round_trip():
    from mbd_b200 import synthetic as sy
    for geo in (_graphene(), sy.cluster(40, seed=2)[0], sy.periodic_box(30, seed=1)[0]):
        back = parse_geometry(write_geometry(geo))
        assert back.names == geo.names and back.n_periodic == geo.n_periodic
        assert np.array_equal(back.coords, geo.coords)
        assert np.array_equal(back.hirshfeld, geo.hirshfeld)
        assert np.array_equal(back.lattice, geo.lattice)


def test_tile_matches_process_py_layout():
    """examples/process.py: copy (i, j) of the cell shifted by i a1 + j a2,
    copies in the order i outer, j inner, lattice vectors a1 * n1, a2 * n2."""
    g = _graphene()
    t = tile(g, (2, 3, 1))
    n = len(g.names)
    assert len(t.names) == 6 * n
    k = 0
    for i in range(2):
        for j in range(3):
            np.testing.assert_array_equal(t.coords[k * n:(k + 1) * n], g.coords + i * g.lattice[0] + j * g.lattice[1])
            np.testing.assert_array_equal(t.hirshfeld[k * n:(k + 1) * n], g.hirshfeld)
            k += 1
    np.testing.assert_array_equal(t.lattice, g.lattice * np.array([[2], [3], [1]]))
    assert tile(g, (1, 1, 1)).coords.tolist() == g.coords.tolist()


def test_tile_refuses_clusters_and_bad_counts():
    from mbd_b200 import synthetic as sy
    with pytest.raises(InputError):
        tile(sy.cluster(10, seed=0)[0], (2, 1, 1))
    with pytest.raises(InputError):
        tile(_graphene(), (0, 1, 1))


def test_network_checkpoint_round_trip_and_checks(tmp_path):
    p = np.random.default_rng(0).standard_normal(1234).astype(np.float32)
    f = tmp_path / "net.bin"
    write_network_file(str(f), p)
    np.testing.assert_array_equal(read_network_file(str(f)), p)
    data = bytearray(f.read_bytes())
    data[40] ^= 0x01                      # one flipped bit in the parameters
    (tmp_path / "bad.bin").write_bytes(bytes(data))
    with pytest.raises(ValueError, match="SHA-256"):
        read_network_file(str(tmp_path / "bad.bin"))
    (tmp_path / "foreign.bin").write_bytes(b"not a network")
    with pytest.raises(ValueError, match="not a network"):
        read_network_file(str(tmp_path / "foreign.bin"))


def test_cli_tile(tmp_path):
    src = tmp_path / "g.in"
    src.write_text(write_geometry(_graphene()))
    out = tmp_path / "g221.in"
    subprocess.run([sys.executable, "-m", "mbd_b200", "tile", str(src), "2", "2", "1", "-o", str(out)], check=True,
                   cwd=ROOT)
    t = parse_geometry(out.read_text())
    assert len(t.names) == 4 * 60 and t.n_periodic == 3


def test_settings_round_trip():
    from mbd_b200 import Settings, parse_settings, write_settings
    st = Settings(xc=2, mbd_supercell_cutoff=12.5, mbd_cfdm_dip_cutoff=0.1 + 0.2, mbd_scs_dip_cutoff=90.0,
                  mbd_scs_vacuum_axis=(False, True, True))
    back = parse_settings(write_settings(st))
    assert (back.xc, back.mbd_supercell_cutoff, back.mbd_cfdm_dip_cutoff, back.mbd_scs_dip_cutoff,
            back.mbd_scs_vacuum_axis) == (2, 12.5, 0.1 + 0.2, 90.0, (False, True, True))
    assert parse_settings(write_settings(Settings())).mbd_scs_vacuum_axis == (False, False, False)


@pytest.mark.parametrize("kind,args", [("cluster", ["--atoms", "40", "--seed", "3"]),
                                       ("box", ["--atoms", "30", "--seed", "2", "--scs-cut", "20", "--cfdm-cut",
                                                "15", "--sc-cut", "5"]),
                                       ("sheet", ["--reps", "3"]),
                                       ("benzene", [])])
def test_cli_generate_writes_the_generators_inputs(tmp_path, kind, args):
    """`generate` writes the seeded generators' geometries and settings in
    pmbd.x's formats; read back they are the generators' own, bit for bit."""
    from mbd_b200 import parse_settings
    from mbd_b200 import synthetic as sy
    g, s = tmp_path / "geometry.in", tmp_path / "setting.in"
    subprocess.run([sys.executable, "-m", "mbd_b200", "generate", kind] + args + ["-o", str(g), "--settings", str(s)],
                   check=True, cwd=ROOT)
    ref_g, ref_s = {"cluster": lambda: sy.cluster(40, seed=3),
                    "box": lambda: sy.periodic_box(30, seed=2, scs_cut=20.0, cfdm_cut=15.0, sc_cut=5.0),
                    "sheet": lambda: sy.graphene_sheet(3),
                    "benzene": lambda: sy.benzene()}[kind]()
    geo, st = parse_geometry(g.read_text()), parse_settings(s.read_text())
    assert geo.names == list(ref_g.names) and geo.n_periodic == ref_g.n_periodic
    assert np.array_equal(geo.coords, ref_g.coords) and np.array_equal(geo.hirshfeld, ref_g.hirshfeld)
    assert np.array_equal(geo.lattice, ref_g.lattice)
    assert (st.xc, st.mbd_supercell_cutoff, st.mbd_cfdm_dip_cutoff, st.mbd_scs_dip_cutoff,
            tuple(st.mbd_scs_vacuum_axis)) == (ref_s.xc, ref_s.mbd_supercell_cutoff, ref_s.mbd_cfdm_dip_cutoff,
                                               ref_s.mbd_scs_dip_cutoff, tuple(bool(v) for v in ref_s.mbd_scs_vacuum_axis))


def test_cli_generate_batch_and_errors(tmp_path):
    from mbd_b200 import synthetic as sy
    out = tmp_path / "batch"
    subprocess.run([sys.executable, "-m", "mbd_b200", "generate", "batch", "--count", "5", "--seed", "4", "-o",
                    str(out)], check=True, cwd=ROOT)
    ref = sy.cluster_batch(count=5, seed=4)
    assert sorted(p.name for p in out.iterdir()) == [f"geometry_{k}.in" for k in range(5)] + ["setting.in"]
    for k, (rg, _) in enumerate(ref):
        geo = parse_geometry((out / f"geometry_{k}.in").read_text())
        assert np.array_equal(geo.coords, rg.coords) and geo.names == list(rg.names)
    bad = subprocess.run([sys.executable, "-m", "mbd_b200", "generate", "cluster", "-o", str(tmp_path / "x.in")],
                         capture_output=True, text=True, cwd=ROOT)
    assert bad.returncode == 1 and "--atoms N" in bad.stderr
