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
