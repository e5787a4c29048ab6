"""CPU-side checks: the C-ABI library loads and exports every declared entry
point, the input readers follow MBD_rsSCS.f90, the synthetic generators meet
their specification.  No compute call is made (no GPU here)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            with open(os.path.join(ROOT, "include", fn)) as fh:
                text = fh.read()
            names |= set(re.findall(r"\b(mbd_rsscs_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    import mbd_b200
    if not os.path.exists(mbd_b200.LIB_PATH):
        from mbd_b200 import build
        build.build(verbose=False)
    lib = ctypes.CDLL(mbd_b200.LIB_PATH)
    declared = _declared_symbols()
    assert declared, "no entry points found in include/*.h"
    for name in sorted(declared):
        assert hasattr(lib, name), name
    assert set(mbd_b200.EXPORTED) <= declared


def test_host_helpers_without_gpu():
    """Entry points that touch no device work on a CPU-only host."""
    from mbd_b200 import engine
    assert engine.element_z("C") == 6
    assert engine.element_z("Ti") == 22
    assert engine.element_z("La") == 0          # no vdW parameters (UTILS.f90:1693)
    assert engine.element_z("Rn") == 86
    lib = engine.load_library()
    a, c, r = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    assert lib.mbd_rsscs_vdw_params(6, ctypes.byref(a), ctypes.byref(c), ctypes.byref(r)) == 0
    assert (a.value, c.value, r.value) == (12.0, float(np.float32(46.6)), float(np.float32(3.59)))
    assert "positive definite" in engine.strerror(3)
    ctx = ctypes.c_void_p()
    # no GPU in this container: creation must fail loudly, never fall back
    if not _has_gpu():
        assert lib.mbd_rsscs_create(ctypes.byref(ctx), 0) == 6


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_table_matches_oracle():
    from mbd_b200 import engine
    from oracle import mbd_oracle as mo
    lib = engine.load_library()
    for sym, (a0, c6, r0) in mo.VDW_PARAMS.items():
        z = engine.element_z(sym)
        assert z > 0, sym
        a, c, r = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        assert lib.mbd_rsscs_vdw_params(z, ctypes.byref(a), ctypes.byref(c), ctypes.byref(r)) == 0
        assert (a.value, c.value, r.value) == (a0, c6, r0), sym


def test_readers_match_reference_semantics():
    from mbd_b200 import InputError, parse_geometry, parse_settings
    g = parse_geometry("2\n comment\nC 0 0 0 0.8\nHe1 1.0d0 0 0 0.9\n"
                       "lattice_vector 10 0 0\nlattice_vector 0 10 0\nlattice_vector 0 0 10\n")
    assert g.names == ["C", "He"] and g.n_periodic == 3
    assert g.coords[1, 0] == 1.0 and g.lattice[2, 2] == 10.0
    s = parse_settings("xc 3\nmbd_scs_vacuum_axis .false. .false. .true.\nnprow 2\nmbd_scs_dip_cutoff 80.d0\n")
    assert s.xc == 3 and s.mbd_scs_vacuum_axis == (False, False, True) and s.mbd_scs_dip_cutoff == 80.0
    assert s.mbd_cfdm_dip_cutoff == 100.0 and s.mbd_supercell_cutoff == 25.0
    with pytest.raises(InputError):
        parse_geometry("3\n\nC 0 0 0 0.8\n")
    with pytest.raises(InputError):
        parse_settings("mbd_scs_vacuum_axis .maybe. .false. .true.\n")


def test_synthetic_generators():
    from mbd_b200 import synthetic as sy
    g, _ = sy.cluster(400, seed=1)
    d = g.coords[:, None, :] - g.coords[None, :, :]
    r = np.sqrt((d * d).sum(-1)) + np.eye(400) * 1e9
    assert r.min() >= 0.95 - 1e-12
    radius = (3 * 400 / (4 * np.pi * 0.1)) ** (1 / 3)
    assert np.all(np.linalg.norm(g.coords, axis=1) <= radius + 1e-12)
    assert set(g.names) <= {"H", "C", "N", "O"}
    assert 0.6 <= g.hirshfeld.min() and g.hirshfeld.max() <= 1.0
    gs, st = sy.graphene_sheet()
    assert len(gs.names) == 128 and st.mbd_scs_vacuum_axis == (False, False, True)
    b, _ = sy.benzene()
    assert len(b.names) == 12 and np.allclose(b.coords[:, 1], 0.0)
    pb, _ = sy.periodic_box(300, seed=2)
    assert pb.n_periodic == 3 and np.isclose(pb.lattice[0, 0] ** 3, 3000.0)
    batch = sy.cluster_batch(count=4, seed=0)
    assert all(20 <= len(gg.names) <= 600 for gg, _ in batch)


@pytest.mark.parametrize("name", ["C6H6", "PBBA"])
def test_report_matches_reference_bytes(name):
    """format_report prints the MBD section of the report with the reference's
    edit descriptors (UTILS.f90:223-331, 753-755, 861): fed the FP64 oracle's
    values, it reproduces the lines of examples/<name>.out byte for byte."""
    import json
    import types

    from mbd_b200 import format_report, parse_geometry
    with open(os.path.join(ROOT, "tests", "golden", name + ".json")) as fh:
        fix = json.load(fh)
    o = fix["oracle"]
    res = types.SimpleNamespace(energy=o["energy"], c6_mol=o["c6_mol"], nimag=o["nimag"],
                                supercell=tuple(o["supercell"]), c6_eff=np.array(o["c6_eff"]),
                                alpha_eff=np.array(o["alpha_eff"]), mol_pol_eig=np.array(o["mol_pol_eig"]))
    lines = format_report(parse_geometry(fix["geometry_in"]), res).splitlines()
    assert lines == fix["printed"]["report_lines"]


def test_fortran_edit_descriptors():
    from mbd_b200 import io
    assert io._fortran_e(65.6629, 15, 6) == "   0.656629E+02"
    assert io._fortran_e(0.0212703, 15, 6) == "   0.212703E-01"
    assert io._fortran_e(-1234.5, 15, 6) == "  -0.123450E+04"
    assert io._fortran_e(0.0, 15, 6) == "   0.000000E+00"
    assert io._fortran_e(0.9999999, 15, 6) == "   0.100000E+01"   # rounding carries into the exponent
    assert io._fortran_f(1622.14013676, 20, 8) == "       1622.14013676"
    assert io._fortran_f(123456.0, 5, 1) == "*****"


def test_frequency_grid_matches_oracle():
    from mbd_b200.engine import frequency_grid
    from oracle import mbd_oracle as mo
    w, wt = frequency_grid()
    np.testing.assert_array_equal(w, mo.CASIMIR_OMEGA)
    np.testing.assert_array_equal(wt, mo.CASIMIR_WEIGHT)
    assert w[0] == 0.0 and wt[0] == 0.0


def test_report_warning_and_supercell_lines():
    """The NIMAG warning (UTILS.f90:861, '(A,I4,A)') and the supercell lines
    (UTILS.f90:753-755) as output_string prints them."""
    import types

    from mbd_b200 import format_report, parse_geometry
    geo = parse_geometry("2\n\nC 0 0 0 0.8\nH 0 0 1.1 0.6\n")
    res = types.SimpleNamespace(energy=-0.5, c6_mol=10.0, nimag=3, supercell=(2, 2, 1),
                                c6_eff=np.array([1.0, 2.0]), alpha_eff=np.array([3.0, 4.0]),
                                mol_pol_eig=np.ones((21, 3)))
    lines = format_report(geo, res, omega_grid=np.zeros(21)).splitlines()
    assert "   | Creating super cell of dimension  2 X   2 X   1 in MBD calculation" in lines
    assert "   | containing     8  atom" in lines
    assert " ***WARNING: found    3 negative eigenvalues in MBD energy calculation." in lines
    assert lines[-1].startswith("   | MBD@rsSCS energy   :")
    assert lines.index(" ***WARNING: found    3 negative eigenvalues in MBD energy calculation.") == len(lines) - 2
