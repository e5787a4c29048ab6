"""Pin the FP64 oracle to the reference's own shipped outputs.

The reference (pmbd.x) ships three reports, examples/{C6H6,graphene_111,PBBA}.out.
Their printed fields are copied into tests/golden/*.json by
tests/golden/make_golden.py; here the oracle must reproduce every printed
digit (values are compared to half a unit in the last printed place).
"""
import json
import os

import numpy as np
import pytest

from oracle import mbd_oracle as mo

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name + ".json")) as fh:
        return json.load(fh)


def run_oracle(fix):
    geo = mo.parse_geometry(fix["geometry_in"])
    st = mo.parse_settings(fix["settings_in"])
    return mo.mbd_at_rsscs(geo, st)


@pytest.mark.parametrize("name", ["C6H6", "PBBA", "graphene_111"])
def test_oracle_reproduces_printed_report(name):
    fix = load(name)
    pr = fix["printed"]
    res = run_oracle(fix)
    # MBD@rsSCS energy, F20.9 (UTILS.f90:330)
    assert abs(res.energy - pr["energy"]) <= 0.5e-9 + 1e-15
    # System C6, f20.8 (UTILS.f90:288)
    assert abs(res.c6_mol - pr["c6_mol"]) <= 0.51e-8 * max(1.0, abs(pr["c6_mol"]) / 1e6)
    # per-atom C6 and alpha, f12.6 (UTILS.f90:310)
    for k, (sym, c6, alpha) in pr["atoms"].items():
        i = int(k) - 1
        assert fix["geometry_in"] and abs(res.c6_eff[i] - c6) <= 0.51e-6
        assert abs(res.alpha_eff[i] - alpha) <= 0.51e-6
    # alpha(iw) table: omega, alpha_iso, three eigenvalues, e15.6 (UTILS.f90:278)
    assert len(pr["pol"]) == 21
    for f, row in enumerate(pr["pol"]):
        assert abs(mo.CASIMIR_OMEGA[f] - row[0]) <= 0.51e-6
        iso = np.sum(res.mol_pol_eig[f]) / 3.0
        for got, want in zip([iso, *res.mol_pol_eig[f]], row[1:]):
            assert abs(got - want) <= 0.51e-6 * abs(want) * 10 + 1e-300


def test_fixture_oracle_section_is_current():
    """The oracle section of each fixture (the GPU parity target) is what the
    oracle computes now."""
    for name in ["C6H6", "H2O", "PBBA"]:
        fix = load(name)
        res = run_oracle(fix)
        o = fix["oracle"]
        assert res.energy == pytest.approx(o["energy"], abs=1e-12)
        assert np.allclose(res.alpha_iw, np.array(o["alpha_iw"]), rtol=1e-12, atol=0)


def test_tiochf_nonpositive_alpha_reported():
    """examples/TiOCHF.in screens several O atoms to alpha <= 0; R_vdW_eff is
    then undefined (UTILS.f90:737) and the reference ships no output."""
    fix = load("TiOCHF")
    assert fix["oracle"]["status"] == "nonpositive_alpha"
    assert fix["oracle"]["energy"] is None
    assert min(fix["oracle"]["alpha_eff"]) < 0.0


def test_unknown_element_stops():
    geo = mo.parse_geometry("1\n\nXx 0 0 0 1.0\n")
    with pytest.raises(mo.UnknownElement):
        mo.mbd_at_rsscs(geo)


def test_settings_parser_first_match_order():
    st = mo.parse_settings(
        "xc 2\nmbd_supercell_cutoff 30.d0\nmbd_cfdm_dip_cutoff 90.0\n"
        "mbd_scs_dip_cutoff 80\nmbd_scs_vacuum_axis .false. .true. .TRUE.\nnprow 3\nnpcol 4\n")
    assert st.xc == 2 and st.mbd_supercell_cutoff == 30.0 and st.mbd_cfdm_dip_cutoff == 90.0
    assert st.mbd_scs_dip_cutoff == 80.0 and st.mbd_scs_vacuum_axis == (False, True, True)
    assert (st.nprow, st.npcol) == (3, 4)
    assert mo.get_beta(2) == mo.get_beta(3) == float(np.float32(0.85))
    assert mo.get_beta(7) == 1.0


def test_image_ranges_graphene():
    fix = load("graphene_111")
    geo = mo.parse_geometry(fix["geometry_in"])
    st = mo.parse_settings(fix["settings_in"])
    sysd = mo._System(geo, st)
    assert list(sysd.scs_rng) == [10, 10, 8]
    assert list(sysd.supercell) == [2, 2, 2]
    assert list(sysd.cfdm_rng) == [5, 4, 4]


def test_zero_damping_skip_changes_no_bit(monkeypatch):
    """Images left out of the short-range sum because their damping factor is
    exactly 0.0 in FP64 contribute exact zeros: the relay matrices are the same
    bit for bit with and without the skip (periodic box, every image of the
    reference's box visited in the second build)."""
    from mbd_b200 import synthetic as sy
    g, s = sy.periodic_box(40, seed=7, scs_cut=40.0, cfdm_cut=20.0, sc_cut=5.0)
    geo = mo.Geometry(list(g.names), g.coords, g.hirshfeld, g.lattice, g.n_periodic)
    st = mo.Settings(mbd_supercell_cutoff=s.mbd_supercell_cutoff, mbd_cfdm_dip_cutoff=s.mbd_cfdm_dip_cutoff,
                     mbd_scs_dip_cutoff=s.mbd_scs_dip_cutoff)
    sysd = mo._System(geo, st)
    fast, _ = mo.relay_matrices(sysd, freqs=[0, 7])
    monkeypatch.setattr(mo, "ZERO_DAMP_X", float("inf"))
    full, _ = mo.relay_matrices(sysd, freqs=[0, 7])
    for f in (0, 7):
        assert np.array_equal(fast[f], full[f])
