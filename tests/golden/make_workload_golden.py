"""Oracle fixtures for the benchmarked workloads (tests/golden/wl_*.npz).

The bench measures seeded synthetic workloads (mbd_b200/synthetic.py) that
are too large for the FP64 oracle to run inside a GPU test: the three
isolated clusters of the headline step (N = 500, 1000, 2000; seeds 0, 1, 2)
and a periodic {H,C,N,O} box at the periodic workload's cut-offs
(120/100/25 A; 256 atoms, seed 3, 2x2x2 supercell).  This script runs the
oracle on them once and stores what the GPU parity tests compare against:

    energy, c6_mol, nimag, supercell, alpha_eff (N), c6_eff (N),
    alpha_iw at frequencies 1, 10, 20 (3 x N), mol_pol_eig (21 x 3),
    and a fingerprint of the generated input (so that a change of the
    generator cannot go unnoticed).

    python tests/golden/make_workload_golden.py            # every case
    python tests/golden/make_workload_golden.py box256_s3  # one case
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from mbd_b200 import synthetic as sy  # noqa: E402
from oracle import mbd_oracle as mo  # noqa: E402

IW_FREQS = (1, 10, 20)

CASES = {
    "cluster500_s0": lambda: sy.cluster(500, seed=0),
    "cluster1000_s1": lambda: sy.cluster(1000, seed=1),
    "cluster2000_s2": lambda: sy.cluster(2000, seed=2),
    "box256_s3": lambda: sy.periodic_box(256, seed=3),
}


def fingerprint(geo, st) -> str:
    """sha256 of the generated input: species, coordinates, Hirshfeld ratios,
    lattice and cut-offs, at full precision."""
    h = hashlib.sha256()
    h.update(" ".join(geo.names).encode())
    for a in (geo.coords, geo.hirshfeld, geo.lattice):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    h.update(repr((geo.n_periodic, st.xc, st.mbd_supercell_cutoff, st.mbd_cfdm_dip_cutoff, st.mbd_scs_dip_cutoff,
                   tuple(st.mbd_scs_vacuum_axis))).encode())
    return h.hexdigest()


def oracle_inputs(geo, st):
    og = mo.Geometry(list(geo.names), geo.coords.copy(), geo.hirshfeld.copy(), geo.lattice.copy(), geo.n_periodic)
    os_ = mo.Settings(xc=st.xc, mbd_supercell_cutoff=st.mbd_supercell_cutoff,
                      mbd_cfdm_dip_cutoff=st.mbd_cfdm_dip_cutoff, mbd_scs_dip_cutoff=st.mbd_scs_dip_cutoff,
                      mbd_scs_vacuum_axis=tuple(st.mbd_scs_vacuum_axis))
    return og, os_


def make(name: str) -> None:
    geo, st = CASES[name]()
    t0 = time.time()
    res = mo.mbd_at_rsscs(*oracle_inputs(geo, st))
    dt = time.time() - t0
    assert res.status == "ok", res.status
    np.savez_compressed(
        os.path.join(HERE, f"wl_{name}.npz"),
        energy=res.energy, c6_mol=res.c6_mol, nimag=res.nimag, supercell=np.array(res.supercell),
        alpha_eff=res.alpha_eff, c6_eff=res.c6_eff, iw_freqs=np.array(IW_FREQS),
        alpha_iw=res.alpha_iw[list(IW_FREQS)], mol_pol_eig=res.mol_pol_eig,
        fingerprint=fingerprint(geo, st), oracle_seconds=dt)
    print(f"{name}: N={len(geo.names)} E={res.energy:.12f} C6={res.c6_mol:.6f} nimag={res.nimag} "
          f"supercell={res.supercell} ({dt:.1f} s)", flush=True)


if __name__ == "__main__":
    for nm in (sys.argv[1:] or list(CASES)):
        make(nm)
