"""Generate the golden fixtures under tests/golden/ from the reference tree.

Run once in a container that has the reference checkout; its root is the
required first argument:

    python tests/golden/make_golden.py <reference checkout>

For every example it writes ``<name>.json`` holding
  * the geometry and settings exactly as the reference run read them
    (examples/<name>.in + the settings used for that run),
  * ``printed``: the values the reference printed in examples/<name>.out
    (C6H6, graphene_111, PBBA), and for the clusters (C6H6, PBBA) the MBD
    report lines themselves (``report_lines``: from "| Many-Body Dispersion"
    to the energy line; the graphene output was written by a version of the
    report code whose headers differ from UTILS.f90:223-331), and
  * ``oracle``: the FP64 oracle's full-precision outputs on the same input
    (used as the parity target for the GPU path; for H2O and TiOCHF, which
    ship no output, this is the only pin).

``--report-only`` adds or refreshes ``report_lines`` in the existing
fixtures without recomputing the oracle.

The settings of the shipped outputs are taken from the headers of the .out
files: C6H6 and PBBA used the defaults (the 2000 A box of C6H6 admits no
image inside any cut-off); graphene_111 used settings.in (supercell 20 A,
cfdm 100 A, scs 120 A, no vacuum axis).
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from oracle import mbd_oracle as mo  # noqa: E402

CASES = {
    # name: (settings source, has printed output)
    "C6H6": (None, True),
    "graphene_111": ("settings.in", True),
    "PBBA": (None, True),
    "H2O": (None, False),
    "TiOCHF": ("settings.in", False),
}


REPORT_CASES = ("C6H6", "PBBA")


def report_lines(out_text: str) -> list:
    """The MBD section of a pmbd.x report: the lines from the section header
    to the energy line that the report code prints (``|`` rows and warnings)."""
    lines = out_text.splitlines()
    start = next(i for i, ln in enumerate(lines) if "| Many-Body Dispersion (MBD@rsSCS) energy" in ln)
    sel = []
    for ln in lines[start:]:
        if ln.lstrip().startswith("|") or ln.startswith(" ***WARNING: found"):
            sel.append(ln)
            if "| MBD@rsSCS energy" in ln:
                break
    return sel


def add_report_lines(ref_root: str) -> None:
    for name in REPORT_CASES:
        path = os.path.join(HERE, name + ".json")
        with open(path) as fh:
            fix = json.load(fh)
        with open(os.path.join(ref_root, "examples", name + ".out")) as fh:
            fix["printed"]["report_lines"] = report_lines(fh.read())
        with open(path, "w") as fh:
            json.dump(fix, fh, indent=1)
        print(f"{name}: {len(fix['printed']['report_lines'])} report lines")


def main(ref_root: str) -> None:
    for name, (settings_file, printed) in CASES.items():
        with open(os.path.join(ref_root, "examples", name + ".in")) as fh:
            geo_text = fh.read()
        st_text = ""
        if settings_file:
            with open(os.path.join(ref_root, settings_file)) as fh:
                st_text = fh.read()
        geo = mo.parse_geometry(geo_text)
        st = mo.parse_settings(st_text)
        t0 = time.time()
        res = mo.mbd_at_rsscs(geo, st)
        dt = time.time() - t0
        fix = {
            "name": name,
            "geometry_in": geo_text,
            "settings_in": st_text,
            "oracle": {
                "energy": res.energy if res.status == "ok" else None,
                "status": res.status,
                "nimag": res.nimag,
                "c6_mol": res.c6_mol,
                "alpha_eff": res.alpha_eff.tolist(),
                "c6_eff": res.c6_eff.tolist(),
                "alpha_iw": res.alpha_iw.tolist(),
                "mol_pol_eig": res.mol_pol_eig.tolist(),
                "supercell": list(res.supercell),
                "seconds": dt,
            },
        }
        if printed:
            with open(os.path.join(ref_root, "examples", name + ".out")) as fh:
                rep = mo.parse_report(fh.read())
            fix["printed"] = {
                "energy": rep["energy"],
                "c6_mol": rep["c6_mol"],
                "atoms": {str(k): v for k, v in rep["atoms"].items()},
                "pol": rep["pol"],
            }
            if name in REPORT_CASES:
                with open(os.path.join(ref_root, "examples", name + ".out")) as fh:
                    fix["printed"]["report_lines"] = report_lines(fh.read())
        with open(os.path.join(HERE, name + ".json"), "w") as fh:
            json.dump(fix, fh, indent=1)
        print(f"{name}: E={res.energy:.12f} C6={res.c6_mol:.8f} nimag={res.nimag} ({dt:.1f}s)")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if not args:
        sys.exit("usage: make_golden.py <reference checkout> [--report-only]")
    root = args[0]
    if "--report-only" in sys.argv:
        add_report_lines(root)
    else:
        main(root)
