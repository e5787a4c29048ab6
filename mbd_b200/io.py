"""Input files and the text report of pmbd.x.

* ``parse_geometry`` reads geometry.in as MBD_rsSCS.f90:66-89 does: atom
  count, a skipped line, ``name x y z hirshfeld`` per atom (Angstrom), then
  optional ``lattice_vector ax ay az`` records that make the system periodic.
* ``parse_settings`` reads setting.in as MBD_rsSCS.f90:98-135: for each line
  the first keyword that occurs as a substring (xc, mbd_supercell_cutoff,
  mbd_cfdm_dip_cutoff, mbd_scs_dip_cutoff, mbd_scs_vacuum_axis, nprow, npcol)
  takes the value(s) after the first token.  ``nprow``/``npcol`` are accepted
  and ignored: there is no process grid.
* ``format_report`` prints the fields of MBD_at_rsSCS's report
  (UTILS.f90:223-331).
* ``write_geometry`` / ``write_settings`` write a Geometry / Settings back in
  those formats and ``tile``
  replicates a periodic geometry into a supercell (the job of the
  reference's examples/process.py, which tiles the 60-atom graphene cell
  into graphene_<i><j>1.in), for any cell and along all three vectors.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

DEFAULT_SC_CUT = 25.0        # UTILS.f90:81
DEFAULT_CFDM_CUT = 100.0     # UTILS.f90:82
DEFAULT_SCS_CUT = 120.0      # UTILS.f90:83


class InputError(ValueError):
    pass


@dataclass
class Settings:
    xc: int = 1
    mbd_supercell_cutoff: float = DEFAULT_SC_CUT
    mbd_cfdm_dip_cutoff: float = DEFAULT_CFDM_CUT
    mbd_scs_dip_cutoff: float = DEFAULT_SCS_CUT
    mbd_scs_vacuum_axis: tuple = (False, False, False)
    nprow: int = 1
    npcol: int = 1
    given: set = field(default_factory=set)   # keywords present in the file


@dataclass
class Geometry:
    names: list
    coords: np.ndarray                    # (N, 3) Angstrom
    hirshfeld: np.ndarray                 # (N,)
    lattice: np.ndarray = field(default_factory=lambda: np.zeros((3, 3)))   # rows = vectors, Angstrom
    n_periodic: int = 0


def _real(tok: str) -> float:
    return float(tok.strip().lower().replace("d", "e"))


def _logical(tok: str) -> bool:
    t = tok.strip().lower().lstrip(".")
    if not t or t[0] not in "tf":
        raise InputError(f"not a Fortran logical: {tok!r}")
    return t[0] == "t"


def _records(text: str):
    for line in text.splitlines():
        yield line.replace(",", " ").split()


def parse_geometry(text: str) -> Geometry:
    lines = text.splitlines()
    try:
        n = int(lines[0].split()[0])
    except (IndexError, ValueError) as exc:
        raise InputError("geometry: first record must hold the atom count") from exc
    if n < 1:
        raise InputError("geometry: atom count must be >= 1")
    names, xyz, hv = [], [], []
    k = 2
    for i in range(n):
        if k >= len(lines):
            raise InputError(f"geometry: expected {n} atoms, found {i}")
        tok = lines[k].replace(",", " ").split()
        k += 1
        if len(tok) < 5:
            raise InputError(f"geometry: atom record {i + 1} needs name x y z hirshfeld")
        names.append(tok[0][:2])                 # CHARACTER*2
        try:
            xyz.append([_real(t) for t in tok[1:4]])
            hv.append(_real(tok[4]))
        except ValueError as exc:
            raise InputError(f"geometry: atom record {i + 1}: {exc}") from exc
    geo = Geometry(names, np.array(xyz, dtype=np.float64), np.array(hv, dtype=np.float64))
    if k < len(lines) and "lattice_vector" in lines[k]:
        geo.n_periodic = 3
        lat = np.zeros((3, 3))
        for i in range(3):
            if k + i >= len(lines):
                raise InputError("geometry: three lattice_vector records required")
            tok = lines[k + i].replace(",", " ").split()
            if len(tok) < 4:
                raise InputError("geometry: lattice_vector needs three components")
            try:
                lat[i] = [_real(t) for t in tok[1:4]]
            except ValueError as exc:
                raise InputError(f"geometry: lattice_vector: {exc}") from exc
        geo.lattice = lat
    return geo


def write_geometry(geo: Geometry) -> str:
    """geometry.in text for `geo` as parse_geometry (MBD_rsSCS.f90:66-89)
    reads it: atom count, a comment line, ``name x y z hirshfeld`` records
    (Angstrom, full double precision), then the three lattice vectors of a
    periodic system."""
    out = [str(len(geo.names)), "geometry written by mbd_b200"]
    for name, xyz, h in zip(geo.names, geo.coords, geo.hirshfeld):
        out.append(f"{name:<2s}  {xyz[0]:.17g}  {xyz[1]:.17g}  {xyz[2]:.17g}  {h:.17g}")
    if geo.n_periodic:
        for a in geo.lattice:
            out.append(f"lattice_vector  {a[0]:.17g}  {a[1]:.17g}  {a[2]:.17g}")
    return "\n".join(out) + "\n"


def write_settings(st: Settings) -> str:
    """setting.in text for `st` as parse_settings (MBD_rsSCS.f90:98-135) reads
    it: one keyword and its value(s) per line, reals in full double precision,
    the vacuum axes as Fortran logicals (nprow / npcol are not written: no
    process grid)."""
    lg = lambda v: ".true." if v else ".false."
    return "\n".join([
        f"xc {int(st.xc)}",
        f"mbd_supercell_cutoff {float(st.mbd_supercell_cutoff):.17g}",
        f"mbd_cfdm_dip_cutoff {float(st.mbd_cfdm_dip_cutoff):.17g}",
        f"mbd_scs_dip_cutoff {float(st.mbd_scs_dip_cutoff):.17g}",
        "mbd_scs_vacuum_axis " + " ".join(lg(v) for v in st.mbd_scs_vacuum_axis),
    ]) + "\n"


def tile(geo: Geometry, reps) -> Geometry:
    """Supercell of a periodic geometry: (n1, n2, n3) copies along the three
    lattice vectors, atoms in the order cell (i, j, k) with k fastest, then
    atom (examples/process.py:10-18 for the graphene cell, there only along
    the first two axes with fixed lattice constants); Hirshfeld ratios copied,
    lattice vectors scaled by the repetitions."""
    n1, n2, n3 = (int(r) for r in reps)
    if not geo.n_periodic:
        raise InputError("tile: the geometry has no lattice vectors")
    if min(n1, n2, n3) < 1:
        raise InputError("tile: repetitions must be >= 1")
    names, xyz, hv = [], [], []
    for i in range(n1):
        for j in range(n2):
            for k in range(n3):
                shift = i * geo.lattice[0] + j * geo.lattice[1] + k * geo.lattice[2]
                names += list(geo.names)
                xyz.append(geo.coords + shift)
                hv.append(geo.hirshfeld)
    lat = geo.lattice * np.array([[n1], [n2], [n3]], dtype=np.float64)
    return Geometry(names, np.concatenate(xyz), np.concatenate(hv), lat, geo.n_periodic)


def parse_settings(text: str) -> Settings:
    s = Settings()
    for tok, line in zip(_records(text), text.splitlines()):
        try:
            if "xc" in line:
                s.xc = int(tok[1]); s.given.add("xc")
            elif "mbd_supercell_cutoff" in line:
                s.mbd_supercell_cutoff = _real(tok[1]); s.given.add("mbd_supercell_cutoff")
            elif "mbd_cfdm_dip_cutoff" in line:
                s.mbd_cfdm_dip_cutoff = _real(tok[1]); s.given.add("mbd_cfdm_dip_cutoff")
            elif "mbd_scs_dip_cutoff" in line:
                s.mbd_scs_dip_cutoff = _real(tok[1]); s.given.add("mbd_scs_dip_cutoff")
            elif "mbd_scs_vacuum_axis" in line:
                s.mbd_scs_vacuum_axis = tuple(_logical(t) for t in tok[1:4]); s.given.add("mbd_scs_vacuum_axis")
            elif "nprow" in line:
                s.nprow = int(tok[1]); s.given.add("nprow")
            elif "npcol" in line:
                s.npcol = int(tok[1]); s.given.add("npcol")
        except (IndexError, ValueError) as exc:
            raise InputError(f"settings: cannot read {line.strip()!r}") from exc
    return s


def _fortran_f(v: float, w: int, d: int) -> str:
    """Fortran Fw.d (asterisks when the number does not fit)."""
    t = f"{v:{w}.{d}f}"
    return t if len(t) <= w else "*" * w


def _fortran_e(v: float, w: int, d: int) -> str:
    """Fortran Ew.d: 0.ddd...E+ee (E dropped for a three-digit exponent)."""
    if v == 0.0 or not np.isfinite(v):
        body = "0." + "0" * d + "E+00" if v == 0.0 else str(v)
    else:
        m, e = f"{abs(v):.{d - 1}E}".split("E")
        digits = m.replace(".", "")
        exp = int(e) + 1
        ee = f"E{exp:+03d}" if abs(exp) <= 99 else f"{exp:+04d}"
        body = ("-" if v < 0 else "") + "0." + digits + ee
    return body.rjust(w) if len(body) <= w else "*" * w


_RULE = "| ---------------------------------------------------------------------------"


def frequency_grid() -> np.ndarray:
    """The 21 imaginary frequencies of the Casimir-Polder integration (omega = 0
    and the 20 Gauss-Legendre nodes, gauss_legendre_grid UTILS.f90:1188-1211),
    in Hartree, as the engine uses them."""
    from .engine import frequency_grid as grid
    return grid()[0]


def format_report(geo: Geometry, res, omega_grid=None) -> str:
    """The MBD section of pmbd.x's report (MBD_at_rsSCS UTILS.f90:223-331 and
    get_mbd_rSCS UTILS.f90:753-755, 861) for a Result, line for line as the
    reference prints it: every line goes through output_string
    (UTILS.f90:1708-1714, list-directed WRITE of TRIM(info_str), hence the
    leading blank) with the reference's edit descriptors."""
    from .engine import N_FREQ
    grid = frequency_grid() if omega_grid is None else omega_grid
    out = []

    def put(text):
        out.append(" " + text.rstrip())

    put("  | Many-Body Dispersion (MBD@rsSCS) energy ")
    put("  | System dynamic molecular polarizability alpha(iw) (bohr^3)")
    put("  " + _RULE)
    put("  |  omega(Ha)   alpha_iso      alpha_xx       alpha_yy       alpha_zz")
    for f in range(N_FREQ):
        ev = res.mol_pol_eig[f]
        vals = (ev.sum() / 3.0, ev[0], ev[1], ev[2])
        put("  | " + _fortran_f(grid[f], 10, 6) + "".join(_fortran_e(x, 15, 6) for x in vals))
    put("  " + _RULE)
    put("  | System C6 coefficient    :  " + _fortran_f(res.c6_mol, 20, 8) + "    hartree bohr^6")
    put("  " + _RULE)
    put("  | Partitioned C6 (hartree bohr^6) | alpha (bohr^3)  of atom in system")
    put("  " + _RULE)
    for i, name in enumerate(geo.names):
        put("  | ATOM " + f"{i + 1:4d}" + "  " + f"{name:2.2s}" + _fortran_f(res.c6_eff[i], 12, 6) + " " * 6 +
            _fortran_f(res.alpha_eff[i], 12, 6))
    put("  " + _RULE)
    sc = res.supercell
    put("  | Creating super cell of dimension" + f"{sc[0]:3d} X {sc[1]:3d} X {sc[2]:3d}" + " in MBD calculation")
    put("  | containing" + f"{len(geo.names) * sc[0] * sc[1] * sc[2]:6d}" + "  atom")
    if res.nimag > 0:
        put("***WARNING: found " + f"{res.nimag:4d}" + " negative eigenvalues in MBD energy calculation.")
    # 27.211 is a REAL*4 literal (UTILS.f90:330)
    put("  | MBD@rsSCS energy   :" + _fortran_f(res.energy, 20, 9) + " Ha     " +
        _fortran_f(res.energy * float(np.float32(27.211)), 20, 9) + " eV")
    return "\n".join(out)
