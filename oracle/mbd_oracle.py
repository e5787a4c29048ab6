"""FP64 CPU oracle for the MBD@rsSCS path of pmbd.x (000Justin000/MBD).

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The product (``mbd_b200``) never calls it
and has no CPU fallback.

It restates, in vectorised numpy + LAPACK (scipy), the algorithm of
``UTILS.f90:153-1320`` (the reference's ``MBD_at_rsSCS``) literally:

* every periodic image inside the box ``ceil(cutoff/|a_k|)`` is tested
  against ``r <= cutoff`` (``UTILS.f90:561-579``, ``610-631``,
  ``1016-1035``, ``1073-1092``) and summed; the only images left out are
  short-range ones whose damping factor ``1 - 1/(1 + exp(-6(x - 1)))`` is
  exactly 0.0 in FP64 (``ZERO_DAMP_X``), which add exact zeros in the
  reference -- ``tests/test_oracle_golden.py`` checks that leaving them out
  changes no bit;
* only the lower triangle of the relay matrix / CFDM Hamiltonian is filled
  (``UTILS.f90:427-431``, ``799-803``) and the dense LAPACK calls read the
  lower triangle (``PDPOTRF('L')``/``PDPOTRS`` at ``UTILS.f90:469,473``,
  ``PDSYEV('N','L')`` at ``UTILS.f90:835``);
* single-precision Fortran literals (``beta=0.83`` ``UTILS.f90:357``, the
  Gauss-Legendre grid ``UTILS.f90:1189-1209`` and the free-atom table
  ``UTILS.f90:1339-1691``) are rounded to float32 before use, exactly as the
  Fortran compiler stores them.

Parity is pinned: ``tests/test_oracle_golden.py`` checks this module against
every value printed in the reference's ``examples/C6H6.out``,
``examples/graphene_111.out`` and ``examples/PBBA.out``.

Third-party dependency of the reference arithmetic: ScaLAPACK/LAPACK from
Intel MKL 2017 (``config/Makefile.in.thinkpad``) or IBM ESSL; not vendored.
Here LAPACK ``dpotrf``/``dpotrs``/``dsyevd``/``dsyev`` come from scipy's
OpenBLAS build.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla
from scipy.special import erf

F32 = lambda v: float(np.float32(v))  # noqa: E731  -- Fortran REAL*4 literal

# --- constants: init_constants, UTILS.f90:78-93 ---------------------------
BOHR = 0.52917721                       # UTILS.f90:85 (double literal)
PI = 3.14159265358979323846             # UTILS.f90:86
OTD = 0.33333333333333333333            # UTILS.f90:87
DEFAULT_SC_CUT = 25.0                   # UTILS.f90:81
DEFAULT_CFDM_CUT = 100.0                # UTILS.f90:82
DEFAULT_SCS_CUT = 120.0                 # UTILS.f90:83
C6_PREFACTOR = 0.954929658551372        # 3/pi as printed, UTILS.f90:288,313
HARTREE_EV = 27.211                     # UTILS.f90:330
N_FREQ = 21

# --- Gauss-Legendre grid, UTILS.f90:1188-1211 (REAL*4 literals) ------------
_GL = [
    (0.0000000, 0.0000000), (0.0392901, 0.0786611), (0.1183580, 0.0796400),
    (0.1989120, 0.0816475), (0.2820290, 0.0847872), (0.3689190, 0.0892294),
    (0.4610060, 0.0952317), (0.5600270, 0.1031720), (0.6681790, 0.1136050),
    (0.7883360, 0.1273500), (0.9243900, 0.1456520), (1.0817900, 0.1704530),
    (1.2684900, 0.2049170), (1.4966100, 0.2544560), (1.7856300, 0.3289620),
    (2.1691700, 0.4480920), (2.7106200, 0.6556060), (3.5457300, 1.0659600),
    (5.0273400, 2.0635700), (8.4489600, 5.6851000), (25.451700, 50.955800),
]
CASIMIR_OMEGA = np.array([F32(w) for w, _ in _GL])
CASIMIR_WEIGHT = np.array([F32(g) for _, g in _GL])

# --- free-atom reference data, get_vdw_param UTILS.f90:1324-1703 ----------
# (symbol, alpha0 [bohr^3], C6 [Ha bohr^6], R0 [bohr]); REAL*4 literals.
_VDW = [
    ("H", 4.5, 6.5, 3.1), ("He", 1.38, 1.46, 2.65), ("Li", 164.2, 1387.0, 4.16),
    ("Be", 38.0, 214.0, 4.17), ("B", 21.0, 99.5, 3.89), ("C", 12.0, 46.6, 3.59),
    ("N", 7.4, 24.2, 3.34), ("O", 5.4, 15.6, 3.19), ("F", 3.8, 9.52, 3.04),
    ("Ne", 2.67, 6.38, 2.91), ("Na", 162.7, 1556.0, 3.73), ("Mg", 71.0, 627.0, 4.27),
    ("Al", 60.0, 528.0, 4.33), ("Si", 37.0, 305.0, 4.2), ("P", 25.0, 185.0, 4.01),
    ("S", 19.6, 134.0, 3.86), ("Cl", 15.0, 94.6, 3.71), ("Ar", 11.1, 64.3, 3.55),
    ("K", 292.9, 3897.0, 3.71), ("Ca", 160.0, 2221.0, 4.65), ("Sc", 120.0, 1383.0, 4.59),
    ("Ti", 98.0, 1044.0, 4.51), ("V", 84.0, 832.0, 4.44), ("Cr", 78.0, 602.0, 3.99),
    ("Mn", 63.0, 552.0, 3.97), ("Fe", 56.0, 482.0, 4.23), ("Co", 50.0, 408.0, 4.18),
    ("Ni", 48.0, 373.0, 3.82), ("Cu", 42.0, 253.0, 3.76), ("Zn", 40.0, 284.0, 4.02),
    ("Ga", 60.0, 498.0, 4.19), ("Ge", 41.0, 354.0, 4.2), ("As", 29.0, 246.0, 4.11),
    ("Se", 25.0, 210.0, 4.04), ("Br", 20.0, 162.0, 3.93), ("Kr", 16.8, 129.6, 3.82),
    ("Rb", 319.2, 4691.0, 3.72), ("Sr", 199.0, 3170.0, 4.54), ("Y", 126.737, 1968.58, 4.8151),
    ("Zr", 119.97, 1677.91, 4.53), ("Nb", 101.603, 1263.61, 4.2365),
    ("Mo", 88.4225785, 1028.73, 4.099), ("Tc", 80.083, 1390.87, 4.076),
    ("Ru", 65.895, 609.754, 3.9953), ("Rh", 56.1, 469.0, 3.95), ("Pd", 23.68, 157.5, 3.66),
    ("Ag", 50.6, 339.0, 3.82), ("Cd", 39.7, 452.0, 3.99), ("In", 70.22, 707.046, 4.23198),
    ("Sn", 55.95, 587.417, 4.303), ("Sb", 43.67197, 459.322, 4.276), ("Te", 37.65, 396.0, 4.22),
    ("I", 35.0, 385.0, 4.17), ("Xe", 27.3, 285.9, 4.08), ("Cs", 427.12, 6582.08, 3.78),
    ("Ba", 275.0, 5727.0, 4.77), ("Hf", 99.52, 1274.8, 4.21), ("Ta", 82.53, 1019.92, 4.15),
    ("W", 71.041, 847.93, 4.08), ("Re", 63.04, 710.2, 4.02), ("Os", 55.055, 596.67, 3.84),
    ("Ir", 42.51, 359.1, 4.0), ("Pt", 39.68, 347.1, 3.92), ("Au", 36.5, 298.0, 3.86),
    ("Hg", 33.9, 392.0, 3.98), ("Tl", 69.92, 717.44, 3.91), ("Pb", 61.8, 697.0, 4.31),
    ("Bi", 49.02, 571.0, 4.32), ("Po", 45.013, 530.92, 4.097), ("At", 38.93, 457.53, 4.07),
    ("Rn", 33.54, 390.63, 4.23),
]
VDW_PARAMS = {s: (F32(a), F32(c), F32(r)) for s, a, c, r in _VDW}


class UnknownElement(ValueError):
    """get_vdw_param's ``case default`` (UTILS.f90:1693-1699) stops the run."""


def get_beta(xc: int) -> float:
    """Range-separation parameter, get_beta UTILS.f90:353-372 (REAL*4 literals)."""
    return {1: F32(0.83), 2: F32(0.85), 3: F32(0.85)}.get(xc, 1.0)


def get_vdw_param(sym: str):
    """Free-atom (alpha0, C6, R0), get_vdw_param UTILS.f90:1324-1703.

    The Fortran argument is CHARACTER*2, so longer names are truncated to two
    characters; the match is case-sensitive."""
    key = sym[:2].strip()
    if key not in VDW_PARAMS:
        raise UnknownElement(f"VdW parameters not defined for atom: {sym}")
    return VDW_PARAMS[key]


# --- inputs ---------------------------------------------------------------
@dataclass
class Settings:
    """setting.in keywords, defaults from init_constants UTILS.f90:78-93."""
    xc: int = 1
    mbd_supercell_cutoff: float = DEFAULT_SC_CUT
    mbd_cfdm_dip_cutoff: float = DEFAULT_CFDM_CUT
    mbd_scs_dip_cutoff: float = DEFAULT_SCS_CUT
    mbd_scs_vacuum_axis: tuple = (False, False, False)
    nprow: int = 1
    npcol: int = 1


@dataclass
class Geometry:
    """geometry.in contents; coordinates and lattice in Angstrom as read."""
    names: list
    coords: np.ndarray                   # (N, 3) Angstrom
    hirshfeld: np.ndarray                # (N,)
    lattice: np.ndarray = field(default_factory=lambda: np.zeros((3, 3)))  # rows = vectors, Angstrom
    n_periodic: int = 0


def _fortran_real(tok: str) -> float:
    return float(tok.lower().replace("d", "e"))


def _fortran_logical(tok: str) -> bool:
    t = tok.strip().lower().lstrip(".")
    return t.startswith("t")


def parse_geometry(text: str) -> Geometry:
    """Geometry reader, MBD_rsSCS.f90:66-89.

    Line 1: atom count; line 2: skipped; then one ``name x y z hirshfeld``
    record per atom; if the next record contains ``lattice_vector`` the
    system is periodic and three ``lattice_vector ax ay az`` records follow
    (each record's vector is a column of ``lattice_vector``)."""
    lines = text.splitlines()
    n = int(lines[0].split()[0])
    names, xyz, hv = [], [], []
    k = 2
    for _ in range(n):
        tok = lines[k].replace(",", " ").split()
        k += 1
        names.append(tok[0][:2])
        xyz.append([_fortran_real(t) for t in tok[1:4]])
        hv.append(_fortran_real(tok[4]))
    geo = Geometry(names, np.array(xyz, dtype=np.float64), np.array(hv, dtype=np.float64))
    if k < len(lines) and "lattice_vector" in lines[k]:
        geo.n_periodic = 3
        lat = np.zeros((3, 3))
        for i in range(3):
            tok = lines[k + i].replace(",", " ").split()
            lat[i] = [_fortran_real(t) for t in tok[1:4]]
        geo.lattice = lat
    return geo


def parse_settings(text: str) -> Settings:
    """Settings parser, MBD_rsSCS.f90:98-135: first-substring-match on each
    line in the order xc, mbd_supercell_cutoff, mbd_cfdm_dip_cutoff,
    mbd_scs_dip_cutoff, mbd_scs_vacuum_axis, nprow, npcol (INDEX >= 1)."""
    s = Settings()
    for line in text.splitlines():
        tok = line.replace(",", " ").split()
        if "xc" in line:
            s.xc = int(tok[1])
        elif "mbd_supercell_cutoff" in line:
            s.mbd_supercell_cutoff = _fortran_real(tok[1])
        elif "mbd_cfdm_dip_cutoff" in line:
            s.mbd_cfdm_dip_cutoff = _fortran_real(tok[1])
        elif "mbd_scs_dip_cutoff" in line:
            s.mbd_scs_dip_cutoff = _fortran_real(tok[1])
        elif "mbd_scs_vacuum_axis" in line:
            s.mbd_scs_vacuum_axis = tuple(_fortran_logical(t) for t in tok[1:4])
        elif "nprow" in line:
            s.nprow = int(tok[1])
        elif "npcol" in line:
            s.npcol = int(tok[1])
    return s


# --- image ranges: UTILS.f90:1215-1320 ------------------------------------
def get_scs_image(lat_bohr, n_periodic, vacuum, scs_cut):
    """Per-axis image range +-ceil(R_scs/|a_k|), 0 on vacuum axes
    (get_scs_image, UTILS.f90:1215-1248).  ``lat_bohr`` rows are vectors."""
    rng = np.zeros(3, dtype=np.int64)
    if n_periodic != 0:
        for k in range(3):
            if not vacuum[k]:
                rng[k] = math.ceil((scs_cut / BOHR) / math.sqrt(float(np.sum(lat_bohr[k] ** 2))))
    return rng


def get_supercell(lat_bohr, n_periodic, vacuum, sc_cut):
    """Supercell multiplicities and lattice (get_supercell, UTILS.f90:1252-1283)."""
    sc = np.ones(3, dtype=np.int64)
    if n_periodic != 0:
        for k in range(3):
            if not vacuum[k]:
                sc[k] = math.ceil((sc_cut / BOHR) / math.sqrt(float(np.sum(lat_bohr[k] ** 2))))
    return sc, lat_bohr * sc[:, None]


def get_cfdm_image(lat_sl_bohr, n_periodic, vacuum, cfdm_cut):
    """Supercell image range (get_cfdm_image, UTILS.f90:1287-1320)."""
    rng = np.zeros(3, dtype=np.int64)
    if n_periodic != 0:
        for k in range(3):
            if not vacuum[k]:
                rng[k] = math.ceil((cfdm_cut / BOHR) / math.sqrt(float(np.sum(lat_sl_bohr[k] ** 2))))
    return rng


def image_vectors(rng, lat_bohr):
    """All translations ``-(i a1 + j a2 + k a3)`` of the image box in the
    reference's loop order (i outer, k inner)."""
    ii, jj, kk = np.meshgrid(np.arange(-rng[0], rng[0] + 1), np.arange(-rng[1], rng[1] + 1),
                             np.arange(-rng[2], rng[2] + 1), indexing="ij")
    n = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1).astype(np.float64)
    return n, -(n @ lat_bohr)


# --- atomic response, get_alpha_and_sgm UTILS.f90:1157-1184 ----------------
def alpha_and_sigma(hirshfeld, c6_free, alpha_free, w):
    w_p = (4.0 / 3.0) * c6_free / (alpha_free * alpha_free)
    a_w = (hirshfeld * alpha_free) / (1.0 + (w * w) / (w_p * w_p))
    sgm = ((a_w / 3.0) * math.sqrt(2.0 / PI)) ** OTD
    return a_w, sgm


# --- dipole tensors ---------------------------------------------------------
def _sym6_from(d, r, a, b):
    """Return the 6 unique components (xx,xy,xz,yy,yz,zz) of a*(d d^T) + b*r^2*I."""
    dx, dy, dz = d
    return np.stack([a * dx * dx + b, a * dx * dy, a * dx * dz,
                     a * dy * dy + b, a * dy * dz, a * dz * dz + b])


def gaussian_dipole_tensor6(d, r, sgm12, rvdw12, beta):
    """Fermi-damped Gaussian dipole tensor, UTILS.f90:637-696.

    T = -(3 d d^T - r^2 I) zeta_l + d d^T zeta_r, times (1 - fermi);
    returns the six unique components, arrays broadcast over the inputs."""
    fermi_param = r / (beta * rvdw12)
    ratio = r / sgm12
    ex = np.exp(-(ratio * ratio))
    zeta_l = (erf(ratio) - (math.sqrt(4.0 / PI) * ratio * ex)) / r ** 5
    zeta_r = (math.sqrt(16.0 / PI) * ex) / (sgm12 * sgm12 * sgm12 * r * r)
    damp = 1.0 - (1.0 / (1.0 + np.exp(-6.0 * (fermi_param - 1.0))))
    a = (-3.0 * zeta_l + zeta_r) * damp
    b = (r * r * zeta_l) * damp
    return _sym6_from(d, r, a, b)


def lr_bare_dipole_tensor6(d, r, rvdw12, beta):
    """Long-range Fermi-damped bare dipole tensor, UTILS.f90:1098-1153:
    T = (r^2 I - 3 d d^T)/r^5 / (1 + exp(-6 (r/(beta R) - 1)))."""
    fermi = 1.0 / (1.0 + np.exp(-6.0 * (r / (beta * rvdw12) - 1.0)))
    inv5 = fermi / r ** 5
    return _sym6_from(d, r, -3.0 * inv5, r * r * inv5)


def _scatter6(mat, rows, cols, t6):
    """Write symmetric 3x3 blocks (6 unique comps, shape (6, P)) at atom-block
    (rows[p], cols[p]) of a 3N x 3N matrix (lower-triangle fill)."""
    comp = [(0, 0, 0), (1, 0, 1), (2, 0, 2), (3, 1, 1), (4, 1, 2), (5, 2, 2)]
    for c, a, b in comp:
        mat[3 * rows + a, 3 * cols + b] = t6[c]
        if a != b:
            mat[3 * rows + b, 3 * cols + a] = t6[c]


class _System:
    """Geometry in bohr plus derived per-atom data and image sets."""

    def __init__(self, geo: Geometry, st: Settings):
        self.names = geo.names
        self.N = len(geo.names)
        self.coords = geo.coords / BOHR                       # MBD_rsSCS.f90:211
        self.lat = geo.lattice / BOHR                         # MBD_rsSCS.f90:212 (rows = vectors)
        self.n_periodic = geo.n_periodic
        self.hirsh = geo.hirshfeld
        self.st = st
        self.beta = get_beta(st.xc)
        p = np.array([get_vdw_param(s) for s in geo.names])
        self.alpha0, self.c6free, self.r0 = p[:, 0], p[:, 1], p[:, 2]
        vac = st.mbd_scs_vacuum_axis
        self.scs_rng = get_scs_image(self.lat, self.n_periodic, vac, st.mbd_scs_dip_cutoff)
        self.supercell, self.lat_sl = get_supercell(self.lat, self.n_periodic, vac, st.mbd_supercell_cutoff)
        self.cfdm_rng = get_cfdm_image(self.lat_sl, self.n_periodic, vac, st.mbd_cfdm_dip_cutoff)
        self.rvdw_iso = (self.hirsh ** OTD) * self.r0         # UTILS.f90:254


def _pair_image_geometry(coords, ii, jj, shifts, cut, self_pairs):
    """Displacements d = r_i - r_j + shift for every (pair, shift), masked by
    r <= cut; for self pairs the zero shift is excluded (UTILS.f90:564)."""
    d0 = coords[ii] - coords[jj]                             # (P, 3)
    d = d0[:, None, :] + shifts[None, :, :]                  # (P, S, 3)
    r = np.sqrt(d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2])
    mask = r <= cut
    if self_pairs:
        mask &= r > 0.0
    p_idx, s_idx = np.nonzero(mask)
    return p_idx, d[p_idx, s_idx].T, r[p_idx, s_idx]


# An image whose Fermi factor 1 - 1/(1 + exp(-6 (r/(beta R) - 1))) rounds to
# exactly 0.0 in FP64 adds an exact zero to the reference's image sum
# (UTILS.f90:692): once exp(-6 (x - 1)) < 2^-53, 1 + exp(...) == 1.0.  Beyond
# x = r/(beta R) > ZERO_DAMP_X, exp(-6 (x - 1)) < exp(-37.5) = 5.2e-17 < 2^-53,
# so the sum does not change bit for bit when those images are left out.
ZERO_DAMP_X = 1.0 + 37.5 / 6.0


def relay_matrices(sysd: _System, freqs=range(N_FREQ), chunk_elems=4_000_000):
    """Lower-filled relay matrices A(iw_f) = alpha^-1 + T_SR for the given
    frequency indices (get_screened_alpha UTILS.f90:415-441 with
    scs_diag_block 543-587 and scs_offdiag_block 591-633).

    Every image of the reference's box that passes ``r <= cutoff`` is summed,
    except those whose short-range damping factor is exactly 0.0 in FP64
    (r > ZERO_DAMP_X * beta * R12): they add exact zeros in the reference.
    Returns (matrices dict f -> (3N,3N) array with lower triangle filled,
    alpha_omega dict f -> (N,))."""
    N = sysd.N
    freqs = list(freqs)
    _, shifts = image_vectors(sysd.scs_rng, sysd.lat)
    cut = sysd.st.mbd_scs_dip_cutoff / BOHR
    beta = sysd.beta
    rzero_atom = ZERO_DAMP_X * beta * sysd.rvdw_iso          # half of a pair's zero-damping radius
    if len(shifts) > 1:
        # images that can bring any pair inside min(cut, zero-damping radius)
        span = np.ptp(sysd.coords, axis=0)
        reach = min(cut, 2.0 * float(np.max(rzero_atom))) + float(np.sqrt(np.sum(span * span)))
        r_sh = np.sqrt(np.sum(shifts * shifts, axis=1))
        shifts = shifts[r_sh <= reach]
    alpha_w, sgm = {}, {}
    for f in freqs:
        alpha_w[f], sgm[f] = alpha_and_sigma(sysd.hirsh, sysd.c6free, sysd.alpha0, CASIMIR_OMEGA[f])
    mats = {f: np.zeros((3 * N, 3 * N)) for f in freqs}
    # off-diagonal pairs i > j, then diagonal self-image terms
    ii, jj = np.tril_indices(N, -1)
    per = max(1, chunk_elems // max(1, len(shifts)))
    for s in range(0, len(ii), per):
        pi_, pj_ = ii[s:s + per], jj[s:s + per]
        p_idx, d, r = _pair_image_geometry(sysd.coords, pi_, pj_, shifts, cut, False)
        keep = r <= rzero_atom[pi_[p_idx]] + rzero_atom[pj_[p_idx]]
        p_idx, d, r = p_idx[keep], d[:, keep], r[keep]
        gi, gj = pi_[p_idx], pj_[p_idx]
        r12 = sysd.rvdw_iso[gi] + sysd.rvdw_iso[gj]
        for f in freqs:
            s12 = np.sqrt(sgm[f][gi] * sgm[f][gi] + sgm[f][gj] * sgm[f][gj])
            t6 = gaussian_dipole_tensor6(d, r, s12, r12, beta)
            acc = np.zeros((6, len(pi_)))
            for c in range(6):
                acc[c] = np.bincount(p_idx, weights=t6[c], minlength=len(pi_))
            _scatter6(mats[f], pi_, pj_, acc)
    # diagonal blocks: images n != 0 of the atom itself, sigma_12 = sigma_i (UTILS.f90:571)
    if len(shifts) > 1:
        r_s = np.sqrt(np.sum(shifts * shifts, axis=1))
        keep = (r_s <= cut) & (r_s > 0.0) & (r_s <= 2.0 * float(np.max(rzero_atom)))
        ds, rs = shifts[keep].T, r_s[keep]
    else:
        ds, rs = np.zeros((3, 0)), np.zeros(0)
    # (atom, image) pairs inside the atom's own zero-damping radius 2 rzero_i
    a_idx, s_idx = np.nonzero(rs[None, :] <= 2.0 * rzero_atom[:, None])
    dd, rr = ds[:, s_idx], rs[s_idx]
    for f in freqs:
        acc = np.zeros((6, N))
        if len(rr):
            t6 = gaussian_dipole_tensor6(dd, rr, sgm[f][a_idx], 2.0 * sysd.rvdw_iso[a_idx], beta)
            for c in range(6):
                acc[c] = np.bincount(a_idx, weights=t6[c], minlength=N)
        inv = 1.0 / alpha_w[f]
        acc[0] += inv
        acc[3] += inv
        acc[5] += inv
        idx = np.arange(N)
        _scatter6(mats[f], idx, idx, acc)
    return mats, alpha_w


def screened_alpha(relay_lower: np.ndarray):
    """Cholesky ('L') + 3-RHS solve and reductions of get_screened_alpha
    (UTILS.f90:469-495): X = A^-1 [I;..;I]; alpha_i = tr X_i / 3; M = sum X_i.
    Returns (alpha (N,), mol_pol (3,3), info)."""
    n = relay_lower.shape[0]
    N = n // 3
    c, info = sla.lapack.dpotrf(relay_lower, lower=1, clean=0)
    b = np.tile(np.eye(3), (N, 1))
    x, info2 = sla.lapack.dpotrs(c, b, lower=1)
    xb = x.reshape(N, 3, 3)
    alpha = (xb[:, 0, 0] / 3.0 + xb[:, 1, 1] / 3.0) + xb[:, 2, 2] / 3.0
    return alpha, xb.sum(axis=0), info if info else info2


def cfdm_hamiltonian(sysd: _System, alpha_eff, c6_eff, chunk_elems=4_000_000):
    """Lower-filled CFDM Hamiltonian (get_mbd_rSCS UTILS.f90:731-807 with
    supercell_*_block 883-994, cfdm_*_block 998-1094, lr_bare_dipole_tensor
    1098-1153).  Layout: row = atom*3*nSL + cell*3 + xyz with
    cell = k*SL_j*SL_i + j*SL_i + i (UTILS.f90:915,921).
    Blocks depend on the atom pair and the cell difference only, so each
    distinct (pair, cell difference) block is evaluated once and placed at
    every (row cell, col cell) with that difference -- identical values."""
    N = sysd.N
    sl = sysd.supercell
    nsl = int(np.prod(sl))
    rvdw_eff = sysd.r0 * ((alpha_eff / sysd.alpha0) ** OTD)             # UTILS.f90:737
    omega = (4.0 / 3.0) * c6_eff / (alpha_eff ** 2.0)                   # UTILS.f90:739
    _, shifts = image_vectors(sysd.cfdm_rng, sysd.lat_sl)
    cut = sysd.st.mbd_cfdm_dip_cutoff / BOHR
    cells = [(i, j, k) for k in range(sl[2]) for j in range(sl[1]) for i in range(sl[0])]
    cell_index = {c: c[2] * sl[1] * sl[0] + c[1] * sl[0] + c[0] for c in cells}
    diffs = sorted({(a[0] - b[0], a[1] - b[1], a[2] - b[2]) for a in cells for b in cells})
    dim = 3 * N * nsl
    H = np.zeros((dim, dim))
    ii, jj = np.tril_indices(N, 0)
    per = max(1, chunk_elems // max(1, len(shifts)))
    for dvec in diffs:
        cshift = np.array(dvec, dtype=np.float64) @ sysd.lat
        zero_diff = dvec == (0, 0, 0)
        for s in range(0, len(ii), per):
            pi_, pj_ = ii[s:s + per], jj[s:s + per]
            # d = (r_i - r_j) + (rdis - cdis).a - n.A_SL
            d0 = (sysd.coords[pi_] - sysd.coords[pj_]) + cshift
            d = d0[:, None, :] + shifts[None, :, :]
            r = np.sqrt(d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2])
            mask = r <= cut
            if zero_diff:
                # same atom & same cell: only images n != 0 (cfdm_diag_block UTILS.f90:1019)
                mask &= ~((pi_ == pj_)[:, None] & (r == 0.0))
            p_idx, s_idx = np.nonzero(mask)
            gi, gj = pi_[p_idx], pj_[p_idx]
            dd, rr = d[p_idx, s_idx].T, r[p_idx, s_idx]
            t6 = lr_bare_dipole_tensor6(dd, rr, rvdw_eff[gi] + rvdw_eff[gj], sysd.beta)
            pref = omega[gi] * omega[gj] * np.sqrt(alpha_eff[gi] * alpha_eff[gj])
            same = gi == gj
            pref[same] = omega[gi[same]] * omega[gi[same]] * alpha_eff[gi[same]]
            t6 = t6 * pref
            acc = np.zeros((6, len(pi_)))
            for c in range(6):
                acc[c] = np.bincount(p_idx, weights=t6[c], minlength=len(pi_))
            if zero_diff:
                diag = pi_ == pj_
                w2 = omega[pi_[diag]] ** 2
                acc[0, diag] += w2
                acc[3, diag] += w2
                acc[5, diag] += w2
            comp = [(0, 0, 0), (1, 0, 1), (2, 0, 2), (3, 1, 1), (4, 1, 2), (5, 2, 2)]
            for rc in cells:
                cc = (rc[0] - dvec[0], rc[1] - dvec[1], rc[2] - dvec[2])
                if cc not in cell_index:
                    continue
                ro = 3 * nsl * pi_ + 3 * cell_index[rc]
                co = 3 * nsl * pj_ + 3 * cell_index[cc]
                for c, a, b in comp:
                    H[ro + a, co + b] = acc[c]
                    if a != b:
                        H[ro + b, co + a] = acc[c]
    return H, omega, rvdw_eff


@dataclass
class Result:
    energy: float
    nimag: int
    info: int
    alpha_eff: np.ndarray          # (N,) screened static polarizability
    c6_eff: np.ndarray             # (N,) screened C6
    alpha_iw: np.ndarray           # (21, N) screened alpha at each frequency (row 0 = static)
    mol_pol: np.ndarray            # (21, 3, 3) molecular polarizability tensors
    mol_pol_eig: np.ndarray        # (21, 3) DSYEV('V','U') eigenvalues
    c6_mol: float
    supercell: tuple
    status: str = "ok"
    omega: np.ndarray = None
    eigenvalues: np.ndarray = None


def mbd_at_rsscs(geo: Geometry, st: Settings | None = None, keep_eigenvalues=False) -> Result:
    """MBD@rsSCS energy, screened alpha and C6 (MBD_at_rsSCS, UTILS.f90:153-349,
    get_mbd_rSCS 700-879)."""
    st = st or Settings()
    sysd = _System(geo, st)
    N = sysd.N
    mats, _ = relay_matrices(sysd)
    alpha_iw = np.zeros((N_FREQ, N))
    mol_pol = np.zeros((N_FREQ, 3, 3))
    mol_eig = np.zeros((N_FREQ, 3))
    mol_c6 = 0.0
    info = 0
    for f in range(N_FREQ):
        a, m, inf = screened_alpha(mats.pop(f))
        info = info or inf
        alpha_iw[f] = a
        mol_pol[f] = m
        ev = sla.eigh(m, lower=False, eigvals_only=True, driver="ev")   # DSYEV('V','U') UTILS.f90:273
        mol_eig[f] = ev
        if f >= 1:
            mol_c6 = mol_c6 + (CASIMIR_WEIGHT[f] * (np.sum(ev) / 3.0) ** 2)    # UTILS.f90:275
    alpha_eff = alpha_iw[0]
    c6_atom = np.zeros(N)
    for f in range(1, N_FREQ):                                          # UTILS.f90:306-308
        c6_atom = c6_atom + (CASIMIR_WEIGHT[f] * alpha_iw[f] ** 2)
    c6_eff = c6_atom * C6_PREFACTOR
    if info != 0 or not np.all(alpha_eff > 0.0):
        # A non-SPD relay (PDPOTRF info ignored at UTILS.f90:469) or a screened
        # alpha <= 0 makes R_vdW_eff = R0 (alpha/alpha0)^(1/3) undefined
        # (UTILS.f90:737); the reference then feeds NaN into PDSYEV.  The
        # restatement stops here and reports why.
        return Result(energy=float("nan"), nimag=0, info=info, alpha_eff=alpha_eff, c6_eff=c6_eff,
                      alpha_iw=alpha_iw, mol_pol=mol_pol, mol_pol_eig=mol_eig,
                      c6_mol=C6_PREFACTOR * mol_c6, supercell=tuple(int(x) for x in sysd.supercell),
                      status="relay_not_spd" if info != 0 else "nonpositive_alpha")
    H, omega, _ = cfdm_hamiltonian(sysd, alpha_eff, c6_eff)
    ev = sla.eigh(H, lower=True, eigvals_only=True, driver="evd")
    e_nonint = float(np.sum(3.0 * omega))
    pos = ev >= 0.0
    nimag = int(np.count_nonzero(~pos))
    e_int = float(np.sum(np.sqrt(ev[pos])))
    nsl = int(np.prod(sysd.supercell))
    energy = (0.5 * e_int) / nsl - (0.5 * e_nonint)                    # UTILS.f90:858
    return Result(energy=energy, nimag=nimag, info=info, alpha_eff=alpha_eff, c6_eff=c6_eff,
                  alpha_iw=alpha_iw, mol_pol=mol_pol, mol_pol_eig=mol_eig,
                  c6_mol=C6_PREFACTOR * mol_c6, supercell=tuple(int(x) for x in sysd.supercell),
                  omega=omega, eigenvalues=ev if keep_eigenvalues else None)


# --- report parsing (for golden fixtures) ----------------------------------
_E_RE = re.compile(r"MBD@rsSCS energy\s*:\s*(-?[0-9.]+)\s*Ha")
_C6_RE = re.compile(r"C6 coefficient\s*:\s*(-?[0-9.]+)")
_ATOM_RE = re.compile(r"\|\s*ATOM\s+(\d+)\s+(\S+)\s+(-?[0-9.]+)\s+(-?[0-9.]+)")
_POL_RE = re.compile(r"^\s*\|\s+([0-9.]+)\s+([0-9.E+-]+)\s+([0-9.E+-]+)\s+([0-9.E+-]+)\s+([0-9.E+-]+)\s*$")


def parse_report(text: str) -> dict:
    """Extract the printed fields of a pmbd.x report (UTILS.f90:278,288,310,330)."""
    out = {"atoms": {}, "pol": []}
    for line in text.splitlines():
        m = _E_RE.search(line)
        if m:
            out["energy"] = float(m.group(1))
        m = _C6_RE.search(line)
        if m:
            out["c6_mol"] = float(m.group(1))
        m = _ATOM_RE.search(line)
        if m:
            out["atoms"][int(m.group(1))] = (m.group(2), float(m.group(3)), float(m.group(4)))
        m = _POL_RE.match(line)
        if m:
            out["pol"].append([float(m.group(k)) for k in range(1, 6)])
    return out
