"""GPU tests of mbd_rsscs_eigh, the eigenvectors of a symmetric matrix (the
PDSYEV call of UTILS.f90:835 with JOBZ = 'V'; the reference asks for 'N').

Every case is checked against LAPACK through numpy: eigenvalues, the
residual H Z - Z diag(w), orthonormality Z^T Z = I and, where eigenvalues
are well separated, the vectors themselves up to sign.  Cases: tiny orders,
random matrices whose order is not a multiple of the 32-column panels or
the 128-reflector blocks, exactly degenerate spectra (clusters solved by
inverse iteration), a block-diagonal matrix whose tridiagonal form splits, a
diagonal and a zero matrix (no reflections at all), and the CFDM
Hamiltonian of the 500-atom fixture cluster, whose MBD energy the vectors'
Rayleigh quotients must reproduce.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
EPS = np.finfo(float).eps


@pytest.fixture(scope="module")
def engine():
    from mbd_b200 import Engine
    eng = Engine(0)
    yield eng
    eng.close()


def _sym(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    return 0.5 * (a + a.T)


def _check(H, w, Z, name=""):
    n = H.shape[0]
    ref = np.linalg.eigvalsh(H)
    scale = max(np.abs(ref).max(), 1e-300)
    slack = max(1.0, np.sqrt(n))
    err_w = np.abs(w - ref).max() / scale
    res = np.abs(H @ Z - Z * w).max() / scale
    orth = np.abs(Z.T @ Z - np.eye(n)).max()
    print(f"{name} n={n}: eigenvalues {err_w:.1e}, residual {res:.1e}, orthogonality {orth:.1e}")
    assert np.all(np.diff(w) >= 0.0)
    assert err_w <= 20 * EPS * slack
    assert res <= 50 * EPS * slack
    assert orth <= 50 * EPS * slack
    return ref


@pytest.mark.parametrize("n", [1, 2, 3, 5, 33, 130, 257, 1000])
def test_random_matches_lapack(engine, n):
    H = _sym(n, seed=n)
    w, Z = engine.eigh(H)
    _check(H, w, Z, "random")
    # separated eigenvalues: the same vectors as LAPACK's up to sign
    ref_w, ref_Z = np.linalg.eigh(H)
    gaps = np.diff(ref_w)
    iso = [k for k in range(n) if (k == 0 or gaps[k - 1] > 1e-6) and (k == n - 1 or gaps[k] > 1e-6)]
    dots = np.abs(np.einsum("ik,ik->k", Z[:, iso], ref_Z[:, iso]))
    assert np.all(np.abs(dots - 1.0) <= 1e-9), dots.min()


def test_lower_triangle_only(engine):
    H = _sym(90, seed=4)
    junk = H.copy()
    junk[np.triu_indices(90, 1)] = 1e30   # the strict upper triangle is not read
    w, Z = engine.eigh(junk)
    _check(H, w, Z, "lower")


def test_degenerate_spectrum(engine):
    """Multiplicities 6, 4, 3 and 2 among simple eigenvalues: every
    eigenspace is spanned orthonormally (projectors equal LAPACK's)."""
    n = 200
    rng = np.random.default_rng(11)
    lam = np.concatenate([np.full(6, -1.5), np.full(4, 0.25), np.full(3, 2.0), np.full(2, 3.5),
                          rng.uniform(-4.0, 4.0, n - 15)])
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    H = (Q * lam) @ Q.T
    H = 0.5 * (H + H.T)
    w, Z = engine.eigh(H)
    _check(H, w, Z, "degenerate")
    for v, mult in ((-1.5, 6), (0.25, 4), (2.0, 3), (3.5, 2)):
        sel = np.abs(w - v) < 1e-9
        assert sel.sum() == mult
        P = Z[:, sel] @ Z[:, sel].T
        Pref = Q[:, lam == v] @ Q[:, lam == v].T
        assert np.abs(P - Pref).max() <= 1e-10


def test_split_tridiagonal(engine):
    """Three identical uncoupled blocks: the reduction's off-diagonal has
    exact zeros and every eigenvalue is triple."""
    B = _sym(40, seed=2)
    H = np.kron(np.eye(3), B)
    w, Z = engine.eigh(H)
    _check(H, w, Z, "split")


def test_diagonal_and_zero(engine):
    D = np.diag(np.linspace(-3.0, 5.0, 77))
    w, Z = engine.eigh(D)
    _check(D, w, Z, "diagonal")
    w0, Z0 = engine.eigh(np.zeros((12, 12)))
    assert np.abs(w0).max() <= 1e-290   # the bisection's interval ends, not exactly 0
    assert np.abs(Z0.T @ Z0 - np.eye(12)).max() <= 1e-13


def test_cfdm_hamiltonian_500_atoms(engine):
    """The CFDM Hamiltonian of the 500-atom fixture cluster (n = 1500): the
    vectors' Rayleigh quotients give the oracle's MBD energy
    (UTILS.f90:839-858) to 1e-9 Ha."""
    from oracle import mbd_oracle as mo
    from tests.golden.make_workload_golden import CASES, oracle_inputs
    geo, st = CASES["cluster500_s0"]()
    og, os_ = oracle_inputs(geo, st)
    fx = np.load(os.path.join(HERE, "golden", "wl_cluster500_s0.npz"))
    H, omega, _ = mo.cfdm_hamiltonian(mo._System(og, os_), fx["alpha_eff"], fx["c6_eff"])
    L = np.tril(H)
    Hs = L + np.tril(L, -1).T
    w, Z = engine.eigh(L)
    _check(Hs, w, Z, "cfdm")
    rq = np.einsum("ik,ik->k", Z, Hs @ Z)
    e = 0.5 * np.sum(np.sqrt(rq[rq >= 0.0])) - 0.5 * np.sum(3.0 * omega)
    assert abs(e - float(fx["energy"])) <= 1e-9
