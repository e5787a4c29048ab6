"""Dense -> band panels by TSQR with Householder reconstruction
(MBD_B200_PANEL_QR=tsqr) against LAPACK and the oracle fixtures.

Covers random symmetric matrices across panel and cluster sizes, a diagonal
matrix (every panel is zero: tau = 0 everywhere), a matrix whose off-diagonal
part has rank 2 (rank-deficient panels), and the headline clusters' energies
in plain FP64 (1e-9 Ha against the oracle)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from mbd_b200 import Engine
    old = os.environ.get("MBD_B200_PANEL_QR")
    os.environ["MBD_B200_PANEL_QR"] = "tsqr"
    try:
        e = Engine(0)
    finally:
        if old is None:
            del os.environ["MBD_B200_PANEL_QR"]
        else:
            os.environ["MBD_B200_PANEL_QR"] = old
    yield e
    e.close()


def _check(w, ref):
    n = len(ref)
    np.testing.assert_allclose(np.sort(w), ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max()) * n)


@pytest.mark.parametrize("n", [64, 97, 300, 1000, 1536, 3000, 6000])
def test_tsqr_random(eng, n):
    rng = np.random.default_rng(n + 1)
    M = rng.standard_normal((n, n))
    S = (M + M.T) / 2
    _check(eng.eigvalsh(np.tril(S)), np.linalg.eigvalsh(S))


def test_tsqr_zero_and_rank_deficient_panels(eng):
    rng = np.random.default_rng(5)
    n = 2000
    d = rng.uniform(-3, 3, n)
    _check(eng.eigvalsh(np.diag(d)), np.sort(d))
    u = rng.standard_normal((n, 2))
    S = np.diag(d) + u @ u.T
    _check(eng.eigvalsh(np.tril(S)), np.linalg.eigvalsh(S))


def test_tsqr_headline_clusters_vs_oracle(eng):
    from tests.golden.make_workload_golden import CASES, fingerprint
    names = ("cluster500_s0", "cluster1000_s1", "cluster2000_s2")
    items = [CASES[nm]() for nm in names]
    res = eng.energy_batch([g for g, _ in items], [s for _, s in items], "plain")
    for nm, (g, s), r in zip(names, items, res):
        fx = np.load(os.path.join(os.path.dirname(__file__), "golden", f"wl_{nm}.npz"))
        assert str(fx["fingerprint"]) == fingerprint(g, s)
        assert r.status == 0 and abs(r.energy - float(fx["energy"])) <= 1e-9
