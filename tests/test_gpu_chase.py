"""Band -> tridiagonal bulge chasing: the cluster-resident kernel (the band
in the distributed shared memory of one thread-block cluster, sweeps advanced
in lock-step wavefront steps) against the flag-synchronised kernel and LAPACK.

Both kernels apply the same reflectors to the same band entries; they take
their sums in different orders, so their eigenvalues agree to rounding (a
schedule error -- a task reading a block before its predecessor wrote it --
shows up as an error many orders of magnitude larger).  Both must match
LAPACK's dsyevd to the tolerance of the eigenvalue parity tests.  Sizes cover
the smallest bands, bands split over one and several CTAs (64-row minimum per
CTA, tasks that straddle two CTAs) and the largest band a 16-CTA cluster
holds here.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _engine(cluster_chase: bool):
    from mbd_b200 import Engine
    old = os.environ.get("MBD_B200_CLUSTER_CHASE")
    os.environ["MBD_B200_CLUSTER_CHASE"] = "1" if cluster_chase else "0"
    try:
        return Engine(0)
    finally:
        if old is None:
            del os.environ["MBD_B200_CLUSTER_CHASE"]
        else:
            os.environ["MBD_B200_CLUSTER_CHASE"] = old


@pytest.fixture(scope="module")
def engines():
    a, b = _engine(True), _engine(False)
    yield a, b
    a.close()
    b.close()


def _sym(n, seed):
    rng = np.random.default_rng(seed)
    M = rng.standard_normal((n, n))
    return (M + M.T) / 2


@pytest.mark.parametrize("n", [3, 4, 33, 63, 64, 65, 97, 128, 129, 300, 700, 1500, 3000, 6000])
def test_cluster_chase_equals_flag_chase_and_lapack(engines, n):
    clu, flag = engines
    S = _sym(n, seed=n)
    w_clu = clu.eigvalsh(np.tril(S))
    w_flag = flag.eigvalsh(np.tril(S))
    ref = np.linalg.eigvalsh(S)
    scale = max(1.0, np.abs(ref).max())
    np.testing.assert_allclose(w_clu, w_flag, rtol=0, atol=1e-14 * scale * n)
    np.testing.assert_allclose(w_clu, ref, rtol=0, atol=1e-12 * scale * n)
    np.testing.assert_allclose(w_flag, ref, rtol=0, atol=1e-12 * scale * n)


def test_cluster_chase_batch_equals_flag_chase(engines):
    """An uneven batch (matrices of 36 .. 6000 rows in one cluster launch,
    the small ones on fewer CTAs of the cluster): energies equal to those of
    the flag-synchronised chase to rounding (1e-9 Ha, the plain-mode bar)."""
    from mbd_b200 import synthetic as sy
    clu, flag = engines
    items = [sy.cluster(n, seed=40 + n) for n in (2000, 12, 25, 140, 700)]
    a = clu.energy_batch([g for g, _ in items], [s for _, s in items], "plain")
    b = flag.energy_batch([g for g, _ in items], [s for _, s in items], "plain")
    for ra, rb in zip(a, b):
        assert ra.status == rb.status == 0
        assert abs(ra.energy - rb.energy) <= 1e-9
        assert ra.nimag == rb.nimag


def test_autotune_choices_and_results():
    """mbd_rsscs_autotune picks, per size class up to the announced size, a
    panel-QR rows-per-CTA target among its candidates and the faster chase
    (flag-synchronised, or cluster-resident at a cluster size that holds the
    band); eigenvalues and energies computed afterwards match LAPACK and the
    oracle fixtures."""
    from mbd_b200 import Engine
    with Engine(0) as eng:
        choices = eng.autotune(3000)
        assert [c["n"] for c in choices] == [512, 1024, 2048, 3000]
        for c in choices:
            assert c["panel_rows_per_cta"] in (48, 96, 192, 384)
            assert c["panel_qr"] in ("householder", "tsqr")
            assert c["dense_to_band_ms"] > 0 and c["flag_chase_ms"] > 0 and c["cluster_chase_ms"] > 0
            if c["chase"] == "flag":
                assert c["chase_ms"] == c["flag_chase_ms"] <= c["cluster_chase_ms"]
            else:
                ctas = int(c["chase"][len("cluster"):])
                assert 1 <= ctas <= 16 and ctas * 378 >= c["n"]
                assert c["chase_ms"] == c["cluster_chase_ms"] < c["flag_chase_ms"]
        S = _sym(3000, seed=77)
        w = eng.eigvalsh(np.tril(S))
        ref = np.linalg.eigvalsh(S)
        np.testing.assert_allclose(w, ref, rtol=0, atol=1e-12 * np.abs(ref).max() * 3000)
        from tests.golden.make_workload_golden import CASES
        geo, st = CASES["cluster1000_s1"]()
        fx = np.load(os.path.join(os.path.dirname(__file__), "golden", "wl_cluster1000_s1.npz"))
        r = eng.energy(geo, st, mode="plain")
        assert r.status == 0 and abs(r.energy - float(fx["energy"])) <= 1e-9
