"""GPU parity of the benchmarked workloads against the FP64 oracle.

The bench times three isolated {H,C,N,O} clusters (N = 500, 1000, 2000;
seeds 0, 1, 2) in one batch, and periodic boxes at cut-offs 120/100/25 A.
The oracle needs seconds to minutes on these, so its results are stored in
tests/golden/wl_*.npz (made by tests/golden/make_workload_golden.py, each
with a fingerprint of the generated input that is checked here first).

Every mode the bench reports is compared, through the C ABI, on exactly the
bench's inputs and call path (one batch: upload, compute, download; a second
compute replays the captured CUDA graph):

* plain FP64:  |E - E_oracle| <= 1e-9 Ha, C6 and alpha within 1e-9 relative;
* mixed (3xTF32 + FP64 refinement) and mixed_learned (network warm start +
  block-CG), with the network on and off: |E - E_oracle| <= 1e-6 Ha, C6
  within 1e-6 relative (the accuracy bars of the mixed forms), plus the
  residual gate: every frequency's relay residual <= 1e-10.

The periodic box (256 atoms, 2x2x2 supercell, 6144-wide Hamiltonian) runs
the image sums out to the periodic workload's full cut-offs.
"""
import os

import numpy as np
import pytest

from tests.golden.make_workload_golden import CASES, fingerprint

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
E_TOL = 1e-6
C6_RTOL = 1e-6
PLAIN_E_TOL = 1e-9
PLAIN_RTOL = 1e-9
CLUSTERS = ("cluster500_s0", "cluster1000_s1", "cluster2000_s2")


def _load(name):
    fx = np.load(os.path.join(GOLDEN, f"wl_{name}.npz"))
    geo, st = CASES[name]()
    assert str(fx["fingerprint"]) == fingerprint(geo, st), f"generator drift for {name}"
    return geo, st, fx


def _check(res, fx, mode):
    e_tol = PLAIN_E_TOL if mode == "plain" else E_TOL
    rtol = PLAIN_RTOL if mode == "plain" else C6_RTOL
    assert res.status == 0, res.status
    assert abs(res.energy - float(fx["energy"])) <= e_tol, (mode, res.energy, float(fx["energy"]))
    assert abs(res.c6_mol - float(fx["c6_mol"])) <= rtol * abs(float(fx["c6_mol"]))
    assert res.nimag == int(fx["nimag"])
    assert list(res.supercell) == [int(x) for x in fx["supercell"]]
    np.testing.assert_allclose(res.c6_eff, fx["c6_eff"], rtol=rtol, atol=0)
    np.testing.assert_allclose(res.alpha_eff, fx["alpha_eff"], rtol=rtol, atol=0)
    np.testing.assert_allclose(res.alpha_iw[list(fx["iw_freqs"])], fx["alpha_iw"], rtol=10 * rtol, atol=1e-12)
    np.testing.assert_allclose(res.mol_pol_eig, fx["mol_pol_eig"], rtol=10 * rtol, atol=1e-10)
    if mode != "plain":
        assert res.refine_iters > 0          # the fast solve passed the residual gate (no fallback)
        assert res.err_est[0] <= 1e-10


@pytest.fixture(scope="module")
def engine():
    """One context with a network trained on small clusters and boxes of the
    workloads' generators (other seeds), as the bench trains it."""
    from mbd_b200 import Engine
    from mbd_b200 import synthetic as sy
    eng = Engine(0)
    rng = np.random.default_rng(4242)
    train = [sy.cluster(int(n), seed=200000 + k) for k, n in enumerate(rng.integers(50, 300, size=24))]
    train += [sy.periodic_box(int(n), seed=300000 + k) for k, n in enumerate(rng.integers(50, 120, size=8))]
    loss = eng.learned_train([g for g, _ in train], [s for _, s in train], epochs=6, lr=1e-3, seed=3)
    assert np.all(np.isfinite(loss))
    yield eng
    eng.close()


def _run_batch(engine, items, mode, network=True):
    """The bench's call path: upload once, compute twice (the second replays
    the captured graph), download."""
    engine.use_network(network)
    try:
        assert engine.upload([g for g, _ in items], [s for _, s in items]) == 0
        for _ in range(2):
            assert engine.compute(mode) == 0
        code, res = engine.download()
        replayed = engine.stats().get("graph_replayed")
    finally:
        engine.use_network(True)
    assert code == 0, code
    return res, replayed


@pytest.mark.parametrize("mode,network", [("plain", True), ("mixed", True), ("mixed_learned", True),
                                          ("mixed_learned", False)])
def test_headline_clusters_vs_oracle(engine, mode, network):
    loaded = [_load(nm) for nm in CLUSTERS]
    res, replayed = _run_batch(engine, [(g, s) for g, s, _ in loaded], mode, network)
    for r, (_, _, fx) in zip(res, loaded):
        _check(r, fx, mode)


@pytest.mark.parametrize("mode,network", [("plain", True), ("mixed", True), ("mixed_learned", True),
                                          ("mixed_learned", False)])
def test_periodic_box_full_cutoffs_vs_oracle(engine, mode, network):
    geo, st, fx = _load("box256_s3")
    assert (st.mbd_scs_dip_cutoff, st.mbd_cfdm_dip_cutoff, st.mbd_supercell_cutoff) == (120.0, 100.0, 25.0)
    res, _ = _run_batch(engine, [(geo, st)], mode, network)
    _check(res[0], fx, mode)


def test_headline_clusters_one_call_each_vs_oracle(engine):
    """mbd_rsscs_energy (one geometry per call, host buffers) on the largest
    headline cluster in the headline mode."""
    geo, st, fx = _load("cluster2000_s2")
    _check(engine.energy(geo, st, mode="mixed_learned"), fx, "mixed_learned")


def test_two_phase_fp32_cg_headline_clusters():
    """The mixed-precision block-CG of the learned mode, forced on
    (MBD_B200_CG_FP32=1; by default it runs where its copy fits: matrix
    passes on an FP32 copy of the relay matrices,
    products in FP32, a restart from the FP64 residual between its two
    phases) on the headline clusters, twice (the second compute replays the
    captured graph with the phase lengths of the first): the mixed forms'
    bars against the oracle fixtures and the FP64 residual gate."""
    from mbd_b200 import Engine
    loaded = [_load(nm) for nm in CLUSTERS]
    old = os.environ.get("MBD_B200_CG_FP32")
    os.environ["MBD_B200_CG_FP32"] = "1"
    try:
        eng = Engine(0)
    finally:
        if old is None:
            del os.environ["MBD_B200_CG_FP32"]
        else:
            os.environ["MBD_B200_CG_FP32"] = old
    with eng:
        eng.use_network(False)
        assert eng.upload([g for g, _, _ in loaded], [s for _, s, _ in loaded]) == 0
        for rep in range(2):
            assert eng.compute("mixed_learned") == 0
            code, res = eng.download()
            assert code == 0
            for r, (_, _, fx) in zip(res, loaded):
                _check(r, fx, "mixed_learned")
        assert eng.stats()["graph_replayed"]
