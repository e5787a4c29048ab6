"""GPU tests of MBD_MODE_MIXED_LEARNED: block-CG relay solve started from a
message-passing network's prediction of each atom's screened-polarizability
block.

* the network's CUDA kernels (forward, loss, backward) against the float64
  numpy restatement in oracle/gnn_oracle.py, on the same inputs;
* the mode's energies, C6 and alpha against the plain FP64 path and the
  oracle, with the network off and on;
* training on the GPU lowers the loss, and the trained network lowers the
  number of CG iterations against starting from zero (the method without it).
"""
import numpy as np
import pytest

from oracle import gnn_oracle as gn

pytestmark = pytest.mark.gpu

E_TOL = 1e-6
C6_RTOL = 1e-6


@pytest.fixture(scope="module")
def engine():
    from mbd_b200 import Engine
    eng = Engine(0)
    yield eng
    eng.close()


def _toy(seed=0, n=16, F=3):
    rng = np.random.default_rng(seed)
    coords = rng.uniform(0.0, 10.0, size=(n, 3))
    off, nbr, d = gn.neighbours(coords)
    species = rng.integers(0, 5, size=n)
    hirsh = rng.uniform(0.6, 1.0, size=n)
    alpha = rng.uniform(1.0, 12.0, size=(F, n))
    omega = np.array([0.0, 0.4, 1.3])[:F]
    x = gn.node_features(species, hirsh, alpha, omega)
    S_true = rng.standard_normal((F * n, 3, 3)) * 0.1 + np.eye(3)
    return x, F, off, nbr, d, S_true


def test_network_kernels_match_cpu_oracle(engine):
    x, F, off, nbr, d, S_true = _toy()
    assert len(nbr) > 20
    rng = np.random.default_rng(3)
    p = (gn.init_params(2) + 0.05 * rng.standard_normal(gn.N_PARAMS)).astype(np.float32).astype(np.float64)
    n = len(off) - 1
    S_ref, _ = gn.forward(p, x, F, off, nbr, d)
    loss_ref, g_ref = gn.loss_and_grad(p, x, F, off, nbr, d, S_true)
    S_gpu, g_gpu, loss_gpu = engine.learned_eval(p, n, F, off, nbr, d, x, S_true)
    np.testing.assert_allclose(S_gpu, S_ref, rtol=2e-4, atol=2e-5)
    assert loss_gpu == pytest.approx(loss_ref, rel=1e-4)
    # every parameter block's gradient, relative to the block's scale (FP32 kernels)
    o = 0
    for name, shp in gn.LAYOUT:
        k = int(np.prod(shp))
        a, b = g_gpu[o:o + k].astype(np.float64), g_ref[o:o + k]
        scale = max(np.abs(b).max(), 1e-6)
        assert np.abs(a - b).max() <= 2e-3 * scale, (name, np.abs(a - b).max(), scale)
        o += k


def test_no_network_is_an_error(engine):
    from mbd_b200 import Engine, MbdError
    from mbd_b200 import synthetic as sy
    with Engine(0) as fresh:
        geo, st = sy.cluster(20, seed=1)
        with pytest.raises(MbdError) as exc:
            fresh.energy(geo, st, mode="mixed_learned")
        assert exc.value.code == 12


def _train_set(count, lo, hi, seed):
    from mbd_b200 import synthetic as sy
    rng = np.random.default_rng(seed)
    return [sy.periodic_box(int(n), seed=seed * 1000 + k, scs_cut=20.0, cfdm_cut=15.0, sc_cut=5.0)
            for k, n in enumerate(rng.integers(lo, hi + 1, size=count))]


@pytest.fixture(scope="module")
def trained(engine):
    items = _train_set(24, 40, 110, seed=5)
    loss = engine.learned_train([g for g, _ in items], [s for _, s in items], epochs=25, lr=3e-3, seed=1)
    return loss


def test_training_lowers_the_loss(trained):
    loss = trained
    assert np.all(np.isfinite(loss))
    assert loss[-1] < 0.5 * loss[0], loss


def test_cg_without_network_matches_plain(engine):
    from mbd_b200 import synthetic as sy
    items = [sy.cluster(n, seed=60 + n) for n in (30, 140)] + _train_set(2, 60, 90, seed=9)
    geos, sets = [g for g, _ in items], [s for _, s in items]
    engine.use_network(False)
    try:
        lr = engine.energy_batch(geos, sets, "mixed_learned")
    finally:
        engine.use_network(True)
    pl = engine.energy_batch(geos, sets, "plain")
    for a, b in zip(lr, pl):
        assert a.status == 0 and b.status == 0
        assert abs(a.energy - b.energy) <= E_TOL
        assert abs(a.c6_mol - b.c6_mol) <= C6_RTOL * abs(b.c6_mol)
        np.testing.assert_allclose(a.alpha_iw, b.alpha_iw, rtol=1e-8)
        assert 0 < a.refine_iters < 64
        assert a.err_est[0] <= 1e-10


def test_network_graph_matches_oracle_neighbours(engine):
    """The network's neighbour lists, built on the GPU at the first learned
    compute of a batch, have the edges of the oracle's brute-force lists: a
    cluster, a periodic box and a sheet (vacuum axis) whose cells are narrower
    than twice the cut-off, so atoms also meet themselves through images."""
    from mbd_b200 import synthetic as sy
    from mbd_b200.engine import BOHR
    items = [sy.cluster(250, seed=4), sy.periodic_box(40, seed=2, scs_cut=20.0, cfdm_cut=15.0, sc_cut=5.0),
             sy.graphene_sheet(3)]
    geos, sets = [g for g, _ in items], [s for _, s in items]
    engine.use_network(False)
    try:
        res = engine.energy_batch(geos, sets, "mixed_learned")
    finally:
        engine.use_network(True)
    assert all(r.status == 0 for r in res)
    expect = []
    for g, s in items:
        lat = g.lattice / BOHR if g.n_periodic else None
        _, nbr, _ = gn.neighbours(g.coords / BOHR, lat, tuple(bool(v) for v in s.mbd_scs_vacuum_axis))
        expect.append(len(nbr))
    assert min(expect) > 0
    assert engine.stats()["network_edges"] == sum(expect), expect


def test_trained_network_saves_cg_iterations(engine, trained):
    """Held-out boxes: the network's warm start needs at least 4 % fewer
    block-CG iterations in total than a zero start, with the same energies
    (measured on a B200: 133 against 140 over the six boxes with FP64 passes,
    142 against 152 counting both phases of the two-phase FP32 form).

    The bar is what a warm start of this accuracy can give: the iteration
    reduces the error by a roughly constant factor rho ~ 0.5 per step, so a
    start with relative block error eps saves about log(eps) / log(rho)
    iterations -- 2 to 3 at the network's ~13 % error (training loss
    ~0.0165, reached with 160 training geometries and not lowered by 2000
    or by 30 epochs), of the 20-30 the solves take."""
    test = _train_set(6, 120, 180, seed=11)
    geos, sets = [g for g, _ in test], [s for _, s in test]
    with_net = engine.energy_batch(geos, sets, "mixed_learned")
    engine.use_network(False)
    try:
        without = engine.energy_batch(geos, sets, "mixed_learned")
    finally:
        engine.use_network(True)
    plain = engine.energy_batch(geos, sets, "plain")
    it_with = sum(r.refine_iters for r in with_net)
    it_without = sum(r.refine_iters for r in without)
    for a, b in zip(with_net, plain):
        assert a.status == 0
        assert abs(a.energy - b.energy) <= E_TOL
        assert abs(a.c6_mol - b.c6_mol) <= C6_RTOL * abs(b.c6_mol)
    print(f"block-CG iterations with the network {it_with}, without {it_without}")
    assert it_with <= 0.96 * it_without, (it_with, it_without)


def test_learned_mode_vs_oracle(engine, trained):
    from oracle import mbd_oracle as mo
    from mbd_b200 import synthetic as sy
    geo, st = sy.cluster(80, seed=3)
    res = engine.energy(geo, st, mode="mixed_learned")
    og = mo.Geometry(list(geo.names), geo.coords.copy(), geo.hirshfeld.copy(), geo.lattice.copy(), geo.n_periodic)
    ref = mo.mbd_at_rsscs(og, mo.Settings())
    assert res.status == 0
    assert abs(res.energy - ref.energy) <= E_TOL
    assert abs(res.c6_mol - ref.c6_mol) <= C6_RTOL * abs(ref.c6_mol)
    np.testing.assert_allclose(res.c6_eff, ref.c6_eff, rtol=C6_RTOL)


def test_params_round_trip(engine, trained):
    p = engine.learned_params()
    assert p.shape == (gn.N_PARAMS,) and np.all(np.isfinite(p))
    engine.set_learned_params(p)
    np.testing.assert_array_equal(engine.learned_params(), p)
