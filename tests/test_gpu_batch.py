"""GPU parity of batched runs: many geometries of uneven size in one call.

A batch runs the relay stages of its geometries concurrently on several
streams and reduces all CFDM Hamiltonians together (the two-stage path: one
bulge-chasing launch for every band; the one-stage path: one grouped launch),
so these tests cover the batch planning (one matrix per CTA group, several
matrices per group when geometries outnumber CTAs, groups of different
widths) and the batched eigenvalue / energy launches against the FP64
oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_TOL = 1e-6
C6_RTOL = 1e-6
PLAIN_E_TOL = 1e-9
PLAIN_RTOL = 1e-9


@pytest.fixture(scope="module")
def engine():
    from mbd_b200 import Engine
    eng = Engine(0)
    yield eng
    eng.close()


def _oracle(geo, st):
    from oracle import mbd_oracle as mo
    og = mo.Geometry(list(geo.names), geo.coords.copy(), geo.hirshfeld.copy(), geo.lattice.copy(), geo.n_periodic)
    os_ = mo.Settings(xc=st.xc, mbd_supercell_cutoff=st.mbd_supercell_cutoff,
                      mbd_cfdm_dip_cutoff=st.mbd_cfdm_dip_cutoff, mbd_scs_dip_cutoff=st.mbd_scs_dip_cutoff,
                      mbd_scs_vacuum_axis=tuple(st.mbd_scs_vacuum_axis))
    return mo.mbd_at_rsscs(og, os_)


def _assert_close(res, ref, mode):
    e_tol = PLAIN_E_TOL if mode == "plain" else E_TOL
    rtol = PLAIN_RTOL if mode == "plain" else C6_RTOL
    assert res.status == 0
    assert abs(res.energy - ref.energy) <= e_tol, (res.energy, ref.energy)
    assert abs(res.c6_mol - ref.c6_mol) <= rtol * abs(ref.c6_mol)
    np.testing.assert_allclose(res.c6_eff, ref.c6_eff, rtol=rtol, atol=0)
    assert res.nimag == ref.nimag


@pytest.mark.parametrize("mode", ["plain", "mixed"])
def test_more_geometries_than_ctas(engine, mode):
    """200 small clusters: more matrices than co-resident CTAs, so CTA groups
    reduce several Hamiltonians one after another."""
    from mbd_b200 import synthetic as sy
    items = sy.cluster_batch(200, nmin=4, nmax=40, seed=7)
    res = engine.energy_batch([g for g, _ in items], [s for _, s in items], mode)
    for (g, s), r in zip(items, res):
        _assert_close(r, _oracle(g, s), mode)


@pytest.mark.parametrize("mode", ["plain", "mixed"])
def test_uneven_batch_vs_oracle(engine, mode):
    """Sizes spread over two orders of magnitude plus a periodic sheet: CTA
    groups of different widths in the same launch."""
    from mbd_b200 import synthetic as sy
    items = [sy.cluster(n, seed=20 + n) for n in (12, 350, 40, 180, 7, 90)]
    items.append(sy.graphene_sheet(reps=4))
    res = engine.energy_batch([g for g, _ in items], [s for _, s in items], mode)
    for (g, s), r in zip(items, res):
        _assert_close(r, _oracle(g, s), mode)


def test_batch_with_failing_member(engine):
    """A geometry with an element outside the table fails alone; the rest of
    the batch is unaffected."""
    from mbd_b200 import Geometry, Settings
    from mbd_b200 import synthetic as sy
    good = [sy.cluster(n, seed=n) for n in (30, 15)]
    bad = Geometry(["C", "La"], np.array([[0, 0, 0], [0, 0, 2.0]]), np.array([0.8, 0.8]))
    geos = [good[0][0], bad, good[1][0]]
    res = engine.energy_batch(geos, [good[0][1], Settings(), good[1][1]], "mixed", check=False)
    assert res[1].status == 2
    for k, (g, s) in zip((0, 2), good):
        _assert_close(res[k], _oracle(g, s), "mixed")


def test_batched_workload_mixed_vs_plain(engine):
    """The 256-cluster batched workload (N ~ U{20..600}): every mixed energy
    within 1e-6 Ha of the plain FP64 one, a sample against the oracle."""
    from mbd_b200 import synthetic as sy
    items = sy.cluster_batch(256)
    geos, sets = [g for g, _ in items], [s for _, s in items]
    mixed = engine.energy_batch(geos, sets, "mixed")
    plain = engine.energy_batch(geos, sets, "plain")
    for rm, rp in zip(mixed, plain):
        assert rm.status == 0 and rp.status == 0
        assert abs(rm.energy - rp.energy) <= E_TOL
        assert abs(rm.c6_mol - rp.c6_mol) <= C6_RTOL * abs(rp.c6_mol)
        assert rm.refine_iters > 0
    sizes = [len(g.names) for g in geos]
    for k in (int(np.argmin(sizes)), int(np.argsort(sizes)[len(sizes) // 2])):
        ref = _oracle(*items[k])
        _assert_close(plain[k], ref, "plain")
        _assert_close(mixed[k], ref, "mixed")


@pytest.mark.parametrize("mode", ["plain", "mixed", "mixed_learned"])
def test_graph_replay_matches_direct_launches(engine, mode, monkeypatch):
    """compute() launches a new batch directly, captures it into a CUDA graph
    on its second call and replays it afterwards; every run equals a context
    that always launches directly.  In the learned mode (block-CG from zero
    here, no network) the graph runs the CG iterations the first compute
    took plus a margin instead of the full schedule."""
    from mbd_b200 import Engine
    from mbd_b200 import synthetic as sy
    items = [sy.cluster(n, seed=40 + n) for n in (25, 140, 60)]
    geos, sets = [g for g, _ in items], [s for _, s in items]
    engine.use_network(False)
    assert engine.upload(geos, sets) == 0
    runs, launches = [], []
    for k in range(3):   # direct launches, capture + replay, replay
        assert engine.compute(mode) == 0
        st = engine.stats()
        assert st["graph_replayed"] == (k > 0)
        launches.append(st["launches"])
        code, res = engine.download()
        assert code == 0
        runs.append(res)
    if mode == "mixed_learned":
        assert launches[1] < launches[0]   # the trimmed CG schedule
        assert [r.refine_iters for r in runs[1]] == [r.refine_iters for r in runs[0]]
    monkeypatch.setenv("MBD_B200_NO_GRAPHS", "1")
    with Engine(0) as direct:
        direct.use_network(False)
        ref = direct.energy_batch(geos, sets, mode)
    for res in runs:
        for a, b in zip(res, ref):
            assert a.energy == b.energy
            np.testing.assert_array_equal(a.alpha_iw, b.alpha_iw)


@pytest.mark.parametrize("mode", ["plain", "mixed", "mixed_learned"])
def test_first_compute_graph_across_batches(mode, monkeypatch):
    """MBD_B200_GRAPH_UPDATE=1, batches of one shape uploaded one after
    another (the structures change, the sizes do not): the first batch
    launches kernel by kernel, every later batch's first compute runs as a
    graph (captured, then written into the previous batch's graph by
    cudaGraphExecUpdate, or instantiated where the driver refuses the
    update), and a batch of another shape launches kernel by kernel again.
    Every batch's results equal a context that always launches directly, bit
    for bit."""
    from mbd_b200 import Engine
    from mbd_b200 import synthetic as sy
    sizes = (25, 140, 60)
    batches = [[sy.cluster(n, seed=1000 * b + n) for n in sizes] for b in range(4)]
    batches.append([sy.cluster(n, seed=77 + n) for n in (30, 90)])
    kinds, updates, runs = [], [], []
    monkeypatch.setenv("MBD_B200_GRAPH_UPDATE", "1")
    with Engine(0) as eng:
        eng.use_network(False)
        for items in batches:
            res = eng.energy_batch([g for g, _ in items], [s for _, s in items], mode)
            st = eng.stats()
            kinds.append(2 if st["first_compute_graph"] else (1 if st["graph_replayed"] else 0))
            updates.append(st["graph_updates"])
            runs.append(res)
    assert kinds == [0, 2, 2, 2, 0], kinds
    assert updates[:2] == [0, 0] and updates[4] == updates[3], updates
    monkeypatch.setenv("MBD_B200_GRAPH_UPDATE", "0")
    monkeypatch.setenv("MBD_B200_NO_GRAPHS", "1")
    with Engine(0) as direct:
        direct.use_network(False)
        for items, res in zip(batches, runs):
            ref = direct.energy_batch([g for g, _ in items], [s for _, s in items], mode)
            for a, b in zip(res, ref):
                assert a.status == 0 and b.status == 0
                assert a.energy == b.energy
                assert a.refine_iters == b.refine_iters
                np.testing.assert_array_equal(a.alpha_iw, b.alpha_iw)


@pytest.mark.parametrize("sizes", [(25, 140, 60, 300, 12), tuple(range(20, 20 + 7 * 40, 7))])
def test_one_stage_reduction_matches_two_stage(engine, sizes, monkeypatch):
    """The grouped one-stage tridiagonalisation (MBD_B200_TWO_STAGE=0; the
    default takes it only for matrices above the two-stage limit) against the
    default two-stage path on the same batches: CTA groups of different
    widths, several matrices per group when geometries outnumber CTAs."""
    from mbd_b200 import Engine
    from mbd_b200 import synthetic as sy
    items = [sy.cluster(n, seed=70 + k) for k, n in enumerate(sizes)]
    geos, sets = [g for g, _ in items], [s for _, s in items]
    two = engine.energy_batch(geos, sets, "plain")
    monkeypatch.setenv("MBD_B200_TWO_STAGE", "0")
    with Engine(0) as one_stage:
        one = one_stage.energy_batch(geos, sets, "plain")
    for a, b in zip(one, two):
        assert a.status == 0 and b.status == 0
        assert abs(a.energy - b.energy) <= PLAIN_E_TOL, (a.energy, b.energy)
        assert a.nimag == b.nimag
