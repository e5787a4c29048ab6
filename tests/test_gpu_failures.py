"""Failure detection on the GPU, in forms that neither fault nor hang it.

* A relay matrix that is not positive definite (a chain of three Cs atoms
  2 A apart: the screened response diverges) is reported as
  MBD_ERR_RELAY_NOT_SPD in every mode.  The reference ignores PDPOTRF's
  info here (UTILS.f90:469) and carries on with a failed factor.
* The residual gate of the mixed and learned relay solves, forced to 0 from
  the host, sends every geometry to the direct FP64 fallback
  (refine_iters = -1), whose results match the oracle at the plain bar.
* A bounded device wait made to run out from the host (the bulge-chasing
  launch's first sweep waits for a count that nothing reaches, with a 50 ms
  limit) ends the compute with MBD_ERR_TIMEOUT; the context then computes
  correctly again.  No kernel traps, faults or spins without a limit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PLAIN_E_TOL = 1e-9
PLAIN_RTOL = 1e-9
MBD_ERR_RELAY_NOT_SPD = 3
MBD_ERR_TIMEOUT = 7


@pytest.fixture(scope="module")
def engine():
    from mbd_b200 import Engine
    eng = Engine(0)
    yield eng
    eng.close()


def _oracle(geo, st):
    from oracle import mbd_oracle as mo
    og = mo.Geometry(list(geo.names), geo.coords.copy(), geo.hirshfeld.copy(), geo.lattice.copy(), geo.n_periodic)
    return mo.mbd_at_rsscs(og, mo.Settings(xc=st.xc))


def _cs_chain():
    from mbd_b200 import Geometry, Settings
    xyz = np.array([[2.0 * i, 0.0, 0.0] for i in range(3)])
    return Geometry(["Cs"] * 3, xyz, np.ones(3)), Settings(xc=1)


@pytest.mark.parametrize("mode", ["plain", "mixed", "mixed_learned"])
def test_non_spd_relay_is_reported(engine, mode):
    geo, st = _cs_chain()
    ref = _oracle(geo, st)
    assert ref.status == "relay_not_spd" and ref.info != 0
    engine.use_network(False)          # the learned mode without a network: block-CG from zero
    try:
        res = engine.energy(geo, st, mode=mode, check=False)
    finally:
        engine.use_network(True)
    assert res.status == MBD_ERR_RELAY_NOT_SPD, res.status
    assert np.isnan(res.energy)
    # the context is still usable
    from mbd_b200 import synthetic as sy
    ok = engine.energy(*sy.benzene(), mode="plain")
    assert ok.status == 0


@pytest.mark.parametrize("mode", ["mixed", "mixed_learned"])
def test_forced_residual_gate_runs_direct_fallback(engine, mode):
    from mbd_b200 import synthetic as sy
    items = [sy.cluster(60, seed=3), sy.cluster(150, seed=8)]
    refs = [_oracle(g, s) for g, s in items]
    engine.set_option("residual_gate", 0.0)
    engine.use_network(False)
    try:
        res = engine.energy_batch([g for g, _ in items], [s for _, s in items], mode)
    finally:
        engine.use_network(True)
        engine.set_option("residual_gate", 1e-10)
    assert engine.get_option("residual_gate") == 1e-10
    for r, ref in zip(res, refs):
        assert r.status == 0
        assert r.refine_iters == -1                      # the direct FP64 solve produced the result
        assert abs(r.energy - ref.energy) <= PLAIN_E_TOL
        np.testing.assert_allclose(r.c6_eff, ref.c6_eff, rtol=PLAIN_RTOL, atol=0)
        np.testing.assert_allclose(r.alpha_iw, ref.alpha_iw, rtol=10 * PLAIN_RTOL, atol=1e-12)


def test_bounded_wait_times_out_and_context_recovers(engine):
    import time

    from mbd_b200 import synthetic as sy
    geo, st = sy.cluster(120, seed=21)
    engine.set_option("wait_limit_s", 0.05)
    engine.set_option("test_stall_wait", 1)
    try:
        t0 = time.perf_counter()
        res = engine.energy(geo, st, mode="plain", check=False)
        took = time.perf_counter() - t0
    finally:
        engine.set_option("test_stall_wait", 0)
        engine.set_option("wait_limit_s", 2.0)
    assert res.status == MBD_ERR_TIMEOUT, res.status
    assert took < 30.0
    # the same context, the same geometry: correct again
    ref = _oracle(geo, st)
    res2 = engine.energy(geo, st, mode="plain")
    assert res2.status == 0
    assert abs(res2.energy - ref.energy) <= PLAIN_E_TOL


def test_option_arguments_are_checked(engine):
    from mbd_b200 import MbdError
    with pytest.raises(MbdError):
        engine.set_option("wait_limit_s", 0.0)
    with pytest.raises(MbdError):
        engine.set_option("residual_gate", -1.0)
    assert engine.get_option("wait_limit_s") == 2.0
    assert engine.get_option("test_stall_wait") == 0.0
