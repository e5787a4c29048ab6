"""CPU checks of the learned warm start's oracle network (oracle/gnn_oracle.py):
its hand-derived gradient against central finite differences, equivariance
of the predicted tensors, and the parameter layout the device kernels use."""
import numpy as np

from oracle import gnn_oracle as gn


def _toy(seed=0, n=14, F=2):
    rng = np.random.default_rng(seed)
    coords = rng.uniform(0.0, 9.0, size=(n, 3))
    off, nbr, d = gn.neighbours(coords)
    species = rng.integers(0, 5, size=n)
    hirsh = rng.uniform(0.6, 1.0, size=n)
    alpha = rng.uniform(1.0, 12.0, size=(F, n))
    omega = np.array([0.0, 0.7])[:F]
    x = gn.node_features(species, hirsh, alpha, omega)
    S_true = rng.standard_normal((F * n, 3, 3)) * 0.1 + np.eye(3)
    return x, F, off, nbr, d, S_true, coords


def _params(seed=1):
    rng = np.random.default_rng(seed)
    p = gn.init_params(seed)
    return p + 0.05 * rng.standard_normal(p.shape)   # every parameter non-zero


def test_parameter_layout():
    assert gn.N_PARAMS == 16274
    p = gn.init_params(3)
    np.testing.assert_array_equal(gn.pack(gn.unpack(p)), p)


def test_gradient_matches_finite_differences():
    x, F, off, nbr, d, S_true, _ = _toy()
    assert len(nbr) > 10
    p = _params()
    loss, g = gn.loss_and_grad(p, x, F, off, nbr, d, S_true)
    rng = np.random.default_rng(5)
    idx = rng.choice(gn.N_PARAMS, size=60, replace=False)
    # every block of the layout at least once
    o = 0
    for name, shp in gn.LAYOUT:
        idx = np.append(idx, o)
        o += int(np.prod(shp))
    eps = 1e-6
    for k in idx:
        pp, pm = p.copy(), p.copy()
        pp[k] += eps
        pm[k] -= eps
        lp, _ = gn.loss_and_grad(pp, x, F, off, nbr, d, S_true)
        lm, _ = gn.loss_and_grad(pm, x, F, off, nbr, d, S_true)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_prediction_is_rotation_equivariant():
    x, F, off, nbr, d, _, coords = _toy(seed=2)
    p = _params(4)
    S, _ = gn.forward(p, x, F, off, nbr, d)
    q, _ = np.linalg.qr(np.random.default_rng(8).standard_normal((3, 3)))
    S_rot, _ = gn.forward(p, x, F, off, nbr, d @ q.T)
    np.testing.assert_allclose(S_rot, q @ S @ q.T, atol=1e-12)
