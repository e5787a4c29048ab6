"""CPU oracle of the learned relay warm start (test infrastructure only).

The reference has no learned component: the relay system
A(iw) X = [I; ...; I] (get_screened_alpha, UTILS.f90:376-539) is solved
directly there.  The engine's MIXED_LEARNED mode solves it by block
conjugate gradients started from a network's prediction of every atom's
3x3 screened-polarizability block X_i = sum_j (A^-1)_ij.  This module is the
float64 numpy restatement of that network -- features, forward pass, loss and
hand-derived backward pass -- against which the CUDA kernels' outputs and
gradients are checked.  Nothing here is used by the product.

Network (per imaginary frequency f and atom i; node = (f, i)):
  x      = [onehot(H, C, N, O, other), h_i, log alpha_i(iw_f), log(1 + w_f)]
  h0     = silu(W0 x + b0)                                   (8 -> 64)
  layer l = 0, 1, 2:
    filt_ij = Wf_l e_ij                                      (16 -> 64)
    m_i     = sum_{j in nbr(i)} filt_ij * h_j                (elementwise)
    u_i     = Wu_l m_i + bu_l
    h_i    <- h_i + silu(u_i)
  s_i    = ws . h_i + bs,   a_i = wa . h_i + ca,   g_ij = wg . e_ij
  S_i    = (1 + s_i) I + sum_j a_j g_ij (u_ij u_ij^T - I/3)
  X_i    = alpha_i(iw_f) S_i
with e_ij = 16 Gaussian radial functions of r_ij times a cosine cut-off and
u_ij the unit vector from i to j.  Loss: mean over nodes of ||S - S_true||_F^2.
"""
from __future__ import annotations

import numpy as np

HIDDEN = 64
N_RBF = 16
N_IN = 8
N_LAYERS = 3
CUTOFF_BOHR = 5.0 / 0.52917721      # 5 Angstrom
SPECIES = {"H": 0, "C": 1, "N": 2, "O": 3}

# flat parameter layout (float32 on the device, same order here)
LAYOUT = [("W0", (HIDDEN, N_IN)), ("b0", (HIDDEN,))]
for _l in range(N_LAYERS):
    LAYOUT += [(f"Wf{_l}", (HIDDEN, N_RBF)), (f"Wu{_l}", (HIDDEN, HIDDEN)), (f"bu{_l}", (HIDDEN,))]
LAYOUT += [("ws", (HIDDEN,)), ("bs", (1,)), ("wa", (HIDDEN,)), ("ca", (1,)), ("wg", (N_RBF,))]
N_PARAMS = int(sum(np.prod(s) for _, s in LAYOUT))


def unpack(flat):
    out, o = {}, 0
    for name, shp in LAYOUT:
        k = int(np.prod(shp))
        out[name] = flat[o:o + k].reshape(shp)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in LAYOUT])


def init_params(seed=0):
    """Deterministic initialisation of the same shape as the engine's (whose
    own generator draws different numbers from the same distributions)."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, shp in LAYOUT:
        if name.startswith("W"):
            fan_in = shp[1]
            d[name] = rng.standard_normal(shp) * np.sqrt(1.0 / fan_in)
        elif name in ("ws", "wa"):
            d[name] = np.zeros(shp)
        elif name == "wg":
            d[name] = rng.standard_normal(shp) * 0.1
        else:
            d[name] = np.zeros(shp)
    return pack(d)


def rbf(r):
    """e(r): 16 Gaussians on [0, cutoff] times 0.5 (cos(pi r / rc) + 1)."""
    mu = np.linspace(0.0, CUTOFF_BOHR, N_RBF)
    width = CUTOFF_BOHR / (N_RBF - 1)
    fc = 0.5 * (np.cos(np.pi * r / CUTOFF_BOHR) + 1.0)
    return np.exp(-0.5 * ((r[:, None] - mu[None, :]) / width) ** 2) * fc[:, None]


def neighbours(coords_bohr, lattice_bohr=None, vacuum=(False, False, False)):
    """CSR neighbour lists within the cut-off: every image r_j + t (t a lattice
    translation along non-vacuum axes) within the cut-off of atom i, except
    atom i itself at t = 0.  An atom can meet another atom, or itself, through
    several images when the cell is narrower than twice the cut-off.
    lattice_bohr rows are the cell vectors.  Returns off, nbr, d
    (d = r_j + t - r_i), edges of atom i in ascending (t, j) order."""
    n = len(coords_bohr)
    shifts = [np.zeros(3)]
    if lattice_bohr is not None:
        a = np.asarray(lattice_bohr, dtype=float)
        vol = abs(np.linalg.det(a))
        rng = []
        for k in range(3):
            if vacuum[k]:
                rng.append(0)
                continue
            area = np.linalg.norm(np.cross(a[(k + 1) % 3], a[(k + 2) % 3]))
            rng.append(int(np.ceil(CUTOFF_BOHR / (vol / area))) + 1)
        shifts = [i * a[0] + j * a[1] + k * a[2]
                  for i in range(-rng[0], rng[0] + 1) for j in range(-rng[1], rng[1] + 1)
                  for k in range(-rng[2], rng[2] + 1)]
    nbr, dv, cnt = [], [], np.zeros(n, dtype=np.int64)
    per_atom = [[] for _ in range(n)]
    for t in shifts:
        diff = coords_bohr[None, :, :] + t[None, None, :] - coords_bohr[:, None, :]
        r = np.linalg.norm(diff, axis=-1)
        mask = (r < CUTOFF_BOHR) & (r > 1e-6)
        for i in range(n):
            js = np.nonzero(mask[i])[0]
            if len(js):
                per_atom[i].append((js, diff[i, js]))
    off = np.zeros(n + 1, dtype=np.int64)
    for i in range(n):
        for js, d in per_atom[i]:
            nbr.append(js)
            dv.append(d)
            cnt[i] += len(js)
        off[i + 1] = off[i] + cnt[i]
    if not nbr:
        return off, np.zeros(0, dtype=np.int64), np.zeros((0, 3))
    return off, np.concatenate(nbr).astype(np.int64), np.concatenate(dv).reshape(-1, 3)


def node_features(species_idx, hirsh, alpha_w, omega):
    """x[f*N + i] for F frequencies: alpha_w (F, N), omega (F,)."""
    F, N = alpha_w.shape
    x = np.zeros((F * N, N_IN))
    oh = np.zeros((N, 5))
    oh[np.arange(N), np.minimum(species_idx, 4)] = 1.0
    for f in range(F):
        x[f * N:(f + 1) * N, 0:5] = oh
        x[f * N:(f + 1) * N, 5] = hirsh
        x[f * N:(f + 1) * N, 6] = np.log(alpha_w[f])
        x[f * N:(f + 1) * N, 7] = np.log1p(omega[f])
    return x


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def _edges(off):
    n = len(off) - 1
    return np.repeat(np.arange(n), np.diff(off))


def forward(flat, x, F, off, nbr, d):
    """Returns S (F*N, 3, 3) and the cache for backward."""
    p = unpack(np.asarray(flat, dtype=np.float64))
    N = len(off) - 1
    src = _edges(off)
    r = np.linalg.norm(d, axis=1)
    e = rbf(r)
    u = d / r[:, None]
    proj = u[:, :, None] * u[:, None, :] - np.eye(3)[None] / 3.0
    pre0 = x @ p["W0"].T + p["b0"]
    h = silu(pre0)
    cache = {"x": x, "pre0": pre0, "hs": [h], "ms": [], "us": [], "filts": [], "e": e, "proj": proj, "src": src}
    for l in range(N_LAYERS):
        filt = e @ p[f"Wf{l}"].T                           # (E, 64)
        m = np.zeros_like(h)
        for f in range(F):
            hj = h[f * N + nbr]                            # (E, 64)
            np.add.at(m[f * N:(f + 1) * N], src, filt * hj)
        uu = m @ p[f"Wu{l}"].T + p[f"bu{l}"]
        h = h + silu(uu)
        cache["filts"].append(filt)
        cache["ms"].append(m)
        cache["us"].append(uu)
        cache["hs"].append(h)
    s = h @ p["ws"] + p["bs"][0]
    a = h @ p["wa"] + p["ca"][0]
    g = e @ p["wg"]
    S = np.zeros((F * N, 3, 3))
    S[:, [0, 1, 2], [0, 1, 2]] = (1.0 + s)[:, None]
    for f in range(F):
        w = a[f * N + nbr] * g                             # (E,)
        np.add.at(S[f * N:(f + 1) * N], src, w[:, None, None] * proj)
    cache.update(s=s, a=a, g=g)
    return S, cache


def loss_and_grad(flat, x, F, off, nbr, d, S_true):
    """Loss = mean_nodes ||S - S_true||_F^2 and d loss / d params (float64)."""
    p = unpack(np.asarray(flat, dtype=np.float64))
    S, c = forward(flat, x, F, off, nbr, d)
    N = len(off) - 1
    M = F * N
    diff = S - S_true
    loss = float(np.sum(diff * diff) / M)
    dS = 2.0 * diff / M
    src, e, proj = c["src"], c["e"], c["proj"]
    h3, a, g = c["hs"][-1], c["a"], c["g"]
    grads = {name: np.zeros(shp) for name, shp in LAYOUT}
    ds = np.trace(dS, axis1=1, axis2=2)
    da = np.zeros(M)
    for f in range(F):
        dw = np.einsum("eab,eab->e", dS[f * N + src], proj)   # d loss / d w_ij
        np.add.at(da[f * N:(f + 1) * N], nbr, dw * g)
        grads["wg"] += (dw * a[f * N + nbr]) @ e
    grads["ws"] = h3.T @ ds
    grads["bs"][0] = ds.sum()
    grads["wa"] = h3.T @ da
    grads["ca"][0] = da.sum()
    dh = ds[:, None] * p["ws"][None, :] + da[:, None] * p["wa"][None, :]
    for l in reversed(range(N_LAYERS)):
        uu, m, filt, h_in = c["us"][l], c["ms"][l], c["filts"][l], c["hs"][l]
        du = dh * dsilu(uu)
        grads[f"Wu{l}"] = du.T @ m
        grads[f"bu{l}"] = du.sum(axis=0)
        dm = du @ p[f"Wu{l}"]
        dh_in = dh.copy()
        dfilt = np.zeros_like(filt)
        for f in range(F):
            dmi = dm[f * N + src]                            # (E, 64)
            np.add.at(dh_in[f * N:(f + 1) * N], nbr, filt * dmi)
            dfilt += dmi * h_in[f * N + nbr]
        grads[f"Wf{l}"] = dfilt.T @ e
        dh = dh_in
    dpre = dh * dsilu(c["pre0"])
    grads["W0"] = dpre.T @ c["x"]
    grads["b0"] = dpre.sum(axis=0)
    return loss, pack(grads)


def adam_step(flat, grad, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (t counts from 1); returns new (flat, m, v)."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return flat - lr * mh / (np.sqrt(vh) + eps), m, v
