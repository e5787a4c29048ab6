"""CPU emulation of split-precision tensor-core GEMMs inside the two-stage
tridiagonalisation, to measure what they would do to the MBD energy.

The engine reduces the CFDM Hamiltonian (the matrix PDSYEV('N','L') takes at
UTILS.f90:835) to a band of half-bandwidth 32 by blocked Householder panels:
Y = A22 V T (SYMM), Z = Y - 1/2 V T^T V^T Y, A22 -= V Z^T + Z V^T (SYR2K),
and chases the band to tridiagonal form in FP64.  The SYMM and SYR2K carry
(4/3) n^3 of the reduction's flops.  This module repeats that reduction in
numpy with those two products computed as a tensor core would in one of the
split-precision schemes -- the FP64 operands rounded to FP32, split into
pieces of p mantissa bits, the products of the leading pieces accumulated in
FP32 -- and the rest (panel QR, compact-WY factor, the small products) in
FP64, then takes the band's eigenvalues in FP64 and forms
E = 1/2 sum_{lambda >= 0} sqrt(lambda) - 1/2 sum 3 omega (UTILS.f90:839-858).

Schemes: "fp64" (the harness itself), "fp32" (SGEMM), "3xtf32" (two TF32
pieces, 10 mantissa bits, three products), "bf16x3" (two BF16 pieces, 7
bits, three products), "bf16x6" (three BF16 pieces, six products).
Test infrastructure only: the engine runs these products in FP64.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla

SCHEMES = {
    # name: (mantissa bits per piece, pieces); None = plain FP64 / FP32
    "fp64": None,
    "fp32": "fp32",
    "3xtf32": (10, 2),
    "bf16x3": (7, 2),
    "bf16x6": (7, 3),
}

BAND = 32


def round_mantissa(x32: np.ndarray, bits: int) -> np.ndarray:
    """FP32 values rounded (to nearest, ties away from zero) to `bits`
    explicit mantissa bits, as a float32 array."""
    drop = 23 - bits
    u = np.ascontiguousarray(x32, dtype=np.float32).view(np.uint32)
    half = np.uint32(1 << (drop - 1))
    mask = np.uint32((0xFFFFFFFF >> drop) << drop)
    return ((u + half) & mask).view(np.float32)


def split(x: np.ndarray, bits: int, pieces: int) -> list[np.ndarray]:
    rem = x.astype(np.float32)
    out = []
    for _ in range(pieces):
        h = round_mantissa(rem, bits)
        out.append(h)
        rem = (rem - h).astype(np.float32)
    return out


def gemm(a: np.ndarray, b: np.ndarray, scheme: str) -> np.ndarray:
    """a @ b (FP64 inputs) computed under `scheme`."""
    cfg = SCHEMES[scheme]
    if cfg is None:
        return a @ b
    if cfg == "fp32":
        return (a.astype(np.float32) @ b.astype(np.float32)).astype(np.float64)
    bits, pieces = cfg
    As, Bs = split(a, bits, pieces), split(b, bits, pieces)
    acc = np.zeros((a.shape[0], b.shape[1]), dtype=np.float32)
    for i in range(pieces):
        for j in range(pieces - i):
            acc += As[i] @ Bs[j]
    return acc.astype(np.float64)


def _panel_qr(P: np.ndarray):
    """Householder QR of the m x 32 panel P: V (unit lower trapezoidal, m x k,
    k = min(m, 32)), T (compact WY, forward columnwise: Q = I - V T V^T) and
    R (k x 32, upper trapezoidal)."""
    qr, tau, _, _ = sla.lapack.dgeqrf(P)
    k = min(P.shape)
    V = np.tril(qr, -1)[:, :k]
    V[np.arange(k), np.arange(k)] = 1.0
    R = np.triu(qr[:k, :])
    T = np.zeros((k, k))
    G = V.T @ V
    for j in range(k):
        T[:j, j] = -tau[j] * (T[:j, :j] @ G[:j, j])
        T[j, j] = tau[j]
    return V, T, R


def band_reduce(H: np.ndarray, scheme: str) -> np.ndarray:
    """Symmetric H (its lower triangle is read) -> symmetric band of
    half-bandwidth 32 with the same eigenvalues, the SYMM and SYR2K under
    `scheme`."""
    L = np.tril(np.asarray(H, dtype=np.float64))
    A = L + np.tril(L, -1).T
    n = A.shape[0]
    for c0 in range(0, n - BAND - 1, BAND):
        r0 = c0 + BAND
        V, T, R = _panel_qr(A[r0:, c0:c0 + BAND])
        A[r0:, c0:c0 + BAND] = 0.0
        A[r0:r0 + R.shape[0], c0:c0 + BAND] = R
        A[c0:c0 + BAND, r0:] = A[r0:, c0:c0 + BAND].T
        A22 = A[r0:, r0:]
        Y = gemm(A22, V, scheme) @ T                     # SYMM (K = m)
        M = T.T @ (V.T @ Y)
        Z = Y - 0.5 * (V @ M)
        L = np.hstack([V, Z])
        Rt = np.hstack([Z, V])
        A22 -= gemm(L, Rt.T, scheme)                      # SYR2K (K = 64)
        A[r0:, r0:] = 0.5 * (A22 + A22.T)
    return A


def energy_from(eigs: np.ndarray, omega: np.ndarray, nsl: int = 1) -> float:
    pos = eigs >= 0.0
    return 0.5 * float(np.sum(np.sqrt(eigs[pos]))) / nsl - 0.5 * float(np.sum(3.0 * omega))


def study(H: np.ndarray, omega: np.ndarray, schemes=("fp64", "fp32", "3xtf32", "bf16x3", "bf16x6")) -> dict:
    """Energy error (Ha) of each scheme against the dense FP64 eigenvalues."""
    e_ref = energy_from(sla.eigh(H, lower=True, eigvals_only=True, driver="evd"), omega)
    out = {"E_ref": e_ref}
    for s in schemes:
        Bm = band_reduce(H, s)
        lam = sla.eigh(Bm, eigvals_only=True, driver="evd")
        out[s] = energy_from(lam, omega) - e_ref
    return out
