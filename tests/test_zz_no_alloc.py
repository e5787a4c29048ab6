"""mbd_rsscs_eigvalsh_noalloc: the eigenvalue entry point for callers that
cannot allocate device memory (a host that owns all GPU memory through its
own pool, or a path where cudaMalloc's synchronisation is not allowed).

It must agree with the allocating entry point mbd_rsscs_eigvalsh on the same
matrices, on two calls in a row (the calls share one fixed scratch array, so
the second call checks that nothing from the first one leaks through), and it
must refuse matrices beyond its fixed maximum.  This file is collected last
on purpose; it passes alone in a fresh process (where its first call does the
one-time scratch set-up) and after the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MBD_ERR_ARG = 1
MBD_ERR_TOO_LARGE = 11


def _sym(n, seed):
    rng = np.random.default_rng(seed)
    M = rng.standard_normal((n, n))
    return (M + M.T) / 2 + np.diag(rng.uniform(0.0, 3.0, n))


def test_noalloc_matches_allocating_entry_point_twice():
    import torch

    from mbd_b200 import Engine, load_library

    lib = load_library()
    fn = lib.mbd_rsscs_eigvalsh_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    max_n = 2048
    with Engine(0) as eng:
        # small, largest, then small again (a smaller call after a larger one
        # must not see the larger call's leftovers in the shared scratch);
        # the last call uses a padded leading dimension
        for call, (n, ld) in enumerate(((700, 700), (max_n, max_n), (700, 702))):
            S = _sym(n, seed=100 + call)
            ref = eng.eigvalsh(np.tril(S))                       # allocating entry point
            lapack = np.linalg.eigvalsh(S)                       # LAPACK on the host
            Hp = np.zeros((n, ld))
            Hp[:, :n] = S
            H = torch.tensor(Hp, dtype=torch.float64, device="cuda")   # caller-owned device buffers
            w = torch.empty(n, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            code = fn(H.data_ptr(), n, ld, w.data_ptr(), torch.cuda.current_stream().cuda_stream)
            assert code == 0, code
            got = w.cpu().numpy()
            # same tolerance as the eigenvalue parity tests
            tol = 1e-12 * max(1.0, np.abs(ref).max()) * n
            np.testing.assert_allclose(got, ref, rtol=0, atol=tol)
            np.testing.assert_allclose(got, lapack, rtol=0, atol=tol)
        big = torch.zeros((max_n + 2, max_n + 2), dtype=torch.float64, device="cuda")
        wb = torch.empty(max_n + 2, dtype=torch.float64, device="cuda")
        assert fn(big.data_ptr(), max_n + 2, max_n + 2, wb.data_ptr(), None) == MBD_ERR_TOO_LARGE
        # an odd leading dimension and a matrix start off the 16-byte grid are refused
        small = torch.zeros((64, 66), dtype=torch.float64, device="cuda")
        ws = torch.empty(64, dtype=torch.float64, device="cuda")
        assert fn(small.data_ptr(), 63, 65, ws.data_ptr(), None) == MBD_ERR_ARG
        assert fn(small.data_ptr() + 8, 64, 64, ws.data_ptr(), None) == MBD_ERR_ARG
