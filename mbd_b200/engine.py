"""ctypes binding of libmbd_b200.so (include/mbd_b200.h).

``Engine`` mirrors the reference's single entry point ``MBD_at_rsSCS``
(UTILS.f90:153-349): give it a geometry and the settings of setting.in and
it returns the MBD@rsSCS energy, the screened polarizabilities alpha(iw),
alpha_eff, C6_eff, the system C6 and NIMAG.  Every call goes through the C
ABI; there is no Python or CPU fallback -- if the CUDA library is missing or
no sm_100 GPU is present, construction raises.
"""
from __future__ import annotations

import ctypes
import functools
import os
from dataclasses import dataclass

import numpy as np

from .io import Geometry, Settings

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmbd_b200.so")

MBD_OK = 0
ERRORS = {
    1: "MBD_ERR_ARG", 2: "MBD_ERR_UNKNOWN_ELEMENT", 3: "MBD_ERR_RELAY_NOT_SPD",
    4: "MBD_ERR_NONPOSITIVE_ALPHA", 5: "MBD_ERR_EIGENSOLVER", 6: "MBD_ERR_DEVICE",
    7: "MBD_ERR_TIMEOUT", 8: "MBD_ERR_OUT_OF_MEMORY", 9: "MBD_ERR_REFINEMENT", 10: "MBD_ERR_NOT_BUILT",
    11: "MBD_ERR_TOO_LARGE", 12: "MBD_ERR_NO_NETWORK",
}
MODES = {"plain": 0, "plain_fp64": 0, "mixed": 1, "mixed_learned": 2, "learned": 2}
N_FREQ = 21
BOHR = 0.52917721          # UTILS.f90:85

EXPORTED = [
    "mbd_rsscs_create", "mbd_rsscs_destroy", "mbd_rsscs_energy", "mbd_rsscs_energy_batch",
    "mbd_rsscs_upload", "mbd_rsscs_compute", "mbd_rsscs_download", "mbd_rsscs_element_z",
    "mbd_rsscs_strerror", "mbd_rsscs_vdw_params", "mbd_rsscs_last_timings", "mbd_rsscs_last_stats",
    "mbd_rsscs_stream", "mbd_rsscs_eigvalsh", "mbd_rsscs_eigvalsh_noalloc", "mbd_rsscs_eigh",
    "mbd_rsscs_learned_param_count", "mbd_rsscs_learned_train", "mbd_rsscs_learned_get_params",
    "mbd_rsscs_learned_set_params", "mbd_rsscs_learned_use_network", "mbd_rsscs_learned_eval",
    "mbd_rsscs_set_option", "mbd_rsscs_get_option", "mbd_rsscs_autotune", "mbd_rsscs_tuning",
]
OPTIONS = {"residual_gate": 1, "wait_limit_s": 2, "test_stall_wait": 3, "fp32_tensor_build": 4}


NETWORK_MAGIC = b"MBDNET\0\0"
NETWORK_VERSION = 1


def write_network_file(path: str, params) -> None:
    """Checkpoint of the learned warm start's network: 8-byte magic, uint32
    format version, uint32 parameter count, the FP32 parameters
    (little-endian, the layout of mbd_rsscs_learned_get_params) and the
    SHA-256 of those parameter bytes."""
    import hashlib
    import struct
    p = np.ascontiguousarray(params, dtype="<f4")
    body = p.tobytes()
    with open(path, "wb") as fh:
        fh.write(NETWORK_MAGIC + struct.pack("<II", NETWORK_VERSION, p.size) + body + hashlib.sha256(body).digest())


def read_network_file(path: str) -> np.ndarray:
    import hashlib
    import struct
    with open(path, "rb") as fh:
        data = fh.read()
    if len(data) < 16 or data[:8] != NETWORK_MAGIC:
        raise ValueError(f"{path}: not a network checkpoint")
    version, count = struct.unpack("<II", data[8:16])
    if version != NETWORK_VERSION:
        raise ValueError(f"{path}: checkpoint format version {version}, expected {NETWORK_VERSION}")
    body = data[16:16 + 4 * count]
    digest = data[16 + 4 * count:]
    if len(body) != 4 * count or hashlib.sha256(body).digest() != digest:
        raise ValueError(f"{path}: checkpoint is truncated or corrupted (SHA-256 mismatch)")
    return np.frombuffer(body, dtype="<f4").astype(np.float32)


class MbdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class CGeom(ctypes.Structure):
    _fields_ = [
        ("n_atoms", ctypes.c_int),
        ("z", ctypes.POINTER(ctypes.c_int)),
        ("coords_bohr", ctypes.POINTER(ctypes.c_double)),
        ("hirshfeld", ctypes.POINTER(ctypes.c_double)),
        ("n_periodic", ctypes.c_int),
        ("lattice_bohr", ctypes.POINTER(ctypes.c_double)),
        ("scs_cut_A", ctypes.c_double),
        ("cfdm_cut_A", ctypes.c_double),
        ("sc_cut_A", ctypes.c_double),
        ("vacuum", ctypes.c_int * 3),
        ("xc", ctypes.c_int),
    ]


class CResult(ctypes.Structure):
    _fields_ = [
        ("energy_Ha", ctypes.c_double),
        ("c6_mol", ctypes.c_double),
        ("nimag", ctypes.c_int),
        ("status", ctypes.c_int),
        ("supercell", ctypes.c_int * 3),
        ("refine_iters", ctypes.c_int),
        ("err_est", ctypes.c_double * 3),
        ("alpha_eff", ctypes.POINTER(ctypes.c_double)),
        ("c6_eff", ctypes.POINTER(ctypes.c_double)),
        ("alpha_iw", ctypes.POINTER(ctypes.c_double)),
        ("molpol_eig", ctypes.POINTER(ctypes.c_double)),
    ]


_LIB = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the CUDA library; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise OSError(f"{path} not found: build it with `python -m mbd_b200.build`")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    lib.mbd_rsscs_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int]
    lib.mbd_rsscs_create.restype = ctypes.c_int
    lib.mbd_rsscs_destroy.argtypes = [vp]
    lib.mbd_rsscs_destroy.restype = None
    lib.mbd_rsscs_energy.argtypes = [vp, ctypes.POINTER(CGeom), ctypes.c_int, ctypes.POINTER(CResult)]
    lib.mbd_rsscs_energy.restype = ctypes.c_int
    lib.mbd_rsscs_energy_batch.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CGeom), ctypes.c_int,
                                           ctypes.POINTER(CResult)]
    lib.mbd_rsscs_energy_batch.restype = ctypes.c_int
    lib.mbd_rsscs_upload.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CGeom)]
    lib.mbd_rsscs_upload.restype = ctypes.c_int
    lib.mbd_rsscs_compute.argtypes = [vp, ctypes.c_int]
    lib.mbd_rsscs_compute.restype = ctypes.c_int
    lib.mbd_rsscs_download.argtypes = [vp, ctypes.POINTER(CResult)]
    lib.mbd_rsscs_download.restype = ctypes.c_int
    lib.mbd_rsscs_element_z.argtypes = [ctypes.c_char_p]
    lib.mbd_rsscs_element_z.restype = ctypes.c_int
    lib.mbd_rsscs_strerror.argtypes = [ctypes.c_int]
    lib.mbd_rsscs_strerror.restype = ctypes.c_char_p
    lib.mbd_rsscs_vdw_params.argtypes = [ctypes.c_int] + [ctypes.POINTER(ctypes.c_double)] * 3
    lib.mbd_rsscs_vdw_params.restype = ctypes.c_int
    lib.mbd_rsscs_frequency_grid.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                             ctypes.c_int]
    lib.mbd_rsscs_frequency_grid.restype = ctypes.c_int
    lib.mbd_rsscs_last_timings.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    lib.mbd_rsscs_last_timings.restype = ctypes.c_int
    lib.mbd_rsscs_last_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    lib.mbd_rsscs_last_stats.restype = ctypes.c_int
    lib.mbd_rsscs_stream.argtypes = [vp]
    lib.mbd_rsscs_stream.restype = ctypes.c_void_p
    lib.mbd_rsscs_eigvalsh.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_double)]
    lib.mbd_rsscs_eigvalsh.restype = ctypes.c_int
    lib.mbd_rsscs_eigh.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    lib.mbd_rsscs_eigh.restype = ctypes.c_int
    fp = ctypes.POINTER(ctypes.c_float)
    ip = ctypes.POINTER(ctypes.c_int)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.mbd_rsscs_learned_param_count.argtypes = []
    lib.mbd_rsscs_learned_param_count.restype = ctypes.c_int
    lib.mbd_rsscs_learned_train.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CGeom), ctypes.c_int, ctypes.c_double,
                                            ctypes.c_int, dp]
    lib.mbd_rsscs_learned_train.restype = ctypes.c_int
    lib.mbd_rsscs_learned_get_params.argtypes = [vp, fp, ctypes.c_int]
    lib.mbd_rsscs_learned_get_params.restype = ctypes.c_int
    lib.mbd_rsscs_learned_set_params.argtypes = [vp, fp, ctypes.c_int]
    lib.mbd_rsscs_learned_set_params.restype = ctypes.c_int
    lib.mbd_rsscs_set_option.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    lib.mbd_rsscs_set_option.restype = ctypes.c_int
    lib.mbd_rsscs_get_option.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.mbd_rsscs_get_option.restype = ctypes.c_int
    lib.mbd_rsscs_autotune.argtypes = [vp, ctypes.c_int]
    lib.mbd_rsscs_autotune.restype = ctypes.c_int
    lib.mbd_rsscs_tuning.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    lib.mbd_rsscs_tuning.restype = ctypes.c_int
    lib.mbd_rsscs_learned_use_network.argtypes = [vp, ctypes.c_int]
    lib.mbd_rsscs_learned_use_network.restype = ctypes.c_int
    lib.mbd_rsscs_learned_eval.argtypes = [vp, fp, ctypes.c_int, ctypes.c_int, ip, ip, fp, fp, fp, fp, fp, dp]
    lib.mbd_rsscs_learned_eval.restype = ctypes.c_int
    _LIB = lib
    return lib


@functools.lru_cache(maxsize=512)
def element_z(symbol: str) -> int:
    return load_library().mbd_rsscs_element_z(symbol.encode())


def strerror(code: int) -> str:
    return load_library().mbd_rsscs_strerror(code).decode()


def frequency_grid():
    """(omega, weight): the 21 imaginary frequencies (Hartree) and Casimir-Polder
    weights the engine integrates with (mbd_rsscs_frequency_grid)."""
    w = np.zeros(21)
    wt = np.zeros(21)
    dp = ctypes.POINTER(ctypes.c_double)
    code = load_library().mbd_rsscs_frequency_grid(w.ctypes.data_as(dp), wt.ctypes.data_as(dp), 21)
    if code != MBD_OK:
        raise MbdError(code, strerror(code))
    return w, wt


@dataclass
class Result:
    energy: float
    c6_mol: float
    nimag: int
    status: int
    supercell: tuple
    refine_iters: int
    err_est: tuple
    alpha_eff: np.ndarray
    c6_eff: np.ndarray
    alpha_iw: np.ndarray      # (21, N)
    mol_pol_eig: np.ndarray   # (21, 3)


class _Packed:
    """Host arrays of one geometry kept alive for the duration of a call."""

    def __init__(self, geo: Geometry, st: Settings, z: np.ndarray | None = None):
        self.z = np.ascontiguousarray(z if z is not None else
                                      np.array([element_z(s) for s in geo.names], dtype=np.int32))
        self.coords = np.ascontiguousarray(geo.coords / BOHR, dtype=np.float64)   # MBD_rsSCS.f90:211
        self.hirsh = np.ascontiguousarray(geo.hirshfeld, dtype=np.float64)
        # lattice(3,3) column-major, columns = vectors == rows of geo.lattice in C order
        self.lat = np.ascontiguousarray(geo.lattice / BOHR, dtype=np.float64)      # MBD_rsSCS.f90:212
        N = len(self.hirsh)
        g = CGeom()
        g.n_atoms = N
        g.z = self.z.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        g.coords_bohr = self.coords.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        g.hirshfeld = self.hirsh.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        g.n_periodic = int(geo.n_periodic)
        g.lattice_bohr = self.lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        g.scs_cut_A = float(st.mbd_scs_dip_cutoff)
        g.cfdm_cut_A = float(st.mbd_cfdm_dip_cutoff)
        g.sc_cut_A = float(st.mbd_supercell_cutoff)
        for k in range(3):
            g.vacuum[k] = int(bool(st.mbd_scs_vacuum_axis[k]))
        g.xc = int(st.xc)
        self.geom = g
        self.out_alpha = np.zeros(N)
        self.out_c6 = np.zeros(N)
        self.out_aiw = np.zeros(N_FREQ * N)
        self.out_eig = np.zeros(N_FREQ * 3)

    def result_struct(self) -> CResult:
        r = CResult()
        r.alpha_eff = self.out_alpha.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        r.c6_eff = self.out_c6.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        r.alpha_iw = self.out_aiw.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        r.molpol_eig = self.out_eig.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        return r

    def to_result(self, r: CResult) -> Result:
        N = len(self.hirsh)
        return Result(
            energy=r.energy_Ha, c6_mol=r.c6_mol, nimag=r.nimag, status=r.status,
            supercell=tuple(r.supercell), refine_iters=r.refine_iters, err_est=tuple(r.err_est),
            alpha_eff=self.out_alpha.copy(), c6_eff=self.out_c6.copy(),
            alpha_iw=self.out_aiw.reshape(N, N_FREQ).T.copy(),
            mol_pol_eig=self.out_eig.reshape(3, N_FREQ).T.copy())


class Engine:
    """One device context (mbd_rsscs_create)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        self.ctx = ctypes.c_void_p()
        code = self.lib.mbd_rsscs_create(ctypes.byref(self.ctx), int(device))
        if code != MBD_OK:
            raise MbdError(code, strerror(code))
        self._packed = []

    def close(self):
        if self.ctx:
            self.lib.mbd_rsscs_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- one geometry (MBD_at_rsSCS) -----------------------------------------
    def energy(self, geo: Geometry, st: Settings | None = None, mode: str = "plain",
               check: bool = True) -> Result:
        return self.energy_batch([geo], [st or Settings()], mode, check)[0]

    # -- many geometries -----------------------------------------------------
    def energy_batch(self, geos, sts, mode: str = "plain", check: bool = True):
        packs = [_Packed(g, s) for g, s in zip(geos, sts)]
        garr = (CGeom * len(packs))(*[p.geom for p in packs])
        rarr = (CResult * len(packs))(*[p.result_struct() for p in packs])
        code = self.lib.mbd_rsscs_energy_batch(self.ctx, len(packs), garr, MODES[mode], rarr)
        res = [p.to_result(rarr[i]) for i, p in enumerate(packs)]
        if check and code != MBD_OK and all(r.status == code for r in res) and code in (6, 8, 10, 1, 12):
            raise MbdError(code, strerror(code))
        return res

    # -- split form for device-resident timing --------------------------------
    def upload(self, geos, sts) -> int:
        self._packed = [_Packed(g, s) for g, s in zip(geos, sts)]
        self._garr = (CGeom * len(self._packed))(*[p.geom for p in self._packed])
        return self.lib.mbd_rsscs_upload(self.ctx, len(self._packed), self._garr)

    def compute(self, mode: str = "plain") -> int:
        return self.lib.mbd_rsscs_compute(self.ctx, MODES[mode])

    def download(self):
        rarr = (CResult * len(self._packed))(*[p.result_struct() for p in self._packed])
        code = self.lib.mbd_rsscs_download(self.ctx, rarr)
        return code, [p.to_result(rarr[i]) for i, p in enumerate(self._packed)]

    def eigvalsh(self, H: np.ndarray) -> np.ndarray:
        """Eigenvalues (ascending) of a symmetric matrix; only its lower
        triangle is read (mbd_rsscs_eigvalsh)."""
        H = np.ascontiguousarray(H, dtype=np.float64)
        n = H.shape[0]
        w = np.zeros(n)
        code = self.lib.mbd_rsscs_eigvalsh(self.ctx, H.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n,
                                           H.shape[1], w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if code != MBD_OK:
            raise MbdError(code, strerror(code))
        return w

    def eigh(self, H: np.ndarray):
        """(w, Z): eigenvalues ascending and orthonormal eigenvectors as the
        columns of Z, H @ Z[:, k] = w[k] Z[:, k] (numpy.linalg.eigh's layout);
        only the lower triangle of H is read (mbd_rsscs_eigh)."""
        H = np.ascontiguousarray(H, dtype=np.float64)
        n = H.shape[0]
        w = np.zeros(n)
        Z = np.zeros((n, n))
        dp = ctypes.POINTER(ctypes.c_double)
        code = self.lib.mbd_rsscs_eigh(self.ctx, H.ctypes.data_as(dp), n, H.shape[1], w.ctypes.data_as(dp),
                                       Z.ctypes.data_as(dp), n)
        if code != MBD_OK:
            raise MbdError(code, strerror(code))
        return w, Z

    # -- learned warm start (MBD_MODE_MIXED_LEARNED) --------------------------
    def learned_train(self, geos, sts, epochs: int = 20, lr: float = 2e-3, seed: int = 0) -> np.ndarray:
        """Trains the context's network on direct relay solutions of the
        given geometries (replaces the uploaded batch); returns the mean
        loss of every epoch."""
        packs = [_Packed(g, s) for g, s in zip(geos, sts)]
        garr = (CGeom * len(packs))(*[p.geom for p in packs])
        loss = np.zeros(epochs)
        code = self.lib.mbd_rsscs_learned_train(self.ctx, len(packs), garr, int(epochs), float(lr), int(seed),
                                                loss.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        self._packed = []
        if code != MBD_OK:
            raise MbdError(code, strerror(code))
        return loss

    def learned_params(self) -> np.ndarray:
        n = self.lib.mbd_rsscs_learned_param_count()
        out = np.zeros(n, dtype=np.float32)
        code = self.lib.mbd_rsscs_learned_get_params(self.ctx, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n)
        if code != MBD_OK:
            raise MbdError(code, strerror(code))
        return out

    def set_learned_params(self, params) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        code = self.lib.mbd_rsscs_learned_set_params(self.ctx, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                     p.size)
        if code != MBD_OK:
            raise MbdError(code, strerror(code))

    def set_option(self, name: str, value: float) -> None:
        """mbd_rsscs_set_option: residual_gate, wait_limit_s, test_stall_wait, fp32_tensor_build."""
        code = self.lib.mbd_rsscs_set_option(self.ctx, OPTIONS[name], float(value))
        if code != MBD_OK:
            raise MbdError(code, strerror(code))

    def get_option(self, name: str) -> float:
        v = ctypes.c_double()
        code = self.lib.mbd_rsscs_get_option(self.ctx, OPTIONS[name], ctypes.byref(v))
        if code != MBD_OK:
            raise MbdError(code, strerror(code))
        return v.value

    def autotune(self, max_n: int) -> list:
        """mbd_rsscs_autotune up to Hamiltonians of max_n rows; returns the
        choices per size class (mbd_rsscs_tuning)."""
        code = self.lib.mbd_rsscs_autotune(self.ctx, int(max_n))
        if code != MBD_OK:
            raise MbdError(code, strerror(code))
        return self.tuning()

    def tuning(self) -> list:
        buf = (ctypes.c_double * 64)()
        k = self.lib.mbd_rsscs_tuning(self.ctx, buf, 64)
        out = []
        for i in range(max(0, k)):
            o = buf[8 * i:8 * i + 8]
            if o[0] <= 0:
                continue
            out.append({"n": int(o[0]), "panel_qr": {0: "householder", 1: "tsqr"}.get(int(o[5]), "default"),
                        "panel_rows_per_cta": int(o[1]),
                        "chase": "flag" if int(o[2]) < 0 else f"cluster{int(o[2])}",
                        "dense_to_band_ms": o[3], "chase_ms": o[4],
                        "flag_chase_ms": o[6], "cluster_chase_ms": o[7]})
        return out

    def save_network(self, path: str) -> None:
        """Write the context's network to `path` (write_network_file)."""
        write_network_file(path, self.learned_params())

    def load_network(self, path: str) -> None:
        """Load a network written by save_network (checked: magic, version,
        parameter count, SHA-256 of the parameters)."""
        self.set_learned_params(read_network_file(path))

    def use_network(self, on: bool) -> None:
        self.lib.mbd_rsscs_learned_use_network(self.ctx, 1 if on else 0)

    def learned_eval(self, params, n_atoms, n_freq, off, nbr, dvec, x, S_true=None):
        """The network's kernels on explicit inputs: returns (S_pred (M,3,3),
        grad or None, loss or None)."""
        f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        P, dv, xx = f32(params), f32(dvec), f32(x)
        o, nb = i32(off), i32(nbr)
        M = n_atoms * n_freq
        S = np.zeros((M, 9), dtype=np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        ip = ctypes.POINTER(ctypes.c_int)
        grad = loss = None
        st_ptr = g_ptr = None
        l_ptr = None
        if S_true is not None:
            St = f32(np.asarray(S_true).reshape(M, 9))
            grad = np.zeros(P.size, dtype=np.float32)
            lbuf = np.zeros(1)
            st_ptr, g_ptr = St.ctypes.data_as(fp), grad.ctypes.data_as(fp)
            l_ptr = lbuf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        code = self.lib.mbd_rsscs_learned_eval(self.ctx, P.ctypes.data_as(fp), int(n_atoms), int(n_freq),
                                               o.ctypes.data_as(ip), nb.ctypes.data_as(ip), dv.ctypes.data_as(fp),
                                               xx.ctypes.data_as(fp), st_ptr, S.ctypes.data_as(fp), g_ptr, l_ptr)
        if code != MBD_OK:
            raise MbdError(code, strerror(code))
        if S_true is not None:
            loss = float(lbuf[0])
        return S.reshape(M, 3, 3), grad, loss

    def stats(self) -> dict:
        buf = (ctypes.c_double * 8)()
        self.lib.mbd_rsscs_last_stats(self.ctx, buf, 8)
        return {"launches": int(buf[0]), "h2d_bytes": int(buf[1]), "d2h_bytes": int(buf[2]),
                "graph_replayed": buf[3] == 1.0, "first_compute_graph": buf[3] == 2.0,
                "network_edges": int(buf[4]), "graph_updates": int(buf[5]),
                "graph_update_result": int(buf[6]), "graph_update_node": int(buf[7])}

    def stream_handle(self) -> int:
        """cudaStream_t of this context (for recording caller-side events)."""
        return int(self.lib.mbd_rsscs_stream(self.ctx) or 0)

    def timings(self) -> dict:
        buf = (ctypes.c_double * 12)()
        self.lib.mbd_rsscs_last_timings(self.ctx, buf, 12)
        keys = ["total", "setup", "relay_build", "relay_factor", "relay_solve", "cfdm_build",
                "tridiag", "eig_energy", "tridiag_dense_to_band", "tridiag_to_tridiagonal",
                "tridiag_one_stage_launch", "tridiag_band_chase_launch"]
        return dict(zip(keys, list(buf)))
