"""ctypes front end of the CPU FP64 oracle (oracle/rsdft_oracle.cpp).

TEST INFRASTRUCTURE ONLY: used by tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py as the checker and the
timed CPU restatement of the reference's CPU path.  The product library never
imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
MDMAX = 12


class OrcProb(C.Structure):
    _fields_ = [
        ("n1", C.c_int), ("n2", C.c_int), ("n3", C.c_int), ("md", C.c_int),
        ("dV", C.c_double),
        ("coef_lap", (C.c_double * MDMAX) * 3),
        ("coef_lap0", C.c_double),
        ("const_k2", C.c_double),
        ("zc_re", (C.c_double * (2 * MDMAX + 1)) * 3),
        ("zc_im", (C.c_double * (2 * MDMAX + 1)) * 3),
        ("pc_c0", C.c_double), ("pc_c", C.c_double * 3),
        ("vloc", C.POINTER(C.c_double)),
        ("nzlma", C.c_int), ("maxmjj", C.c_int),
        ("mjj", C.POINTER(C.c_int)), ("jjp", C.POINTER(C.c_int)),
        ("uv_re", C.POINTER(C.c_double)), ("uv_im", C.POINTER(C.c_double)),
        ("npair", C.c_int),
        ("pairs", C.POINTER(C.c_int)), ("dij", C.POINTER(C.c_double)),
        ("ncg", C.c_int), ("mloop", C.c_int),
        ("is_complex", C.c_int),
        ("cggs", C.c_int),
        ("ggg_x", C.c_double * 3),
        ("coef_nab", (C.c_double * MDMAX) * 3),
    ]


def build() -> str:
    """Compile liborc.so in place (make); returns its path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liborc.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liborc.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        P = C.POINTER(OrcProb)
        vp = C.c_void_p
        for name in ("orc_hpsi_d", "orc_hpsi_z", "orc_precond_d", "orc_precond_z"):
            getattr(_LIB, name).argtypes = [P, vp, vp, C.c_int]
        for name in ("orc_cg_d", "orc_cg_z", "orc_residual_d", "orc_residual_z"):
            getattr(_LIB, name).argtypes = [P, vp, C.c_int, vp, vp]
        for name in ("orc_gs_d", "orc_gs_z"):
            getattr(_LIB, name).argtypes = [P, vp, C.c_int]
        for name in ("orc_sd_d", "orc_sd_z"):
            getattr(_LIB, name).argtypes = [P, vp, C.c_int, vp]
            getattr(_LIB, name).restype = C.c_int
        for name in ("orc_sweep_d", "orc_sweep_z"):
            getattr(_LIB, name).argtypes = [P, vp, C.c_int, C.c_int, vp, vp]
            getattr(_LIB, name).restype = C.c_int
        _LIB.orc_dense_kinetic_d.argtypes = [P, vp]
        _LIB.orc_set_threads.argtypes = [C.c_int]
    return _LIB


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


class Oracle:
    """Oracle bound to one k-point of a :class:`rsdft_develop_b200.synth.Problem`."""

    def __init__(self, prob, k: int = 0, ncg: int = 3, mloop: int = 3, nonlocal_on: bool = True, cggs: int = 0):
        self.prob = prob
        self.k = k
        p = OrcProb()
        p.n1, p.n2, p.n3 = prob.n
        p.md = prob.md
        p.dV = prob.dV
        kin = prob.kin
        for d in range(3):
            for m in range(prob.md):
                p.coef_lap[d][m] = kin["coef_lap"][d, m]
            for m in range(2 * prob.md + 1):
                p.zc_re[d][m] = kin["zcoef_kin"][k, d, m].real
                p.zc_im[d][m] = kin["zcoef_kin"][k, d, m].imag
        p.coef_lap0 = kin["coef_lap0"]
        p.const_k2 = kin["const_k2"][k]
        ggg = np.asarray(kin.get("ggg", np.ones(3)), np.float64)
        if ggg.size >= 6 and np.any(ggg[3:6] != 0.0):
            for q in range(3):
                p.ggg_x[q] = float(ggg[3 + q])
            for d in range(3):
                for m in range(prob.md):
                    p.coef_nab[d][m] = kin["coef_nab"][d, m]
        h = prob.h
        p.pc_c0 = 3.0 / h ** 2
        for d in range(3):
            p.pc_c[d] = -0.5 / h ** 2
        self._keep = []

        def ptr(a, ct):
            a = np.ascontiguousarray(a)
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(ct))

        p.vloc = ptr(prob.vloc.astype(np.float64), C.c_double)
        p.nzlma = prob.nzlma if nonlocal_on else 0
        p.maxmjj = prob.maxmjj
        p.mjj = ptr(prob.mjj.astype(np.int32), C.c_int)
        p.jjp = ptr(prob.jjp.astype(np.int32), C.c_int)
        uv = prob.uvk[k]
        p.uv_re = ptr(np.real(uv).astype(np.float64), C.c_double)
        p.uv_im = ptr(np.imag(uv).astype(np.float64), C.c_double) if prob.is_complex else None
        p.npair = prob.pairs.shape[0] if nonlocal_on else 0
        p.pairs = ptr(prob.pairs.astype(np.int32), C.c_int)
        p.dij = ptr(prob.dij.astype(np.float64), C.c_double)
        p.ncg = ncg
        p.mloop = mloop
        p.is_complex = 1 if prob.is_complex else 0
        p.cggs = int(cggs)
        self.p = p
        self.dtype = np.complex128 if prob.is_complex else np.float64
        self.sfx = "z" if prob.is_complex else "d"

    def _arr(self, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        return a

    def hpsi(self, psi: np.ndarray) -> np.ndarray:
        psi = self._arr(psi)
        nb = psi.shape[0] if psi.ndim == 2 else 1
        out = np.zeros_like(psi)
        getattr(lib(), "orc_hpsi_" + self.sfx)(C.byref(self.p), psi.ctypes.data, out.ctypes.data, nb)
        return out

    def precond(self, g: np.ndarray) -> np.ndarray:
        g = self._arr(g)
        nb = g.shape[0] if g.ndim == 2 else 1
        pg = g.copy()
        getattr(lib(), "orc_precond_" + self.sfx)(C.byref(self.p), g.ctypes.data, pg.ctypes.data, nb)
        return pg

    def cg(self, psi: np.ndarray):
        u = self._arr(psi).copy()
        nb = u.shape[0]
        esp = np.zeros(nb)
        res = np.zeros(nb)
        getattr(lib(), "orc_cg_" + self.sfx)(C.byref(self.p), u.ctypes.data, nb, esp.ctypes.data,
                                             res.ctypes.data)
        return u, esp, res

    def gram_schmidt(self, psi: np.ndarray) -> np.ndarray:
        u = self._arr(psi).copy()
        getattr(lib(), "orc_gs_" + self.sfx)(C.byref(self.p), u.ctypes.data, u.shape[0])
        return u

    def subspace_diag(self, psi: np.ndarray):
        u = self._arr(psi).copy()
        esp = np.zeros(u.shape[0])
        info = getattr(lib(), "orc_sd_" + self.sfx)(C.byref(self.p), u.ctypes.data, u.shape[0],
                                                   esp.ctypes.data)
        if info != 0:
            raise RuntimeError(f"oracle eigensolver info={info}")
        return u, esp

    def residual(self, psi: np.ndarray):
        u = self._arr(psi)
        nb = u.shape[0]
        esp = np.zeros(nb)
        res = np.zeros(nb)
        getattr(lib(), "orc_residual_" + self.sfx)(C.byref(self.p), u.ctypes.data, nb,
                                                   esp.ctypes.data, res.ctypes.data)
        return esp, res

    def sweep(self, psi: np.ndarray, nsweep: int):
        u = self._arr(psi).copy()
        nb = u.shape[0]
        esp = np.zeros(nb)
        res = np.zeros(nb)
        info = getattr(lib(), "orc_sweep_" + self.sfx)(C.byref(self.p), u.ctypes.data, nb, nsweep,
                                                      esp.ctypes.data, res.ctypes.data)
        if info != 0:
            raise RuntimeError(f"oracle sweep info={info}")
        return u, esp, res

    def dense_kinetic(self) -> np.ndarray:
        ng = self.prob.ng
        H = np.zeros((ng, ng))
        lib().orc_dense_kinetic_d(C.byref(self.p), H.ctypes.data)
        return H
