"""Python host mirror of RSDFT's band-update module interfaces over the C ABI.

The reference's Fortran procedures and their counterparts here:

=====================================================  ===================================
reference (RSDFT_DEVELOP)                              this module
=====================================================  ===================================
``hamiltonian(tpsi, htpsi, n, k, s)``                  :meth:`BandUpdate.hamiltonian`
(src/hamiltonian_module.f90:44-46,118-172)
``conjugate_gradient(n1, n2, k, s, unk, esp, res)``    :meth:`BandUpdate.conjugate_gradient`
(src/conjugate_gradient/cg_module.f90:53-109)
``gram_schmidt(n0, n1, k, s)``                         :meth:`BandUpdate.gram_schmidt`
(src/gram_schmidt/gram_schmidt_module.f90:35-79)
``subspace_diag(k, s, unk, esp)``                      :meth:`BandUpdate.subspace_diag`
(src/subspace_diag/subspace_diag_module.f90:17-32)
``calc_sweep`` (src/sweep_module.f90:64-248)           :meth:`BandUpdate.calc_sweep`
=====================================================  ===================================

k and s are 1-based as in the reference.  Every call goes to ``librsdft_b200.so``;
there is no CPU fallback: a missing or unloadable library raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import synth

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librsdft_b200.so")

PREC_FP64, PREC_MIXED = 0, 1
PC_NONE, PC_HPRSDFT, PC_LEARNED = 0, 4, 100
MEM_HOST, MEM_DEVICE = 0, 1
MDMAX = 12

ERRORS = {
    -1: "RSDFT_ERR_ARG", -2: "RSDFT_ERR_OOM", -3: "RSDFT_ERR_CUDA", -4: "RSDFT_ERR_NOT_SPD",
    -5: "RSDFT_ERR_EIG", -6: "RSDFT_ERR_TIMEOUT", -7: "RSDFT_ERR_STATE", -8: "RSDFT_ERR_UNSUPPORTED",
    -9: "RSDFT_ERR_NUMERIC",
}

# Every symbol declared in include/rsdft_b200.h (checked by tests).
EXPORTS = [
    "rsdft_gpu_init", "rsdft_gpu_finalize", "rsdft_gpu_last_error", "rsdft_gpu_get_stream",
    "rsdft_gpu_synchronize", "rsdft_gpu_set_kpoint", "rsdft_gpu_set_vloc", "rsdft_gpu_set_projectors",
    "rsdft_gpu_set_uvk_d", "rsdft_gpu_set_uvk_z", "rsdft_gpu_set_wf_d", "rsdft_gpu_get_wf_d",
    "rsdft_gpu_set_wf_z", "rsdft_gpu_get_wf_z", "rsdft_gpu_random_wf", "rsdft_gpu_write_wf", "rsdft_gpu_read_wf",
    "rsdft_gpu_hamiltonian_d",
    "rsdft_gpu_hamiltonian_z", "rsdft_gpu_hamiltonian_f", "rsdft_gpu_hamiltonian_c",
    "rsdft_gpu_conjugate_gradient", "rsdft_gpu_gram_schmidt", "rsdft_gpu_subspace_diag",
    "rsdft_gpu_residual", "rsdft_gpu_precond_d", "rsdft_gpu_precond_f", "rsdft_gpu_set_pc_form", "rsdft_gpu_sweep", "rsdft_gpu_profile",
    "rsdft_gpu_profile_get", "rsdft_gpu_kernel_launches", "rsdft_gpu_selftest_gemm", "rsdft_gpu_set_gemm_terms", "rsdft_gpu_set_gemm_tile", "rsdft_gpu_set_nl_form", "rsdft_gpu_set_stencil_form", "rsdft_gpu_init_sweep", "rsdft_gpu_set_wait_polls", "rsdft_gpu_set_precision", "rsdft_gpu_set_cggs", "rsdft_gpu_set_sweep_check", "rsdft_gpu_set_gemm_schedule",
    "rsdft_gpu_hamiltonian_noalloc_d",
    "rsdft_gpu_set_vion", "rsdft_gpu_set_rho", "rsdft_gpu_get_rho", "rsdft_gpu_density", "rsdft_gpu_normalize_density",
    "rsdft_gpu_potential", "rsdft_gpu_init_mixing", "rsdft_gpu_sqerr", "rsdft_gpu_mix_density", "rsdft_gpu_xc_pbe",
    "rsdft_gpu_lpc_init", "rsdft_gpu_lpc_set_weights", "rsdft_gpu_lpc_get_weights", "rsdft_gpu_lpc_forward",
    "rsdft_gpu_lpc_loss_grad", "rsdft_gpu_lpc_dataset", "rsdft_gpu_lpc_harvest", "rsdft_gpu_lpc_dataset_get",
    "rsdft_gpu_lpc_dataset_add", "rsdft_gpu_lpc_train", "rsdft_gpu_lpc_precond_f", "rsdft_gpu_lpc_status",
    "rsdft_gpu_lpc_inference",
]
LPC_NWEIGHTS = 14688


class RsdftError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("n1", C.c_int), ("n2", C.c_int), ("n3", C.c_int), ("md", C.c_int),
        ("hgrid", C.c_double * 3), ("dv", C.c_double),
        ("coef_lap", (C.c_double * MDMAX) * 3), ("coef_lap0", C.c_double),
        ("ggg", C.c_double * 3),
        ("nk", C.c_int), ("nspin", C.c_int), ("mb", C.c_int), ("is_complex", C.c_int),
        ("precision", C.c_int), ("pc_mode", C.c_int), ("ncg", C.c_int), ("mloop", C.c_int),
        ("cg_block", C.c_int),
    ]


_LIB = None


def load_library(path: str = LIB_PATH):
    """Load librsdft_b200.so (build it in place first if absent); never falls back."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        from . import build as _build
        _build.build()
    lib = C.CDLL(path)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    sig = {
        "rsdft_gpu_init": [C.POINTER(Params)], "rsdft_gpu_finalize": [],
        "rsdft_gpu_get_stream": [C.POINTER(C.c_void_p)], "rsdft_gpu_synchronize": [],
        "rsdft_gpu_set_kpoint": [i, vp, d, i], "rsdft_gpu_set_vloc": [vp, i, i],
        "rsdft_gpu_set_projectors": [i, i, vp, vp, vp, i, vp, vp],
        "rsdft_gpu_set_uvk_d": [i, vp], "rsdft_gpu_set_uvk_z": [i, vp],
        "rsdft_gpu_set_wf_d": [i, i, vp, i, i], "rsdft_gpu_get_wf_d": [i, i, vp, i, i],
        "rsdft_gpu_set_wf_z": [i, i, vp, i, i], "rsdft_gpu_get_wf_z": [i, i, vp, i, i],
        "rsdft_gpu_random_wf": [i, i, C.c_uint64],
        "rsdft_gpu_write_wf": [C.c_char_p, i, vp, vp, vp, vp], "rsdft_gpu_read_wf": [C.c_char_p, vp],
        "rsdft_gpu_set_vion": [vp, i], "rsdft_gpu_set_rho": [vp, i], "rsdft_gpu_get_rho": [vp, vp, vp],
        "rsdft_gpu_density": [vp], "rsdft_gpu_normalize_density": [d], "rsdft_gpu_potential": [vp],
        "rsdft_gpu_init_mixing": [i, d], "rsdft_gpu_sqerr": [vp], "rsdft_gpu_mix_density": [vp],
        "rsdft_gpu_xc_pbe": [vp, vp, vp],
        "rsdft_gpu_hamiltonian_d": [i, i, vp, vp, i, i, i], "rsdft_gpu_hamiltonian_z": [i, i, vp, vp, i, i, i],
        "rsdft_gpu_hamiltonian_f": [i, i, vp, vp, i, i, i], "rsdft_gpu_hamiltonian_c": [i, i, vp, vp, i, i, i],
        "rsdft_gpu_conjugate_gradient": [i, i, vp, vp], "rsdft_gpu_gram_schmidt": [i, i],
        "rsdft_gpu_subspace_diag": [i, i, vp], "rsdft_gpu_residual": [i, i, vp, vp],
        "rsdft_gpu_precond_d": [i, vp, vp, i, i, i],
        "rsdft_gpu_precond_f": [i, vp, vp, i, i, i],
        "rsdft_gpu_set_pc_form": [i],
        "rsdft_gpu_sweep": [i, d, C.POINTER(C.c_int), vp, vp],
        "rsdft_gpu_selftest_gemm": [i, i, C.c_longlong, i, C.POINTER(C.c_double)],
        "rsdft_gpu_set_gemm_terms": [i, i], "rsdft_gpu_set_gemm_tile": [i], "rsdft_gpu_set_nl_form": [i],
        "rsdft_gpu_set_stencil_form": [i],
        "rsdft_gpu_set_wait_polls": [i], "rsdft_gpu_set_precision": [i], "rsdft_gpu_set_cggs": [i],
        "rsdft_gpu_set_sweep_check": [i], "rsdft_gpu_set_gemm_schedule": [d, d],
        "rsdft_gpu_init_sweep": [i],
        "rsdft_gpu_hamiltonian_noalloc_d": [i, i, vp, vp, i, i],
        "rsdft_gpu_lpc_init": [C.c_ulonglong], "rsdft_gpu_lpc_set_weights": [vp, i],
        "rsdft_gpu_lpc_get_weights": [vp, i], "rsdft_gpu_lpc_forward": [vp, vp, i, i, i, i, i, i],
        "rsdft_gpu_lpc_loss_grad": [vp, vp, i, i, i, C.POINTER(C.c_double), vp, i],
        "rsdft_gpu_lpc_dataset": [i, i],
        "rsdft_gpu_lpc_harvest": [i, i, i, d, i, C.c_ulonglong, C.POINTER(C.c_int)],
        "rsdft_gpu_lpc_dataset_get": [i, i, vp, vp],
        "rsdft_gpu_lpc_dataset_add": [vp, vp, i, C.POINTER(C.c_int)],
        "rsdft_gpu_lpc_train": [i, i, i, d, C.c_ulonglong, vp],
        "rsdft_gpu_lpc_precond_f": [vp, vp, i, i], "rsdft_gpu_lpc_inference": [i],
        "rsdft_gpu_lpc_status": [C.POINTER(C.c_int)] * 4,
        "rsdft_gpu_profile": [i], "rsdft_gpu_profile_get": [C.c_char_p, C.POINTER(C.c_double),
                                                            C.POINTER(C.c_longlong), C.POINTER(C.c_double),
                                                            C.POINTER(C.c_double)],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    lib.rsdft_gpu_last_error.restype = C.c_char_p
    lib.rsdft_gpu_last_error.argtypes = []
    lib.rsdft_gpu_kernel_launches.restype = C.c_longlong
    lib.rsdft_gpu_kernel_launches.argtypes = []
    _LIB = lib
    return lib


def _call(fn, *args):
    r = fn(*args)
    if r != 0:
        raise RsdftError(r, load_library().rsdft_gpu_last_error().decode())
    return r


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class BandUpdate:
    """One library context holding the operator of a synthetic problem and its wavefunctions."""

    def __init__(self, prob: "synth.Problem", precision: int = PREC_FP64, pc_mode: int = PC_HPRSDFT,
                 ncg: int = 3, mloop: int = 3, cg_block: int = 0, nonlocal_on: bool = True,
                 nspin: int = 1):
        ggg = np.asarray(prob.kin["ggg"], np.float64)
        if ggg.size > 3 and np.any(ggg[3:] != 0.0):
            raise NotImplementedError("non-orthogonal cell: the device stencil has no cross-derivative "
                                      "terms (ggg(4:6) of init_kinetic)")
        self.lib = load_library()
        self.prob = prob
        self.cplx = prob.is_complex
        p = Params()
        p.n1, p.n2, p.n3 = prob.n
        p.md = prob.md
        for d in range(3):
            p.hgrid[d] = prob.h
            p.ggg[d] = prob.kin["ggg"][d]
            for m in range(prob.md):
                p.coef_lap[d][m] = prob.kin["coef_lap"][d, m]
        p.dv = prob.dV
        p.coef_lap0 = prob.kin["coef_lap0"]
        p.nk = prob.nk
        p.nspin = nspin
        p.mb = prob.nband
        p.is_complex = 1 if self.cplx else 0
        p.precision = precision
        p.pc_mode = pc_mode
        p.ncg, p.mloop, p.cg_block = ncg, mloop, cg_block
        self.params = p
        self.precision = precision
        _call(self.lib.rsdft_gpu_init, C.byref(p))
        self._open = True
        for k in range(prob.nk):
            nabk = np.zeros((3, MDMAX))
            nabk[:, :prob.md] = prob.kin["coef_nabk"][k]
            _call(self.lib.rsdft_gpu_set_kpoint, k + 1, _ptr(nabk), float(prob.kin["const_k2"][k]), int(prob.nband_k[k]))
        for s in range(1, nspin + 1):
            v = np.ascontiguousarray(prob.vloc, dtype=np.float64)
            _call(self.lib.rsdft_gpu_set_vloc, _ptr(v), prob.ng, s)
        if nonlocal_on and prob.nzlma > 0:
            self._set_projectors()
        else:
            _call(self.lib.rsdft_gpu_set_projectors, 0, 0, None, None, None, 0, None, None)

    def set_vloc(self, vloc: np.ndarray, s: int = 1):
        """Local potential of spin s (Vloc(:, s) of the reference, src/localpot_module.f90)."""
        v = np.ascontiguousarray(vloc, dtype=np.float64)
        assert v.size == self.prob.ng
        _call(self.lib.rsdft_gpu_set_vloc, _ptr(v), self.prob.ng, s)

    def set_kpoint_operator(self, prob: "synth.Problem", ik: int, k: int = 1, nonlocal_on: bool = True):
        """Point k-point slot k of this context at k-point ik of prob (same grid, atoms and Dij):
        its kinetic coefficients (coef_nabk, const_k2) and projector phases uVk."""
        nabk = np.zeros((3, MDMAX))
        nabk[:, :prob.md] = prob.kin["coef_nabk"][ik]
        _call(self.lib.rsdft_gpu_set_kpoint, k, _ptr(nabk), float(prob.kin["const_k2"][ik]), self.nband(k))
        if nonlocal_on and prob.nzlma > 0:
            u = np.ascontiguousarray(prob.uvk[ik], np.complex128)
            _call(self.lib.rsdft_gpu_set_uvk_z, k, _ptr(u))

    def _set_projectors(self):
        pr = self.prob
        mjj = np.ascontiguousarray(pr.mjj, np.int32)
        jjp = np.ascontiguousarray(pr.jjp, np.int32)
        amap = np.ascontiguousarray(pr.amap, np.int32)
        pairs = np.ascontiguousarray(pr.pairs, np.int32)
        dij = np.ascontiguousarray(pr.dij, np.float64)
        _call(self.lib.rsdft_gpu_set_projectors, pr.nzlma, pr.maxmjj, _ptr(mjj), _ptr(jjp), _ptr(amap),
              pairs.shape[0], _ptr(pairs), _ptr(dij))
        for k in range(pr.nk):
            if self.cplx:
                u = np.ascontiguousarray(pr.uvk[k], np.complex128)
                _call(self.lib.rsdft_gpu_set_uvk_z, k + 1, _ptr(u))
            else:
                u = np.ascontiguousarray(pr.uvk[k], np.float64)
                _call(self.lib.rsdft_gpu_set_uvk_d, k + 1, _ptr(u))

    # ---- context ----
    def close(self):
        if getattr(self, "_open", False):
            self.lib.rsdft_gpu_finalize()
            self._open = False

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def synchronize(self):
        _call(self.lib.rsdft_gpu_synchronize)

    def stream(self) -> int:
        s = C.c_void_p()
        _call(self.lib.rsdft_gpu_get_stream, C.byref(s))
        return s.value or 0

    # ---- wavefunctions ----
    def nband(self, k: int = 1) -> int:
        return int(self.prob.nband_k[k - 1])

    def set_wf(self, unk: np.ndarray, k: int = 1, s: int = 1):
        nb = unk.shape[0]
        if self.cplx:
            a = np.ascontiguousarray(unk, np.complex128)
            _call(self.lib.rsdft_gpu_set_wf_z, k, s, _ptr(a), self.prob.ng, nb)
        else:
            a = np.ascontiguousarray(unk, np.float64)
            _call(self.lib.rsdft_gpu_set_wf_d, k, s, _ptr(a), self.prob.ng, nb)

    def get_wf(self, k: int = 1, s: int = 1) -> np.ndarray:
        nb = self.nband(k)
        if self.cplx:
            a = np.zeros((nb, self.prob.ng), np.complex128)
            _call(self.lib.rsdft_gpu_get_wf_z, k, s, _ptr(a), self.prob.ng, nb)
        else:
            a = np.zeros((nb, self.prob.ng), np.float64)
            _call(self.lib.rsdft_gpu_get_wf_d, k, s, _ptr(a), self.prob.ng, nb)
        return a

    def set_wf_host(self, ptr: int, nb: int, k: int = 1, s: int = 1):
        """set_wf from a raw host pointer (e.g. pinned memory) holding nb bands of ML0 points."""
        fn = self.lib.rsdft_gpu_set_wf_z if self.cplx else self.lib.rsdft_gpu_set_wf_d
        _call(fn, k, s, C.c_void_p(ptr), self.prob.ng, nb)

    def get_wf_host(self, ptr: int, nb: int, k: int = 1, s: int = 1):
        """get_wf into a raw host pointer (e.g. pinned memory) with room for nb bands."""
        fn = self.lib.rsdft_gpu_get_wf_z if self.cplx else self.lib.rsdft_gpu_get_wf_d
        _call(fn, k, s, C.c_void_p(ptr), self.prob.ng, nb)

    def random_wf(self, seed: int, k: int = 1, s: int = 1):
        _call(self.lib.rsdft_gpu_random_wf, k, s, C.c_uint64(seed))

    # ---- the four module procedures ----
    def write_wf(self, path: str, oc: int = 1, occ=None, aa=None, bb=None, kbb=None):
        """write_wf_simple: the resident bands of every (k, s) in the reference's wf file format
        (oc 1/3: FP64 records, 4/5: FP32 records)."""
        def opt(x, shape):
            if x is None:
                return None
            return np.asfortranarray(np.asarray(x, dtype=np.float64).reshape(shape, order="F"))
        nk = int(self.prob.nk)
        mb = int(max(self.prob.nband_k))
        ns = int(self.params.nspin)
        o, a_, b_, k_ = opt(occ, (mb, nk, ns)), opt(aa, (3, 3)), opt(bb, (3, 3)), opt(kbb, (3, nk))
        _call(self.lib.rsdft_gpu_write_wf, path.encode(), int(oc), *(None if x is None else x.ctypes.data_as(C.c_void_p)
                                                                    for x in (o, a_, b_, k_)))

    def read_wf(self, path: str) -> np.ndarray:
        """read_wf_simple: a wf file (this library's or the reference's) into the resident bands;
        returns the file's occupations occ(MB, MK, MS) (Fortran order)."""
        nk = int(self.prob.nk)
        # the band count of the file is read from its header record (third record)
        with open(path, "rb") as f:
            import struct
            recs = []
            for _ in range(3):
                (m,) = struct.unpack("<i", f.read(4))
                recs.append(f.read(m))
                f.read(4)
        newfmt = struct.unpack("<i", recs[0][:4])[0] < 0
        mb = struct.unpack("<i", (recs[2] if newfmt else recs[1])[:4])[0]
        occ = np.zeros((mb, nk, int(self.params.nspin)), order="F")
        _call(self.lib.rsdft_gpu_read_wf, path.encode(), occ.ctypes.data_as(C.c_void_p))
        return occ

    # ---- SCF pieces ----
    def set_vion(self, vion: np.ndarray):
        v = np.ascontiguousarray(vion, dtype=np.float64)
        _call(self.lib.rsdft_gpu_set_vion, _ptr(v), self.prob.ng)

    def set_rho(self, rho: np.ndarray):
        r = np.ascontiguousarray(rho, dtype=np.float64).reshape(-1)
        assert r.size == self.prob.ng * self.params.nspin
        _call(self.lib.rsdft_gpu_set_rho, _ptr(r), self.prob.ng)

    def get_rho(self):
        ns = int(self.params.nspin)
        rho = np.zeros((ns, self.prob.ng))
        vh = np.zeros(self.prob.ng)
        vxc = np.zeros((ns, self.prob.ng))
        _call(self.lib.rsdft_gpu_get_rho, _ptr(rho), _ptr(vh), _ptr(vxc))
        return rho, vh, vxc

    def density(self, occ: np.ndarray):
        """occ: (nspin, nk, mb) occupations (k weights and spin factor included)."""
        o = np.ascontiguousarray(occ, dtype=np.float64)
        assert o.shape == (int(self.params.nspin), int(self.prob.nk), int(self.params.mb))
        _call(self.lib.rsdft_gpu_density, _ptr(o))

    def normalize_density(self, nelec: float):
        _call(self.lib.rsdft_gpu_normalize_density, float(nelec))

    def potential(self) -> np.ndarray:
        ene = np.zeros(4)
        _call(self.lib.rsdft_gpu_potential, _ptr(ene))
        return ene

    def init_mixing(self, mmix: int = 4, beta: float = 1.1):
        _call(self.lib.rsdft_gpu_init_mixing, int(mmix), float(beta))

    def sqerr(self) -> np.ndarray:
        e = np.zeros(2 * int(self.params.nspin))
        _call(self.lib.rsdft_gpu_sqerr, _ptr(e))
        return e

    def xc_pbe(self, rho: np.ndarray):
        """GGA-PBE V_xc (nspin, ng) and (E_x, E_c) of the host density rho (nspin, ng) on the device."""
        ns = int(self.params.nspin)
        r = np.ascontiguousarray(rho, dtype=np.float64).reshape(ns, self.prob.ng)
        v = np.zeros((ns, self.prob.ng))
        e = np.zeros(2)
        _call(self.lib.rsdft_gpu_xc_pbe, _ptr(r), _ptr(v), _ptr(e))
        return v, float(e[0]), float(e[1])

    def mix_density(self) -> float:
        b = np.zeros(1)
        _call(self.lib.rsdft_gpu_mix_density, _ptr(b))
        return float(b[0])

    def hamiltonian(self, tpsi: np.ndarray, k: int = 1, s: int = 1, fp32: bool = False) -> np.ndarray:
        """htpsi = H tpsi for a host block tpsi[nb][ML0] (hamiltonian(tpsi,htpsi,n,k,s))."""
        tpsi = np.atleast_2d(tpsi)
        nb = tpsi.shape[0]
        ng = self.prob.ng
        if self.cplx:
            dt = np.complex64 if fp32 else np.complex128
            fn = self.lib.rsdft_gpu_hamiltonian_c if fp32 else self.lib.rsdft_gpu_hamiltonian_z
        else:
            dt = np.float32 if fp32 else np.float64
            fn = self.lib.rsdft_gpu_hamiltonian_f if fp32 else self.lib.rsdft_gpu_hamiltonian_d
        a = np.ascontiguousarray(tpsi, dt)
        out = np.zeros_like(a)
        _call(fn, k, s, _ptr(a), _ptr(out), ng, nb, MEM_HOST)
        return out

    def hamiltonian_device(self, tpsi_ptr: int, htpsi_ptr: int, nb: int, k: int = 1, s: int = 1,
                           fp32: bool = False):
        """Device-pointer form (both pointers from the caller's CUDA allocation)."""
        if self.cplx:
            fn = self.lib.rsdft_gpu_hamiltonian_c if fp32 else self.lib.rsdft_gpu_hamiltonian_z
        else:
            fn = self.lib.rsdft_gpu_hamiltonian_f if fp32 else self.lib.rsdft_gpu_hamiltonian_d
        _call(fn, k, s, C.c_void_p(tpsi_ptr), C.c_void_p(htpsi_ptr), self.prob.ng, nb, MEM_DEVICE)

    def hamiltonian_noalloc_device(self, tpsi_ptr: int, htpsi_ptr: int, nb: int, k: int = 1, s: int = 1):
        """hamiltonian on caller-owned device blocks without any device allocation: the nonlocal
        scratch is a fixed 4 MiB array inside the library (for callers that cannot let a library
        call cudaMalloc).  nb x projector slots must stay <= 524288; concurrent calls race."""
        _call(self.lib.rsdft_gpu_hamiltonian_noalloc_d, k, s, C.c_void_p(tpsi_ptr), C.c_void_p(htpsi_ptr),
              self.prob.ng, nb)

    def precond(self, gk: np.ndarray, k: int = 1) -> np.ndarray:
        g = np.ascontiguousarray(np.atleast_2d(gk), np.float64)
        out = np.zeros_like(g)
        _call(self.lib.rsdft_gpu_precond_d, k, _ptr(g), _ptr(out), self.prob.ng, g.shape[0], MEM_HOST)
        return out

    def precond_f32(self, gk: np.ndarray, k: int = 1) -> np.ndarray:
        """precond_hprsdft on FP32 bands (the mixed-precision CG's evaluation)."""
        g = np.ascontiguousarray(np.atleast_2d(gk), np.float32)
        out = np.zeros_like(g)
        _call(self.lib.rsdft_gpu_precond_f, k, _ptr(g), _ptr(out), self.prob.ng, g.shape[0], MEM_HOST)
        return out

    def conjugate_gradient(self, k: int = 1, s: int = 1):
        nb = self.nband(k)
        esp = np.zeros(nb)
        res = np.zeros(nb)
        _call(self.lib.rsdft_gpu_conjugate_gradient, k, s, _ptr(esp), _ptr(res))
        return esp, res

    def gram_schmidt(self, n0: int = 1, n1: int | None = None, k: int = 1, s: int = 1):
        if n0 != 1 or (n1 is not None and n1 != self.nband(k)):
            raise RsdftError(-1, "gram_schmidt orthonormalises bands 1..nband")
        _call(self.lib.rsdft_gpu_gram_schmidt, k, s)

    def subspace_diag(self, k: int = 1, s: int = 1) -> np.ndarray:
        esp = np.zeros(self.nband(k))
        _call(self.lib.rsdft_gpu_subspace_diag, k, s, _ptr(esp))
        return esp

    def residual(self, k: int = 1, s: int = 1):
        nb = self.nband(k)
        esp = np.zeros(nb)
        res = np.zeros(nb)
        _call(self.lib.rsdft_gpu_residual, k, s, _ptr(esp), _ptr(res))
        return esp, res

    def set_precision(self, precision: int):
        """Switch between PREC_MIXED and PREC_FP64, converting the resident wavefunctions (the
        FP64 final polish of a mixed-precision solve is set_precision(PREC_FP64) + calc_sweep)."""
        _call(self.lib.rsdft_gpu_set_precision, int(precision))
        self.precision = precision

    def sweep_check(self, iconv_check: int):
        """Convergence test of calc_sweep: 0 FP64 residual <= tol, 2 eigenvalue change < tol
        (the reference's conv_check_2)."""
        _call(self.lib.rsdft_gpu_set_sweep_check, int(iconv_check))

    def init_sweep(self, mb_ref: int = 0):
        """Check convergence on bands 1..mb_ref (0: all), as init_sweep(..., mb_ref, ...)."""
        _call(self.lib.rsdft_gpu_init_sweep, int(mb_ref))

    def calc_sweep(self, nsweep: int, tol: float = 0.0):
        """CG -> GS -> SD sweeps over all (k, s) until max FP64 residual <= tol."""
        nk, mb = self.prob.nk, self.prob.nband
        esp = np.zeros((self.params.nspin, nk, mb))
        res = np.zeros((self.params.nspin, nk, mb))
        it = C.c_int(0)
        _call(self.lib.rsdft_gpu_sweep, nsweep, float(tol), C.byref(it), _ptr(esp), _ptr(res))
        return it.value, esp, res

    # ---- learned preconditioner ----
    def lpc_init(self, seed: int = 1):
        _call(self.lib.rsdft_gpu_lpc_init, int(seed))

    def lpc_set_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, np.float32).ravel()
        _call(self.lib.rsdft_gpu_lpc_set_weights, _ptr(w), w.size)

    def lpc_get_weights(self) -> np.ndarray:
        w = np.zeros(LPC_NWEIGHTS, np.float32)
        _call(self.lib.rsdft_gpu_lpc_get_weights, _ptr(w), w.size)
        return w

    def lpc_forward(self, x: np.ndarray, periodic: bool = False) -> np.ndarray:
        """Network output for x of shape (nb, n3, n2, n1) (no input scaling)."""
        x = np.ascontiguousarray(x, np.float32)
        nb, n3, n2, n1 = x.shape
        y = np.zeros_like(x)
        _call(self.lib.rsdft_gpu_lpc_forward, _ptr(x), _ptr(y), nb, n1, n2, n3, 1 if periodic else 0, MEM_HOST)
        return y

    def lpc_loss_grad(self, x: np.ndarray, t: np.ndarray, margin: int):
        """(loss, dloss/dw) for patches x, t of shape (nb, n, n, n)."""
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        nb, n = x.shape[0], x.shape[1]
        loss = C.c_double(0.0)
        g = np.zeros(LPC_NWEIGHTS, np.float32)
        _call(self.lib.rsdft_gpu_lpc_loss_grad, _ptr(x), _ptr(t), nb, n, margin, C.byref(loss), _ptr(g), MEM_HOST)
        return loss.value, g

    def lpc_dataset(self, capacity: int, patch: int = 16):
        _call(self.lib.rsdft_gpu_lpc_dataset, int(capacity), int(patch))

    def lpc_harvest(self, npatch: int, sigma: float = 2.5, iters: int = 30, seed: int = 1, k: int = 1,
                    s: int = 1) -> int:
        """Cut (gradient, screened-kinetic correction) patch pairs from the resident bands."""
        added = C.c_int(0)
        _call(self.lib.rsdft_gpu_lpc_harvest, k, s, int(npatch), float(sigma), int(iters), int(seed),
              C.byref(added))
        return added.value

    def lpc_dataset_get(self, first: int, count: int, patch: int):
        x = np.zeros((count, patch, patch, patch), np.float32)
        t = np.zeros_like(x)
        _call(self.lib.rsdft_gpu_lpc_dataset_get, first, count, _ptr(x), _ptr(t))
        return x, t

    def lpc_dataset_add(self, x: np.ndarray, t: np.ndarray) -> int:
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        added = C.c_int(0)
        _call(self.lib.rsdft_gpu_lpc_dataset_add, _ptr(x), _ptr(t), x.shape[0], C.byref(added))
        return added.value

    def lpc_train(self, epochs: int, batch: int = 32, lr: float = 2e-3, margin: int = 4, seed: int = 1):
        losses = np.zeros(epochs)
        _call(self.lib.rsdft_gpu_lpc_train, int(margin), int(epochs), int(batch), float(lr), int(seed),
              _ptr(losses))
        return losses

    def lpc_precond(self, g: np.ndarray) -> np.ndarray:
        """Learned preconditioner on full bands (nb, ng), FP32."""
        g = np.ascontiguousarray(np.atleast_2d(g), np.float32)
        out = np.zeros_like(g)
        _call(self.lib.rsdft_gpu_lpc_precond_f, _ptr(g), _ptr(out), g.shape[0], MEM_HOST)
        return out

    def lpc_inference(self, fp32: bool):
        """Evaluate the network on CUDA cores in FP32 (True) or on the tensor cores (False, default)."""
        _call(self.lib.rsdft_gpu_lpc_inference, 1 if fp32 else 0)

    def lpc_status(self):
        """(weights ready, PC mode in use by CG, learned-to-plain fallbacks, harvested pairs)."""
        v = [C.c_int(0) for _ in range(4)]
        _call(self.lib.rsdft_gpu_lpc_status, *[C.byref(x) for x in v])
        return tuple(x.value for x in v)

    # ---- measurement ----
    def profile(self, on):
        """Per-kernel CUDA-event timing: False/0 off, True/1 every kernel family, 2 the hpsi
        stencil only."""
        _call(self.lib.rsdft_gpu_profile, int(on))

    def profile_get(self, name: str):
        """(total ms, launches, algorithmic bytes, algorithmic flops) of a kernel family."""
        ms = C.c_double(0.0)
        n = C.c_longlong(0)
        by = C.c_double(0.0)
        fl = C.c_double(0.0)
        _call(self.lib.rsdft_gpu_profile_get, name.encode(), C.byref(ms), C.byref(n), C.byref(by), C.byref(fl))
        return ms.value, n.value, by.value, fl.value

    def selftest_gemm(self, m: int, n: int, k: int, op: int) -> float:
        """Relative error of the split-BF16 tensor-core GEMM against cuBLAS DGEMM."""
        e = C.c_double(0.0)
        _call(self.lib.rsdft_gpu_selftest_gemm, m, n, k, op, C.byref(e))
        return e.value

    def pc_form(self, form) -> None:
        """FP32 precond_hprsdft evaluation inside CG: 3 (the default) the s-step form in separate
        passes with the CG direction formed by its last pass, 1 (or True) the same leaving Pg for
        separate direction passes, 2 the fused z-streamed s-step form, 0 (or False) the
        recurrence form."""
        _call(self.lib.rsdft_gpu_set_pc_form, int(form))

    def stencil_form(self, vloc_global: bool) -> None:
        """Real build's hpsi stencil: V_loc rows staged in shared memory (False, the default) or
        read from L2 by the consumer threads (True)."""
        _call(self.lib.rsdft_gpu_set_stencil_form, int(bool(vloc_global)))

    def nl_form(self, fused: bool) -> None:
        """Nonlocal term of the real hpsi: inside the stencil (fused) or by a scatter after it."""
        _call(self.lib.rsdft_gpu_set_nl_form, 1 if fused else 0)

    def cggs(self, iswitch: int) -> None:
        """SWGS: orthogonalise CG's preconditioned gradients against the lower bands (1) or all
        other bands (2), or not at all (0, the default)."""
        _call(self.lib.rsdft_gpu_set_cggs, int(iswitch))

    def wait_polls(self, polls: int) -> None:
        """Polls of the hpsi stencil's bounded waits (0: give up at once; < 0: the default)."""
        _call(self.lib.rsdft_gpu_set_wait_polls, int(polls))

    def gemm_tile(self, wide: bool = True, tri: int = 1, update: bool = False) -> None:
        """Three-term GEMM tiles: 128 x 256 over K blocks of 32 (default) or 128 x 128 over 64;
        tri: 1 the overlap S by upper-triangle tiles (default), 2 S and Hsub, 0 neither;
        update: the band rotation in update form.  The defaults are the library's."""
        flags = (1 if wide else 0) | (0 if update else 4)
        if tri:
            flags |= 2 | (8 if tri == 2 else 0)
        _call(self.lib.rsdft_gpu_set_gemm_tile, flags)

    def gemm_schedule(self, res_sm: float, res_rot: float) -> None:
        """Two BF16 terms in the overlap/Hsub (rotation) contractions of a sweep while CG's
        largest residual is above res_sm (res_rot); 0 switches a threshold off."""
        _call(self.lib.rsdft_gpu_set_gemm_schedule, float(res_sm), float(res_rot))

    def gemm_terms(self, overlap: int, rotation: int) -> None:
        """BF16 terms (2 or 3) of the mixed-precision overlap/Hsub and rotation contractions."""
        _call(self.lib.rsdft_gpu_set_gemm_terms, overlap, rotation)

    def kernel_launches(self) -> int:
        return int(self.lib.rsdft_gpu_kernel_launches())
